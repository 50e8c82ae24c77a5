// Host-side scene recording: the reference's Canvas for the vector path.
//
// Record layouts and allocation rules follow src/canvas/paths.rs:65-156
// (path records, backdrop pool, segment slices), src/shared/brush.rs:249-340
// (brush blob), src/canvas/compile.rs:39-331 and
// src/shared/execution/batches.rs (draw batches, painter order).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <atomic>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/tileink.h"
#include "../../include/tileink_canvas.h"
#include "../../include/tileink_diff.h"
#include "flatten_core.h"
#include "host.h"
#include "planner.h"
#include "stroke_core.h"

namespace {

using tkf::Pt;

// A flattened point together with its weights over the four control points of
// the cubic being flattened: every point the flattener emits is a fixed linear
// combination of them once the subdivision is fixed.
struct WPt {
    Pt v;
    double w[4];
};
inline WPt operator+(const WPt& a, const WPt& b) {
    return {a.v + b.v, {a.w[0] + b.w[0], a.w[1] + b.w[1], a.w[2] + b.w[2], a.w[3] + b.w[3]}};
}
inline WPt operator-(const WPt& a, const WPt& b) {
    return {a.v - b.v, {a.w[0] - b.w[0], a.w[1] - b.w[1], a.w[2] - b.w[2], a.w[3] - b.w[3]}};
}
inline WPt operator*(const WPt& a, double s) { return {a.v * s, {a.w[0] * s, a.w[1] * s, a.w[2] * s, a.w[3] * s}}; }
inline const Pt& val(const WPt& p) { return p.v; }

enum Verb : uint8_t { MOVE, LINE, QUAD, CUBIC, CLOSE };
struct El {
    Verb verb;
    Pt p[3];
};

}  // namespace

struct tk_path {
    std::vector<El> els;
};

namespace {

// Flattening: the shared host/device flattener (flatten_core.h).
using tkf::flatten_cubic;
using tkf::flatten_quad;

// PathFlatten::flatten (src/shared/path_flatten.rs:20-82): closes open
// contours whose gap exceeds 1e-6 and drops edges with length^2 <= 1e-24.
void flatten_path(const tk_path& path, double tol, uint32_t path_id, std::vector<tk_line>& out) {
    bool has_start = false;
    Pt start{0, 0}, last{0, 0};
    auto push = [&](Pt a, Pt b) {
        double dx = a.x - b.x, dy = a.y - b.y;
        if (!(dx * dx + dy * dy > 1.0e-12 * 1.0e-12)) return;
        out.push_back(tk_line{path_id, 0.0f, {float(a.x), float(a.y)}, {float(b.x), float(b.y)}});
    };
    auto open_close = [&]() {
        if (!has_start) return;
        double dx = start.x - last.x, dy = start.y - last.y;
        if (dx * dx + dy * dy > 1.0e-6 * 1.0e-6) push(last, start);
    };
    auto emit = [&](Pt p) {
        push(last, p);
        last = p;
    };
    for (const El& e : path.els) {
        switch (e.verb) {
            case MOVE:
                open_close();
                start = last = e.p[0];
                has_start = true;
                break;
            case LINE:
                if (has_start) emit(e.p[0]);
                else { start = last = e.p[0]; has_start = true; }
                break;
            case QUAD:
                if (!has_start) { start = last = e.p[0]; has_start = true; }
                flatten_quad(last, e.p[0], e.p[1], tol, emit);
                break;
            case CUBIC: {
                if (!has_start) { start = last = e.p[0]; has_start = true; }
                Pt c[4] = {last, e.p[0], e.p[1], e.p[2]};
                flatten_cubic(c, tol, emit);
                break;
            }
            case CLOSE:
                if (has_start) {
                    push(last, start);
                    last = start;
                }
                break;
        }
    }
    open_close();
}

// Tight bounding box of the curves (kurbo BezPath::bounding_box).
struct Box {
    double x0 = std::numeric_limits<double>::infinity(), y0 = x0, x1 = -x0, y1 = -x0;
    void add(Pt p) {
        x0 = std::min(x0, p.x); y0 = std::min(y0, p.y);
        x1 = std::max(x1, p.x); y1 = std::max(y1, p.y);
    }
    bool empty() const { return !(x1 >= x0 && y1 >= y0); }
};
void quad_extrema(Pt p0, Pt p1, Pt p2, Box& b) {
    for (int axis = 0; axis < 2; ++axis) {
        double a = axis ? p0.y : p0.x, m = axis ? p1.y : p1.x, c = axis ? p2.y : p2.x;
        double den = a - 2.0 * m + c;
        if (den != 0.0) {
            double t = (a - m) / den;
            if (t > 0.0 && t < 1.0) b.add(quad_eval(p0, p1, p2, t));
        }
    }
}
void cubic_extrema(const Pt c[4], Box& b) {
    for (int axis = 0; axis < 2; ++axis) {
        double p0 = axis ? c[0].y : c[0].x, p1 = axis ? c[1].y : c[1].x;
        double p2 = axis ? c[2].y : c[2].x, p3 = axis ? c[3].y : c[3].x;
        double qa = -p0 + 3.0 * p1 - 3.0 * p2 + p3, qb = 2.0 * (p0 - 2.0 * p1 + p2), qc = p1 - p0;
        double ts[2];
        int nt = 0;
        if (std::fabs(qa) < 1e-12) {
            if (qb != 0.0) ts[nt++] = -qc / qb;
        } else {
            double disc = qb * qb - 4.0 * qa * qc;
            if (disc >= 0.0) {
                double r = std::sqrt(disc);
                ts[nt++] = (-qb - r) / (2.0 * qa);
                ts[nt++] = (-qb + r) / (2.0 * qa);
            }
        }
        for (int k = 0; k < nt; ++k)
            if (ts[k] > 0.0 && ts[k] < 1.0) b.add(cubic_eval(c, ts[k]));
    }
}
Box path_bbox(const tk_path& path) {
    Box b;
    Pt last{0, 0};
    for (const El& e : path.els) {
        switch (e.verb) {
            case MOVE: case LINE: b.add(e.p[0]); last = e.p[0]; break;
            case QUAD: b.add(e.p[1]); quad_extrema(last, e.p[0], e.p[1], b); last = e.p[1]; break;
            case CUBIC: {
                Pt c[4] = {last, e.p[0], e.p[1], e.p[2]};
                b.add(e.p[2]);
                cubic_extrema(c, b);
                last = e.p[2];
                break;
            }
            case CLOSE: break;
        }
    }
    return b;
}

tk_path transform_path(const tk_path& p, const double m[6]) {
    tk_path out = p;
    for (El& e : out.els)
        for (Pt& q : e.p) q = {m[0] * q.x + m[2] * q.y + m[4], m[1] * q.x + m[3] * q.y + m[5]};
    return out;
}

// --------------------------------------------------------------------------
// Stroking with round joins and round caps (stroke_core.h, shared with the
// device stroker). The centerline is recorded as elements in local units:
// a polyline starts at its first drawing element with a TK_EL_MOVE at the
// current point (so a lone move_to strokes nothing), and a close marks it
// closed and returns the current point to its start. Element `path` fields
// hold the polyline index.
// --------------------------------------------------------------------------
void record_centerlines(const tk_path& path, double tol, uint32_t stroke, std::vector<tk_flatten_el>& els,
                        std::vector<tk_stroke_polyline>& polys) {
    bool open = false;
    Pt last{0, 0}, front{0, 0};
    auto element = [&](uint32_t verb, std::initializer_list<Pt> pts) {
        tk_flatten_el e{};
        e.verb = verb;
        e.path = uint32_t(polys.size() - 1);
        e.tolerance = tol;
        int k = 0;
        for (const Pt& p : pts) {
            e.p[k][0] = p.x;
            e.p[k][1] = p.y;
            ++k;
        }
        els.push_back(e);
        ++polys.back().element_count;
    };
    auto begin = [&]() {
        if (open) return;
        polys.push_back({stroke, uint32_t(els.size()), 0u, 0u});
        element(TK_EL_MOVE, {last});
        front = last;
        open = true;
    };
    for (const El& e : path.els) {
        switch (e.verb) {
            case MOVE: open = false; last = e.p[0]; break;
            case LINE: begin(); element(TK_EL_LINE, {last, e.p[0]}); last = e.p[0]; break;
            case QUAD: begin(); element(TK_EL_QUAD, {last, e.p[0], e.p[1]}); last = e.p[1]; break;
            case CUBIC: begin(); element(TK_EL_CUBIC, {last, e.p[0], e.p[1], e.p[2]}); last = e.p[2]; break;
            case CLOSE:
                if (open) {
                    polys.back().closed = 1u;
                    last = front;
                    open = false;
                }
                break;
        }
    }
}

// The outline lines of a stroke's polylines, in the device stroker's order:
// polyline by polyline, loop by loop, unit by unit.
void outline_lines(const std::vector<tk_flatten_el>& els, const tk_stroke_polyline* polys, uint32_t npl,
                   const tk_stroke_desc& S, std::vector<tk_line>& out) {
    struct Push {
        std::vector<tk_line>& out;
        uint32_t path;
        void operator()(Pt a, Pt b) {
            out.push_back(tk_line{path, 0.0f, {float(a.x), float(a.y)}, {float(b.x), float(b.y)}});
        }
    } push{out, S.path};
    tkf::Affine xf;
    std::memcpy(xf.t, S.transform, sizeof(xf.t));
    std::vector<Pt> v;
    auto add = [&](Pt p) { v.push_back(p); };
    for (uint32_t k = 0; k < npl; ++k) {
        const tk_stroke_polyline& P = polys[k];
        v.clear();
        for (uint32_t e = P.element0; e < P.element0 + P.element_count; ++e) tkf::element_points(els[e], add);
        const bool closed = P.closed != 0u;
        const uint32_t n = tkf::dedupe_polyline(v, uint32_t(v.size()), closed);
        const uint32_t loops = tkf::outline_loops(n, closed), units = tkf::outline_units(n, closed);
        for (uint32_t loop = 0; loop < loops; ++loop)
            for (uint32_t u = 0; u < units; ++u) {
                tkf::EdgeChain<Push> chain{xf, push};
                tkf::outline_unit(v, n, closed, loop, u, S.half_width, S.tolerance, chain);
            }
    }
}

// --------------------------------------------------------------------------
// Brushes (src/shared/brush.rs:249-340, 638-767; src/shared/pixel.rs:14-21).
// --------------------------------------------------------------------------
inline uint32_t u8_sat(float v) {
    if (!(v > 0.0f)) return 0u;
    if (v >= 255.0f) return 255u;
    return uint32_t(v);
}
inline uint32_t premul_f32_to_u32(const float c[4]) {
    return u8_sat(c[0] * 255.0f + 0.5f) | (u8_sat(c[1] * 255.0f + 0.5f) << 8) | (u8_sat(c[2] * 255.0f + 0.5f) << 16) |
           (u8_sat(c[3] * 255.0f + 0.5f) << 24);
}
inline uint32_t premul_color(const float rgba[4]) {
    float p[4] = {rgba[0] * rgba[3], rgba[1] * rgba[3], rgba[2] * rgba[3], rgba[3]};
    return premul_f32_to_u32(p);
}
size_t quantize_ramp_size(float span, size_t stops) {
    size_t span_samples = size_t(std::ceil(std::max(span, 1.0f) * 2.0f));
    size_t stop_samples = (std::max<size_t>(stops, 2) - 1) * 16;
    size_t target = std::min<size_t>(std::max<size_t>(std::max(span_samples, stop_samples), 64), 4096);
    size_t p = 1;
    while (p < target) p <<= 1;
    return std::min<size_t>(p, 4096);
}
// Ramp of premultiplied colors (build_ramp, src/shared/brush.rs:638-689):
// each entry is peniko's premultiplied sRGB interpolation between its two
// stops, as the `color` crate evaluates it: premul = p1 + (p2 - p1) * t and
// alpha = a1 + t * (a2 - a1), un-premultiplied (scale by 1 / alpha, by 1 at
// alpha 0) and premultiplied again before the RGBA8 store.
std::vector<uint32_t> build_ramp(const tk_gradient_stop* stops, uint32_t n, size_t size) {
    size = std::max<size_t>(size, 2);
    std::vector<uint32_t> ramp(size, 0u);
    if (n == 0) return ramp;
    std::vector<tk_gradient_stop> s(stops, stops + n);
    std::stable_sort(s.begin(), s.end(), [](const tk_gradient_stop& a, const tk_gradient_stop& b) { return a.offset < b.offset; });
    for (size_t ix = 0; ix < size; ++ix) {
        float t = float(ix) / float(size - 1);
        size_t upper = 0;
        while (upper < s.size() && s[upper].offset < t) ++upper;
        const tk_gradient_stop& l = upper == 0 ? s[0] : (upper >= s.size() ? s.back() : s[upper - 1]);
        const tk_gradient_stop& r = upper == 0 ? s[0] : (upper >= s.size() ? s.back() : s[upper]);
        float span = r.offset - l.offset;
        float lt = std::fabs(span) <= 1.1920929e-7f ? 0.0f : std::min(std::max((t - l.offset) / span, 0.0f), 1.0f);
        float lp[4] = {l.rgba[0] * l.rgba[3], l.rgba[1] * l.rgba[3], l.rgba[2] * l.rgba[3], l.rgba[3]};
        float rp[4] = {r.rgba[0] * r.rgba[3], r.rgba[1] * r.rgba[3], r.rgba[2] * r.rgba[3], r.rgba[3]};
        const float alpha = lp[3] + lt * (rp[3] - lp[3]);
        const float inv = alpha == 0.0f ? 1.0f : 1.0f / alpha;
        float c[4];
        for (int k = 0; k < 3; ++k) {
            const float premul = lp[k] + (rp[k] - lp[k]) * lt;
            c[k] = (premul * inv) * alpha;
        }
        c[3] = alpha;
        ramp[ix] = premul_f32_to_u32(c);
    }
    return ramp;
}
inline uint32_t fbits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

std::pair<uint32_t, uint32_t> push_brush(std::vector<uint32_t>& blob, const tk_brush_desc& b) {
    uint32_t offset = uint32_t(blob.size());
    uint32_t data[TK_BRUSH_HEADER_WORDS] = {TK_BRUSH_SOLID, TK_EXTEND_PAD, 0, 0, 0, 0, 0, 255, 0};
    uint32_t params[TK_BRUSH_PARAM_WORDS] = {};
    const float ident[6] = {1, 0, 0, 1, 0, 0};
    std::vector<uint32_t> ramp;
    if (b.kind == TK_BRUSH_KIND_SOLID) {
        data[4] = premul_color(b.rgba);
    } else if (b.kind == TK_BRUSH_KIND_LINEAR) {
        data[0] = TK_BRUSH_LINEAR;
        data[1] = b.extend;
        params[0] = fbits(b.p0[0]); params[1] = fbits(b.p0[1]);
        params[2] = fbits(b.p1[0]); params[3] = fbits(b.p1[1]);
        for (int k = 0; k < 6; ++k) params[4 + k] = fbits(ident[k]);
        float span = std::hypot(b.p1[0] - b.p0[0], b.p1[1] - b.p0[1]);
        ramp = build_ramp(b.stops, b.stop_count, quantize_ramp_size(span, b.stop_count));
    } else {
        data[0] = TK_BRUSH_RADIAL;
        data[1] = b.extend;
        params[0] = fbits(b.p0[0]); params[1] = fbits(b.p0[1]);
        params[2] = fbits(b.p1[0]); params[3] = fbits(b.p1[1]);
        params[4] = fbits(b.r0); params[5] = fbits(b.r1);
        for (int k = 0; k < 6; ++k) params[6 + k] = fbits(ident[k]);
        float cs = std::hypot(b.p1[0] - b.p0[0], b.p1[1] - b.p0[1]);
        float span = std::max(cs + std::fabs(b.r0) + std::fabs(b.r1), std::fabs(b.r1 - b.r0));
        ramp = build_ramp(b.stops, b.stop_count, quantize_ramp_size(span, b.stop_count));
    }
    if (!ramp.empty()) {
        data[2] = TK_BRUSH_HEADER_WORDS + TK_BRUSH_PARAM_WORDS;
        data[3] = uint32_t(ramp.size());
    }
    blob.insert(blob.end(), data, data + TK_BRUSH_HEADER_WORDS);
    blob.insert(blob.end(), params, params + TK_BRUSH_PARAM_WORDS);
    blob.insert(blob.end(), ramp.begin(), ramp.end());
    return {offset, uint32_t(blob.size()) - offset};
}

struct Cmd {
    enum Kind { DRAW, CLIP, BLUR, OPACITY } kind;
    uint32_t draw;
    float sigma;
    uint32_t children;
    uint32_t payload = 0u;     // OPACITY: opacity_f32_to_u8 of the layer's opacity; BLUR: sampling
    int32_t progressive = -1;  // BLUR of a progressive blur: its index in the canvas's progressive blurs
    int32_t filter = -1;       // BLUR of a filter layer: its index in the canvas's filter layers
};

// One recorded Canvas call with its original geometry, for replay into
// another canvas under an extra transform (a retained scene node's content).
// A glyph image with its texels shared, so that replay into another canvas
// registers the same image there.
struct GlyphImage {
    tk_glyph_image desc{};  // data_offset: where the owning canvas put the texels
    std::shared_ptr<const std::vector<uint32_t>> texels;
};

struct RecCmd {
    enum Kind : uint8_t {
        FILL, STROKE, CLIP, BLUR, POP, SDF, SDF_CLIP, IMAGE, OPACITY, GLYPHS, GLYPH_RUN, PROGRESSIVE, FILTER
    } kind = FILL;
    // FILTER: the chain as recorded (logical units), the region in shape.p0 /
    // p1, and the chain's transfer tables and kernels (f32 bits) in chain order
    std::vector<tk_canvas_filter> chain;
    std::vector<uint32_t> tables;
    bool fixed = false;
    bool region_path = false;  // FILTER: the region is `path` under the transform
    // GLYPH_RUN: the glyphs (image = index into run_images or TK_INVALID_INDEX),
    // their images and the optional clip rect
    std::vector<tk_glyph> run_glyphs;
    std::vector<GlyphImage> run_images;
    bool has_clip = false;
    int32_t clip[4] = {0, 0, 0, 0};
    tk_path path;
    tk_sdf_shape shape{};
    // IMAGE: the rect in shape.p0 / p1, the image's texels and brush options;
    // BLUR: `sampling` is the TK_BLUR_SAMPLING word
    std::shared_ptr<const std::vector<uint32_t>> texels;
    uint32_t iw = 0, ih = 0, extend = 0, sampling = 0, opacity = 255;
    bool has_brush = false;
    tk_brush_desc brush{};
    std::vector<tk_gradient_stop> stops;
    bool has_transform = false;
    double t[6] = {1, 0, 0, 1, 0, 0};
    uint32_t rule = 0;
    double tolerance = 0.1, width = 0.0;
    float sigma = 0.0f;  // BLUR: sigma; OPACITY: opacity
};

RecCmd rec_cmd(RecCmd::Kind kind, const tk_path* path, const tk_brush_desc* brush, const double* transform) {
    RecCmd r;
    r.kind = kind;
    if (path) r.path = *path;
    if (brush) {
        r.has_brush = true;
        r.brush = *brush;
        if (brush->stop_count && brush->stops) r.stops.assign(brush->stops, brush->stops + brush->stop_count);
        r.brush.stops = nullptr;
    }
    if (transform) {
        r.has_transform = true;
        std::memcpy(r.t, transform, sizeof(r.t));
    }
    return r;
}

}  // namespace

struct tk_canvas {
    uint32_t W = 0, H = 0, tw = 0, th = 0;
    float scale = 1.0f;
    bool host_plan = true;
    uint32_t clear = 0u;
    std::vector<tk_line> lines;
    std::vector<tk_path_record> paths;
    std::vector<tk_draw_record> draws;
    std::vector<uint32_t> brush;
    std::vector<uint32_t> sdf, shadow;  // SDF and SDF shadow records (Canvas::sdf_blob, sdf_shadow_blob)
    // registered images (Canvas::scene_images) and their texture table
    std::vector<std::shared_ptr<const std::vector<uint32_t>>> images;
    std::vector<tk_image_desc> image_table;
    // the text blob: glyph images (with their texels concatenated), runs and glyphs
    std::vector<GlyphImage> glyph_image_src;
    std::vector<tk_glyph_image> glyph_images;
    std::vector<uint32_t> glyph_texels;
    std::vector<tk_glyph_run> glyph_runs;
    std::vector<tk_glyph> glyphs;
    std::vector<tk_progressive_blur> progressive;  // device-pixel progressive blurs
    std::vector<tk_filter_layer> filter_layers;    // filter layers and their chains' filters
    std::vector<tk_filter> filters;
    std::vector<uint32_t> filter_words;            // transfer tables and convolution kernels
    uint32_t backdrop_pool = 0, tile_cnt = 0;
    std::vector<std::vector<Cmd>> lists{std::vector<Cmd>{}};
    std::vector<uint32_t> stack{0};
    // compiled plan
    bool dirty = true;
    std::vector<tk_layer_record> layers;
    std::vector<tk_op> ops;
    std::vector<uint32_t> order, batch_ids;
    // differentiable parameters (fills of recorded paths)
    std::vector<double> points;
    std::vector<float> colors;
    // device flattening: fills are kept as elements and strokes as centerline
    // elements, flattened (and stroked) at upload
    bool device_flatten = false;
    std::vector<tk_flatten_el> els;
    std::vector<uint32_t> path_els;  // per path: first element, element count
    std::vector<tk_flatten_el> stroke_els;
    std::vector<tk_stroke_polyline> polylines;
    std::vector<tk_stroke_desc> strokes;
    // command log for replay (tk_canvas_set_keep_commands)
    bool keep = false;
    std::vector<RecCmd> log;
    // why the last compile failed (empty: it did not)
    std::string compile_error;
};

namespace {

// flatten_path's walk with every flattening step recorded as an element
// carrying its start point instead of being flattened here.
void record_elements(const tk_path& path, double tol, uint32_t path_id, std::vector<tk_flatten_el>& out) {
    bool has_start = false;
    Pt start{0, 0}, last{0, 0};
    auto element = [&](uint32_t verb, std::initializer_list<Pt> pts) {
        tk_flatten_el e{};
        e.verb = verb;
        e.path = path_id;
        e.tolerance = tol;
        int k = 0;
        for (const Pt& p : pts) {
            e.p[k][0] = p.x;
            e.p[k][1] = p.y;
            ++k;
        }
        out.push_back(e);
    };
    auto open_close = [&]() {
        if (!has_start) return;
        double dx = start.x - last.x, dy = start.y - last.y;
        if (dx * dx + dy * dy > 1.0e-6 * 1.0e-6) element(TK_EL_LINE, {last, start});
    };
    for (const El& e : path.els) {
        switch (e.verb) {
            case MOVE:
                open_close();
                start = last = e.p[0];
                has_start = true;
                break;
            case LINE:
                if (has_start) {
                    element(TK_EL_LINE, {last, e.p[0]});
                    last = e.p[0];
                } else {
                    start = last = e.p[0];
                    has_start = true;
                }
                break;
            case QUAD:
                if (!has_start) { start = last = e.p[0]; has_start = true; }
                element(TK_EL_QUAD, {last, e.p[0], e.p[1]});
                last = e.p[1];
                break;
            case CUBIC:
                if (!has_start) { start = last = e.p[0]; has_start = true; }
                element(TK_EL_CUBIC, {last, e.p[0], e.p[1], e.p[2]});
                last = e.p[2];
                break;
            case CLOSE:
                if (has_start) {
                    element(TK_EL_LINE, {last, start});
                    last = start;
                }
                break;
        }
    }
    open_close();
}

// The device transform: the canvas scale times the path's transform.
void device_transform(const tk_canvas* c, const double* transform, double dev[6]) {
    const double s = double(c->scale);
    double m[6] = {1, 0, 0, 1, 0, 0};
    if (transform) std::memcpy(m, transform, sizeof(m));
    for (int k = 0; k < 6; ++k) dev[k] = s * m[k];
}

int64_t add_path(tk_canvas* c, const Box& bb, uint32_t line_start, uint32_t line_count, const tk_brush_desc* brush,
                 uint32_t rule, uint32_t tag, bool emit_command);

int64_t push_path_with_tag(tk_canvas* c, const tk_path& src, const tk_brush_desc* brush, const double* transform,
                           uint32_t rule, double tolerance, uint32_t tag, bool emit_command) {
    const uint32_t line_start = uint32_t(c->lines.size());
    const uint32_t path_id = uint32_t(c->paths.size());
    const double s = double(c->scale);
    double dev[6];
    device_transform(c, transform, dev);
    tk_path path = transform_path(src, dev);
    const uint32_t el0 = uint32_t(c->els.size());
    if (c->device_flatten) record_elements(path, tolerance * s, path_id, c->els);
    else flatten_path(path, tolerance * s, path_id, c->lines);
    c->path_els.push_back(el0);
    c->path_els.push_back(uint32_t(c->els.size()) - el0);
    return add_path(c, path_bbox(path), line_start, uint32_t(c->lines.size()) - line_start, brush, rule, tag,
                    emit_command);
}

// The path and draw records of a path whose lines are
// lines[line_start, + line_count) (none yet when the device makes them),
// with pixel bounds from `bb`.
int64_t add_path(tk_canvas* c, const Box& bb, uint32_t line_start, uint32_t line_count, const tk_brush_desc* brush,
                 uint32_t rule, uint32_t tag, bool emit_command) {
    const uint32_t path_id = uint32_t(c->paths.size());
    tk_pixel_bounds pb{0, 0, 0, 0};
    if (!bb.empty()) pb = {int32_t(std::floor(bb.x0)), int32_t(std::floor(bb.y0)), int32_t(std::ceil(bb.x1)), int32_t(std::ceil(bb.y1))};
    // PixelBounds::tile_bbox (src/shared/bounds.rs:113-128)
    uint32_t tx0 = std::min(uint32_t(std::max(pb.x0, 0)) / TK_TILE_SIZE, c->tw);
    uint32_t ty0 = std::min(uint32_t(std::max(pb.y0, 0)) / TK_TILE_SIZE, c->th);
    uint32_t tx1 = std::min((uint32_t(std::max(pb.x1, 0)) + TK_TILE_SIZE - 1) / TK_TILE_SIZE, c->tw);
    uint32_t ty1 = std::min((uint32_t(std::max(pb.y1, 0)) + TK_TILE_SIZE - 1) / TK_TILE_SIZE, c->th);
    uint32_t stride = tx1 > tx0 ? tx1 - tx0 : 0u, height = ty1 > ty0 ? ty1 - ty0 : 0u;
    uint32_t capacity = 0;
    if (c->host_plan) {
        for (uint32_t l = 0; l < line_count; ++l)
            capacity += tk_plan_line_tile_count(&c->lines[line_start + l], tx0, ty0, tx1, ty1);
    }
    tk_path_record rec{};
    rec.path_id = path_id;
    rec.line_count = line_count;
    rec.line_start = line_start;
    rec.data_offset = c->backdrop_pool;
    rec.data_len = stride * height;
    rec.tile_x0 = tx0; rec.tile_y0 = ty0; rec.tile_x1 = tx1; rec.tile_y1 = ty1;
    rec.segment_start = c->tile_cnt;
    rec.segment_capacity = capacity;
    rec.transform = tk_affine{1, 0, 0, 1, 0, 0};
    c->backdrop_pool += stride * height;
    c->tile_cnt += capacity;
    c->paths.push_back(rec);
    tk_brush_desc transparent{};
    transparent.kind = TK_BRUSH_KIND_SOLID;
    auto br = push_brush(c->brush, brush ? *brush : transparent);
    tk_draw_record d{};
    d.path_id = path_id;
    d.glyph_run_id = TK_INVALID_INDEX;
    d.sdf_offset = TK_INVALID_INDEX;
    d.sdf_shadow_offset = TK_INVALID_INDEX;
    d.brush_offset = br.first;
    d.brush_len = br.second;
    d.tag = tag;
    d.fill_rule = rule;
    d.pixel_bounds = pb;
    d.local_pixel_bounds = pb;
    d.transform = tk_affine{1, 0, 0, 1, 0, 0};
    d.inverse_transform = tk_affine{1, 0, 0, 1, 0, 0};
    uint32_t draw_ix = uint32_t(c->draws.size());
    c->draws.push_back(d);
    if (emit_command) c->lists[c->stack.back()].push_back({Cmd::DRAW, draw_ix, 0.0f, 0u});
    c->dirty = true;
    return draw_ix;
}

void paint_bounds(const tk_canvas* c, uint32_t list, tk_pixel_bounds& b, bool& any) {
    for (const Cmd& cmd : c->lists[list]) {
        if (cmd.kind == Cmd::DRAW) {
            const tk_pixel_bounds& p = c->draws[cmd.draw].pixel_bounds;
            if (p.x0 >= p.x1 || p.y0 >= p.y1) continue;
            if (!any) { b = p; any = true; }
            else { b.x0 = std::min(b.x0, p.x0); b.y0 = std::min(b.y0, p.y0); b.x1 = std::max(b.x1, p.x1); b.y1 = std::max(b.y1, p.y1); }
        } else {
            paint_bounds(c, cmd.children, b, any);
        }
    }
}

struct Compiled {
    struct Op {
        tk_op op;
        std::vector<uint32_t> draws;
        std::vector<tk_layer_record> stack;
    };
    std::vector<Op> ops;
};

// command_list_has_single_stack (src/canvas/compile.rs:355-378): every draw
// under `list` sits in one command list once clip and opacity layers are
// entered; a blur group below splits the draws into separate surfaces.
bool single_stack(const tk_canvas* c, uint32_t list, uint32_t stack, int64_t& first) {
    for (const Cmd& cmd : c->lists[list]) {
        if (cmd.kind == Cmd::DRAW) {
            if (first < 0) first = stack;
            else if (first != int64_t(stack)) return false;
        } else if (cmd.kind == Cmd::CLIP || cmd.kind == Cmd::OPACITY) {
            if (!single_stack(c, cmd.children, cmd.children, first)) return false;
        } else {
            return false;
        }
    }
    return true;
}

void compile_into(const tk_canvas* c, uint32_t list, std::vector<tk_layer_record>& stack, Compiled& out) {
    std::vector<uint32_t> pending;
    auto flush = [&]() {
        if (pending.empty()) return;
        Compiled::Op op{};
        op.op.kind = TK_OP_DRAW_BATCH;
        op.draws = std::move(pending);
        op.stack = stack;
        pending.clear();
        out.ops.push_back(std::move(op));
    };
    for (const Cmd& cmd : c->lists[list]) {
        if (cmd.kind == Cmd::DRAW) {
            pending.push_back(cmd.draw);
        } else if (cmd.kind == Cmd::CLIP) {
            flush();
            stack.push_back({TK_LAYER_CLIP, cmd.draw, 0u});
            compile_into(c, cmd.children, stack, out);
            stack.pop_back();
        } else if (cmd.kind == Cmd::OPACITY) {
            // A path-masked opacity layer fuses into the batch's layer stack
            // when its subtree draws in one stack (Canvas::can_fuse,
            // src/canvas/compile.rs:342-353); fine opens and closes the group
            // per batch (BEGIN_OPACITY / END_OPACITY).
            int64_t first = -1;
            if (!single_stack(c, cmd.children, cmd.children, first))
                throw std::runtime_error(
                    "an opacity layer over draws in several layer stacks needs an offscreen group, which this "
                    "path does not build");
            flush();
            stack.push_back({TK_LAYER_OPACITY, cmd.draw, cmd.payload});
            compile_into(c, cmd.children, stack, out);
            stack.pop_back();
        } else {
            flush();
            Compiled::Op begin{};
            begin.op.kind = TK_OP_BLUR_BEGIN;
            begin.op.sigma = cmd.sigma;
            begin.op.batch_id = cmd.payload;  // the blur's sampling
            begin.stack = stack;  // outer clips
            tk_pixel_bounds pb{0, 0, 0, 0};
            bool any = false;
            paint_bounds(c, cmd.children, pb, any);
            int32_t out_r = int32_t(std::ceil(std::max(cmd.sigma, 0.0f) * 3.0f));
            if (cmd.progressive >= 0) {
                // sample_outset (shared/layer/filter/progressive.rs:95-103):
                // the upper pyramid level's support with its reconstruction
                begin.op.kind = TK_OP_PROGRESSIVE_BEGIN;
                begin.op.batch_id = uint32_t(cmd.progressive);
                out_r = cmd.sigma > 0.0f ? int32_t(std::ceil(20.0f * cmd.sigma + 8.0f)) : 0;
            }
            if (cmd.filter >= 0) {
                // output bounds: the surface clipped to the canvas
                // (filter_surface_bounds, shared/layer/filter.rs:510-527)
                const int32_t* sf = c->filter_layers[size_t(cmd.filter)].surface;
                begin.op.kind = TK_OP_FILTER_BEGIN;
                begin.op.batch_id = uint32_t(cmd.filter);
                begin.op.bounds[0] = std::max(sf[0], 0);
                begin.op.bounds[1] = std::max(sf[1], 0);
                begin.op.bounds[2] = std::min(sf[2], int32_t(c->W));
                begin.op.bounds[3] = std::min(sf[3], int32_t(c->H));
                if (begin.op.bounds[2] < begin.op.bounds[0] || begin.op.bounds[3] < begin.op.bounds[1])
                    begin.op.bounds[0] = begin.op.bounds[1] = begin.op.bounds[2] = begin.op.bounds[3] = 0;
                any = false;
            }
            if (any) {
                begin.op.bounds[0] = std::max(pb.x0 - out_r, 0);
                begin.op.bounds[1] = std::max(pb.y0 - out_r, 0);
                begin.op.bounds[2] = std::min(pb.x1 + out_r, int32_t(c->W));
                begin.op.bounds[3] = std::min(pb.y1 + out_r, int32_t(c->H));
            }
            out.ops.push_back(std::move(begin));
            std::vector<tk_layer_record> inner;
            compile_into(c, cmd.children, inner, out);
            Compiled::Op end{};
            end.op.kind = TK_OP_BLUR_END;
            out.ops.push_back(std::move(end));
        }
    }
    flush();
}

void compile(tk_canvas* c) {
    if (!c->dirty) return;
    Compiled comp;
    std::vector<tk_layer_record> stack;
    c->compile_error.clear();
    try {
        compile_into(c, 0, stack, comp);
    } catch (const std::exception& e) {
        c->compile_error = e.what();
        return;
    }
    // coalesce adjacent batches with equal stacks (execution/batches.rs)
    std::vector<Compiled::Op> merged;
    for (auto& op : comp.ops) {
        if (op.op.kind == TK_OP_DRAW_BATCH && !merged.empty() && merged.back().op.kind == TK_OP_DRAW_BATCH) {
            const auto& a = merged.back().stack;
            bool same = a.size() == op.stack.size();
            for (size_t i = 0; same && i < a.size(); ++i)
                same = a[i].tag == op.stack[i].tag && a[i].draw == op.stack[i].draw && a[i].payload == op.stack[i].payload;
            if (same) {
                merged.back().draws.insert(merged.back().draws.end(), op.draws.begin(), op.draws.end());
                continue;
            }
        }
        merged.push_back(std::move(op));
    }
    c->layers.clear();
    c->ops.clear();
    c->order.clear();
    c->batch_ids.assign(c->draws.size(), TK_INVALID_INDEX);
    uint32_t next_batch = 0;
    for (auto& op : merged) {
        tk_op o = op.op;
        o.layer_start = uint32_t(c->layers.size());
        c->layers.insert(c->layers.end(), op.stack.begin(), op.stack.end());
        o.layer_end = uint32_t(c->layers.size());
        if (o.kind == TK_OP_DRAW_BATCH) {
            o.batch_id = next_batch++;
            for (uint32_t d : op.draws) {
                c->order.push_back(d);
                c->batch_ids[d] = o.batch_id;
            }
        }
        c->ops.push_back(o);
    }
    c->dirty = false;
}


// ---------------------------------------------------------------------------
// SDF shapes: physical geometry (canvas/surface.rs:193-245, 435-555), pixel
// bounds (src/shared/sdf/{rect,circle,line,shadow}.rs) and the 17-word
// records (src/shared/gpu_sdf.rs:48-260).
// ---------------------------------------------------------------------------
// Rust's float-to-int `as` cast: saturating, NaN to 0.
int32_t sat_i32(double v) {
    if (v != v) return 0;
    if (v <= -2147483648.0) return INT32_MIN;
    if (v >= 2147483647.0) return INT32_MAX;
    return int32_t(v);
}
tk_pixel_bounds box_bounds(double x0, double y0, double x1, double y1) {
    return {sat_i32(std::floor(x0)), sat_i32(std::floor(y0)), sat_i32(std::ceil(x1)), sat_i32(std::ceil(y1))};
}
// shadow_bounds (src/shared/sdf/shadow.rs:35-43), in f32
tk_pixel_bounds shadow_bounds(const tk_pixel_bounds& b, const float opt[4]) {
    const float outset = opt[2] * 4.0f + 1.0f;
    return {sat_i32(std::floor(float(b.x0) + opt[0] - outset)), sat_i32(std::floor(float(b.y0) + opt[1] - outset)),
            sat_i32(std::ceil(float(b.x1) + opt[0] + outset)), sat_i32(std::ceil(float(b.y1) + opt[1] + outset))};
}
// Circle::bounds (src/shared/sdf/circle.rs:13-20), in f32
tk_pixel_bounds circle_bounds(double cx, double cy, float r) {
    return {sat_i32(std::floor(float(cx) - r)), sat_i32(std::floor(float(cy) - r)), sat_i32(std::ceil(float(cx) + r)),
            sat_i32(std::ceil(float(cy) + r))};
}
// Line::bounds (src/shared/sdf/line.rs:51-83)
tk_pixel_bounds line_bounds(double sx, double sy, double ex, double ey, float width, uint32_t cap) {
    const double half = double(width) * 0.5;
    const double dx = ex - sx, dy = ey - sy, len = std::hypot(dx, dy);
    if (len == 0.0) return box_bounds(sx - half, sy - half, sx + half, sy + half);
    const double ux = dx / len, uy = dy / len;
    double x0 = sx, y0 = sy, x1 = ex, y1 = ey;
    if (cap == TK_SDF_CAP_SQUARE) {
        x0 -= ux * half;
        y0 -= uy * half;
        x1 += ux * half;
        y1 += uy * half;
    }
    return box_bounds(std::min(x0, x1) - half, std::min(y0, y1) - half, std::max(x0, x1) + half,
                      std::max(y0, y1) + half);
}

// The physical record and bounds of `s` (logical); false when the shape draws
// nothing (the reference's None).
bool encode_sdf(const tk_canvas* c, const tk_sdf_shape& s, uint32_t rec[TK_SDF_RECORD_WORDS], tk_pixel_bounds& pb) {
    const float sc = c->scale;
    const double sd = double(sc);
    std::memset(rec, 0, TK_SDF_RECORD_WORDS * 4);
    rec[0] = s.kind;
    auto put = [&](int i, float v) { rec[i] = fbits(v); };
    const bool shadow = s.kind == TK_SDF_RECT_SHADOW || s.kind == TK_SDF_CIRCLE_SHADOW ||
                        s.kind == TK_SDF_LINE_SHADOW || s.kind == TK_SDF_CALLOUT_SHADOW || s.kind == TK_SDF_ARC_SHADOW;
    float opt[4] = {0, 0, 0, 0};
    if (shadow) {  // ShadowOptions::normalized, then physical_shadow_options
        const float intensity = std::min(std::max(s.shadow[3], 0.0f), 1.0f);
        if (!(intensity > 0.0f)) return false;
        opt[0] = s.shadow[0] * sc;
        opt[1] = s.shadow[1] * sc;
        opt[2] = std::max(s.shadow[2], 0.0f) * sc;
        opt[3] = intensity;
        for (int k = 0; k < 4; ++k) put(13 + k, opt[k]);
    }
    const double x0 = s.p0[0] * sd, y0 = s.p0[1] * sd, x1 = s.p1[0] * sd, y1 = s.p1[1] * sd;
    switch (s.kind) {
        case TK_SDF_RECT:
        case TK_SDF_RECT_STROKE:
        case TK_SDF_RECT_SHADOW: {
            const double ax0 = std::min(x0, x1), ay0 = std::min(y0, y1), ax1 = std::max(x0, x1), ay1 = std::max(y0, y1);
            put(1, float(ax0));
            put(2, float(ay0));
            put(3, float(ax1));
            put(4, float(ay1));
            for (int k = 0; k < 4; ++k) put(5 + k, s.radii[k] * sc);
            pb = box_bounds(ax0, ay0, ax1, ay1);
            if (s.kind == TK_SDF_RECT_STROKE) {
                float half[4];  // StrokeWidths::half of the physical clamped widths
                bool any = false;
                for (int k = 0; k < 4; ++k) {
                    const float w = std::max(s.widths[k], 0.0f);
                    any = any || w != 0.0f;
                    half[k] = std::max(w * sc, 0.0f) * 0.5f;
                }
                if (!any) return false;
                for (int k = 0; k < 4; ++k) put(9 + k, half[k]);
                // RectStroke::bounds: the outer rectangle (top, right, bottom, left)
                pb = box_bounds(ax0 - double(half[3]), ay0 - double(half[0]), ax1 + double(half[1]),
                                ay1 + double(half[2]));
            }
            if (shadow) pb = shadow_bounds(pb, opt);
            return true;
        }
        case TK_SDF_CIRCLE:
        case TK_SDF_CIRCLE_STROKE:
        case TK_SDF_CIRCLE_SHADOW: {
            const float r = float(s.radius) * sc;
            put(1, float(x0));
            put(2, float(y0));
            put(3, r);
            pb = circle_bounds(x0, y0, r);
            if (s.kind == TK_SDF_CIRCLE_STROKE) {
                if (!(s.width > 0.0)) return false;
                const float hw = float(s.width * 0.5) * sc;
                for (int k = 0; k < 4; ++k) put(9 + k, hw);
                pb = circle_bounds(x0, y0, r + std::max(hw, 0.0f));
            }
            if (shadow) pb = shadow_bounds(pb, opt);
            return true;
        }
        case TK_SDF_LINE:
        case TK_SDF_LINE_SHADOW: {
            // Line::is_empty (src/shared/sdf/line.rs:45-49)
            const float w = float(s.width);
            if (s.cap > TK_SDF_CAP_ROUND) return false;
            if (w <= 0.0f || !(w == w) || (s.cap == TK_SDF_CAP_BUTT && s.p0[0] == s.p1[0] && s.p0[1] == s.p1[1]))
                return false;
            const float pw = w * sc;
            put(1, float(x0));
            put(2, float(y0));
            put(3, float(x1));
            put(4, float(y1));
            put(5, pw);
            put(6, float(s.cap));
            pb = line_bounds(x0, y0, x1, y1, pw, s.cap);
            if (shadow) pb = shadow_bounds(pb, opt);
            return true;
        }
        case TK_SDF_DASH_LINE: {
            // DashLine::is_empty (src/shared/sdf/line.rs:140-148) on the logical line
            const float w = float(s.width), dash = s.dash[0], gap = s.dash[1], off = s.dash[2];
            if (s.cap > TK_SDF_CAP_ROUND || !(gap >= 0.0f) || !(dash == dash) || !(off == off)) return false;
            if (w <= 0.0f || !(w == w) || (s.cap == TK_SDF_CAP_BUTT && s.p0[0] == s.p1[0] && s.p0[1] == s.p1[1]))
                return false;
            if (dash <= 0.0f) return false;
            const double len = std::hypot(s.p1[0] - s.p0[0], s.p1[1] - s.p0[1]);
            if (len > 0.0 && gap > 0.0f) {  // has_visible_dash
                const double cycle = double(dash) + double(gap);
                double o = std::fmod(double(off), cycle);
                if (o < 0.0) o += cycle;  // f64::rem_euclid
                if (!(o < double(dash) || cycle - o < len)) return false;
            }
            const float pw = w * sc;
            put(1, float(x0));
            put(2, float(y0));
            put(3, float(x1));
            put(4, float(y1));
            put(5, pw);
            put(6, float(s.cap));
            put(7, dash * sc);
            put(8, gap * sc);
            put(9, off * sc);
            pb = line_bounds(x0, y0, x1, y1, pw, s.cap);
            return true;
        }
        case TK_SDF_TRIANGLE: {
            // Triangle::is_empty / bounds (src/shared/sdf/triangle.rs:37-66)
            const float corner = float(s.radius);
            const double v[6] = {s.p0[0], s.p0[1], s.p1[0], s.p1[1], s.p2[0], s.p2[1]};
            for (double q : v)
                if (!std::isfinite(q)) return false;
            const double area = (v[2] - v[0]) * (v[5] - v[1]) - (v[3] - v[1]) * (v[4] - v[0]);
            if (!std::isfinite(corner) || corner < 0.0f || !std::isfinite(area) || area == 0.0) return false;
            double p[6];
            for (int k = 0; k < 6; ++k) p[k] = v[k] * sd;
            const float pc = corner * sc;
            put(1, float(p[0]));
            put(2, float(p[1]));
            put(3, float(p[2]));
            put(4, float(p[3]));
            put(5, float(p[4]));
            put(6, float(p[5]));
            put(7, pc);
            const double r = double(pc);
            pb = box_bounds(std::min(std::min(p[0], p[2]), p[4]) - r, std::min(std::min(p[1], p[3]), p[5]) - r,
                            std::max(std::max(p[0], p[2]), p[4]) + r, std::max(std::max(p[1], p[3]), p[5]) + r);
            return true;
        }
        case TK_SDF_CHECKERBOARD: {
            // Checkerboard::is_empty / bounds (src/shared/sdf/checkerboard.rs:32-58)
            const float cell = float(s.radius);
            if (!std::isfinite(s.p0[0]) || !std::isfinite(s.p0[1]) || !std::isfinite(s.p1[0]) ||
                !std::isfinite(s.p1[1]) || !std::isfinite(cell) || cell <= 0.0f || s.p0[0] == s.p1[0] ||
                s.p0[1] == s.p1[1])
                return false;
            const double ax0 = std::min(x0, x1), ay0 = std::min(y0, y1), ax1 = std::max(x0, x1), ay1 = std::max(y0, y1);
            put(1, float(ax0));
            put(2, float(ay0));
            put(3, float(ax1));
            put(4, float(ay1));
            put(5, cell * sc);
            pb = box_bounds(ax0, ay0, ax1, ay1);
            return true;
        }
        case TK_SDF_ARC:
        case TK_SDF_ARC_SHADOW: {
            // Rc::is_empty / bounds (src/shared/sdf/arc.rs:43-98) of the physical arc
            const float r = float(s.radius), wd = float(s.width), start = s.angle[0], sweep = s.angle[1];
            if (s.cap > TK_SDF_CAP_ROUND || r <= 0.0f || wd <= 0.0f || sweep == 0.0f) return false;
            const float pr = r * sc, pw = wd * sc, cx = float(x0), cy = float(y0), half = pw * 0.5f;
            put(1, cx);
            put(2, cy);
            put(3, pr);
            put(4, pw);
            put(5, start);
            put(6, sweep);
            put(7, float(s.cap));
            const float tau = 6.2831855f;
            if (std::fabs(sweep) >= tau) {
                const float rr = pr + half;
                pb = {sat_i32(std::floor(cx - rr)), sat_i32(std::floor(cy - rr)), sat_i32(std::ceil(cx + rr)),
                      sat_i32(std::ceil(cy + rr))};
            } else {
                float bx0 = INFINITY, by0 = INFINITY, bx1 = -INFINITY, by1 = -INFINITY;
                auto include = [&](float a) {
                    const float px = cx + pr * std::cos(a), py = cy + pr * std::sin(a);
                    bx0 = std::min(bx0, px);
                    by0 = std::min(by0, py);
                    bx1 = std::max(bx1, px);
                    by1 = std::max(by1, py);
                };
                auto norm = [&](float a) { return a - std::floor(a / tau) * tau; };  // normalize_angle
                include(start);
                include(start + sweep);
                const float axes[4] = {0.0f, 1.5707964f, 3.1415927f, 3.1415927f + 1.5707964f};
                for (float a : axes)
                    if (sweep >= 0.0f ? norm(a - start) <= sweep : norm(start - a) <= -sweep) include(a);
                const float outset = half + 1.0f;
                pb = {sat_i32(std::floor(bx0 - outset)), sat_i32(std::floor(by0 - outset)),
                      sat_i32(std::ceil(bx1 + outset)), sat_i32(std::ceil(by1 + outset))};
            }
            if (shadow) pb = shadow_bounds(pb, opt);
            return true;
        }
        case TK_SDF_STAR:
        case TK_SDF_STAR_STROKE: {
            // Star::is_empty / expanded_bounds (src/shared/sdf/star.rs:37-90) of the physical star
            const float outer = float(s.radius), inner = s.widths[0], corner = s.widths[1], rot = s.angle[0];
            if (!std::isfinite(s.p0[0]) || !std::isfinite(s.p0[1]) || !std::isfinite(outer) || outer <= 0.0f ||
                !std::isfinite(inner) || inner <= 0.0f || inner >= outer || !std::isfinite(corner) || corner < 0.0f ||
                !std::isfinite(rot))
                return false;
            float half = 0.0f;
            if (s.kind == TK_SDF_STAR_STROKE) {
                const float hl = float(s.width) * 0.5f;
                if (!std::isfinite(hl) || hl <= 0.0f) return false;
                half = hl * sc;
            }
            const float po = outer * sc, pi_ = inner * sc, pc = corner * sc;
            put(1, float(x0));
            put(2, float(y0));
            put(3, po);
            put(4, pi_);
            put(5, pc);
            put(6, rot);
            put(9, half);
            double bx0 = INFINITY, by0 = INFINITY, bx1 = -INFINITY, by1 = -INFINITY;
            for (int i = 0; i < 10; ++i) {
                const double rr = double(i % 2 == 0 ? po : pi_);
                const double a = double(rot) + double(i) * 3.14159265358979323846 / 5.0;
                const double px = x0 + rr * std::cos(a), py = y0 + rr * std::sin(a);
                bx0 = std::min(bx0, px);
                by0 = std::min(by0, py);
                bx1 = std::max(bx1, px);
                by1 = std::max(by1, py);
            }
            const double e = double(pc) + double(half);
            pb = box_bounds(bx0 - e, by0 - e, bx1 + e, by1 + e);
            return true;
        }
        case TK_SDF_CALLOUT:
        case TK_SDF_CALLOUT_STROKE:
        case TK_SDF_CALLOUT_SHADOW: {
            // Callout::is_empty / physical / expanded_bounds (src/shared/sdf/callout.rs:83-195)
            const bool visible = !(s.flags & TK_SDF_CALLOUT_TAIL_HIDDEN);
            const float br = float(s.radius);
            const float off = s.widths[0], tw = s.widths[1], tl = s.widths[2], tr = s.widths[3];
            const double lx0 = std::min(s.p0[0], s.p1[0]), ly0 = std::min(s.p0[1], s.p1[1]);
            const double lx1 = std::max(s.p0[0], s.p1[0]), ly1 = std::max(s.p0[1], s.p1[1]);
            if (!std::isfinite(lx0) || !std::isfinite(ly0) || !std::isfinite(lx1) || !std::isfinite(ly1) ||
                lx0 >= lx1 || ly0 >= ly1 || !std::isfinite(br) || br < 0.0f || s.cap > 3u)
                return false;
            if (visible && (!std::isfinite(off) || !std::isfinite(tw) || tw <= 0.0f || !std::isfinite(tl) ||
                            tl <= 0.0f || !std::isfinite(tr) || tr < 0.0f))
                return false;
            float half = 0.0f;
            if (s.kind == TK_SDF_CALLOUT_STROKE) {  // CalloutStroke::is_empty
                const float hl = float(s.width) * 0.5f;
                if (!std::isfinite(hl) || hl <= 0.0f) return false;
                half = hl * sc;
            }
            const double ax0 = std::min(x0, x1), ay0 = std::min(y0, y1), ax1 = std::max(x0, x1), ay1 = std::max(y0, y1);
            const float ptl = visible ? tl * sc : 0.0f;
            put(1, float(ax0));
            put(2, float(ay0));
            put(3, float(ax1));
            put(4, float(ay1));
            put(5, br * sc);
            put(6, visible ? off * sc : 0.0f);
            put(7, visible ? tw * sc : 0.0f);
            put(8, ptl);
            put(9, visible ? tr * sc : 0.0f);
            put(10, visible ? float(s.cap) : 2.0f);  // a hidden tail is CalloutTail::hidden(): bottom, zeros
            put(11, half);
            put(12, visible ? 1.0f : 0.0f);
            double bx0 = ax0, by0 = ay0, bx1 = ax1, by1 = ay1;
            if (visible) {
                const double t = double(ptl);
                if (s.cap == 0u) by0 -= t;
                else if (s.cap == 1u) bx1 += t;
                else if (s.cap == 2u) by1 += t;
                else bx0 -= t;
            }
            const double extra = double(std::max(half, 0.0f));
            pb = box_bounds(bx0 - extra, by0 - extra, bx1 + extra, by1 + extra);
            if (shadow) pb = shadow_bounds(pb, opt);
            return true;
        }
        case TK_SDF_CANDLESTICK: {
            // physical_sdf (canvas/surface.rs:459-469, scaled_positive_u32 canvas.rs:214-219)
            // and CandleStick::bounds (src/shared/sdf/candlestick.rs:58-70)
            auto scaled_u32 = [&](float w) {
                const float v = std::min(std::max(std::round(w * sc), 1.0f), 4294967295.0f);
                return float(uint32_t(v));
            };
            const float cx = float(s.p0[0]) * sc, high = float(s.p0[1]) * sc, low = float(s.p2[0]) * sc;
            const float top = float(s.p1[0]) * sc, bottom = float(s.p1[1]) * sc;
            const float bw = scaled_u32(s.widths[0]), ww = scaled_u32(s.widths[1]);
            put(1, cx);
            put(2, high);
            put(3, low);
            put(4, top);
            put(5, bottom);
            put(6, bw);
            put(7, ww);
            const float bh = bw * 0.5f, wh = ww * 0.5f;
            float by0 = std::min(top, bottom), by1 = std::max(top, bottom);
            if (by0 == by1) {
                by0 -= 0.5f;
                by1 += 0.5f;
            }
            pb = {sat_i32(std::floor(std::min(cx - bh, cx - wh))), sat_i32(std::floor(std::min(by0, std::min(high, low)))),
                  sat_i32(std::ceil(std::max(cx + bh, cx + wh))), sat_i32(std::ceil(std::max(by1, std::max(high, low))))};
            return true;
        }
        default:
            return false;
    }
}

}  // namespace

extern "C" {

tk_path* tk_path_new(void) { return new tk_path(); }
void tk_path_free(tk_path* p) { delete p; }
void tk_path_move_to(tk_path* p, double x, double y) { p->els.push_back({MOVE, {{x, y}, {}, {}}}); }
void tk_path_line_to(tk_path* p, double x, double y) { p->els.push_back({LINE, {{x, y}, {}, {}}}); }
void tk_path_quad_to(tk_path* p, double x1, double y1, double x2, double y2) {
    p->els.push_back({QUAD, {{x1, y1}, {x2, y2}, {}}});
}
void tk_path_cubic_to(tk_path* p, double x1, double y1, double x2, double y2, double x3, double y3) {
    p->els.push_back({CUBIC, {{x1, y1}, {x2, y2}, {x3, y3}}});
}
void tk_path_close(tk_path* p) { p->els.push_back({CLOSE, {{}, {}, {}}}); }

uint64_t tk_path_flatten(const tk_path* p, float tolerance, uint32_t path_id, tk_line* out, uint64_t cap) {
    std::vector<tk_line> lines;
    flatten_path(*p, double(tolerance), path_id, lines);
    if (out) std::memcpy(out, lines.data(), std::min<uint64_t>(cap, lines.size()) * sizeof(tk_line));
    return lines.size();
}

tk_canvas* tk_canvas_new(uint32_t lw, uint32_t lh, float scale) {
    if (!(scale > 0.0f) || !std::isfinite(scale)) return nullptr;
    auto* c = new tk_canvas();
    c->scale = scale;
    c->W = uint32_t(std::ceil(double(lw) * scale));
    c->H = uint32_t(std::ceil(double(lh) * scale));
    c->tw = (c->W + TK_TILE_SIZE - 1) / TK_TILE_SIZE;
    c->th = (c->H + TK_TILE_SIZE - 1) / TK_TILE_SIZE;
    return c;
}
void tk_canvas_free(tk_canvas* c) { delete c; }
void tk_canvas_set_host_segment_plan(tk_canvas* c, int32_t enabled) { c->host_plan = enabled != 0; }
void tk_canvas_set_device_flatten(tk_canvas* c, int32_t enabled) {
    c->device_flatten = enabled != 0;
    if (c->device_flatten) c->host_plan = false;  // segment capacities come from the device
}
int32_t tk_canvas_flatten_desc(const tk_canvas* c, tk_flatten_desc* out) {
    if (!c || !out) return TK_E_INVALID;
    out->elements = c->els.data();
    out->element_count = c->els.size();
    out->path_elements = c->path_els.data();
    out->stroke_elements = c->stroke_els.data();
    out->stroke_element_count = c->stroke_els.size();
    out->polylines = c->polylines.data();
    out->polyline_count = uint32_t(c->polylines.size());
    out->stroke_count = uint32_t(c->strokes.size());
    out->strokes = c->strokes.data();
    return TK_OK;
}
void tk_canvas_set_clear_color(tk_canvas* c, uint32_t premul) { c->clear = premul; }

int64_t tk_canvas_push_path(tk_canvas* c, const tk_path* path, const tk_brush_desc* brush, const double* transform,
                            uint32_t fill_rule, double tolerance) {
    if (!c || !path || fill_rule > 1u || !(tolerance > 0.0)) return -1;
    const int64_t draw = push_path_with_tag(c, *path, brush, transform, fill_rule, tolerance, TK_DRAW_BRUSH, true);
    if (c->keep) {
        RecCmd r = rec_cmd(RecCmd::FILL, path, brush, transform);
        r.rule = fill_rule;
        r.tolerance = tolerance;
        c->log.push_back(std::move(r));
    }
    return draw;
}
int64_t tk_canvas_push_glyph_outlines(tk_canvas* c, const tk_path* path, const tk_brush_desc* brush,
                                      const double* transform, double tolerance) {
    if (!c || !path || !(tolerance > 0.0)) return -1;
    const int64_t draw =
        push_path_with_tag(c, *path, brush, transform, TK_FILL_NONZERO, tolerance, TK_DRAW_PATH_GLYPH, true);
    if (c->keep) {
        RecCmd r = rec_cmd(RecCmd::GLYPHS, path, brush, transform);
        r.tolerance = tolerance;
        c->log.push_back(std::move(r));
    }
    return draw;
}
int64_t tk_canvas_push_stroke(tk_canvas* c, const tk_path* path, const tk_brush_desc* brush, double width,
                              const double* transform, double tolerance) {
    if (!c || !path || !(width > 0.0) || !(tolerance > 0.0)) return -1;
    // Strokes are outlined in the path's local space, then transformed
    // (kurbo::stroke before the transform, src/canvas/primitives/paths.rs:24-48).
    tk_stroke_desc S{};
    S.path = uint32_t(c->paths.size());
    S.half_width = 0.5 * width;
    S.tolerance = tolerance;
    device_transform(c, transform, S.transform);
    // Bounds: the transformed centerline's tight box grown by the half width
    // and the flattening tolerance, stretched by the transform; it holds the
    // outline, which lies within half_width of the flattened centerline.
    Box bb = path_bbox(transform_path(*path, S.transform));
    if (!bb.empty()) {
        const double g = (S.half_width + tolerance) * tkf::max_stretch(S.transform) * (1.0 + 1e-12) + 1e-6;
        bb.x0 -= g;
        bb.y0 -= g;
        bb.x1 += g;
        bb.y1 += g;
    }
    const uint32_t line_start = uint32_t(c->lines.size());
    if (c->device_flatten) {
        S.polyline0 = uint32_t(c->polylines.size());
        record_centerlines(*path, tolerance, uint32_t(c->strokes.size()), c->stroke_els, c->polylines);
        S.polyline_count = uint32_t(c->polylines.size()) - S.polyline0;
        c->strokes.push_back(S);
    } else {
        std::vector<tk_flatten_el> els;
        std::vector<tk_stroke_polyline> polys;
        record_centerlines(*path, tolerance, 0u, els, polys);
        outline_lines(els, polys.data(), uint32_t(polys.size()), S, c->lines);
    }
    c->path_els.push_back(uint32_t(c->els.size()));  // no fill elements
    c->path_els.push_back(0u);
    if (c->keep) {
        RecCmd r = rec_cmd(RecCmd::STROKE, path, brush, transform);
        r.width = width;
        r.tolerance = tolerance;
        c->log.push_back(std::move(r));
    }
    return add_path(c, bb, line_start, uint32_t(c->lines.size()) - line_start, brush, TK_FILL_NONZERO, TK_DRAW_BRUSH,
                    true);
}
}  // extern "C"

namespace {
// The SDF draw of `shape` with `tag`; -2 when it draws nothing, -1 on error.
int64_t add_sdf_draw(tk_canvas* c, const tk_sdf_shape* shape, const tk_brush_desc* brush, uint32_t tag,
                     bool emit_command, const uint32_t* brush_words = nullptr);
int32_t add_glyph_image(tk_canvas* c, const tk_glyph_image& d, std::shared_ptr<const std::vector<uint32_t>> texels) {
    for (size_t k = 0; k < c->glyph_image_src.size(); ++k) {  // one entry per cached glyph image
        const tk_glyph_image& e = c->glyph_image_src[k].desc;
        if (c->glyph_image_src[k].texels == texels && e.left == d.left && e.top == d.top && e.width == d.width &&
            e.height == d.height && e.content == d.content)
            return int32_t(k);
    }
    if (c->glyph_texels.size() + texels->size() > 0xFFFFFFFFull) return -1;
    GlyphImage g{d, texels};
    g.desc.data_offset = uint32_t(c->glyph_texels.size());
    c->glyph_texels.insert(c->glyph_texels.end(), texels->begin(), texels->end());
    c->glyph_images.push_back(g.desc);
    c->glyph_image_src.push_back(std::move(g));
    return int32_t(c->glyph_images.size() - 1);
}
int32_t add_image(tk_canvas* c, std::shared_ptr<const std::vector<uint32_t>> texels, uint32_t w, uint32_t h) {
    for (size_t k = 0; k < c->images.size(); ++k)  // register_scene_image: one entry per image
        if (c->images[k] == texels) return int32_t(k);
    c->images.push_back(texels);
    c->image_table.push_back(tk_image_desc{texels->data(), w, h});
    return int32_t(c->images.size() - 1);
}
}  // namespace

extern "C" {

int64_t tk_canvas_push_sdf(tk_canvas* c, const tk_sdf_shape* shape, const tk_brush_desc* brush) {
    if (!c || !shape) return -1;
    if (c->keep) {
        RecCmd r = rec_cmd(RecCmd::SDF, nullptr, brush, nullptr);
        r.shape = *shape;
        c->log.push_back(std::move(r));
    }
    return add_sdf_draw(c, shape, brush, TK_DRAW_BRUSH, true);
}

int32_t tk_canvas_add_glyph_image(tk_canvas* c, int32_t left, int32_t top, uint32_t width, uint32_t height,
                                  uint32_t content, const uint32_t* texels) {
    if (!c || !texels || width == 0u || height == 0u || width > TK_MAX_IMAGE_DIMENSION ||
        height > TK_MAX_IMAGE_DIMENSION || content > TK_GLYPH_LINEAR_SUBPIXEL_MASK)
        return -1;
    tk_glyph_image d{left, top, width, height, content, 0u};
    const size_t n = size_t(width) * height;
    return add_glyph_image(c, d, std::make_shared<const std::vector<uint32_t>>(texels, texels + n));
}

int64_t tk_canvas_push_glyph_run(tk_canvas* c, const tk_glyph* glyphs, uint32_t count, const tk_brush_desc* brush,
                                 const int32_t* clip) {
    if (!c || !glyphs || count == 0u) return -1;
    // the run's bounds: the union of its glyph images (a glyph without an
    // image draws nothing), then the clip (push_text_layout_clipped)
    int64_t x0 = INT64_MAX, y0 = INT64_MAX, x1 = INT64_MIN, y1 = INT64_MIN;
    for (uint32_t k = 0; k < count; ++k) {
        const tk_glyph& g = glyphs[k];
        if (g.image == TK_INVALID_INDEX) continue;
        if (g.image >= c->glyph_images.size()) return -1;
        const tk_glyph_image& im = c->glyph_images[g.image];
        const int64_t gx0 = int64_t(g.x) + im.left, gy0 = int64_t(g.y) - im.top;
        x0 = std::min(x0, gx0);
        y0 = std::min(y0, gy0);
        x1 = std::max(x1, gx0 + int64_t(im.width));
        y1 = std::max(y1, gy0 + int64_t(im.height));
    }
    if (clip) {
        x0 = std::max<int64_t>(x0, clip[0]);
        y0 = std::max<int64_t>(y0, clip[1]);
        x1 = std::min<int64_t>(x1, clip[2]);
        y1 = std::min<int64_t>(y1, clip[3]);
    }
    if (x1 <= x0 || y1 <= y0 || x0 < INT32_MIN || y0 < INT32_MIN || x1 > INT32_MAX || y1 > INT32_MAX) return -1;
    if (c->keep) {
        RecCmd r = rec_cmd(RecCmd::GLYPH_RUN, nullptr, brush, nullptr);
        std::vector<uint32_t> local(c->glyph_images.size(), TK_INVALID_INDEX);
        for (uint32_t k = 0; k < count; ++k) {
            tk_glyph g = glyphs[k];
            if (g.image != TK_INVALID_INDEX) {
                if (local[g.image] == TK_INVALID_INDEX) {
                    local[g.image] = uint32_t(r.run_images.size());
                    r.run_images.push_back(c->glyph_image_src[g.image]);
                }
                g.image = local[g.image];
            }
            r.run_glyphs.push_back(g);
        }
        if (clip) {
            r.has_clip = true;
            std::memcpy(r.clip, clip, sizeof(r.clip));
        }
        c->log.push_back(std::move(r));
    }
    const uint32_t run = uint32_t(c->glyph_runs.size());
    c->glyph_runs.push_back(tk_glyph_run{uint32_t(c->glyphs.size()), count});
    c->glyphs.insert(c->glyphs.end(), glyphs, glyphs + count);
    tk_brush_desc transparent{};
    transparent.kind = TK_BRUSH_KIND_SOLID;
    const std::pair<uint32_t, uint32_t> br = push_brush(c->brush, brush ? *brush : transparent);
    // push_text_layout_inner's draw record (canvas/primitives/text.rs:80-96)
    tk_draw_record d{};
    d.path_id = TK_INVALID_INDEX;
    d.glyph_run_id = run;
    d.sdf_offset = TK_INVALID_INDEX;
    d.sdf_shadow_offset = TK_INVALID_INDEX;
    d.brush_offset = br.first;
    d.brush_len = br.second;
    d.tag = TK_DRAW_BRUSH;
    d.fill_rule = TK_FILL_NONZERO;
    d.pixel_bounds = tk_pixel_bounds{int32_t(x0), int32_t(y0), int32_t(x1), int32_t(y1)};
    d.local_pixel_bounds = d.pixel_bounds;
    d.transform = tk_affine{1, 0, 0, 1, 0, 0};
    d.inverse_transform = tk_affine{1, 0, 0, 1, 0, 0};
    const uint32_t draw_ix = uint32_t(c->draws.size());
    c->draws.push_back(d);
    c->lists[c->stack.back()].push_back({Cmd::DRAW, draw_ix, 0.0f, 0u});
    c->dirty = true;
    return draw_ix;
}

int32_t tk_canvas_add_image(tk_canvas* c, const uint32_t* premul_rgba8, uint32_t width, uint32_t height) {
    if (!c || !premul_rgba8 || width == 0u || height == 0u || width > TK_MAX_IMAGE_DIMENSION ||
        height > TK_MAX_IMAGE_DIMENSION)
        return -1;
    const size_t n = size_t(width) * height;
    return add_image(c, std::make_shared<const std::vector<uint32_t>>(premul_rgba8, premul_rgba8 + n), width, height);
}

int64_t tk_canvas_push_image(tk_canvas* c, const double rect[4], uint32_t image, uint32_t extend,
                             uint32_t sampling, uint32_t opacity) {
    if (!c || !rect || image >= c->images.size() || extend > TK_EXTEND_REFLECT || sampling > TK_PATTERN_BILINEAR ||
        opacity > 255u)
        return -1;
    // image_rect_is_valid / rect_is_valid_image_target (shared/brush.rs:627-634)
    const double x0 = rect[0], y0 = rect[1], x1 = rect[2], y1 = rect[3];
    if (!std::isfinite(x0) || !std::isfinite(y0) || !std::isfinite(x1) || !std::isfinite(y1) || !(x1 - x0 > 0.0) ||
        !(y1 - y0 > 0.0))
        return -1;
    const tk_image_desc& im = c->image_table[image];
    if (c->keep) {
        RecCmd r = rec_cmd(RecCmd::IMAGE, nullptr, nullptr, nullptr);
        r.shape.p0[0] = x0;
        r.shape.p0[1] = y0;
        r.shape.p1[0] = x1;
        r.shape.p1[1] = y1;
        r.texels = c->images[image];
        r.iw = im.width;
        r.ih = im.height;
        r.extend = extend;
        r.sampling = sampling;
        r.opacity = opacity;
        c->log.push_back(std::move(r));
    }
    // Brush::for_rect_resource (shared/brush.rs:557-580), then physical_brush's
    // scale_brush_transform(transform, 1 / scale) (canvas/surface.rs:395-400, canvas.rs:203-212)
    const float sx = 1.0f / float(x1 - x0), sy = 1.0f / float(y1 - y0);
    const float inv_scale = 1.0f / c->scale;
    const float t[6] = {sx * inv_scale, 0.0f * inv_scale, 0.0f * inv_scale, sy * inv_scale, -float(x0) * sx,
                        -float(y0) * sy};
    uint32_t words[TK_BRUSH_HEADER_WORDS + TK_BRUSH_PARAM_WORDS] = {};
    words[0] = TK_BRUSH_PATTERN_RESOURCE;
    words[1] = extend;
    words[4] = TK_BRUSH_TEXTURE_PLACEMENT_BIT | image;
    words[5] = im.width;
    words[6] = im.height;
    words[7] = opacity;
    words[8] = sampling;
    for (int k = 0; k < 6; ++k) words[TK_BRUSH_HEADER_WORDS + k] = fbits(t[k]);
    // Canvas::push_rect(rect, Radius::ZERO, brush)
    tk_sdf_shape shape{};
    shape.kind = TK_SDF_RECT;
    shape.p0[0] = x0;
    shape.p0[1] = y0;
    shape.p1[0] = x1;
    shape.p1[1] = y1;
    return add_sdf_draw(c, &shape, nullptr, TK_DRAW_BRUSH, true, words);
}

int32_t tk_canvas_push_clip_sdf_layer(tk_canvas* c, const tk_sdf_shape* shape) {
    if (!c || !shape) return -1;
    const uint32_t k = shape->kind;
    if (k == TK_SDF_RECT_SHADOW || k == TK_SDF_CIRCLE_SHADOW || k == TK_SDF_LINE_SHADOW || k == TK_SDF_ARC_SHADOW ||
        k == TK_SDF_CALLOUT_SHADOW)
        return -1;  // shadows are not clips
    // push_clip_sdf_layer (canvas/layers.rs:64-78): a transparent clip draw outside the draw order
    const int64_t draw = add_sdf_draw(c, shape, nullptr, TK_DRAW_CLIP, false);
    if (draw < 0) return -1;  // a shape that draws nothing is no clip
    if (c->keep) {
        RecCmd r = rec_cmd(RecCmd::SDF_CLIP, nullptr, nullptr, nullptr);
        r.shape = *shape;
        c->log.push_back(std::move(r));
    }
    const uint32_t child = uint32_t(c->lists.size());
    c->lists.emplace_back();
    c->lists[c->stack.back()].push_back({Cmd::CLIP, uint32_t(draw), 0.0f, child});
    c->stack.push_back(child);
    return 0;
}

}  // extern "C"

namespace {
int64_t add_sdf_draw(tk_canvas* c, const tk_sdf_shape* shape, const tk_brush_desc* brush, uint32_t tag,
                     bool emit_command, const uint32_t* brush_words) {
    const uint32_t k = shape->kind;
    if (k != TK_SDF_RECT && k != TK_SDF_RECT_STROKE && k != TK_SDF_RECT_SHADOW && k != TK_SDF_CIRCLE &&
        k != TK_SDF_CIRCLE_STROKE && k != TK_SDF_CIRCLE_SHADOW && k != TK_SDF_LINE && k != TK_SDF_LINE_SHADOW &&
        k != TK_SDF_DASH_LINE && k != TK_SDF_TRIANGLE && k != TK_SDF_CHECKERBOARD && k != TK_SDF_CANDLESTICK &&
        k != TK_SDF_CALLOUT && k != TK_SDF_CALLOUT_STROKE && k != TK_SDF_CALLOUT_SHADOW && k != TK_SDF_ARC &&
        k != TK_SDF_ARC_SHADOW && k != TK_SDF_STAR && k != TK_SDF_STAR_STROKE)
        return -1;
    // CandleStick::new and DashLine::new reject these (the reference panics)
    if (k == TK_SDF_CANDLESTICK && !(shape->widths[0] > 0.0f && shape->widths[1] > 0.0f)) return -1;
    if (k == TK_SDF_DASH_LINE && !(shape->dash[1] >= 0.0f)) return -1;
    uint32_t rec[TK_SDF_RECORD_WORDS];
    tk_pixel_bounds pb{0, 0, 0, 0};
    if (!encode_sdf(c, *shape, rec, pb)) return -2;
    const bool shadow = k == TK_SDF_RECT_SHADOW || k == TK_SDF_CIRCLE_SHADOW || k == TK_SDF_LINE_SHADOW ||
                        k == TK_SDF_CALLOUT_SHADOW || k == TK_SDF_ARC_SHADOW;
    std::vector<uint32_t>& blob = shadow ? c->shadow : c->sdf;
    const uint32_t off = uint32_t(blob.size());
    blob.insert(blob.end(), rec, rec + TK_SDF_RECORD_WORDS);
    tk_brush_desc transparent{};
    transparent.kind = TK_BRUSH_KIND_SOLID;
    std::pair<uint32_t, uint32_t> br;
    if (brush_words) {  // a prebuilt image pattern brush
        br = {uint32_t(c->brush.size()), TK_BRUSH_HEADER_WORDS + TK_BRUSH_PARAM_WORDS};
        c->brush.insert(c->brush.end(), brush_words, brush_words + br.second);
    } else {
        br = push_brush(c->brush, brush ? *brush : transparent);
    }
    // push_physical_sdf_record / push_physical_sdf_shadow_record (canvas/paths.rs:207-300)
    tk_draw_record d{};
    d.path_id = TK_INVALID_INDEX;
    d.glyph_run_id = TK_INVALID_INDEX;
    d.sdf_offset = shadow ? TK_INVALID_INDEX : off;
    d.sdf_len = shadow ? 0u : TK_SDF_RECORD_WORDS;
    d.sdf_shadow_offset = shadow ? off : TK_INVALID_INDEX;
    d.sdf_shadow_len = shadow ? TK_SDF_RECORD_WORDS : 0u;
    d.brush_offset = br.first;
    d.brush_len = br.second;
    d.tag = tag;
    d.fill_rule = TK_FILL_NONZERO;
    d.pixel_bounds = pb;
    d.local_pixel_bounds = pb;
    d.transform = tk_affine{1, 0, 0, 1, 0, 0};
    d.inverse_transform = tk_affine{1, 0, 0, 1, 0, 0};
    const uint32_t draw_ix = uint32_t(c->draws.size());
    c->draws.push_back(d);
    if (emit_command) c->lists[c->stack.back()].push_back({Cmd::DRAW, draw_ix, 0.0f, 0u});
    c->dirty = true;
    return draw_ix;
}
}  // namespace

extern "C" {
int32_t tk_canvas_push_clip_layer(tk_canvas* c, const tk_path* path, const double* transform, uint32_t rule,
                                  double tolerance) {
    if (!c || !path || rule > 1u || !(tolerance > 0.0)) return -1;
    int64_t draw = push_path_with_tag(c, *path, nullptr, transform, rule, tolerance, TK_DRAW_CLIP, false);
    uint32_t child = uint32_t(c->lists.size());
    c->lists.emplace_back();
    c->lists[c->stack.back()].push_back({Cmd::CLIP, uint32_t(draw), 0.0f, child});
    c->stack.push_back(child);
    if (c->keep) {
        RecCmd r = rec_cmd(RecCmd::CLIP, path, nullptr, transform);
        r.rule = rule;
        r.tolerance = tolerance;
        c->log.push_back(std::move(r));
    }
    return 0;
}
int32_t tk_canvas_push_progressive_blur_group(tk_canvas* c, double start_x, double start_y, double end_x,
                                              double end_y, float max_std_dev, uint32_t quality) {
    if (!c || quality > TK_PROGRESSIVE_HIGH) return -1;
    // ProgressiveBlur::scaled (the canvas scale), then projection()
    // (shared/layer/filter/progressive.rs:71-93)
    const double s = double(c->scale);
    const double sx = start_x * s, sy = start_y * s, ex = end_x * s, ey = end_y * s;
    const float sd = max_std_dev * c->scale;
    const double dx = ex - sx, dy = ey - sy, length2 = dx * dx + dy * dy;
    if (!std::isfinite(sd) || !(sd >= 0.0f && sd <= 65536.0f) || !std::isfinite(length2)) return -1;
    tk_progressive_blur pb{float(sx), float(sy), 0.0f, 0.0f, sd, quality};
    if (length2 != 0.0) {
        pb.dir_x = float(dx / length2);
        pb.dir_y = float(dy / length2);
    }
    if (!std::isfinite(pb.start_x) || !std::isfinite(pb.start_y) || !std::isfinite(pb.dir_x) ||
        !std::isfinite(pb.dir_y))
        return -1;
    const uint32_t child = uint32_t(c->lists.size());
    c->lists.emplace_back();
    Cmd cmd{Cmd::BLUR, 0u, sd, child, 0u};
    cmd.progressive = int32_t(c->progressive.size());
    c->progressive.push_back(pb);
    c->lists[c->stack.back()].push_back(cmd);
    c->stack.push_back(child);
    c->dirty = true;
    if (c->keep) {
        RecCmd r = rec_cmd(RecCmd::PROGRESSIVE, nullptr, nullptr, nullptr);
        r.shape.p0[0] = start_x;
        r.shape.p0[1] = start_y;
        r.shape.p1[0] = end_x;
        r.shape.p1[1] = end_y;
        r.sigma = max_std_dev;
        r.sampling = quality;
        c->log.push_back(std::move(r));
    }
    return 0;
}

namespace {
// region_bounds (shared/layer/filter.rs:578-597): a device-space box floored /
// ceiled to whole pixels (an empty box gives an empty region at the origin)
bool region_pixel_bounds(double x0, double y0, double x1, double y1, double b[4]) {
    const double v[4] = {x0, y0, x1, y1};
    for (int k = 0; k < 4; ++k) {
        if (!std::isfinite(v[k])) return false;
        b[k] = (k < 2) ? std::floor(v[k]) : std::ceil(v[k]);
        b[k] = std::min(std::max(b[k], -2147483648.0), 2147483647.0);
    }
    return true;
}

// A filter layer over region pixel bounds b: the chain made physical, the
// surface grown by its reach, the command pushed (recording is the caller's).
int32_t push_filter_layer_bounds(tk_canvas* c, const tk_canvas_filter* filters, uint32_t count, const double b[4],
                                 int32_t fixed_region) {
    // physical_filter (canvas/surface.rs:247-326): offsets scale with the
    // canvas; filter_offset_to_pixel_delta (filter.rs:490-494) rounds them to
    // whole pixels; filter_outset (filter.rs:533-575) sums the chain's reach
    std::vector<tk_filter> chain(count);
    std::vector<uint32_t> words;  // the chain's transfer tables and convolution kernels
    uint64_t reach = 0;
    for (uint32_t k = 0; k < count; ++k) {
        const tk_canvas_filter& f = filters[k];
        tk_filter& g = chain[k];
        g = tk_filter{};
        g.kind = f.kind;
        if (f.kind < TK_FILTER_BRIGHTNESS || f.kind > TK_FILTER_BLUR || !std::isfinite(f.amount)) return -1;
        if (f.kind == TK_FILTER_BLUR) {
            // Filter::Blur scaled by the canvas (surface.rs:284-292); reach
            // blur_outset(max(sx, sy)) = ceil(3 max)
            const float sx = std::max(f.dx * c->scale, 0.0f), sy = std::max(f.dy * c->scale, 0.0f);
            if (!std::isfinite(sx) || !std::isfinite(sy) || sx > 1.0e4f || sy > 1.0e4f) return -1;
            g.std_dev = sx;
            reach += uint64_t(std::ceil(std::max(sx, sy) * 3.0f));
        }
        if (f.kind == TK_FILTER_COMPONENT_TRANSFER) {
            if (!f.table) return -1;
            for (uint32_t k2 = 0; k2 < TK_TRANSFER_TABLE_WORDS; ++k2)
                if (f.table[k2] > 255u) return -1;
            g.color = uint32_t(c->filter_words.size() + words.size());
            words.insert(words.end(), f.table, f.table + TK_TRANSFER_TABLE_WORDS);
        }
        if (f.kind == TK_FILTER_CONVOLVE) {
            // ConvolveMatrix (filter.rs:611-628): the kernel copied as f32 bits
            const uint64_t taps = uint64_t(f.columns) * f.rows;
            if (taps > TK_CONVOLVE_MAX_TAPS || (taps && !f.kernel) || f.edge_mode > TK_CONVOLVE_EDGE_WRAP ||
                !std::isfinite(f.divisor) || !std::isfinite(f.bias) || (taps && (f.target_x >= f.columns ||
                                                                                f.target_y >= f.rows)))
                return -1;
            g.color = uint32_t(c->filter_words.size() + words.size());
            for (uint64_t t = 0; t < taps; ++t) {
                if (!std::isfinite(f.kernel[t])) return -1;
                uint32_t w;
                std::memcpy(&w, &f.kernel[t], 4);
                words.push_back(w);
            }
            g.columns = f.columns;
            g.rows = f.rows;
            g.target_x = f.target_x;
            g.target_y = f.target_y;
            g.edge_mode = f.edge_mode;
            g.preserve_alpha = f.preserve_alpha ? 1u : 0u;
            g.divisor = f.divisor;
            g.bias = f.bias;
        }
        if (f.kind == TK_FILTER_FLOOD || f.kind == TK_FILTER_DROP_SHADOW) {
            for (float v : f.rgba)
                if (!std::isfinite(v)) return -1;
            g.color = premul_color(f.rgba);  // the solid brush's colour word
        }
        if (f.kind == TK_FILTER_DROP_SHADOW) {
            // physical_filter scales offset and deviation; shadow.rs rounds the
            // offset (half away from zero); filter_outset adds blur_outset
            // (ceil(3 std_dev)) and the offset's reach (filter.rs:566-571)
            const float ox = f.dx * c->scale, oy = f.dy * c->scale, sd = f.std_dev * c->scale;
            if (!std::isfinite(ox) || !std::isfinite(oy) || !std::isfinite(sd) || std::fabs(ox) > 1.0e6f ||
                std::fabs(oy) > 1.0e6f || sd > 1.0e4f)
                return -1;
            g.dx = int32_t(std::round(ox));
            g.dy = int32_t(std::round(oy));
            g.std_dev = sd;
            reach += uint64_t(std::ceil(std::max(sd, 0.0f) * 3.0f)) +
                     uint64_t(std::max(std::ceil(std::fabs(ox)), std::ceil(std::fabs(oy))));
        }
        g.amount = f.kind == TK_FILTER_BLUR ? std::max(f.dy * c->scale, 0.0f) : f.amount;  // BLUR: y deviation
        if (f.kind == TK_FILTER_OFFSET) {
            const float dx = f.dx * c->scale, dy = f.dy * c->scale;
            if (!std::isfinite(dx) || !std::isfinite(dy) || std::fabs(dx) > 1.0e6f || std::fabs(dy) > 1.0e6f)
                return -1;
            g.dx = int32_t(std::ceil(dx - 0.5f));
            g.dy = int32_t(std::ceil(dy - 0.5f));
            reach += uint64_t(std::max(std::ceil(std::fabs(dx)), std::ceil(std::fabs(dy))));
        }
        if (f.kind == TK_FILTER_ERODE || f.kind == TK_FILTER_DILATE) {
            // the radii scale with the canvas and round up to whole pixels
            // (effects.rs:169-221); a dilation reaches max(rx, ry) further
            const float rx = f.dx * c->scale, ry = f.dy * c->scale;
            if (!std::isfinite(rx) || !std::isfinite(ry) || rx > 1.0e6f || ry > 1.0e6f) return -1;
            g.dx = int32_t(std::ceil(std::max(rx, 0.0f)));
            g.dy = int32_t(std::ceil(std::max(ry, 0.0f)));
            if (f.kind == TK_FILTER_DILATE) reach += uint64_t(std::ceil(std::max(std::max(rx, ry), 0.0f)));
        }
        if (f.kind == TK_FILTER_COLOR_MATRIX)
            for (int m = 0; m < 20; ++m) {
                if (!std::isfinite(f.matrix[m])) return -1;
                g.matrix[m] = f.matrix[m];
            }
    }
    if (fixed_region) reach = 0;
    const double r = double(std::min<uint64_t>(reach, 0xFFFFFFFFull));
    tk_filter_layer L{uint32_t(c->filters.size()), count, {0, 0, 0, 0}};
    L.surface[0] = int32_t(std::max(b[0] - r, -2147483648.0));
    L.surface[1] = int32_t(std::max(b[1] - r, -2147483648.0));
    L.surface[2] = int32_t(std::min(b[2] + r, 2147483647.0));
    L.surface[3] = int32_t(std::min(b[3] + r, 2147483647.0));
    c->filters.insert(c->filters.end(), chain.begin(), chain.end());
    c->filter_words.insert(c->filter_words.end(), words.begin(), words.end());
    const uint32_t child = uint32_t(c->lists.size());
    c->lists.emplace_back();
    Cmd cmd{Cmd::BLUR, 0u, 0.0f, child, 0u};
    cmd.filter = int32_t(c->filter_layers.size());
    c->filter_layers.push_back(L);
    c->lists[c->stack.back()].push_back(cmd);
    c->stack.push_back(child);
    c->dirty = true;
    return 0;
}
}  // namespace

int32_t tk_canvas_push_filter_layer(tk_canvas* c, const tk_canvas_filter* filters, uint32_t count, const double rect[4],
                                    int32_t fixed_region) {
    if (!c || (count && !filters) || !rect) return -1;
    // physical_region (canvas/surface.rs:197-205,370-386)
    const double s = double(c->scale);
    double b[4];
    if (!region_pixel_bounds(rect[0] * s, rect[1] * s, rect[2] * s, rect[3] * s, b)) return -1;
    if (push_filter_layer_bounds(c, filters, count, b, fixed_region) != 0) return -1;
    if (c->keep) {
        RecCmd rc = rec_cmd(RecCmd::FILTER, nullptr, nullptr, nullptr);
        rc.chain.assign(filters, filters + count);
        // the recorded tables and kernels point into this canvas's own copies
        rc.tables.clear();
        for (uint32_t k = 0; k < count; ++k) {
            if (filters[k].kind == TK_FILTER_COMPONENT_TRANSFER)
                rc.tables.insert(rc.tables.end(), filters[k].table, filters[k].table + TK_TRANSFER_TABLE_WORDS);
            if (filters[k].kind == TK_FILTER_CONVOLVE)
                for (uint64_t t = 0; t < uint64_t(filters[k].columns) * filters[k].rows; ++t) {
                    uint32_t w;
                    std::memcpy(&w, &filters[k].kernel[t], 4);
                    rc.tables.push_back(w);
                }
        }
        rc.fixed = fixed_region != 0;
        rc.shape.p0[0] = rect[0];
        rc.shape.p0[1] = rect[1];
        rc.shape.p1[0] = rect[2];
        rc.shape.p1[1] = rect[3];
        c->log.push_back(std::move(rc));
    }
    return 0;
}

int32_t tk_canvas_push_filter_layer_path(tk_canvas* c, const tk_canvas_filter* filters, uint32_t count,
                                         const tk_path* path, const double* transform, int32_t fixed_region) {
    if (!c || (count && !filters) || !path) return -1;
    // Region::Path: its bounds are the tight box of the path under the device
    // transform (physical_region, canvas/surface.rs:376-384; region_bounds)
    double dev[6];
    device_transform(c, transform, dev);
    const Box bb = path_bbox(transform_path(*path, dev));
    double b[4] = {0.0, 0.0, 0.0, 0.0};
    if (!bb.empty() && !region_pixel_bounds(bb.x0, bb.y0, bb.x1, bb.y1, b)) return -1;
    if (push_filter_layer_bounds(c, filters, count, b, fixed_region) != 0) return -1;
    if (c->keep) {
        RecCmd rc = rec_cmd(RecCmd::FILTER, path, nullptr, transform);
        rc.region_path = true;
        rc.chain.assign(filters, filters + count);
        rc.fixed = fixed_region != 0;
        for (uint32_t k = 0; k < count; ++k) {
            if (filters[k].kind == TK_FILTER_COMPONENT_TRANSFER)
                rc.tables.insert(rc.tables.end(), filters[k].table, filters[k].table + TK_TRANSFER_TABLE_WORDS);
            if (filters[k].kind == TK_FILTER_CONVOLVE)
                for (uint64_t t = 0; t < uint64_t(filters[k].columns) * filters[k].rows; ++t) {
                    uint32_t w;
                    std::memcpy(&w, &filters[k].kernel[t], 4);
                    rc.tables.push_back(w);
                }
        }
        c->log.push_back(std::move(rc));
    }
    return 0;
}

int32_t tk_canvas_push_blur_group_sampled(tk_canvas* c, float sigma, uint32_t sampling) {
    float physical = sigma * c->scale;
    if (!(sigma >= 0.0f) || !std::isfinite(physical)) return -1;
    const uint32_t factor = sampling & 255u, down = (sampling >> 8) & 255u, up = (sampling >> 16) & 255u;
    if ((sampling >> 24) != 0u || factor > TK_BLUR_MAX_FACTOR || down > TK_BLUR_DOWNSAMPLE_BOX ||
        up > TK_BLUR_UPSAMPLE_BILINEAR)
        return -1;
    uint32_t child = uint32_t(c->lists.size());
    c->lists.emplace_back();
    c->lists[c->stack.back()].push_back({Cmd::BLUR, 0u, physical, child, factor > 1u ? sampling : 0u});
    c->stack.push_back(child);
    c->dirty = true;
    if (c->keep) {
        RecCmd r = rec_cmd(RecCmd::BLUR, nullptr, nullptr, nullptr);
        r.sigma = sigma;
        r.sampling = factor > 1u ? sampling : 0u;
        c->log.push_back(std::move(r));
    }
    return 0;
}
int32_t tk_canvas_push_blur_group(tk_canvas* c, float sigma) { return tk_canvas_push_blur_group_sampled(c, sigma, 0u); }
int32_t tk_canvas_push_opacity_layer(tk_canvas* c, const tk_path* path, const double* transform, double tolerance,
                                     float opacity) {
    if (!c || !path || !(tolerance > 0.0) || !std::isfinite(opacity)) return -1;
    // push_layer_path(DrawTag::Opacity, .., FillRule::NonZero, ..) (canvas/layers.rs:122-140)
    int64_t draw = push_path_with_tag(c, *path, nullptr, transform, TK_FILL_NONZERO, tolerance, TK_DRAW_OPACITY, false);
    if (draw < 0) return -1;
    // opacity_f32_to_u8 (src/shared/pixel.rs:3-6): the stack record's payload
    const uint32_t alpha = uint32_t(std::min(std::max(opacity, 0.0f), 1.0f) * 255.0f + 0.5f);
    uint32_t child = uint32_t(c->lists.size());
    c->lists.emplace_back();
    c->lists[c->stack.back()].push_back({Cmd::OPACITY, uint32_t(draw), 0.0f, child, alpha});
    c->stack.push_back(child);
    c->dirty = true;
    if (c->keep) {
        RecCmd r = rec_cmd(RecCmd::OPACITY, path, nullptr, transform);
        r.tolerance = tolerance;
        r.sigma = opacity;
        c->log.push_back(std::move(r));
    }
    return 0;
}
const char* tk_canvas_last_error(const tk_canvas* c) { return c ? c->compile_error.c_str() : ""; }
int32_t tk_canvas_pop_layer(tk_canvas* c) {
    if (c->stack.size() <= 1) return -1;
    c->stack.pop_back();
    c->dirty = true;
    if (c->keep) c->log.push_back(rec_cmd(RecCmd::POP, nullptr, nullptr, nullptr));
    return 0;
}

void tk_canvas_set_keep_commands(tk_canvas* c, int32_t enabled) {
    if (c) c->keep = enabled != 0;
}

int32_t tk_canvas_scene(tk_canvas* c, tk_scene_desc* out) {
    if (!c || !out) return -1;
    compile(c);
    if (!c->compile_error.empty()) return -1;
    std::memset(out, 0, sizeof(*out));
    out->width = c->W;
    out->height = c->H;
    out->clear_color = c->clear;
    out->flags = c->host_plan ? 0u : TK_SCENE_SEGMENTS_FROM_DEVICE;
    out->lines = c->lines.data();
    out->line_count = c->lines.size();
    out->paths = c->paths.data();
    out->path_count = uint32_t(c->paths.size());
    out->draws = c->draws.data();
    out->draw_count = uint32_t(c->draws.size());
    out->brush_blob = c->brush.data();
    out->brush_word_count = c->brush.size();
    out->sdf_blob = c->sdf.data();
    out->sdf_word_count = c->sdf.size();
    out->sdf_shadow_blob = c->shadow.data();
    out->sdf_shadow_word_count = c->shadow.size();
    out->images = c->image_table.data();
    out->image_count = uint32_t(c->image_table.size());
    out->glyph_runs = c->glyph_runs.data();
    out->glyph_run_count = uint32_t(c->glyph_runs.size());
    out->glyphs = c->glyphs.data();
    out->glyph_count = uint32_t(c->glyphs.size());
    out->glyph_images = c->glyph_images.data();
    out->glyph_image_count = uint32_t(c->glyph_images.size());
    out->glyph_texels = c->glyph_texels.data();
    out->glyph_texel_count = c->glyph_texels.size();
    out->progressive_blurs = c->progressive.data();
    out->progressive_count = uint32_t(c->progressive.size());
    out->filter_layers = c->filter_layers.data();
    out->filter_layer_count = uint32_t(c->filter_layers.size());
    out->filters = c->filters.data();
    out->filter_count = uint32_t(c->filters.size());
    out->filter_words = c->filter_words.data();
    out->filter_word_count = uint32_t(c->filter_words.size());
    out->layers = c->layers.data();
    out->layer_count = uint32_t(c->layers.size());
    out->draw_order = c->order.data();
    out->draw_order_count = uint32_t(c->order.size());
    out->draw_batch_ids = c->batch_ids.data();
    out->ops = c->ops.data();
    out->op_count = uint32_t(c->ops.size());
    return 0;
}

uint64_t tk_canvas_param_points(const tk_canvas* c, double* out) {
    if (out) std::memcpy(out, c->points.data(), c->points.size() * sizeof(double));
    return c->points.size();
}
uint64_t tk_canvas_param_colors(const tk_canvas* c, float* out) {
    if (out) std::memcpy(out, c->colors.data(), c->colors.size() * sizeof(float));
    return c->colors.size();
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Seeded synthetic workloads (the five measured configurations).
// ---------------------------------------------------------------------------
#include <random>

namespace {

struct Rng {
    std::mt19937_64 g;
    explicit Rng(uint64_t seed) : g(seed) {}
    double u01() { return double(g() >> 11) * (1.0 / 9007199254740992.0); }
    double uniform(double a, double b) { return a + (b - a) * u01(); }
    uint32_t range(uint32_t a, uint32_t b) { return a + uint32_t(g() % uint64_t(b - a + 1)); }
    double normal() {
        double u1 = std::max(u01(), 1e-300), u2 = u01();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
    }
    float f32(double lo, double hi) { return float(uniform(lo, hi)); }
};

tk_brush_desc solid(float r, float g, float b, float a) {
    tk_brush_desc d{};
    d.kind = TK_BRUSH_KIND_SOLID;
    d.rgba[0] = r; d.rgba[1] = g; d.rgba[2] = b; d.rgba[3] = a;
    return d;
}

// Random closed path of `n` cubic segments with f32 control points drawn by `pt`.
template <class P>
void random_cubic_path(tk_path* p, uint32_t n, P&& pt, std::vector<double>* record) {
    auto put = [&](double x, double y) { if (record) { record->push_back(x); record->push_back(y); } };
    auto a = pt();
    tk_path_move_to(p, a.first, a.second);
    put(a.first, a.second);
    for (uint32_t k = 0; k < n; ++k) {
        auto c1 = pt(), c2 = pt(), c3 = pt();
        tk_path_cubic_to(p, c1.first, c1.second, c2.first, c2.second, c3.first, c3.second);
        put(c1.first, c1.second); put(c2.first, c2.second); put(c3.first, c3.second);
    }
    tk_path_close(p);
}

void gen_uniform_fills(tk_canvas* c, Rng& r, uint32_t w, uint32_t h, uint32_t paths, uint32_t seg_lo, uint32_t seg_hi,
                       float alpha_lo, bool record) {
    for (uint32_t i = 0; i < paths; ++i) {
        tk_path* p = tk_path_new();
        uint32_t n = r.range(seg_lo, seg_hi);
        auto pt = [&]() { return std::make_pair(double(r.f32(0.0, w)), double(r.f32(0.0, h))); };
        random_cubic_path(p, n, pt, record ? &c->points : nullptr);
        float rgb[3] = {float(r.range(0, 255)) / 255.0f, float(r.range(0, 255)) / 255.0f, float(r.range(0, 255)) / 255.0f};
        float a = r.f32(alpha_lo, 1.0);
        tk_brush_desc b = solid(rgb[0], rgb[1], rgb[2], a);
        if (record) { c->colors.insert(c->colors.end(), {rgb[0], rgb[1], rgb[2], a}); }
        tk_canvas_push_path(c, p, &b, nullptr, TK_FILL_NONZERO, 0.1);
        tk_path_free(p);
    }
}

tk_brush_desc random_paint(Rng& r, double cx, double cy, std::vector<tk_gradient_stop>& stops) {
    double kind = r.u01();
    auto color = [&](float* out) {
        out[0] = float(r.range(0, 255)) / 255.0f;
        out[1] = float(r.range(0, 255)) / 255.0f;
        out[2] = float(r.range(0, 255)) / 255.0f;
        out[3] = r.f32(0.3, 1.0);
    };
    if (kind < 0.5) {
        tk_brush_desc b{};
        b.kind = TK_BRUSH_KIND_SOLID;
        color(b.rgba);
        return b;
    }
    uint32_t ns = r.range(2, 6);
    stops.resize(ns);
    for (uint32_t k = 0; k < ns; ++k) {
        stops[k].offset = ns == 1 ? 0.0f : (k == 0 ? 0.0f : (k + 1 == ns ? 1.0f : r.f32(0.0, 1.0)));
        color(stops[k].rgba);
    }
    tk_brush_desc b{};
    b.stop_count = ns;
    b.stops = stops.data();
    b.extend = r.range(0, 2);
    if (kind < 0.75) {
        b.kind = TK_BRUSH_KIND_LINEAR;
        b.p0[0] = float(cx + 300.0 * r.normal()); b.p0[1] = float(cy + 300.0 * r.normal());
        b.p1[0] = float(cx + 300.0 * r.normal()); b.p1[1] = float(cy + 300.0 * r.normal());
    } else {
        b.kind = TK_BRUSH_KIND_RADIAL;
        b.p0[0] = float(cx + 100.0 * r.normal()); b.p0[1] = float(cy + 100.0 * r.normal());
        b.p1[0] = float(cx + 100.0 * r.normal()); b.p1[1] = float(cy + 100.0 * r.normal());
        b.r0 = r.f32(0.0, 50.0);
        b.r1 = r.f32(100.0, 600.0);
    }
    return b;
}

// Config 2: mixed fills/strokes clustered around Gaussian centers, half
// nonzero / half even-odd, solid/linear/radial paint, 10% of paths in clip
// layers nested 1-4 deep.
void gen_mixed(tk_canvas* c, Rng& r, uint32_t w, uint32_t h, uint32_t paths) {
    const uint32_t centers = 200;
    const double sd = 300.0 * std::min(w, h) / 4096.0;
    std::vector<std::pair<double, double>> ctr(centers);
    for (auto& q : ctr) q = {r.uniform(0.0, w), r.uniform(0.0, h)};
    std::vector<tk_gradient_stop> stops;
    auto random_segments = [&](tk_path* p, uint32_t n, double cx, double cy, bool close) {
        auto pt = [&]() { return std::make_pair(double(float(cx + sd * r.normal())), double(float(cy + sd * r.normal()))); };
        auto a = pt();
        tk_path_move_to(p, a.first, a.second);
        for (uint32_t k = 0; k < n; ++k) {
            if (r.u01() < 0.5) {
                auto c1 = pt(), c2 = pt(), c3 = pt();
                tk_path_cubic_to(p, c1.first, c1.second, c2.first, c2.second, c3.first, c3.second);
            } else {
                auto c1 = pt(), c2 = pt();
                tk_path_quad_to(p, c1.first, c1.second, c2.first, c2.second);
            }
        }
        if (close) tk_path_close(p);
    };
    uint32_t i = 0;
    const double group_start = 0.0241;  // ~10% of paths end up clipped
    while (i < paths) {
        uint32_t depth = 0, group = 1;
        if (r.u01() < group_start) {
            depth = r.range(1, 4);
            group = std::min(r.range(1, 8), paths - i);
        }
        auto k = ctr[r.range(0, centers - 1)];
        for (uint32_t d = 0; d < depth; ++d) {
            tk_path* cp = tk_path_new();
            random_segments(cp, r.range(4, 16), k.first, k.second, true);
            tk_canvas_push_clip_layer(c, cp, nullptr, TK_FILL_NONZERO, 0.1);
            tk_path_free(cp);
        }
        for (uint32_t g = 0; g < group; ++g, ++i) {
            auto q = g == 0 ? k : ctr[r.range(0, centers - 1)];
            if (depth) q = k;
            tk_path* p = tk_path_new();
            bool fill = r.u01() < 0.6;
            random_segments(p, r.range(4, 64), q.first, q.second, fill);
            tk_brush_desc b = random_paint(r, q.first, q.second, stops);
            if (fill) {
                uint32_t rule = r.u01() < 0.5 ? TK_FILL_NONZERO : TK_FILL_EVEN_ODD;
                tk_canvas_push_path(c, p, &b, nullptr, rule, 0.1);
            } else {
                tk_canvas_push_stroke(c, p, &b, r.uniform(0.5, 8.0), nullptr, 0.1);
            }
            tk_path_free(p);
        }
        for (uint32_t d = 0; d < depth; ++d) tk_canvas_pop_layer(c);
    }
}

// Config 3: glyph-like paths (2-4 closed quadratic contours in a unit em box,
// inner contours reversed so nonzero fill leaves holes) on baseline rows.
void gen_glyphs(tk_canvas* c, Rng& r, uint32_t w, uint32_t h, uint32_t count) {
    tk_brush_desc black = solid(0.0f, 0.0f, 0.0f, 1.0f);
    double x = 2.0, baseline = 0.0, row_em = 0.0;
    for (uint32_t i = 0; i < count; ++i) {
        double em = r.uniform(8.0, 64.0);
        if (x + 0.7 * em > w || baseline == 0.0) {
            baseline += row_em > 0.0 ? 1.2 * row_em : 0.0;
            if (baseline == 0.0 || baseline > h + 8.0) baseline = r.uniform(40.0, 70.0);
            x = r.uniform(0.0, 8.0);
            row_em = 0.0;
        }
        row_em = std::max(row_em, em);
        double ox = x + r.uniform(0.0, 1.0), oy = baseline + r.uniform(0.0, 1.0);
        tk_path* p = tk_path_new();
        uint32_t contours = r.range(2, 4);
        double cx = 0.5, cy = 0.45, rx = r.uniform(0.25, 0.4), ry = r.uniform(0.3, 0.42);
        for (uint32_t k = 0; k < contours; ++k) {
            double ccx = cx, ccy = cy, crx = rx, cry = ry;
            bool inner = k > 0;
            if (inner) {
                crx = r.uniform(0.04, 0.12);
                cry = r.uniform(0.04, 0.12);
                ccx = cx + r.uniform(-0.5, 0.5) * (rx - crx);
                ccy = cy + r.uniform(-0.5, 0.5) * (ry - cry);
            }
            uint32_t n = r.range(6, 24);
            auto at = [&](double ang, double rad_scale) {
                double sgn = inner ? -1.0 : 1.0;
                double px = ccx + crx * rad_scale * std::cos(sgn * ang), py = ccy + cry * rad_scale * std::sin(sgn * ang);
                return std::make_pair(ox + float(px * em), oy + float((py - 0.9) * em));
            };
            double jit = 0.08;
            auto s = at(0.0, 1.0);
            tk_path_move_to(p, s.first, s.second);
            for (uint32_t q = 0; q < n; ++q) {
                double a0 = 2.0 * M_PI * q / n, a1 = 2.0 * M_PI * (q + 1) / n;
                auto cpt = at(0.5 * (a0 + a1), (1.0 / std::cos(M_PI / n)) * (1.0 + r.uniform(-jit, jit)));
                auto end = q + 1 == n ? s : at(a1, 1.0 + r.uniform(-jit, jit));
                tk_path_quad_to(p, cpt.first, cpt.second, end.first, end.second);
            }
            tk_path_close(p);
        }
        tk_canvas_push_glyph_outlines(c, p, &black, nullptr, 0.1);  // text as outlines: PathGlyph draws
        tk_path_free(p);
        x += 0.62 * em;
    }
}

}  // namespace

extern "C" tk_canvas* tk_generate(uint32_t config, uint64_t seed, const tk_gen_params* o) {
    tk_gen_params z{};
    if (!o) o = &z;
    auto pick = [](uint32_t v, uint32_t d) { return v ? v : d; };
    tk_canvas* c = nullptr;
    switch (config) {
        case 1: {
            uint32_t w = pick(o->width, 640), h = pick(o->height, 360);
            c = tk_canvas_new(w, h, 1.0f);
            c->host_plan = !(o->flags & 1u);
            if (o->flags & 2u) tk_canvas_set_device_flatten(c, 1);
            c->clear = 0xFFFFFFFFu;
            Rng r(seed);
            gen_uniform_fills(c, r, w, h, pick(o->paths, 240), 8, 40, 0.3f, true);
            break;
        }
        case 2: {
            uint32_t w = pick(o->width, 4096), h = pick(o->height, 4096);
            c = tk_canvas_new(w, h, 1.0f);
            c->host_plan = !(o->flags & 1u);
            if (o->flags & 2u) tk_canvas_set_device_flatten(c, 1);
            c->clear = 0xFFFFFFFFu;
            Rng r(seed);
            gen_mixed(c, r, w, h, pick(o->paths, 50000));
            break;
        }
        case 3: {
            uint32_t w = pick(o->width, 1920), h = pick(o->height, 1080);
            c = tk_canvas_new(w, h, 1.0f);
            c->host_plan = !(o->flags & 1u);
            if (o->flags & 2u) tk_canvas_set_device_flatten(c, 1);
            c->clear = 0xFFFFFFFFu;
            Rng r(seed);
            gen_glyphs(c, r, w, h, pick(o->paths, 20000));
            break;
        }
        case 4: {
            Rng r(seed * 0x9E3779B97F4A7C15ull + o->variant + 1);
            uint32_t w = o->width ? o->width : uint32_t(std::lround(std::exp(r.uniform(std::log(64.0), std::log(1024.0)))));
            uint32_t h = o->height ? o->height : uint32_t(std::lround(std::exp(r.uniform(std::log(64.0), std::log(1024.0)))));
            uint32_t n = o->paths ? o->paths : uint32_t(std::lround(std::exp(r.uniform(std::log(10.0), std::log(2000.0)))));
            c = tk_canvas_new(w, h, 1.0f);
            c->host_plan = !(o->flags & 1u);
            if (o->flags & 2u) tk_canvas_set_device_flatten(c, 1);
            c->clear = 0xFFFFFFFFu;
            gen_uniform_fills(c, r, w, h, n, 8, 40, 0.3f, false);
            break;
        }
        case 5: {
            uint32_t w = pick(o->width, 1024), h = pick(o->height, 1024);
            c = tk_canvas_new(w, h, 1.0f);
            c->host_plan = !(o->flags & 1u);
            if (o->flags & 2u) tk_canvas_set_device_flatten(c, 1);
            c->clear = 0xFFFFFFFFu;
            Rng r(seed);
            Rng jr(seed ^ 0x6A09E667F3BCC909ull);  // jitter stream, independent of the scene stream
            float sigma = o->sigma > 0.0f ? o->sigma : 4.0f;
            tk_canvas_push_blur_group(c, sigma);
            uint32_t paths = pick(o->paths, 256);
            for (uint32_t i = 0; i < paths; ++i) {
                tk_path* p = tk_path_new();
                auto pt = [&]() { return std::make_pair(double(r.f32(0.0, w)), double(r.f32(0.0, h))); };
                std::vector<double> pts;
                random_cubic_path(p, 12, pt, &pts);
                if (o->jitter > 0.0f) {
                    tk_path_free(p);
                    p = tk_path_new();
                    for (double& v : pts) v = double(float(v + o->jitter * jr.normal()));
                    tk_path_move_to(p, pts[0], pts[1]);
                    for (size_t k = 2; k + 5 < pts.size(); k += 6)
                        tk_path_cubic_to(p, pts[k], pts[k + 1], pts[k + 2], pts[k + 3], pts[k + 4], pts[k + 5]);
                    tk_path_close(p);
                }
                c->points.insert(c->points.end(), pts.begin(), pts.end());
                float rgba[4] = {r.f32(0.0, 1.0), r.f32(0.0, 1.0), r.f32(0.0, 1.0), r.f32(0.0, 1.0)};
                c->colors.insert(c->colors.end(), rgba, rgba + 4);
                tk_brush_desc b = solid(rgba[0], rgba[1], rgba[2], rgba[3]);
                tk_canvas_push_path(c, p, &b, nullptr, TK_FILL_NONZERO, 0.1);
                tk_path_free(p);
            }
            tk_canvas_pop_layer(c);
            break;
        }
        default:
            return nullptr;
    }
    return c;
}

// The differentiable scene's flattening: flatten_path on move_to, cubic_to...,
// close, with every point carrying its weights over the four control points of
// its cubic (WPt), so that d(line endpoint)/d(control point) is known.
namespace {
// One path of the differentiable flattening: its lines in order, each handed
// to emit(line, base0, w0[4], base1, w1[4]) with its endpoints' control-point
// base indices and weights.
template <class Emit>
void diff_flatten_path(const tk_diff_scene* sc, uint32_t path, Emit&& emit) {
    const uint32_t n = sc->cubics_per_path, per = 1u + 3u * n;
    const double tol = double(sc->tolerance);
    struct Node {
        WPt p;
        uint32_t base;  // global index of the first of the four control points the weights refer to
    };
    const float* P = sc->points + size_t(2) * per * path;
    auto pt = [&](uint32_t j) { return Pt{double(P[2 * j]), double(P[2 * j + 1])}; };
    const uint32_t first = path * per;
    const Node start{{pt(0), {1.0, 0.0, 0.0, 0.0}}, first};
    Node last = start;
    auto push = [&](const Node& a, const Node& b) {
        double dx = a.p.v.x - b.p.v.x, dy = a.p.v.y - b.p.v.y;
        if (!(dx * dx + dy * dy > 1.0e-12 * 1.0e-12)) return;
        emit(tk_line{path, 0.0f, {float(a.p.v.x), float(a.p.v.y)}, {float(b.p.v.x), float(b.p.v.y)}}, a.base,
             a.p.w, b.base, b.p.w);
    };
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t base = first + 3u * k;
        // c[0] is the previous cubic's exact end point, pt(3k)
        const WPt c[4] = {{pt(3 * k), {1, 0, 0, 0}}, {pt(3 * k + 1), {0, 1, 0, 0}},
                          {pt(3 * k + 2), {0, 0, 1, 0}}, {pt(3 * k + 3), {0, 0, 0, 1}}};
        flatten_cubic(c, tol, [&](const WPt& q) {
            const Node nd{q, base};
            push(last, nd);
            last = nd;
        });
    }
    push(last, start);
}

// f(p) for every path p on host threads.
template <class F>
void for_each_path(uint32_t np, F&& f) {
    const uint32_t nt = std::max<uint32_t>(1u, std::min<uint32_t>(np, std::thread::hardware_concurrency()));
    std::atomic<uint32_t> next{0};
    auto work = [&]() {
        for (uint32_t p; (p = next.fetch_add(1)) < np;) f(p);
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
}
}  // namespace

void tk_diff_flatten_all(const tk_diff_scene* sc, std::vector<tk_line>& lines, std::vector<uint32_t>& ep_point,
                         std::vector<float>& ep_w) {
    lines.clear();
    ep_point.clear();
    ep_w.clear();
    if (!sc || !sc->points || sc->cubics_per_path == 0 || sc->path_count == 0) return;
    // paths are independent: count every path's lines on host threads, then
    // each thread writes its paths at their offsets (the vectors keep their
    // capacity between calls, so a steady caller touches no fresh pages)
    const uint32_t np = sc->path_count;
    std::vector<uint64_t> off(np + 1, 0);
    for_each_path(np, [&](uint32_t p) {
        uint64_t n = 0;
        diff_flatten_path(sc, p, [&](const tk_line&, uint32_t, const double*, uint32_t, const double*) { ++n; });
        off[p + 1] = n;
    });
    for (uint32_t p = 0; p < np; ++p) off[p + 1] += off[p];
    lines.resize(off[np]);
    ep_point.resize(2 * off[np]);
    ep_w.resize(8 * off[np]);
    for_each_path(np, [&](uint32_t p) {
        uint64_t at = off[p];
        diff_flatten_path(sc, p, [&](const tk_line& l, uint32_t b0, const double* w0, uint32_t b1, const double* w1) {
            lines[at] = l;
            ep_point[2 * at] = b0;
            ep_point[2 * at + 1] = b1;
            for (int i = 0; i < 4; ++i) {
                ep_w[8 * at + i] = float(w0[i]);
                ep_w[8 * at + 4 + i] = float(w1[i]);
            }
            ++at;
        });
    });
}

uint64_t tk_diff_flatten(const tk_diff_scene* sc, tk_line* lines, uint32_t* endpoint_point, float* endpoint_weights,
                         uint64_t capacity) {
    std::vector<tk_line> L;
    std::vector<uint32_t> E;
    std::vector<float> Wt;
    tk_diff_flatten_all(sc, L, E, Wt);
    const uint64_t k = std::min<uint64_t>(capacity, L.size());
    if (lines) std::copy(L.begin(), L.begin() + k, lines);
    if (endpoint_point) std::copy(E.begin(), E.begin() + 2 * k, endpoint_point);
    if (endpoint_weights) std::copy(Wt.begin(), Wt.begin() + 8 * k, endpoint_weights);
    return L.size();
}

// ---------------------------------------------------------------------------
// Replay and retained scenes (RetainedScene, src/retained_scene/scene.rs and
// transaction.rs; the materializer's damage, src/render/incremental.rs).
// ---------------------------------------------------------------------------

namespace {

// The affine map `outer` applied after `inner` (x' = a x + c y + e,
// y' = b x + d y + f).
void affine_after(const double o[6], const double i[6], double out[6]) {
    out[0] = o[0] * i[0] + o[2] * i[1];
    out[1] = o[1] * i[0] + o[3] * i[1];
    out[2] = o[0] * i[2] + o[2] * i[3];
    out[3] = o[1] * i[2] + o[3] * i[3];
    out[4] = o[0] * i[4] + o[2] * i[5] + o[4];
    out[5] = o[1] * i[4] + o[3] * i[5] + o[5];
}

int32_t replay_one(tk_canvas* dst, const RecCmd& r, const double* node_t) {
    double m[6];
    const double* t = nullptr;
    if (node_t && r.has_transform) {
        affine_after(node_t, r.t, m);
        t = m;
    } else if (node_t) {
        t = node_t;
    } else if (r.has_transform) {
        t = r.t;
    }
    tk_brush_desc b = r.brush;
    b.stops = r.stops.empty() ? nullptr : r.stops.data();
    const tk_brush_desc* bp = r.has_brush ? &b : nullptr;
    switch (r.kind) {
        case RecCmd::FILL: return tk_canvas_push_path(dst, &r.path, bp, t, r.rule, r.tolerance) < 0 ? -1 : 0;
        case RecCmd::GLYPHS: return tk_canvas_push_glyph_outlines(dst, &r.path, bp, t, r.tolerance) < 0 ? -1 : 0;
        case RecCmd::GLYPH_RUN: {
            // glyph runs take whole-pixel translations only (bitmap glyphs
            // have no transformed path, canvas/primitives/text.rs:7-10)
            double dx = 0.0, dy = 0.0;
            if (t) {
                if (t[0] != 1.0 || t[1] != 0.0 || t[2] != 0.0 || t[3] != 1.0) return -1;
                dx = t[4] * double(dst->scale);
                dy = t[5] * double(dst->scale);
                if (dx != std::floor(dx) || dy != std::floor(dy) || std::fabs(dx) > 1.0e9 || std::fabs(dy) > 1.0e9)
                    return -1;
            }
            std::vector<uint32_t> ids(r.run_images.size());
            for (size_t k = 0; k < r.run_images.size(); ++k) {
                const int32_t id = add_glyph_image(dst, r.run_images[k].desc, r.run_images[k].texels);
                if (id < 0) return -1;
                ids[k] = uint32_t(id);
            }
            std::vector<tk_glyph> gl = r.run_glyphs;
            for (tk_glyph& g : gl) {
                if (g.image != TK_INVALID_INDEX) g.image = ids[g.image];
                g.x += int32_t(dx);
                g.y += int32_t(dy);
            }
            int32_t cl[4];
            if (r.has_clip) {
                cl[0] = r.clip[0] + int32_t(dx);
                cl[1] = r.clip[1] + int32_t(dy);
                cl[2] = r.clip[2] + int32_t(dx);
                cl[3] = r.clip[3] + int32_t(dy);
            }
            return tk_canvas_push_glyph_run(dst, gl.data(), uint32_t(gl.size()), bp, r.has_clip ? cl : nullptr) < 0
                       ? -1
                       : 0;
        }
        case RecCmd::STROKE: return tk_canvas_push_stroke(dst, &r.path, bp, r.width, t, r.tolerance) < 0 ? -1 : 0;
        case RecCmd::CLIP: return tk_canvas_push_clip_layer(dst, &r.path, t, r.rule, r.tolerance);
        case RecCmd::OPACITY: return tk_canvas_push_opacity_layer(dst, &r.path, t, r.tolerance, r.sigma);
        case RecCmd::BLUR: return tk_canvas_push_blur_group_sampled(dst, r.sigma, r.sampling);
        case RecCmd::PROGRESSIVE: {
            // ProgressiveBlur::translated (canvas/offset.rs:153-154): translations only
            double dx = 0.0, dy = 0.0;
            if (t) {
                if (t[0] != 1.0 || t[1] != 0.0 || t[2] != 0.0 || t[3] != 1.0) return -1;
                dx = t[4];
                dy = t[5];
            }
            return tk_canvas_push_progressive_blur_group(dst, r.shape.p0[0] + dx, r.shape.p0[1] + dy,
                                                         r.shape.p1[0] + dx, r.shape.p1[1] + dy, r.sigma,
                                                         r.sampling);
        }
        case RecCmd::FILTER: {
            // a rect region moves with a translation; under any other
            // transform it becomes the transformed rectangle path, and a path
            // region composes the transform (effect_placement.rs:57-118)
            double rect[4] = {r.shape.p0[0], r.shape.p0[1], r.shape.p1[0], r.shape.p1[1]};
            const bool moved = t && (t[0] != 1.0 || t[1] != 0.0 || t[2] != 0.0 || t[3] != 1.0);
            if (t && !moved) {
                rect[0] += t[4];
                rect[1] += t[5];
                rect[2] += t[4];
                rect[3] += t[5];
            }
            std::vector<tk_canvas_filter> chain = r.chain;
            size_t word = 0;
            for (tk_canvas_filter& f : chain) {
                if (f.kind == TK_FILTER_COMPONENT_TRANSFER) {
                    f.table = r.tables.data() + word;
                    word += TK_TRANSFER_TABLE_WORDS;
                }
                if (f.kind == TK_FILTER_CONVOLVE) {
                    f.kernel = reinterpret_cast<const float*>(r.tables.data() + word);
                    word += size_t(f.columns) * f.rows;
                }
            }
            if (r.region_path || moved) {
                tk_path region;
                if (r.region_path) {
                    region = r.path;
                } else {
                    region.els.push_back(El{MOVE, {Pt{rect[0], rect[1]}}});
                    region.els.push_back(El{LINE, {Pt{rect[2], rect[1]}}});
                    region.els.push_back(El{LINE, {Pt{rect[2], rect[3]}}});
                    region.els.push_back(El{LINE, {Pt{rect[0], rect[3]}}});
                    region.els.push_back(El{CLOSE, {}});
                }
                return tk_canvas_push_filter_layer_path(dst, chain.data(), uint32_t(chain.size()), &region, t,
                                                        r.fixed ? 1 : 0);
            }
            return tk_canvas_push_filter_layer(dst, chain.data(), uint32_t(chain.size()), rect, r.fixed ? 1 : 0);
        }
        case RecCmd::POP: return tk_canvas_pop_layer(dst);
        case RecCmd::SDF:
        case RecCmd::SDF_CLIP: {
            // SDF records carry no draw transform: they replay under translations
            tk_sdf_shape sh = r.shape;
            if (t) {
                if (t[0] != 1.0 || t[1] != 0.0 || t[2] != 0.0 || t[3] != 1.0) return -1;
                sh.p0[0] += t[4];
                sh.p0[1] += t[5];
                sh.p1[0] += t[4];
                sh.p1[1] += t[5];
                if (sh.kind == TK_SDF_CANDLESTICK) {  // y values in p1, p2[0]
                    sh.p1[0] += t[5] - t[4];
                    sh.p2[0] += t[5];
                } else {
                    sh.p2[0] += t[4];
                    sh.p2[1] += t[5];
                }
            }
            return r.kind == RecCmd::SDF_CLIP ? tk_canvas_push_clip_sdf_layer(dst, &sh)
                                              : (tk_canvas_push_sdf(dst, &sh, bp) == -1 ? -1 : 0);
        }
        case RecCmd::IMAGE: {
            // the brush maps the image into the rect: a translated rect carries it along
            double rect[4] = {r.shape.p0[0], r.shape.p0[1], r.shape.p1[0], r.shape.p1[1]};
            if (t) {
                if (t[0] != 1.0 || t[1] != 0.0 || t[2] != 0.0 || t[3] != 1.0) return -1;
                rect[0] += t[4];
                rect[1] += t[5];
                rect[2] += t[4];
                rect[3] += t[5];
            }
            const int32_t ix = add_image(dst, r.texels, r.iw, r.ih);
            return tk_canvas_push_image(dst, rect, uint32_t(ix), r.extend, r.sampling, r.opacity) == -1 ? -1 : 0;
        }
    }
    return -1;
}

bool has_layers(const std::vector<RecCmd>& log) {
    for (const RecCmd& r : log)
        if (r.kind == RecCmd::CLIP || r.kind == RecCmd::BLUR || r.kind == RecCmd::PROGRESSIVE || r.kind == RecCmd::FILTER ||
            r.kind == RecCmd::SDF_CLIP ||
            r.kind == RecCmd::OPACITY)
            return true;
    return false;
}

using Content = std::shared_ptr<const std::vector<RecCmd>>;

struct RNode {
    uint64_t id;
    Content content;
    bool layered;
    bool has_t;
    double t[6];
    uint64_t rev;
};

struct Drawn {
    uint64_t rev;
    bool layered;
    std::vector<tk_pixel_bounds> rects;
};

}  // namespace

struct tk_retained {
    uint32_t lw = 0, lh = 0;
    float scale = 1.0f;
    uint32_t clear = 0;
    bool device_flatten = false;
    std::vector<RNode> nodes;  // painter order
    uint64_t version = 0, next_rev = 1;
    bool materialized = false, pending_all = true;
    std::vector<int32_t> pending_rects;
    std::unordered_map<uint64_t, Drawn> drawn;  // per node at the last materialization
    tk_canvas* canvas = nullptr;
    std::vector<int32_t> damage;
};

namespace {

int64_t find_node(const tk_retained* rs, uint64_t id) {
    for (size_t k = 0; k < rs->nodes.size(); ++k)
        if (rs->nodes[k].id == id) return int64_t(k);
    return -1;
}

// A node's content: the canvas's command log, which must be kept and close
// every layer it opens.
bool content_of(const tk_canvas* c, Content& out, bool& layered) {
    if (!c || !c->keep || c->stack.size() != 1) return false;
    out = std::make_shared<const std::vector<RecCmd>>(c->log);
    layered = has_layers(c->log);
    return true;
}

void set_node_transform(RNode& n, const double* t) {
    n.has_t = t != nullptr;
    if (t) std::memcpy(n.t, t, sizeof(n.t));
}

void touched(tk_retained* rs, RNode& n) {
    n.rev = rs->next_rev++;
    ++rs->version;
}

}  // namespace

extern "C" {

int32_t tk_canvas_replay(tk_canvas* dst, const tk_canvas* src, const double* transform) {
    if (!dst || !src || !src->keep || src->stack.size() != 1) return -1;
    for (const RecCmd& r : src->log)
        if (replay_one(dst, r, transform) != 0) return -1;
    return 0;
}

tk_retained* tk_retained_new(uint32_t logical_width, uint32_t logical_height, float scale) {
    if (!(scale > 0.0f) || !std::isfinite(scale) || !logical_width || !logical_height) return nullptr;
    auto* rs = new tk_retained();
    rs->lw = logical_width;
    rs->lh = logical_height;
    rs->scale = scale;
    return rs;
}
void tk_retained_free(tk_retained* rs) {
    if (!rs) return;
    tk_canvas_free(rs->canvas);
    delete rs;
}
void tk_retained_set_clear_color(tk_retained* rs, uint32_t premul) {
    if (!rs || rs->clear == premul) return;
    rs->clear = premul;
    rs->pending_all = true;
    ++rs->version;
}
void tk_retained_set_device_flatten(tk_retained* rs, int32_t enabled) {
    if (rs) rs->device_flatten = enabled != 0;  // the same lines either way: no damage
}
uint64_t tk_retained_version(const tk_retained* rs) { return rs ? rs->version : 0; }

int32_t tk_retained_insert(tk_retained* rs, uint64_t id, const tk_canvas* content, const double* transform,
                           uint64_t before) {
    if (!rs || id == 0 || find_node(rs, id) >= 0) return -1;
    RNode n{};
    n.id = id;
    if (!content_of(content, n.content, n.layered)) return -1;
    set_node_transform(n, transform);
    size_t at = rs->nodes.size();
    if (before) {
        const int64_t k = find_node(rs, before);
        if (k < 0) return -1;
        at = size_t(k);
    }
    touched(rs, n);
    rs->nodes.insert(rs->nodes.begin() + int64_t(at), std::move(n));
    return 0;
}
int32_t tk_retained_replace(tk_retained* rs, uint64_t id, const tk_canvas* content) {
    const int64_t k = rs ? find_node(rs, id) : -1;
    if (k < 0) return -1;
    RNode& n = rs->nodes[size_t(k)];
    Content c;
    bool layered = false;
    if (!content_of(content, c, layered)) return -1;
    n.content = std::move(c);
    n.layered = layered;
    touched(rs, n);
    return 0;
}
int32_t tk_retained_set_transform(tk_retained* rs, uint64_t id, const double* transform) {
    const int64_t k = rs ? find_node(rs, id) : -1;
    if (k < 0) return -1;
    RNode& n = rs->nodes[size_t(k)];
    set_node_transform(n, transform);
    touched(rs, n);
    return 0;
}
int32_t tk_retained_move_before(tk_retained* rs, uint64_t id, uint64_t sibling) {
    const int64_t k = rs ? find_node(rs, id) : -1;
    if (k < 0 || sibling == id) return -1;
    if (sibling && find_node(rs, sibling) < 0) return -1;
    RNode n = std::move(rs->nodes[size_t(k)]);
    rs->nodes.erase(rs->nodes.begin() + k);
    size_t at = rs->nodes.size();
    if (sibling) at = size_t(find_node(rs, sibling));
    touched(rs, n);
    rs->nodes.insert(rs->nodes.begin() + int64_t(at), std::move(n));
    return 0;
}
int32_t tk_retained_remove(tk_retained* rs, uint64_t id) {
    const int64_t k = rs ? find_node(rs, id) : -1;
    if (k < 0) return -1;
    rs->nodes.erase(rs->nodes.begin() + k);
    ++rs->version;
    return 0;
}
int32_t tk_retained_invalidate_rect(tk_retained* rs, const int32_t rect[4]) {
    if (!rs || !rect) return -1;
    rs->pending_rects.insert(rs->pending_rects.end(), rect, rect + 4);
    ++rs->version;
    return 0;
}
int32_t tk_retained_invalidate_all(tk_retained* rs) {
    if (!rs) return -1;
    rs->pending_all = true;
    ++rs->version;
    return 0;
}

tk_canvas* tk_retained_materialize(tk_retained* rs, tk_damage* damage) {
    if (!rs) return nullptr;
    tk_canvas* c = tk_canvas_new(rs->lw, rs->lh, rs->scale);
    if (!c) return nullptr;
    c->host_plan = false;
    if (rs->device_flatten) tk_canvas_set_device_flatten(c, 1);
    c->clear = rs->clear;
    std::unordered_map<uint64_t, Drawn> now;
    for (const RNode& n : rs->nodes) {
        const size_t d0 = c->draws.size();
        for (const RecCmd& r : *n.content) {
            if (replay_one(c, r, n.has_t ? n.t : nullptr) != 0) {
                tk_canvas_free(c);
                return nullptr;
            }
        }
        Drawn d{n.rev, n.layered, {}};
        for (size_t k = d0; k < c->draws.size(); ++k) {
            const tk_pixel_bounds& b = c->draws[k].pixel_bounds;
            if (b.x1 > b.x0 && b.y1 > b.y0) d.rects.push_back(b);
        }
        now.emplace(n.id, std::move(d));
    }
    // Damage: the draw rectangles, before and after, of every node inserted,
    // changed, moved or removed since the last materialization. A change to a
    // node with clip or blur layers can merge or split the draw batches of
    // other nodes (and so where pixels are stored as RGBA8 between them),
    // which a rectangle does not bound: such changes damage everything.
    bool full = !rs->materialized || rs->pending_all;
    rs->damage.clear();
    auto add = [&](const std::vector<tk_pixel_bounds>& rects) {
        for (const tk_pixel_bounds& b : rects) rs->damage.insert(rs->damage.end(), {b.x0, b.y0, b.x1, b.y1});
    };
    if (!full) {
        for (const auto& kv : now) {
            auto it = rs->drawn.find(kv.first);
            if (it == rs->drawn.end()) {
                full = full || kv.second.layered;
                add(kv.second.rects);
            } else if (it->second.rev != kv.second.rev) {
                full = full || kv.second.layered || it->second.layered;
                add(it->second.rects);
                add(kv.second.rects);
            }
        }
        for (const auto& kv : rs->drawn) {
            if (now.count(kv.first)) continue;
            full = full || kv.second.layered;
            add(kv.second.rects);
        }
        rs->damage.insert(rs->damage.end(), rs->pending_rects.begin(), rs->pending_rects.end());
    }
    if (full) rs->damage.clear();
    rs->drawn = std::move(now);
    rs->pending_rects.clear();
    rs->pending_all = false;
    rs->materialized = true;
    tk_canvas_free(rs->canvas);
    rs->canvas = c;
    if (damage) {
        damage->full = full ? 1u : 0u;
        damage->rect_count = uint32_t(rs->damage.size() / 4);
        damage->rects = rs->damage.empty() ? nullptr : rs->damage.data();
    }
    return c;
}

}  // extern "C"
