// C ABI of the B200 tile rasterization path: context, scene upload,
// frame driver, readback, debug readback and stage harnesses.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tileink.h"
#include "../../include/tileink_canvas.h"
#include "../../include/tileink_diff.h"
#include "flatten_core.h"
#include "host.h"
#include "kernels.h"

namespace {

struct Fail {
    int32_t code;
    std::string msg;
};

#define TK_CUDA(call)                                                                                   \
    do {                                                                                                \
        cudaError_t e_ = (call);                                                                        \
        if (e_ != cudaSuccess) throw Fail{TK_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

// Device buffer that only grows; owns its allocation (freed when released,
// reassigned by a move, or destroyed).
template <class T>
struct DBuf {
    T* ptr = nullptr;
    size_t cap = 0;  // elements
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : ptr(o.ptr), cap(o.cap) {
        o.ptr = nullptr;
        o.cap = 0;
    }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) {
            release();
            ptr = o.ptr;
            cap = o.cap;
            o.ptr = nullptr;
            o.cap = 0;
        }
        return *this;
    }
    ~DBuf() { release(); }
    void reserve(size_t n) {
        if (n <= cap && ptr) return;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
        size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
        cudaError_t e = cudaMalloc(&ptr, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            ptr = nullptr;
            throw Fail{TK_E_ALLOC, "device allocation of " + std::to_string(bytes) + " bytes failed"};
        }
        cap = std::max<size_t>(n, 1);
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        cap = 0;
    }
};

// Scratch of device flattening and stroking, kept between uploads (grow-only)
// so that a scene re-uploaded every frame does not allocate.
struct FlattenScratch {
    DBuf<tk_flatten_el> els, sels;
    DBuf<uint32_t> path_els, offsets, sums, words, soff, ssums, poly_n, line_off, unit_lines;
    DBuf<tk_stroke_polyline> polys;
    DBuf<tk_stroke_desc> strokes;
    DBuf<unsigned long long> wide;
    DBuf<tkf::Pt> pts;
    void release() {
        for (auto* b : {&path_els, &offsets, &sums, &words, &soff, &ssums, &poly_n, &line_off, &unit_lines}) b->release();
        els.release();
        sels.release();
        polys.release();
        strokes.release();
        wide.release();
        pts.release();
    }
};

struct Pass {
    uint32_t order0 = 0, draw_n = 0, batch0 = 0, batch_n = 0;
    std::vector<tk::PassBatch> batches;
    DBuf<tk::PassBatch> d_batches;
    DBuf<uint32_t> bin_lists, bin_counts;
    DBuf<tk_tile_record> tiles;
    DBuf<tk_ptcl_record> ptcl;
    uint64_t ptcl_needed = 0;  // known after the first frame, 0 = unknown
    uint64_t ptcl_used = 0;
    DBuf<uint32_t> glyph_list;  // text scenes: the glyph indices PTCL_GLYPH records name
    uint64_t glyph_needed = 0, glyph_used = 0;
};

// A new upload's passes take over the device buffers of the last upload's
// passes, position by position (grow-only, so re-uploading a scene allocates
// nothing); the buffers of passes the new scene does not have are freed.
void adopt_pass_buffers(std::vector<Pass>& now, std::vector<Pass>& old) {
    for (size_t i = 0; i < now.size() && i < old.size(); ++i) {
        now[i].d_batches = std::move(old[i].d_batches);
        now[i].bin_lists = std::move(old[i].bin_lists);
        now[i].bin_counts = std::move(old[i].bin_counts);
        now[i].tiles = std::move(old[i].tiles);
        now[i].ptcl = std::move(old[i].ptcl);
        now[i].glyph_list = std::move(old[i].glyph_list);
    }
    old.clear();
}

enum StepKind { STEP_PASS, STEP_BLUR_BEGIN, STEP_BLUR_END };
struct Step {
    StepKind kind;
    uint32_t pass;
    float sigma;
    int32_t bounds[4];
    uint32_t sampling = 0u;  // BLUR_BEGIN: TK_BLUR_SAMPLING_* word (0: full resolution)
    bool progressive = false;  // BLUR_BEGIN of a progressive blur group
    tk_progressive_blur prog{};
    std::vector<tk_filter> chain;  // BLUR_BEGIN of a filter layer: its chain (filter is set)
    bool filter = false;
    bool shadow = false;  // the chain has a drop shadow (a second scratch surface)
};

// State of the last differentiable forward, kept for its backward.
struct DiffState {
    bool ready = false;
    uint32_t width = 0, height = 0, paths = 0, points = 0, pass = 0;
    uint64_t lines = 0;
    int32_t radius = 0;
    float sigma = 0.0f;
    float4 bg{};
    std::vector<float> colors;  // straight RGBA per path
    DBuf<float4> colp, target, layer, t1, blurred, gI, d0, d1;
    DBuf<float2> scratch, line_acc;
    DBuf<float> color_acc, dpoints, taps, dtaps, ep_w;
    DBuf<uint32_t> ep_point;
    DBuf<double> sums;  // [0] loss [1] dL/dsigma
    // the forward's host flattening and its device check, kept between calls
    std::vector<tk_line> h_lines, h_dev_lines;
    std::vector<uint32_t> h_ep_point;
    std::vector<float> h_ep_w;
};

}  // namespace

struct tk_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    // A second stream for the scene records an upload copies while the main
    // stream flattens on the device, and the events that order the two.
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_main = nullptr, ev_copy = nullptr;
    std::string error;
    // scene
    bool have_scene = false;
    uint32_t width = 0, height = 0, tw = 0, th = 0, clear = 0, flags = 0;
    uint64_t line_count = 0, brush_words = 0, pool_len = 0, host_segment_capacity = 0;
    uint64_t sdf_words = 0, sdf_shadow_base = 0;  // SDF buffer: sdf_blob, then sdf_shadow_blob
    bool sdf_ext = false;                          // a candlestick, dash line, triangle or checkerboard
    bool text = false;                             // glyph outline fills or glyph runs
    uint32_t path_count = 0, draw_count = 0, layer_count = 0, order_count = 0;
    std::vector<tk_path_record> h_paths;
    std::vector<tk::ScanItem> h_items;
    std::vector<Pass> passes;
    std::vector<Step> steps;
    uint64_t tile_draw_refs = 0;
    // device scene
    DBuf<tk_line> lines;
    DBuf<tk_path_record> paths;
    DBuf<tk_draw_record> draws;
    DBuf<uint32_t> brush, sdf, batch_ids, order;
    DBuf<uint32_t> texels;  // the scene's images, concatenated
    DBuf<uint4> image_tab;  // per image: first texel, width, height
    // the text blob (glyph runs)
    uint32_t glyph_run_count = 0;
    DBuf<tk_glyph_run> glyph_runs;
    DBuf<tk_glyph> glyphs;
    DBuf<tk_glyph_image> glyph_images;
    DBuf<uint32_t> glyph_texels;
    DBuf<uint32_t> filter_words;  // filter layers' transfer tables and convolution kernels
    DBuf<tk_layer_record> layers;
    DBuf<tk::ScanItem> items;
    DBuf<unsigned long long> item_desc, tile_desc, stats;
    DBuf<int32_t> backdrops;
    // misc: [0] error [1] ticket [2] seg total [3] ptcl total [4] emit ticket
    // [5] delta total check [6] glyph list total
    DBuf<uint32_t> counts, cursors, bumps, misc;
    DBuf<tk_segment_range> ranges;
    DBuf<tk::SegmentRec> segments;
    DBuf<tk::PaintInfo> paints;  // per draw, built at upload
    uint64_t segment_needed = 0;  // device plan: total from the last frame
    DBuf<uint32_t> image, temp, low;  // target, blur temporary, reduced-resolution blur surface
    tk::ProgressiveScratch prog_scratch;  // progressive blur levels (grown on demand)
    std::vector<DBuf<uint32_t>> surfaces;
    bool rendered = false;
    // paths by decreasing line count: the order scan_emit's warps take them
    DBuf<uint32_t> emit_order;
    // line index per emitted segment (differentiable mode only)
    DBuf<uint32_t> seg_line;
    bool want_seg_line = false;
    DiffState diff;
    // pool-scan work item size in tiles (whole bbox rows up to this many)
    uint32_t scan_item_elems = tk::kScanItemElems;
    // batched mode: several canvases in one pass, rendered by one graph launch
    bool batched = false;
    std::vector<tk::BatchScene> h_scenes;
    std::vector<tk_batch_info> h_batch_info;
    DBuf<tk::BatchScene> d_scenes;
    DBuf<uint32_t> bin_scene, tile_scene;
    uint32_t total_bins = 0, total_tiles = 0;
    uint64_t total_pixels = 0;
    cudaGraphExec_t graph_exec = nullptr;
    // stage timing
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
    FlattenScratch flat;
    // incremental rendering: whether `image` holds the last single-scene
    // frame (and its size and clear colour), and the redrawn tiles of the
    // frame in progress (null outside tk_render_incremental)
    bool history = false;
    uint32_t history_w = 0, history_h = 0, history_clear = 0;
    std::vector<uint8_t> h_active;
    std::vector<uint32_t> h_active_list;
    DBuf<uint8_t> tile_active;
    DBuf<uint32_t> tile_list;
    const uint8_t* active_mask = nullptr;
    const uint32_t* active_list = nullptr;
    uint32_t active_n = 0;
    // band split (tk_set_band): tile rows [band_y0, band_y1) of the frame;
    // paths are clamped to them at upload
    bool band = false;
    uint32_t band_y0 = 0, band_y1 = 0;
    std::vector<tk_path_record> band_paths;
    // the scan buffers hold the scan of the uploaded scene (nothing has
    // been uploaded or scanned into them since), except for the paths in
    // `rescan`, whose records or lines a delta upload replaced
    bool scan_valid = false;
    std::vector<uint32_t> rescan;
    DBuf<uint32_t> rescan_list;
    DBuf<tk::ScanItem> rescan_items;
    DBuf<unsigned long long> rescan_desc;
    // device segment plans: the rescanned paths keep their planned slices
    // only if their counted totals still fill them exactly (checked after
    // counting; otherwise the whole scene is scanned)
    bool rescan_check = false;
    uint32_t last_scan_paths = 0;  // paths the last scan covered
};

namespace {

int32_t fail(tk_ctx* c, const Fail& f) {
    if (c) c->error = f.msg;
    return f.code;
}

template <class F>
int32_t guarded(tk_ctx* c, F&& f) {
    if (!c) return TK_E_INVALID;
    try {
        TK_CUDA(cudaSetDevice(c->device));
        f();
        return TK_OK;
    } catch (const Fail& e) {
        return fail(c, e);
    } catch (const std::exception& e) {
        return fail(c, Fail{TK_E_INVALID, e.what()});
    }
}

void invalid(const std::string& m) { throw Fail{TK_E_INVALID, m}; }

template <class T>
void upload(DBuf<T>& b, const T* src, size_t n, cudaStream_t st) {
    b.reserve(n);
    if (n) TK_CUDA(cudaMemcpyAsync(b.ptr, src, n * sizeof(T), cudaMemcpyHostToDevice, st));
}

// Host validation of a scene against the contracts the kernels rely on.
void validate_and_plan(tk_ctx* c, const tk_scene_desc& d) {
    if (d.width == 0 || d.height == 0) invalid("empty canvas");
    uint32_t tw = (d.width + TK_TILE_SIZE - 1) / TK_TILE_SIZE, th = (d.height + TK_TILE_SIZE - 1) / TK_TILE_SIZE;
    if (uint64_t(tw) * th > 0x7FFFFFFFull || tw > 65535u || th > 65535u) invalid("canvas too large");
    if ((d.line_count && !d.lines) || (d.path_count && !d.paths) || (d.draw_count && !d.draws) ||
        (d.brush_word_count && !d.brush_blob) || (d.layer_count && !d.layers) ||
        (d.sdf_word_count && !d.sdf_blob) || (d.sdf_shadow_word_count && !d.sdf_shadow_blob) ||
        (d.image_count && !d.images) ||
        (d.draw_order_count && !d.draw_order) || (d.draw_count && !d.draw_batch_ids) || (d.op_count && !d.ops))
        invalid("null array with nonzero count");
    bool device_plan = (d.flags & TK_SCENE_SEGMENTS_FROM_DEVICE) != 0u;
    // Paths: line ranges partition the line array in path order; bbox inside
    // the canvas; data_len matches the bbox.
    uint64_t next_line = 0, pool = 0, seg_cap = 0;
    uint32_t next_data = d.path_count ? d.paths[0].data_offset : 0u;
    c->h_items.clear();
    for (uint32_t p = 0; p < d.path_count; ++p) {
        const tk_path_record& r = d.paths[p];
        if (r.line_start != next_line) invalid("path " + std::to_string(p) + ": lines are not consecutive per path");
        next_line += r.line_count;
        if (r.tile_x1 > tw || r.tile_y1 > th) invalid("path " + std::to_string(p) + ": tile bbox outside the canvas");
        uint32_t stride = r.tile_x1 > r.tile_x0 ? r.tile_x1 - r.tile_x0 : 0u;
        uint32_t height = r.tile_y1 > r.tile_y0 ? r.tile_y1 - r.tile_y0 : 0u;
        if (uint64_t(stride) * height != r.data_len) invalid("path " + std::to_string(p) + ": data_len != bbox tiles");
        if (stride > tk::kScanItemElems) invalid("path bbox wider than 4096 tiles");
        if (device_plan && r.data_offset != next_data)
            invalid("device segment planning needs contiguous backdrop slices in path order");
        next_data = r.data_offset + r.data_len;
        pool = std::max<uint64_t>(pool, uint64_t(r.data_offset) + r.data_len);
        if (pool > 0xFFFFFFFFull) invalid("backdrop pool exceeds u32 indexing");
        seg_cap = std::max<uint64_t>(seg_cap, uint64_t(r.segment_start) + r.segment_capacity);
        if (r.data_len) {
            uint32_t rows_per = std::max<uint32_t>(1u, c->scan_item_elems / stride);
            for (uint32_t row = 0; row < height; row += rows_per)
                c->h_items.push_back({p, row, std::min(rows_per, height - row), row == 0u ? 1u : 0u});
        }
    }
    if (next_line != d.line_count) invalid("path line ranges do not cover the line array");
    if (seg_cap > 0xFFFFFFFFull) invalid("segment capacity exceeds u32 indexing");
    if (d.sdf_word_count + d.sdf_shadow_word_count > 0xFFFFFFFFull) invalid("SDF blobs exceed u32 indexing");
    uint64_t texel_words = 0;
    for (uint32_t k = 0; k < d.image_count; ++k) {
        const tk_image_desc& im = d.images[k];
        if (!im.premul_rgba8 || im.width == 0u || im.height == 0u) invalid("image " + std::to_string(k) + " is empty");
        if (im.width > TK_MAX_IMAGE_DIMENSION || im.height > TK_MAX_IMAGE_DIMENSION)
            invalid("image " + std::to_string(k) + " exceeds the 2D texture limit of " +
                    std::to_string(TK_MAX_IMAGE_DIMENSION));
        texel_words += uint64_t(im.width) * im.height;
    }
    if (texel_words > 0xFFFFFFFFull) invalid("images exceed u32 indexing");
    // the text blob: runs inside the glyphs, glyphs naming images, images
    // inside the texels
    if ((d.glyph_run_count && !d.glyph_runs) || (d.glyph_count && !d.glyphs) ||
        (d.glyph_image_count && !d.glyph_images) || (d.glyph_texel_count && !d.glyph_texels))
        invalid("null text blob array with nonzero count");
    if (d.glyph_texel_count > 0xFFFFFFFFull) invalid("glyph texels exceed u32 indexing");
    for (uint32_t k = 0; k < d.glyph_run_count; ++k)
        if (uint64_t(d.glyph_runs[k].first) + d.glyph_runs[k].count > d.glyph_count)
            invalid("glyph run " + std::to_string(k) + " outside the glyphs");
    for (uint32_t k = 0; k < d.glyph_count; ++k)
        if (d.glyphs[k].image != TK_INVALID_INDEX && d.glyphs[k].image >= d.glyph_image_count)
            invalid("glyph " + std::to_string(k) + ": image out of range");
    for (uint32_t k = 0; k < d.glyph_image_count; ++k) {
        const tk_glyph_image& im = d.glyph_images[k];
        if (im.content > TK_GLYPH_LINEAR_SUBPIXEL_MASK) invalid("glyph image " + std::to_string(k) + ": bad content");
        if (im.width > TK_MAX_IMAGE_DIMENSION || im.height > TK_MAX_IMAGE_DIMENSION ||
            uint64_t(im.data_offset) + uint64_t(im.width) * im.height > d.glyph_texel_count)
            invalid("glyph image " + std::to_string(k) + " outside the glyph texels");
    }
    bool sdf_ext = false;
    bool text = false;
    // Draws: path fills/clips, and brush draws of the SDF kinds this library
    // renders (one complete record each, src/shared/gpu_sdf.rs:27-46).
    for (uint32_t i = 0; i < d.draw_count; ++i) {
        const tk_draw_record& r = d.draws[i];
        const auto at = [i] { return "draw " + std::to_string(i); };  // built only for a message
        if (r.tag == TK_DRAW_PATH_GLYPH || r.glyph_run_id != TK_INVALID_INDEX) text = true;
        if (r.glyph_run_id != TK_INVALID_INDEX) {
            // a glyph run draw (canvas/primitives/text.rs:80-96)
            if (r.glyph_run_id >= d.glyph_run_count) invalid(at() + ": glyph run out of range");
            if (r.tag != TK_DRAW_BRUSH || r.path_id != TK_INVALID_INDEX || r.sdf_offset != TK_INVALID_INDEX ||
                r.sdf_shadow_offset != TK_INVALID_INDEX)
                invalid(at() + ": a glyph run draw is a brush draw without a path or SDF record");
        }
        const bool plain = r.sdf_offset != TK_INVALID_INDEX, shadow = r.sdf_shadow_offset != TK_INVALID_INDEX;
        if (plain || shadow) {
            if (plain && shadow) invalid(at() + ": both an SDF and a shadow record");
            if (r.tag != TK_DRAW_BRUSH && !(r.tag == TK_DRAW_CLIP && plain))
                invalid(at() + ": SDF groups and shadow clips are outside this path");
            if (r.path_id != TK_INVALID_INDEX) invalid(at() + ": an SDF draw with a path");
            const uint64_t off = plain ? r.sdf_offset : r.sdf_shadow_offset;
            const uint64_t len = plain ? r.sdf_len : r.sdf_shadow_len;
            const uint64_t words = plain ? d.sdf_word_count : d.sdf_shadow_word_count;
            if (len != TK_SDF_RECORD_WORDS || off + len > words) invalid(at() + ": SDF record outside its blob");
            const uint32_t kind = (plain ? d.sdf_blob : d.sdf_shadow_blob)[off];
            const bool ext = plain ? (kind == TK_SDF_CANDLESTICK || kind == TK_SDF_DASH_LINE || kind == TK_SDF_TRIANGLE ||
                                      kind == TK_SDF_CHECKERBOARD || kind == TK_SDF_CALLOUT ||
                                      kind == TK_SDF_CALLOUT_STROKE || kind == TK_SDF_ARC ||
                                      kind == TK_SDF_STAR || kind == TK_SDF_STAR_STROKE)
                                   : (kind == TK_SDF_CALLOUT_SHADOW || kind == TK_SDF_ARC_SHADOW);
            const bool ok = ext || (plain ? (kind == TK_SDF_RECT || kind == TK_SDF_CIRCLE || kind == TK_SDF_RECT_STROKE ||
                                             kind == TK_SDF_CIRCLE_STROKE || kind == TK_SDF_LINE)
                                          : (kind == TK_SDF_RECT_SHADOW || kind == TK_SDF_CIRCLE_SHADOW ||
                                             kind == TK_SDF_LINE_SHADOW));
            if (!ok) invalid(at() + ": SDF kind " + std::to_string(kind) + " is not supported");
            sdf_ext = sdf_ext || ext;
        }
        // image pattern brushes (shared/brush/sample.hlsli:32-41): texture-table
        // placement of a registered image, sized as that image
        const uint64_t bo = r.brush_offset;
        if (bo != TK_INVALID_INDEX && bo < d.brush_word_count && d.brush_blob[bo] == TK_BRUSH_PATTERN_RESOURCE) {
            if (bo + TK_BRUSH_HEADER_WORDS + TK_BRUSH_PARAM_WORDS > d.brush_word_count)
                invalid(at() + ": image brush outside the brush blob");
            const uint32_t* w = d.brush_blob + bo;
            const uint32_t ix = w[4] & ~TK_BRUSH_TEXTURE_PLACEMENT_BIT;
            if (!(w[4] & TK_BRUSH_TEXTURE_PLACEMENT_BIT)) invalid(at() + ": atlas image placement is outside this path");
            if (ix >= d.image_count) invalid(at() + ": image index out of range");
            if (w[5] != d.images[ix].width || w[6] != d.images[ix].height)
                invalid(at() + ": image brush size differs from its image");
            if (!plain) invalid(at() + ": image patterns fill SDF rects only");
            if (w[1] > TK_EXTEND_REFLECT || w[7] > 255u || w[8] > TK_PATTERN_BILINEAR)
                invalid(at() + ": bad image brush extend, opacity or sampling");
        }
        if (r.tag != TK_DRAW_BRUSH && r.tag != TK_DRAW_CLIP && r.tag != TK_DRAW_OPACITY && r.tag != TK_DRAW_BLEND &&
            r.tag != TK_DRAW_ISOLATE && r.tag != TK_DRAW_PATH_GLYPH)
            invalid("draw " + std::to_string(i) + ": unsupported tag");
        if (r.tag == TK_DRAW_PATH_GLYPH && r.path_id == TK_INVALID_INDEX)
            invalid("draw " + std::to_string(i) + ": a glyph outline draw without a path");
        if (r.path_id != TK_INVALID_INDEX && r.path_id >= d.path_count) invalid("draw path out of range");
        if (r.fill_rule > 1u) invalid("bad fill rule");
    }
    for (uint32_t i = 0; i < d.layer_count; ++i) {
        if (d.layers[i].tag == TK_LAYER_BLEND) invalid("blend layers are outside this path");
        if (d.layers[i].tag > TK_LAYER_BLEND) invalid("bad layer tag");
        if (d.layers[i].draw >= d.draw_count) invalid("layer draw out of range");
        const tk_draw_record& ld = d.draws[d.layers[i].draw];
        const bool sdf_clip = ld.sdf_offset != TK_INVALID_INDEX && ld.tag == TK_DRAW_CLIP;
        if (sdf_clip ? d.layers[i].tag != TK_LAYER_CLIP : ld.path_id == TK_INVALID_INDEX)
            invalid("layer draws must be path draws, or SDF draws of clip layers");
    }
    // Painter order grouped by batch in op order.
    std::vector<uint32_t> batch_draws;
    for (uint32_t k = 0; k < d.draw_order_count; ++k) {
        uint32_t di = d.draw_order[k];
        if (di >= d.draw_count) invalid("draw order out of range");
        uint32_t b = d.draw_batch_ids[di];
        if (b == TK_INVALID_INDEX) invalid("ordered draw without a batch");
        if (b + 1 > batch_draws.size()) batch_draws.resize(b + 1, 0u);
        if (k && d.draw_batch_ids[d.draw_order[k - 1]] > b) invalid("draw order is not grouped by batch");
        batch_draws[b]++;
    }
    // Ops -> passes and steps. The last scene's passes keep their device
    // buffers until the new passes take them over (or free them on a throw).
    std::vector<Pass> old_passes;
    old_passes.swap(c->passes);
    c->steps.clear();
    uint32_t order_pos = 0, depth = 0;
    int64_t last_batch = -1;
    bool open = false;
    for (uint32_t i = 0; i < d.op_count; ++i) {
        const tk_op& op = d.ops[i];
        if (op.kind == TK_OP_DRAW_BATCH) {
            if (int64_t(op.batch_id) != last_batch + 1) invalid("batch ids must be consecutive in op order");
            last_batch = op.batch_id;
            if (op.layer_start > op.layer_end || op.layer_end > d.layer_count) invalid("bad batch layer range");
            if (!open) {
                c->passes.emplace_back();
                Pass& p = c->passes.back();
                p.order0 = order_pos;
                p.batch0 = op.batch_id;
                c->steps.push_back({STEP_PASS, uint32_t(c->passes.size() - 1), 0.0f, {0, 0, 0, 0}});
                open = true;
            }
            Pass& p = c->passes.back();
            uint32_t n = op.batch_id < batch_draws.size() ? batch_draws[op.batch_id] : 0u;
            p.batches.push_back({op.batch_id, op.layer_start, op.layer_end, 0u});
            p.batch_n++;
            p.draw_n += n;
            order_pos += n;
        } else if (op.kind == TK_OP_BLUR_BEGIN) {
            open = false;
            if (op.layer_end > op.layer_start) invalid("blur groups under clip layers are outside this path");
            if (!(op.sigma >= 0.0f) || !std::isfinite(op.sigma)) invalid("bad blur sigma");
            // BLUR_BEGIN's batch_id word carries the blur's sampling
            const uint32_t factor = op.batch_id & 255u, down = (op.batch_id >> 8) & 255u, up = (op.batch_id >> 16) & 255u;
            if ((op.batch_id >> 24) != 0u || down > 1u || up > 1u || factor > TK_BLUR_MAX_FACTOR)
                invalid("bad blur sampling");
            Step s{STEP_BLUR_BEGIN, 0u, op.sigma, {op.bounds[0], op.bounds[1], op.bounds[2], op.bounds[3]},
                   factor > 1u ? op.batch_id : 0u};
            c->steps.push_back(s);
            ++depth;
        } else if (op.kind == TK_OP_PROGRESSIVE_BEGIN) {
            open = false;
            if (op.layer_end > op.layer_start) invalid("blur groups under clip layers are outside this path");
            if (op.batch_id >= d.progressive_count || !d.progressive_blurs) invalid("progressive blur out of range");
            const tk_progressive_blur& pb = d.progressive_blurs[op.batch_id];
            // projection() and the device-space limit (progressive.rs:71-93)
            if (!std::isfinite(pb.start_x) || !std::isfinite(pb.start_y) || !std::isfinite(pb.dir_x) ||
                !std::isfinite(pb.dir_y) || !(pb.max_std_dev >= 0.0f && pb.max_std_dev <= 65536.0f) ||
                pb.quality > TK_PROGRESSIVE_HIGH)
                invalid("bad progressive blur");
            Step s{STEP_BLUR_BEGIN, 0u, pb.max_std_dev, {op.bounds[0], op.bounds[1], op.bounds[2], op.bounds[3]}, 0u};
            s.progressive = true;
            s.prog = pb;
            c->steps.push_back(s);
            ++depth;
        } else if (op.kind == TK_OP_FILTER_BEGIN) {
            open = false;
            if (op.layer_end > op.layer_start) invalid("filter layers under clip layers are outside this path");
            if (op.batch_id >= d.filter_layer_count || !d.filter_layers) invalid("filter layer out of range");
            const tk_filter_layer& L = d.filter_layers[op.batch_id];
            if (uint64_t(L.first) + L.count > d.filter_count || (L.count && !d.filters))
                invalid("filter layer chain outside the filters");
            // output bounds: the surface clipped to the canvas (filter.rs:510-527)
            const int32_t ob[4] = {std::max(L.surface[0], 0), std::max(L.surface[1], 0),
                                   int32_t(std::min<int64_t>(L.surface[2], d.width)),
                                   int32_t(std::min<int64_t>(L.surface[3], d.height))};
            Step s{STEP_BLUR_BEGIN, 0u, 0.0f, {ob[0], ob[1], ob[2], ob[3]}, 0u};
            s.filter = true;
            bool spatial = false, shadow = false;
            for (uint32_t k = L.first; k < L.first + L.count; ++k) {
                const tk_filter& f = d.filters[k];
                if (f.kind < TK_FILTER_BRIGHTNESS || f.kind > TK_FILTER_BLUR || !std::isfinite(f.amount))
                    invalid("filter " + std::to_string(k) + ": bad kind or amount");
                if (f.kind == TK_FILTER_COMPONENT_TRANSFER) {
                    if (uint64_t(f.color) + TK_TRANSFER_TABLE_WORDS > d.filter_word_count || !d.filter_words)
                        invalid("filter " + std::to_string(k) + ": transfer table outside the filter words");
                    const uint32_t* t = d.filter_words + f.color;
                    for (uint32_t e = 0; e < TK_TRANSFER_TABLE_WORDS; ++e)
                        if (t[e] > 255u) invalid("filter " + std::to_string(k) + ": transfer table entry above 255");
                }
                if (f.kind == TK_FILTER_BLUR) {
                    if (!(f.std_dev >= 0.0f && f.std_dev <= 1.0e4f && f.amount >= 0.0f && f.amount <= 1.0e4f))
                        invalid("filter " + std::to_string(k) + ": blur deviations outside [0, 1e4]");
                    if (f.std_dev > 0.0f || f.amount > 0.0f) spatial = true;
                }
                if (f.kind == TK_FILTER_CONVOLVE) {
                    const uint64_t taps = uint64_t(f.columns) * f.rows;
                    if (taps > TK_CONVOLVE_MAX_TAPS || f.edge_mode > TK_CONVOLVE_EDGE_WRAP || f.preserve_alpha > 1u ||
                        !std::isfinite(f.divisor) || !std::isfinite(f.bias) ||
                        (taps && (f.target_x >= f.columns || f.target_y >= f.rows)) ||
                        (taps && (uint64_t(f.color) + taps > d.filter_word_count || !d.filter_words)))
                        invalid("filter " + std::to_string(k) + ": bad convolution kernel");
                    if (taps) spatial = true;
                }
                if (f.kind == TK_FILTER_DROP_SHADOW) {
                    if (!(f.std_dev >= 0.0f && f.std_dev <= 1.0e4f) || f.dx < -1000000 || f.dx > 1000000 ||
                        f.dy < -1000000 || f.dy > 1000000)
                        invalid("filter " + std::to_string(k) + ": drop shadow offset or deviation out of range");
                    spatial = true;
                    shadow = true;
                }
                if (f.kind == TK_FILTER_COLOR_MATRIX)
                    for (float v : f.matrix)
                        if (!std::isfinite(v)) invalid("filter " + std::to_string(k) + ": non-finite matrix");
                const bool morph = f.kind == TK_FILTER_ERODE || f.kind == TK_FILTER_DILATE;
                if (morph && (f.dx < 0 || f.dy < 0 || f.dx > 1000000 || f.dy > 1000000))
                    invalid("filter " + std::to_string(k) + ": morphology radii outside [0, 1e6]");
                if ((f.kind == TK_FILTER_OFFSET || morph) && (f.dx != 0 || f.dy != 0)) spatial = true;
                s.chain.push_back(f);
            }
            // The reference renders the group into a surface of the layer's
            // surface bounds, which may reach past the canvas; an offset or a
            // morphology reads such pixels, and this path's surfaces are the
            // canvas, so those layers are refused.
            if (spatial && (L.surface[0] < 0 || L.surface[1] < 0 || L.surface[2] > int64_t(d.width) ||
                            L.surface[3] > int64_t(d.height)))
                invalid("an offset, morphology, drop shadow or convolution filter layer whose surface reaches past "
                        "the canvas is outside this path");
            s.shadow = shadow;
            c->steps.push_back(std::move(s));
            ++depth;
        } else if (op.kind == TK_OP_BLUR_END) {
            open = false;
            if (depth == 0) invalid("unbalanced BLUR_END");
            --depth;
            c->steps.push_back({STEP_BLUR_END, 0u, 0.0f, {0, 0, 0, 0}});
        } else {
            invalid("bad op kind");
        }
    }
    if (depth) invalid("unbalanced BLUR_BEGIN");
    if (order_pos != d.draw_order_count) invalid("draw order does not match the batches");
    adopt_pass_buffers(c->passes, old_passes);
    c->width = d.width;
    c->height = d.height;
    c->tw = tw;
    c->th = th;
    c->clear = d.clear_color;
    c->flags = d.flags;
    c->line_count = d.line_count;
    c->path_count = d.path_count;
    c->draw_count = d.draw_count;
    c->layer_count = d.layer_count;
    c->order_count = d.draw_order_count;
    c->brush_words = d.brush_word_count;
    c->sdf_words = d.sdf_word_count + d.sdf_shadow_word_count;
    c->sdf_shadow_base = d.sdf_word_count;
    c->sdf_ext = sdf_ext;
    c->glyph_run_count = d.glyph_run_count;
    c->text = text;
    c->pool_len = pool;
    c->host_segment_capacity = seg_cap;
    c->h_paths.assign(d.paths, d.paths + d.path_count);
    // bbox tile references (binning work measure)
    uint64_t refs = 0;
    for (uint32_t k = 0; k < d.draw_order_count; ++k) {
        const tk_pixel_bounds& pb = d.draws[d.draw_order[k]].pixel_bounds;
        auto tmin = [](int32_t v, uint32_t lim) { return v > 0 ? std::min(uint32_t(v) / TK_TILE_SIZE, lim) : 0u; };
        auto tmax = [](int32_t v, uint32_t lim) {
            return v > 0 ? std::min((uint32_t(v) + TK_TILE_SIZE - 1) / TK_TILE_SIZE, lim) : 0u;
        };
        uint32_t x0 = tmin(pb.x0, tw), x1 = tmax(pb.x1, tw), y0 = tmin(pb.y0, th), y1 = tmax(pb.y1, th);
        if (x1 > x0 && y1 > y0) refs += uint64_t(x1 - x0) * (y1 - y0);
    }
    c->tile_draw_refs = refs;
}

tk::SceneView view(tk_ctx* c) {
    tk::SceneView s{};
    s.lines = c->lines.ptr;
    s.line_count = c->line_count;
    s.paths = c->paths.ptr;
    s.path_count = c->path_count;
    s.draws = c->draws.ptr;
    s.draw_count = c->draw_count;
    s.brush = c->brush.ptr;
    s.brush_words = c->brush_words;
    s.sdf = c->sdf.ptr;
    s.sdf_words = c->sdf_words;
    s.sdf_shadow_base = c->sdf_shadow_base;
    s.sdf_ext = c->sdf_ext;
    s.text = c->text;
    s.texels = c->texels.ptr;
    if (c->glyph_run_count) {
        s.glyph_runs = c->glyph_runs.ptr;
        s.glyphs = c->glyphs.ptr;
        s.glyph_images = c->glyph_images.ptr;
        s.glyph_texels = c->glyph_texels.ptr;
        s.glyph_run_count = c->glyph_run_count;
    }
    s.layers = c->layers.ptr;
    s.batch_ids = c->batch_ids.ptr;
    s.order = c->order.ptr;
    s.width = c->width;
    s.height = c->height;
    s.tw = c->tw;
    s.th = c->th;
    s.backdrops = c->backdrops.ptr;
    s.counts = c->counts.ptr;
    s.ranges = c->ranges.ptr;
    s.cursors = c->cursors.ptr;
    s.pool_len = c->pool_len;
    s.segments = c->segments.ptr;
    s.segment_capacity = c->segments.cap;
    s.error = c->misc.ptr;
    s.seg_line = c->want_seg_line ? c->seg_line.ptr : nullptr;
    s.paints = c->paints.ptr;
    s.emit_order = c->emit_order.ptr;
    s.emit_ticket = c->misc.ptr + 4;
    return s;
}

tk::PassView pass_view(tk_ctx* c, Pass& p) {
    tk::PassView v{};
    v.order0 = p.order0;
    v.draw_n = p.draw_n;
    v.batches = p.d_batches.ptr;
    v.batch0 = p.batch0;
    v.batch_n = p.batch_n;
    v.nbx = (c->tw + 15) / 16;
    v.nby = (c->th + 15) / 16;
    v.bin_lists = p.bin_lists.ptr;
    v.bin_counts = p.bin_counts.ptr;
    v.tiles = p.tiles.ptr;
    v.ptcl = p.ptcl.ptr;
    v.ptcl_capacity = p.ptcl.ptr ? p.ptcl.cap : 0;
    v.tile_desc = c->tile_desc.ptr;
    v.ticket = c->misc.ptr + 1;
    v.ptcl_total = c->misc.ptr + 3;
    v.glyph_list = p.glyph_list.ptr;
    v.glyph_capacity = p.glyph_list.ptr ? p.glyph_list.cap : 0;
    v.glyph_total = c->misc.ptr + 6;
    v.stats = c->stats.ptr;
    if (c->batched) {
        v.scenes = c->d_scenes.ptr;
        v.bin_scene = c->bin_scene.ptr;
        v.tile_scene = c->tile_scene.ptr;
        v.total_bins = c->total_bins;
        v.total_tiles = c->total_tiles;
        v.scene_count = uint32_t(c->h_scenes.size());
    }
    v.tile_active = c->active_mask;
    v.tile_list = c->active_list;
    v.tile_list_n = c->active_n;
    return v;
}

uint32_t read_word(tk_ctx* c, const uint32_t* dptr) {
    uint32_t v = 0;
    TK_CUDA(cudaMemcpyAsync(&v, dptr, 4, cudaMemcpyDeviceToHost, c->stream));
    TK_CUDA(cudaStreamSynchronize(c->stream));
    return v;
}

// Paths by decreasing line count (stable), for scan_emit's path queue.
void upload_emit_order(tk_ctx* c) {
    // Paths longest first, ties in path order: a stable sort by descending
    // line count, done as an LSD radix sort of the inverted counts (16 bits a
    // pass; the high pass only when some count reaches 2^16).
    const uint32_t n = uint32_t(c->h_paths.size());
    std::vector<uint32_t> key(n), order(n), tmp(n);
    uint32_t most = 0;
    for (uint32_t i = 0; i < n; ++i) {
        key[i] = ~c->h_paths[i].line_count;
        most = std::max(most, c->h_paths[i].line_count);
        order[i] = i;
    }
    std::vector<uint32_t> count(65537);
    for (uint32_t shift = 0; shift < (most >> 16 ? 32u : 16u); shift += 16) {
        std::fill(count.begin(), count.end(), 0u);
        for (uint32_t i = 0; i < n; ++i) ++count[((key[order[i]] >> shift) & 0xFFFFu) + 1u];
        for (uint32_t k = 1; k < 65537; ++k) count[k] += count[k - 1];
        for (uint32_t i = 0; i < n; ++i) tmp[count[(key[order[i]] >> shift) & 0xFFFFu]++] = order[i];
        order.swap(tmp);
    }
    upload(c->emit_order, order.data(), order.size(), c->stream);
}

void flatten_on_device(tk_ctx* c, const tk_scene_desc& d, const tk_flatten_desc& fl,
                       const std::function<void()>& side_copies);

// Waits for both streams when an upload leaves, so that no copy still reads
// the caller's host arrays (on a throw as well; the normal path checks the
// main stream's status itself).
struct UploadJoin {
    tk_ctx* c;
    ~UploadJoin() {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamSynchronize(c->stream);
    }
};

// The scene of one band of tile rows: every path's tile bbox clamped to the
// band's rows (tile rows are independent after the scan: a backdrop is the
// row-wise cumsum of its own row's deltas, and the scan's tile walk and
// clipped segments depend on the line and the tile only), backdrop slices
// repacked in path order and segments planned on the device. Paths that miss
// the band keep their lines but get an empty bbox, so the scan skips them.
tk_scene_desc band_scene(tk_ctx* c, const tk_scene_desc& d) {
    tk_scene_desc b = d;
    c->band_paths.resize(d.path_count);
    tk_band_paths(d.paths, d.path_count, c->band_y0, c->band_y1, c->band_paths.data());
    b.paths = c->band_paths.data();
    b.flags |= TK_SCENE_SEGMENTS_FROM_DEVICE;
    return b;
}

// line_dirty (a delta upload): per path, whether its lines are uploaded; the
// other paths' lines are already on the device at the same positions.
void do_upload(tk_ctx* c, const tk_scene_desc& scene, const tk_flatten_desc* fl = nullptr,
               const std::vector<uint8_t>* line_dirty = nullptr) {
    if (c->band) {
        const uint32_t th = (scene.height + TK_TILE_SIZE - 1) / TK_TILE_SIZE;
        if (c->band_y1 > th) invalid("band rows beyond the canvas");
    }
    const tk_scene_desc d = c->band ? band_scene(c, scene) : scene;
    // A failed upload leaves no renderable scene behind.
    c->have_scene = false;
    c->scan_valid = false;
    c->rendered = false;
    c->diff.ready = false;
    c->want_seg_line = false;
    c->batched = false;
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    c->graph_exec = nullptr;
    validate_and_plan(c, d);
    cudaStream_t st = c->stream, cs = c->copy_stream;
    UploadJoin join{c};
    // The records nothing reads before the paint table go up on the copy
    // stream, after the main stream's earlier work (the last frame may still
    // read these buffers); with device flattening they overlap its kernels.
    std::vector<uint4> tab(d.image_count);  // the texture table: per image its first texel and size
    auto side_copies = [&] {
        TK_CUDA(cudaEventRecord(c->ev_main, st));
        TK_CUDA(cudaStreamWaitEvent(cs, c->ev_main, 0));
        upload(c->draws, d.draws, d.draw_count, cs);
        upload(c->brush, d.brush_blob, d.brush_word_count, cs);
        c->sdf.reserve(c->sdf_words);
        if (d.sdf_word_count)
            TK_CUDA(cudaMemcpyAsync(c->sdf.ptr, d.sdf_blob, d.sdf_word_count * 4, cudaMemcpyHostToDevice, cs));
        if (d.sdf_shadow_word_count)
            TK_CUDA(cudaMemcpyAsync(c->sdf.ptr + d.sdf_word_count, d.sdf_shadow_blob, d.sdf_shadow_word_count * 4,
                                    cudaMemcpyHostToDevice, cs));
        uint64_t texel_words = 0;
        for (uint32_t k = 0; k < d.image_count; ++k) {
            tab[k] = make_uint4(uint32_t(texel_words), d.images[k].width, d.images[k].height, 0u);
            texel_words += uint64_t(d.images[k].width) * d.images[k].height;
        }
        c->texels.reserve(texel_words);
        for (uint32_t k = 0; k < d.image_count; ++k)
            TK_CUDA(cudaMemcpyAsync(c->texels.ptr + tab[k].x, d.images[k].premul_rgba8,
                                    uint64_t(tab[k].y) * tab[k].z * 4, cudaMemcpyHostToDevice, cs));
        upload(c->image_tab, tab.data(), tab.size(), cs);
        upload(c->glyph_runs, d.glyph_runs, d.glyph_run_count, cs);
        upload(c->glyphs, d.glyphs, d.glyph_count, cs);
        upload(c->glyph_images, d.glyph_images, d.glyph_image_count, cs);
        upload(c->glyph_texels, d.glyph_texels, d.glyph_texel_count, cs);
        upload(c->filter_words, d.filter_words, d.filter_word_count, cs);
        TK_CUDA(cudaEventRecord(c->ev_copy, cs));
    };
    upload(c->paths, d.paths, d.path_count, st);
    if (fl) {
        flatten_on_device(c, d, *fl, side_copies);  // the host lines, then the device lines
    } else if (line_dirty) {  // the changed paths' line ranges, runs coalesced
        c->lines.reserve(d.line_count);
        for (uint32_t p = 0; p < d.path_count;) {
            if (!(*line_dirty)[p]) { ++p; continue; }
            uint32_t q = p;
            while (q < d.path_count && (*line_dirty)[q]) ++q;
            const uint64_t a = d.paths[p].line_start, b = uint64_t(d.paths[q - 1].line_start) + d.paths[q - 1].line_count;
            if (b > a)
                TK_CUDA(cudaMemcpyAsync(c->lines.ptr + a, d.lines + a, (b - a) * sizeof(tk_line),
                                        cudaMemcpyHostToDevice, st));
            p = q;
        }
    } else {
        upload(c->lines, d.lines, d.line_count, st);
    }
    if (!fl) side_copies();
    TK_CUDA(cudaStreamWaitEvent(st, c->ev_copy, 0));
    c->paints.reserve(d.draw_count);
    tk::launch_paint_table(c->draws.ptr, d.draw_count, c->brush.ptr, d.brush_word_count,
                           uint32_t(c->sdf_shadow_base), c->image_tab.ptr, d.image_count, c->paints.ptr, st);
    upload(c->layers, d.layers, d.layer_count, st);
    upload(c->batch_ids, d.draw_batch_ids, d.draw_count, st);
    upload(c->order, d.draw_order, d.draw_order_count, st);
    upload(c->items, c->h_items.data(), c->h_items.size(), st);
    upload_emit_order(c);
    c->item_desc.reserve(c->h_items.size());
    c->backdrops.reserve(c->pool_len);
    c->counts.reserve(c->pool_len);
    c->cursors.reserve(c->pool_len);
    c->ranges.reserve(c->pool_len);
    c->bumps.reserve(c->path_count);
    c->misc.reserve(8);
    c->stats.reserve(4);
    uint32_t T = c->tw * c->th;
    c->tile_desc.reserve((T + 4095) / 4096 + 1);
    if (uint64_t(c->width) * c->height > c->image.cap) c->history = false;  // reallocated below
    c->image.reserve(uint64_t(c->width) * c->height);
    bool device_plan = (c->flags & TK_SCENE_SEGMENTS_FROM_DEVICE) != 0u;
    c->segment_needed = device_plan ? 0 : c->host_segment_capacity;
    if (!device_plan) c->segments.reserve(c->host_segment_capacity + 1);
    uint32_t nbins = ((c->tw + 15) / 16) * ((c->th + 15) / 16);
    for (Pass& p : c->passes) {
        upload(p.d_batches, p.batches.data(), p.batches.size(), st);
        p.bin_lists.reserve(uint64_t(nbins) * std::max<uint32_t>(p.draw_n, 1));
        p.bin_counts.reserve(nbins);
        p.tiles.reserve(T);
        p.ptcl_needed = 0;
        p.glyph_needed = 0;
    }
    size_t blur_depth = 0, cur = 0;
    for (const Step& s : c->steps) {
        if (s.kind == STEP_BLUR_BEGIN) blur_depth = std::max(blur_depth, ++cur);
        if (s.kind == STEP_BLUR_END) --cur;
    }
    if (c->surfaces.size() < blur_depth) c->surfaces.resize(blur_depth);
    for (size_t i = 0; i < blur_depth; ++i) c->surfaces[i].reserve(uint64_t(c->width) * c->height);
    if (blur_depth) c->temp.reserve(uint64_t(c->width) * c->height);
    bool reduced = false;
    for (const Step& s : c->steps) reduced = reduced || s.sampling != 0u || s.shadow;
    if (reduced) c->low.reserve(uint64_t(c->width) * c->height);
    if (c->band && blur_depth) invalid("band rendering takes scenes without blur layers (their reach crosses bands)");
    TK_CUDA(cudaMemsetAsync(c->misc.ptr, 0, 8 * sizeof(uint32_t), st));
    TK_CUDA(cudaGetLastError());
    TK_CUDA(cudaStreamSynchronize(st));  // every copy of the caller's arrays is done
    c->have_scene = true;
    c->rendered = false;
}

void check_error_word(tk_ctx* c) {
    uint32_t e = read_word(c, c->misc.ptr);
    if (!e) return;
    std::string m = "device error flags " + std::to_string(e) + ":";
    if (e & tk::ERR_LOOKBACK_TIMEOUT) m += " look-back wait gave up;";
    if (e & tk::ERR_LINE_PATH_MISMATCH) m += " a line's path_id does not match its path's line range;";
    if (e & tk::ERR_SEGMENT_OVERFLOW) m += " segment capacity exceeded (segment_capacity below the scanned count);";
    if (e & tk::ERR_PTCL_OVERFLOW) m += " PTCL capacity exceeded;";
    if (e & tk::ERR_STACK_DEPTH) m += " clip/group stack deeper than supported;";
    if (e & tk::ERR_UNSUPPORTED) m += " unsupported particle;";
    TK_CUDA(cudaMemsetAsync(c->misc.ptr, 0, 4, c->stream));
    throw Fail{(e & (tk::ERR_SEGMENT_OVERFLOW | tk::ERR_PTCL_OVERFLOW)) ? TK_E_CAPACITY
               : (e & tk::ERR_LOOKBACK_TIMEOUT)                         ? TK_E_TIMEOUT
                                                                        : TK_E_INVALID,
               m};
}

struct StageMark {
    tk_ctx* c;
    int stage;
    cudaEvent_t a = nullptr;
    StageMark(tk_ctx* ctx, int s) : c(ctx), stage(s) {
        if (!c->timing) return;
        a = next_event(c);
        cudaEventRecord(a, c->stream);
    }
    ~StageMark() {
        if (!a) return;
        cudaEvent_t b = next_event(c);
        cudaEventRecord(b, c->stream);
        c->marks.push_back({stage, {a, b}});
    }
    static cudaEvent_t next_event(tk_ctx* c) {
        if (c->ev_used == c->ev_pool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            c->ev_pool.push_back(e);
        }
        return c->ev_pool[c->ev_used++];
    }
};

void run_pass(tk_ctx* c, Pass& p, uint32_t* target, bool fine = true) {
    cudaStream_t st = c->stream;
    tk::SceneView s = view(c);
    tk::PassView v = pass_view(c, p);
    {
        StageMark m(c, 4);
        tk::launch_bins(s, v, st);
    }
    {
        StageMark m(c, 5);
        tk::launch_coarse(s, v, false, st);
        tk::launch_tile_prefix(s, v, st);
    }
    const bool text = c->glyph_run_count != 0u;
    if (c->active_mask) {  // incremental frame: size for its tiles, keep the full-frame size unknown
        uint32_t total = read_word(c, c->misc.ptr + 3);
        p.ptcl.reserve(uint64_t(total) + 1);
        p.ptcl_used = total;
        if (text) {
            const uint32_t glyphs = read_word(c, c->misc.ptr + 6);
            p.glyph_list.reserve(uint64_t(glyphs) + 1);
            p.glyph_used = glyphs;
        }
        v = pass_view(c, p);
    } else {
        if (p.ptcl_needed == 0) {  // first frame of this scene: size the PTCL buffer (and the glyph lists)
            uint32_t total = read_word(c, c->misc.ptr + 3);
            p.ptcl_needed = uint64_t(total) + 1;
            p.ptcl.reserve(p.ptcl_needed);
            if (text) {
                p.glyph_needed = uint64_t(read_word(c, c->misc.ptr + 6)) + 1;
                p.glyph_list.reserve(p.glyph_needed);
            }
            v = pass_view(c, p);
        }
        p.ptcl_used = p.ptcl_needed - 1;
        p.glyph_used = text ? p.glyph_needed - 1 : 0;
    }
    {
        StageMark m(c, 6);
        tk::launch_coarse(s, v, true, st);
    }
    if (!fine) return;
    {
        StageMark m(c, 7);
        tk::launch_fine(s, v, target, st);
    }
}

void scan_phase(tk_ctx* c);

// The scan of the paths a delta upload replaced (scene_scan.rs:116-192's
// selected paths): their slices cleared and counted, their pool scan items,
// their segments emitted; every other path's scan output stays as it is.
void scan_phase_partial(tk_ctx* c) {
    cudaStream_t st = c->stream;
    tk::SceneView s = view(c);
    c->ev_used = 0;
    c->marks.clear();
    c->scan_valid = false;
    const uint32_t n = uint32_t(c->rescan.size());
    upload(c->rescan_list, c->rescan.data(), n, st);
    std::vector<uint8_t> sel(c->path_count, 0u);
    for (uint32_t p : c->rescan) sel[p] = 1u;
    std::vector<tk::ScanItem> items;
    for (const tk::ScanItem& it : c->h_items)
        if (sel[it.path]) items.push_back(it);
    upload(c->rescan_items, items.data(), items.size(), st);
    c->rescan_desc.reserve(std::max<size_t>(items.size(), 1));
    {
        StageMark m(c, 0);
        TK_CUDA(cudaMemsetAsync(c->stats.ptr, 0, 4 * sizeof(unsigned long long), st));
    }
    {
        StageMark m(c, 1);
        tk::launch_scan_count_paths(s, c->rescan_list.ptr, n, st);
    }
    {
        StageMark m(c, 2);
        tk::launch_pool_scan(s, c->rescan_items.ptr, uint32_t(items.size()), c->rescan_desc.ptr, false, 0u,
                             c->misc.ptr + 2, st);
        tk::launch_path_totals(s, c->bumps.ptr, false, c->misc.ptr + 2, st);
    }
    if (c->rescan_check) {
        // device plans: a replaced path whose segment total changed moves
        // every later path's slice, so the scene is scanned whole
        tk::launch_check_path_totals(s, c->bumps.ptr, c->rescan_list.ptr, n, c->misc.ptr + 5, st);
        c->rescan_check = false;
        if (read_word(c, c->misc.ptr + 5)) {
            c->rescan.clear();
            c->segment_needed = 0;
            scan_phase(c);
            return;
        }
    }
    const bool device_plan = (c->flags & TK_SCENE_SEGMENTS_FROM_DEVICE) != 0u;
    s.segment_capacity = device_plan ? c->segment_needed - 1 : c->host_segment_capacity;
    {
        StageMark m(c, 3);
        tk::launch_scan_emit_paths(s, c->rescan_list.ptr, n, st);
    }
    c->last_scan_paths = n;
    c->rescan.clear();
    c->scan_valid = true;
}

// Pool clear, scan_count, pool scan, path totals and scan_emit; only the
// paths a delta upload replaced when the rest of the scan is in place.
void scan_phase(tk_ctx* c) {
    if (!c->have_scene) throw Fail{TK_E_STATE, "no scene uploaded"};
    if (c->scan_valid && !c->rescan.empty()) {
        scan_phase_partial(c);
        return;
    }
    c->rescan.clear();
    c->rescan_check = false;
    c->last_scan_paths = c->path_count;
    c->scan_valid = false;
    cudaStream_t st = c->stream;
    bool device_plan = (c->flags & TK_SCENE_SEGMENTS_FROM_DEVICE) != 0u;
    tk::SceneView s = view(c);
    c->ev_used = 0;
    c->marks.clear();
    {
        StageMark m(c, 0);
        if (c->pool_len) {
            TK_CUDA(cudaMemsetAsync(c->backdrops.ptr, 0, c->pool_len * 4, st));
            TK_CUDA(cudaMemsetAsync(c->counts.ptr, 0, c->pool_len * 4, st));
        }
        TK_CUDA(cudaMemsetAsync(c->stats.ptr, 0, 4 * sizeof(unsigned long long), st));
    }
    {
        StageMark m(c, 1);
        tk::launch_scan_count(s, st);
    }
    const uint32_t device_base = 0u;  // Canvas segment slices start at 0 (canvas/paths.rs:117)
    {
        StageMark m(c, 2);
        tk::launch_pool_scan(s, c->items.ptr, uint32_t(c->h_items.size()), c->item_desc.ptr, device_plan, device_base,
                             c->misc.ptr + 2, st);
        tk::launch_path_totals(s, c->bumps.ptr, device_plan, c->misc.ptr + 2, st);
    }
    if (device_plan && c->segment_needed == 0) {
        uint32_t total = read_word(c, c->misc.ptr + 2);
        c->segment_needed = uint64_t(total) + 1;
        c->segments.reserve(c->segment_needed);
        s = view(c);
    }
    if (c->want_seg_line) {  // the line of every segment (differentiable mode)
        c->seg_line.reserve(device_plan ? c->segment_needed : std::max<uint64_t>(c->host_segment_capacity, 1));
        s = view(c);
    }
    s.segment_capacity = device_plan ? c->segment_needed - 1 : c->host_segment_capacity;
    {
        StageMark m(c, 3);
        tk::launch_scan_emit(s, st);
    }
    c->scan_valid = true;
}

void do_render(tk_ctx* c) {
    c->history = false;
    scan_phase(c);
    cudaStream_t st = c->stream;
    tk::launch_fill(c->image.ptr, uint64_t(c->width) * c->height, c->clear, st);
    std::vector<uint32_t*> targets{c->image.ptr};
    std::vector<const Step*> open;
    for (const Step& step : c->steps) {
        if (step.kind == STEP_PASS) {
            run_pass(c, c->passes[step.pass], targets.back());
        } else if (step.kind == STEP_BLUR_BEGIN) {
            uint32_t* surf = c->surfaces[targets.size() - 1].ptr;
            tk::launch_fill(surf, uint64_t(c->width) * c->height, 0u, st);
            targets.push_back(surf);
            open.push_back(&step);
        } else {
            const Step& b = *open.back();
            open.pop_back();
            uint32_t* surf = targets.back();
            targets.pop_back();
            // Output bounds and the surface region they read from
            // (shared/layer/filter.rs:510-531,599-601).
            int32_t W = int32_t(c->width), H = int32_t(c->height);
            int32_t ob[4] = {std::max(b.bounds[0], 0), std::max(b.bounds[1], 0), std::min(b.bounds[2], W),
                             std::min(b.bounds[3], H)};
            int32_t rad = int32_t(std::ceil(std::fmax(b.sigma, 0.0f) * 3.0f));
            int32_t sx0 = std::max(b.bounds[0] - rad, 0), sy0 = std::max(b.bounds[1] - rad, 0);
            int32_t sx1 = std::min(b.bounds[2] + rad, W), sy1 = std::min(b.bounds[3] + rad, H);
            StageMark m(c, 8);
            if (b.filter) {
                // the chain over the layer's bounds (render/filter_program/effects.rs:3-268)
                if (ob[2] > ob[0] && ob[3] > ob[1])
                    tk::launch_filter_chain(surf, c->temp.ptr, b.shadow ? c->low.ptr : nullptr, c->filter_words.ptr,
                                            c->width, c->height, ob, b.chain.data(), uint32_t(b.chain.size()), st);
            } else if (b.progressive) {
                // Filter::ProgressiveBlur over the output bounds
                // (native/runtime/program/filter/progressive/mod.rs:44-146)
                if (ob[2] > ob[0] && ob[3] > ob[1] && b.prog.max_std_dev > 0.0f) {
                    const int32_t rc = tk::launch_progressive_blur(surf, c->width, c->height, ob, b.prog,
                                                                   c->prog_scratch, st);
                    if (rc == -1) throw Fail{TK_E_CAPACITY, "progressive blur level count overflow"};
                    if (rc == -2) throw Fail{TK_E_ALLOC, "progressive blur levels: out of device memory"};
                }
            } else if (b.sampling != 0u && ob[2] > ob[0] && ob[3] > ob[1] && b.sigma > 0.0f) {
                // BlurSampling with factor > 1 (render/filter_program/blur.rs:194-212):
                // reduce, blur at sigma / factor, restore, over the output bounds
                tk::launch_blur_downsampled(surf, c->low.ptr, c->temp.ptr, c->width, c->height, ob, b.sigma,
                                            b.sampling, st);
            } else if (ob[2] > ob[0] && ob[3] > ob[1] && b.sigma > 0.0f) {
                tk::BlurParams bp{};
                bp.width = c->width;
                bp.height = c->height;
                bp.region[0] = uint32_t(sx0);
                bp.region[1] = uint32_t(sy0);
                bp.region[2] = uint32_t(sx1 - sx0);
                bp.region[3] = uint32_t(sy1 - sy0);
                bp.bounds[0] = sx0;
                bp.bounds[1] = sy0;
                bp.bounds[2] = sx1;
                bp.bounds[3] = sy1;
                bp.sigma = b.sigma;
                bp.axis = 0;
                tk::launch_blur(surf, c->temp.ptr, bp, st);
                bp.axis = 1;
                tk::launch_blur(c->temp.ptr, surf, bp, st);
            }
            if (ob[2] > ob[0] && ob[3] > ob[1]) tk::launch_composite(targets.back(), surf, c->width, ob, st);
        }
    }
    TK_CUDA(cudaGetLastError());
    c->rendered = true;
    c->history = true;
    c->history_w = c->width;
    c->history_h = c->height;
    c->history_clear = c->clear;
}

// The incremental frame: a full scan, then coarse and fine of the active
// tiles only, over the previous frame (scenes without blur layers: one pass
// per batch group straight into the image).
void do_render_tiles(tk_ctx* c, bool reuse_scan = false) {
    c->history = false;
    if (reuse_scan && c->scan_valid && c->rescan.empty()) {  // the uploaded scene's scan is still in place
        c->ev_used = 0;
        c->marks.clear();
    } else {
        scan_phase(c);
    }
    cudaStream_t st = c->stream;
    const uint32_t T = c->tw * c->th;
    upload(c->tile_active, c->h_active.data(), T, st);
    upload(c->tile_list, c->h_active_list.data(), c->h_active_list.size(), st);
    tk::launch_fill_tiles(c->image.ptr, c->width, c->height, c->tw, c->tile_list.ptr,
                          uint32_t(c->h_active_list.size()), c->clear, st);
    c->active_mask = c->tile_active.ptr;
    c->active_list = c->tile_list.ptr;
    c->active_n = uint32_t(c->h_active_list.size());
    struct Reset {
        tk_ctx* c;
        ~Reset() {
            c->active_mask = nullptr;
            c->active_list = nullptr;
            c->active_n = 0;
        }
    } reset{c};
    for (const Step& step : c->steps) run_pass(c, c->passes[step.pass], c->image.ptr);
    TK_CUDA(cudaGetLastError());
    c->rendered = true;
    c->history = true;
    c->history_w = c->width;
    c->history_h = c->height;
    c->history_clear = c->clear;
}

// The band's frame: the scan of the band scene, then coarse and fine of the
// band's tiles only (the other rows of the image are left as they are).
void do_render_band(tk_ctx* c) {
    const uint32_t T = c->tw * c->th;
    c->h_active.assign(T, 0u);
    c->h_active_list.clear();
    for (uint32_t ty = c->band_y0; ty < c->band_y1; ++ty) {
        std::memset(c->h_active.data() + size_t(ty) * c->tw, 1, c->tw);
        for (uint32_t tx = 0; tx < c->tw; ++tx) c->h_active_list.push_back(ty * c->tw + tx);
    }
    do_render_tiles(c);
    c->history = false;
}

void drop_graph(tk_ctx* c) {
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    c->graph_exec = nullptr;
}

// Pool-scan work items from the current paths and work item size.
void rebuild_items(tk_ctx* c) {
    c->h_items.clear();
    for (uint32_t p = 0; p < uint32_t(c->h_paths.size()); ++p) {
        const tk_path_record& r = c->h_paths[p];
        const uint32_t stride = r.tile_x1 > r.tile_x0 ? r.tile_x1 - r.tile_x0 : 0u;
        const uint32_t height = r.tile_y1 > r.tile_y0 ? r.tile_y1 - r.tile_y0 : 0u;
        if (!r.data_len) continue;
        const uint32_t rows_per = std::max<uint32_t>(1u, c->scan_item_elems / stride);
        for (uint32_t row = 0; row < height; row += rows_per)
            c->h_items.push_back({p, row, std::min(rows_per, height - row), row == 0u ? 1u : 0u});
    }
    upload(c->items, c->h_items.data(), c->h_items.size(), c->stream);
    c->item_desc.reserve(c->h_items.size());
}

// Lines of the element paths flattened on the device after the host lines;
// their path records get their line ranges on the device.
// side_copies runs once the element counts are back: the scene records then
// go up on the copy stream while the stroking and emit kernels run.
void flatten_on_device(tk_ctx* c, const tk_scene_desc& d, const tk_flatten_desc& fl,
                       const std::function<void()>& side_copies) {
    if (!(d.flags & TK_SCENE_SEGMENTS_FROM_DEVICE)) invalid("device flattening needs device segment planning");
    if ((fl.element_count && !fl.elements) || (d.path_count && !fl.path_elements)) invalid("null flatten arrays");
    // Element ranges are checked here; the elements themselves (verb,
    // tolerance >= 1e-3 px, coordinates within 1e6 px, owning path) on the
    // device, which skips and reports any that fail.
    std::vector<uint8_t> taken(d.path_count, 0);  // paths whose lines come from the device
    for (uint32_t p = 0; p < d.path_count; ++p) {
        const uint64_t e0 = fl.path_elements[2 * p], ne = fl.path_elements[2 * p + 1];
        if (!ne) continue;
        if (e0 + ne > fl.element_count) invalid("path " + std::to_string(p) + ": elements out of range");
        if (d.paths[p].line_count) invalid("path " + std::to_string(p) + ": both lines and elements");
        taken[p] = 1;
    }
    // Strokes and their polylines are checked here (ranges, ownership, sizes);
    // their elements on the device like the fills'.
    const uint32_t ns = fl.stroke_count, npl = fl.polyline_count;
    const uint64_t nse = fl.stroke_element_count;
    if ((ns && !fl.strokes) || (npl && !fl.polylines) || (nse && !fl.stroke_elements)) invalid("null stroke arrays");
    for (uint32_t s = 0; s < ns; ++s) {
        const tk_stroke_desc& S = fl.strokes[s];
        const auto at = [s] { return "stroke " + std::to_string(s) + ": "; };  // built only for a message
        if (S.path >= d.path_count) invalid(at() + "path out of range");
        if (taken[S.path] || d.paths[S.path].line_count) invalid(at() + "its path already has lines or elements");
        taken[S.path] = 1;
        if (!(S.half_width > 0.0 && S.half_width <= 1e6)) invalid(at() + "half width outside (0, 1e6]");
        if (!(S.tolerance >= 1e-3 && S.tolerance <= 1e6)) invalid(at() + "tolerance outside [1e-3, 1e6]");
        for (double t : S.transform)
            if (!(std::fabs(t) <= 1e6)) invalid(at() + "transform entries must be finite, within 1e6");
        if (uint64_t(S.polyline0) + S.polyline_count > npl) invalid(at() + "polylines out of range");
        for (uint32_t k = S.polyline0; k < S.polyline0 + S.polyline_count; ++k)
            if (fl.polylines[k].stroke != s) invalid(at() + "polyline " + std::to_string(k) + " belongs elsewhere");
    }
    for (uint32_t k = 0; k < npl; ++k) {
        const tk_stroke_polyline& P = fl.polylines[k];
        if (P.stroke >= ns) invalid("polyline " + std::to_string(k) + ": stroke out of range");
        if (!P.element_count || uint64_t(P.element0) + P.element_count > nse)
            invalid("polyline " + std::to_string(k) + ": elements out of range");
    }
    if (nse > 0xFFFFFFFFull) invalid("stroke element count exceeds u32 indexing");
    cudaStream_t st = c->stream;
    const uint64_t n = fl.element_count;
    FlattenScratch& F = c->flat;
    auto &els = F.els, &sels = F.sels;
    auto &path_els = F.path_els, &offsets = F.offsets, &sums = F.sums, &words = F.words, &soff = F.soff,
         &ssums = F.ssums, &poly_n = F.poly_n, &line_off = F.line_off;
    auto& polys = F.polys;
    auto& strokes = F.strokes;
    auto& wide = F.wide;
    auto& pts = F.pts;
    upload(els, fl.elements, n, st);
    upload(path_els, fl.path_elements, 2ull * d.path_count, st);
    upload(sels, fl.stroke_elements, nse, st);
    upload(polys, fl.polylines, npl, st);
    upload(strokes, fl.strokes, ns, st);
    offsets.reserve(n);
    sums.reserve(tk::flatten_block_sums(n));
    soff.reserve(nse);
    ssums.reserve(tk::flatten_block_sums(std::max<uint64_t>(nse, npl)));
    poly_n.reserve(npl);
    line_off.reserve(npl);
    // words: [0] fill lines [1] error [2] stroke points [3] stroke lines
    words.reserve(4);
    wide.reserve(2);  // exact sums: [0] stroke points [1] stroke lines
    TK_CUDA(cudaMemsetAsync(words.ptr, 0, 4 * sizeof(uint32_t), st));
    TK_CUDA(cudaMemsetAsync(wide.ptr, 0, 2 * sizeof(unsigned long long), st));
    tk::launch_flatten_count(els.ptr, n, offsets.ptr, sums.ptr, words.ptr, words.ptr + 1, st);
    tk::launch_stroke_count(sels.ptr, nse, soff.ptr, ssums.ptr, words.ptr + 2, wide.ptr, words.ptr + 1, st);
    uint32_t w[4] = {0, 0, 0, 0};
    unsigned long long wsum[2] = {0, 0};
    TK_CUDA(cudaMemcpyAsync(w, words.ptr, sizeof(w), cudaMemcpyDeviceToHost, st));
    TK_CUDA(cudaMemcpyAsync(wsum, wide.ptr, sizeof(wsum), cudaMemcpyDeviceToHost, st));
    TK_CUDA(cudaStreamSynchronize(st));
    side_copies();
    if (wsum[0] > 0xFFFFFFFFull) invalid("stroke centerline points exceed u32 indexing");
    tk::StrokeView sv{sels.ptr, nse,        soff.ptr, words.ptr + 2, nullptr,     0,
                      polys.ptr, npl,       strokes.ptr, ns,         poly_n.ptr, line_off.ptr, words.ptr + 1,
                      nullptr};
    if (npl) {
        pts.reserve(std::max<uint64_t>(w[2], 1));
        sv.pts = pts.ptr;
        sv.pt_cap = w[2];
        F.unit_lines.reserve(std::max<uint64_t>(2ull * w[2], 1));  // two unit slots per raw point
        sv.unit_lines = F.unit_lines.ptr;
        tk::launch_stroke_outline_count(sv, ssums.ptr, words.ptr + 3, wide.ptr + 1, st);
        TK_CUDA(cudaMemcpyAsync(w, words.ptr, sizeof(w), cudaMemcpyDeviceToHost, st));
        TK_CUDA(cudaMemcpyAsync(wsum, wide.ptr, sizeof(wsum), cudaMemcpyDeviceToHost, st));
        TK_CUDA(cudaStreamSynchronize(st));
    }
    const uint64_t host_lines = d.line_count, fill_lines = w[0], stroke_lines = wsum[1];
    const uint64_t total = host_lines + fill_lines + stroke_lines;
    if (total > 0xFFFFFFFFull) invalid("line count exceeds u32 indexing");
    c->lines.reserve(total);
    if (host_lines) TK_CUDA(cudaMemcpyAsync(c->lines.ptr, d.lines, host_lines * sizeof(tk_line), cudaMemcpyHostToDevice, st));
    tk::launch_flatten_emit(els.ptr, n, offsets.ptr, words.ptr, c->paths.ptr, d.path_count, path_els.ptr, c->lines.ptr,
                            host_lines, host_lines + fill_lines, words.ptr + 1, st);
    tk::launch_stroke_emit(sv, words.ptr + 3, c->paths.ptr, c->lines.ptr, host_lines + fill_lines, total, st);
    TK_CUDA(cudaGetLastError());
    uint32_t err = 0;
    TK_CUDA(cudaMemcpyAsync(&err, words.ptr + 1, 4, cudaMemcpyDeviceToHost, st));
    TK_CUDA(cudaMemcpyAsync(c->h_paths.data(), c->paths.ptr, d.path_count * sizeof(tk_path_record),
                            cudaMemcpyDeviceToHost, st));
    TK_CUDA(cudaStreamSynchronize(st));
    if (err) {
        std::string m = "device flattening rejected the elements:";
        if (err & tk::ERR_UNSUPPORTED) m += " bad verb, tolerance below 1e-3 px or coordinates beyond 1e6 px;";
        if (err & tk::ERR_LINE_PATH_MISMATCH)
            m += " an element's path or polyline index differs from its owner, or a polyline does not start with a move;";
        if (err & tk::ERR_SEGMENT_OVERFLOW) m += " lines past the counted total;";
        throw Fail{TK_E_INVALID, m};
    }
    c->line_count = total;
}

// Merges one-pass scenes into one batched pass: arrays concatenated with their
// indices offset, one BatchScene per canvas.
void do_batch_upload(tk_ctx* c, const tk_scene_desc* scenes, uint32_t n) {
    c->history = false;  // the image becomes the batch's canvases
    c->scan_valid = false;
    c->have_scene = false;
    c->rendered = false;
    c->diff.ready = false;
    c->want_seg_line = false;
    c->batched = false;
    drop_graph(c);
    if (n == 0 || !scenes) invalid("empty batch");
    // Lines, the bulk of a batch, go straight from each scene's array into the
    // device buffer; their path ids are rebased on the device.
    std::vector<uint64_t> line_base;
    std::vector<uint32_t> line_path_base;
    uint64_t total_lines = 0;
    std::vector<tk_path_record> paths;
    std::vector<tk_draw_record> draws;
    std::vector<uint32_t> brush, sdf, shadow, order, batch_ids, bin_scene, tile_scene;
    std::vector<tk_layer_record> layers;
    std::vector<tk::PassBatch> batches;
    std::vector<tk::BatchScene> table;
    std::vector<tk_batch_info> info;
    uint64_t pool = 0, segs = 0, list = 0, pixels = 0;
    uint32_t tiles = 0, bins = 0, batch_base = 0;
    bool ext = false;  // some scene has SDF records of an extended kind
    bool text = false;  // some scene has glyph outline fills
    for (uint32_t s = 0; s < n; ++s) {
        const tk_scene_desc& d = scenes[s];
        if (d.flags & TK_SCENE_SEGMENTS_FROM_DEVICE) invalid("batched scenes use host segment planning");
        if (d.image_count) invalid("scene " + std::to_string(s) + ": image patterns are not batched");
        if (d.glyph_run_count) invalid("scene " + std::to_string(s) + ": glyph runs are not batched");
        validate_and_plan(c, d);
        ext = ext || c->sdf_ext;
        text = text || c->text;
        uint32_t npass = 0;
        for (const Step& st : c->steps) {
            if (st.kind != STEP_PASS) invalid("scene " + std::to_string(s) + ": blur groups are not batched");
            ++npass;
        }
        if (npass > 1) invalid("scene " + std::to_string(s) + ": batched scenes have one target pass");
        tk_batch_info bi{};
        bi.width = d.width;
        bi.height = d.height;
        bi.tile_base = tiles;
        bi.tile_count = c->tw * c->th;
        bi.path_base = uint32_t(paths.size());
        bi.draw_base = uint32_t(draws.size());
        bi.batch_base = batch_base;
        bi.line_base = uint32_t(total_lines);
        bi.layer_base = uint32_t(layers.size());
        bi.segment_base = segs;
        bi.pool_base = pool;
        bi.image_offset = pixels;
        line_base.push_back(total_lines);
        line_path_base.push_back(bi.path_base);
        total_lines += d.line_count;
        for (uint32_t i = 0; i < d.path_count; ++i) {
            tk_path_record p = d.paths[i];
            p.path_id += bi.path_base;
            p.line_start += bi.line_base;
            p.data_offset += uint32_t(bi.pool_base);
            p.segment_start += uint32_t(bi.segment_base);
            paths.push_back(p);
        }
        const uint32_t brush_base = uint32_t(brush.size());
        const uint32_t sdf_base = uint32_t(sdf.size()), shadow_base = uint32_t(shadow.size());
        for (uint32_t i = 0; i < d.draw_count; ++i) {
            tk_draw_record r = d.draws[i];
            if (r.path_id != TK_INVALID_INDEX) r.path_id += bi.path_base;
            if (r.brush_offset != TK_INVALID_INDEX) r.brush_offset += brush_base;
            if (r.sdf_offset != TK_INVALID_INDEX) r.sdf_offset += sdf_base;
            if (r.sdf_shadow_offset != TK_INVALID_INDEX) r.sdf_shadow_offset += shadow_base;
            draws.push_back(r);
            batch_ids.push_back(d.draw_batch_ids[i] == TK_INVALID_INDEX ? TK_INVALID_INDEX
                                                                        : d.draw_batch_ids[i] + batch_base);
        }
        brush.insert(brush.end(), d.brush_blob, d.brush_blob + d.brush_word_count);
        sdf.insert(sdf.end(), d.sdf_blob, d.sdf_blob + d.sdf_word_count);
        shadow.insert(shadow.end(), d.sdf_shadow_blob, d.sdf_shadow_blob + d.sdf_shadow_word_count);
        if (sdf.size() + shadow.size() > 0xFFFFFFFFull) invalid("batch SDF blobs exceed u32 indexing");
        for (uint32_t i = 0; i < d.layer_count; ++i) {
            tk_layer_record L = d.layers[i];
            L.draw += bi.draw_base;
            layers.push_back(L);
        }
        const uint32_t order0 = uint32_t(order.size());
        for (uint32_t i = 0; i < d.draw_order_count; ++i) order.push_back(d.draw_order[i] + bi.draw_base);
        uint32_t nb = 0;
        if (npass)
            for (const tk::PassBatch& b : c->passes[0].batches) {
                batches.push_back({b.batch_id + batch_base, b.layer_start + bi.layer_base, b.layer_end + bi.layer_base,
                                   0u});
                nb = std::max(nb, b.batch_id + 1u);
            }
        for (uint32_t i = 0; i < d.op_count; ++i)
            if (d.ops[i].kind == TK_OP_DRAW_BATCH) nb = std::max(nb, d.ops[i].batch_id + 1u);
        tk::BatchScene sc{};
        sc.tile_base = tiles;
        sc.bin_base = bins;
        sc.list_base = list;
        sc.tw = c->tw;
        sc.th = c->th;
        sc.nbx = (c->tw + 15) / 16;
        sc.order0 = order0;
        sc.draw_n = npass ? c->passes[0].draw_n : 0u;
        sc.width = d.width;
        sc.height = d.height;
        sc.clear = d.clear_color;
        sc.image_offset = pixels;
        const uint32_t nbins = sc.nbx * ((c->th + 15) / 16);
        for (uint32_t b = 0; b < nbins; ++b) bin_scene.push_back(s);
        for (uint32_t t = 0; t < sc.tw * sc.th; ++t) tile_scene.push_back(s);
        table.push_back(sc);
        info.push_back(bi);
        tiles += sc.tw * sc.th;
        bins += nbins;
        list += uint64_t(nbins) * sc.draw_n;
        pixels += uint64_t(d.width) * d.height;
        pool += c->pool_len;
        segs += c->host_segment_capacity;
        batch_base += nb;
        if (pool > 0xFFFFFFFFull || segs > 0xFFFFFFFFull || total_lines > 0xFFFFFFFFull)
            invalid("batch exceeds u32 indexing");
    }
    // merged scene state
    cudaStream_t st = c->stream;
    c->lines.reserve(total_lines);
    for (uint32_t s = 0; s < n; ++s)
        if (scenes[s].line_count)
            TK_CUDA(cudaMemcpyAsync(c->lines.ptr + line_base[s], scenes[s].lines, scenes[s].line_count * sizeof(tk_line),
                                    cudaMemcpyHostToDevice, st));
    DBuf<uint64_t> d_line_base;
    DBuf<uint32_t> d_path_base;
    upload(d_line_base, line_base.data(), line_base.size(), st);
    upload(d_path_base, line_path_base.data(), line_path_base.size(), st);
    tk::launch_rebase_lines(c->lines.ptr, total_lines, d_line_base.ptr, d_path_base.ptr, n, st);
    TK_CUDA(cudaStreamSynchronize(st));
    d_line_base.release();
    d_path_base.release();
    c->flags = 0;
    c->line_count = total_lines;
    c->path_count = uint32_t(paths.size());
    c->draw_count = uint32_t(draws.size());
    c->layer_count = uint32_t(layers.size());
    c->order_count = uint32_t(order.size());
    c->brush_words = brush.size();
    c->sdf_shadow_base = sdf.size();
    c->sdf_ext = ext;
    c->text = text;
    sdf.insert(sdf.end(), shadow.begin(), shadow.end());
    c->sdf_words = sdf.size();
    c->pool_len = pool;
    c->host_segment_capacity = segs;
    c->h_paths = paths;
    c->width = c->height = 0;
    c->tw = tiles;
    c->th = 1;
    c->steps.assign(1, Step{STEP_PASS, 0u, 0.0f, {0, 0, 0, 0}});
    std::vector<Pass> old_passes;
    old_passes.swap(c->passes);
    c->passes.emplace_back();
    adopt_pass_buffers(c->passes, old_passes);
    Pass& p = c->passes.back();
    p.order0 = 0;
    p.draw_n = uint32_t(order.size());
    p.batch0 = 0;
    p.batch_n = uint32_t(batches.size());
    p.batches = batches;
    upload(c->paths, paths.data(), paths.size(), st);
    upload(c->draws, draws.data(), draws.size(), st);
    upload(c->brush, brush.data(), brush.size(), st);
    upload(c->sdf, sdf.data(), sdf.size(), st);
    c->paints.reserve(draws.size());
    tk::launch_paint_table(c->draws.ptr, uint32_t(draws.size()), c->brush.ptr, brush.size(),
                           uint32_t(c->sdf_shadow_base), nullptr, 0u, c->paints.ptr, st);
    upload(c->layers, layers.data(), layers.size(), st);
    upload(c->batch_ids, batch_ids.data(), batch_ids.size(), st);
    upload(c->order, order.data(), order.size(), st);
    rebuild_items(c);
    upload_emit_order(c);
    c->backdrops.reserve(pool);
    c->counts.reserve(pool);
    c->cursors.reserve(pool);
    c->ranges.reserve(pool);
    c->bumps.reserve(c->path_count);
    c->misc.reserve(8);
    c->stats.reserve(4);
    c->tile_desc.reserve((tiles + 4095) / 4096 + 1);
    c->image.reserve(pixels);
    c->segment_needed = segs;
    c->segments.reserve(segs + 1);
    upload(p.d_batches, p.batches.data(), p.batches.size(), st);
    p.bin_lists.reserve(std::max<uint64_t>(list, 1));
    p.bin_counts.reserve(bins);
    p.tiles.reserve(tiles);
    p.ptcl_needed = 0;
    upload(c->d_scenes, table.data(), table.size(), st);
    upload(c->bin_scene, bin_scene.data(), bin_scene.size(), st);
    upload(c->tile_scene, tile_scene.data(), tile_scene.size(), st);
    c->h_scenes = table;
    c->h_batch_info = info;
    c->total_bins = bins;
    c->total_tiles = tiles;
    c->total_pixels = pixels;
    TK_CUDA(cudaMemsetAsync(c->misc.ptr, 0, 8 * sizeof(uint32_t), st));
    TK_CUDA(cudaGetLastError());
    c->batched = true;
    c->have_scene = true;
}

// The batched frame: scan, clear every canvas, bins, coarse, fine.
void batch_frame(tk_ctx* c) {
    scan_phase(c);
    tk::launch_fill_scenes(c->image.ptr, c->d_scenes.ptr, uint32_t(c->h_scenes.size()), c->stream);
    run_pass(c, c->passes[0], c->image.ptr);
}

void do_batch_render(tk_ctx* c) {
    if (!c->have_scene || !c->batched) throw Fail{TK_E_STATE, "no batch uploaded"};
    cudaStream_t st = c->stream;
    if (!c->graph_exec) {
        // First frame sizes the PTCL (a host read-back) and is this render's
        // frame; the same launch sequence is then captured once (capture
        // runs nothing) and replayed by the renders after it.
        bool rendered_now = false;
        if (c->passes[0].ptcl_needed == 0) {
            batch_frame(c);
            check_error_word(c);
            rendered_now = true;
        }
        const bool timing = c->timing;
        c->timing = false;
        cudaGraph_t g = nullptr;
        TK_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
            batch_frame(c);
        } catch (...) {
            cudaStreamEndCapture(st, &g);
            if (g) cudaGraphDestroy(g);
            c->timing = timing;
            throw;
        }
        c->timing = timing;
        TK_CUDA(cudaStreamEndCapture(st, &g));
        cudaError_t e = cudaGraphInstantiate(&c->graph_exec, g, 0);
        cudaGraphDestroy(g);
        TK_CUDA(e);
        if (rendered_now) {
            c->rendered = true;
            return;
        }
    }
    TK_CUDA(cudaGraphLaunch(c->graph_exec, st));
    c->rendered = true;
}

}  // namespace

extern "C" {

const char* tk_version(void) { return "tileink_b200 0.1 (sm_100a)"; }

int32_t tk_ctx_create(int32_t device, tk_ctx** out) {
    if (!out) return TK_E_INVALID;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return TK_E_CUDA;
    }
    auto* c = new tk_ctx();
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_main, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_copy, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (c->ev_copy) cudaEventDestroy(c->ev_copy);
        if (c->ev_main) cudaEventDestroy(c->ev_main);
        if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
        return TK_E_CUDA;
    }
    *out = c;
    return TK_OK;
}

void tk_ctx_destroy(tk_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    c->lines.release(); c->paths.release(); c->draws.release(); c->brush.release(); c->sdf.release();
    c->batch_ids.release(); c->order.release(); c->layers.release(); c->items.release();
    c->item_desc.release(); c->tile_desc.release(); c->stats.release(); c->backdrops.release();
    c->counts.release(); c->cursors.release(); c->bumps.release(); c->misc.release();
    c->ranges.release(); c->segments.release(); c->image.release(); c->temp.release();
    tk::release_progressive(c->prog_scratch);
    for (auto& s : c->surfaces) s.release();
    for (auto& p : c->passes) {
        p.d_batches.release(); p.bin_lists.release(); p.bin_counts.release(); p.tiles.release(); p.ptcl.release();
    }
    c->seg_line.release();
    c->emit_order.release();
    drop_graph(c);
    c->d_scenes.release(); c->bin_scene.release(); c->tile_scene.release();
    c->flat.release();
    c->paints.release();
    c->tile_active.release();
    c->tile_list.release();
    DiffState& D = c->diff;
    D.colp.release(); D.target.release(); D.layer.release(); D.t1.release(); D.blurred.release(); D.gI.release();
    D.d0.release(); D.d1.release(); D.scratch.release(); D.line_acc.release(); D.color_acc.release();
    D.dpoints.release(); D.taps.release(); D.dtaps.release(); D.ep_w.release(); D.ep_point.release();
    D.sums.release();
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    cudaStreamSynchronize(c->copy_stream);
    cudaEventDestroy(c->ev_main);
    cudaEventDestroy(c->ev_copy);
    cudaStreamDestroy(c->copy_stream);
    cudaStreamDestroy(c->stream);
    delete c;
}

const char* tk_last_error(const tk_ctx* c) { return c ? c->error.c_str() : "null context"; }
void* tk_ctx_stream(tk_ctx* c) { return c ? (void*)c->stream : nullptr; }

int32_t tk_synchronize(tk_ctx* c) {
    return guarded(c, [&] { TK_CUDA(cudaStreamSynchronize(c->stream)); });
}

int32_t tk_scene_upload(tk_ctx* c, const tk_scene_desc* d) {
    if (!d) return fail(c, Fail{TK_E_INVALID, "null scene"});
    return guarded(c, [&] { do_upload(c, *d); });
}

int32_t tk_scene_upload_delta(tk_ctx* c, const tk_scene_desc* d, const uint32_t* changed, uint32_t changed_count,
                              uint32_t* rescan_paths) {
    if (!d) return fail(c, Fail{TK_E_INVALID, "null scene"});
    return guarded(c, [&] {
        if (changed_count && !changed) invalid("null changed-path list");
        const bool device_plan = (c->flags & TK_SCENE_SEGMENTS_FROM_DEVICE) != 0u;
        const bool can = c->have_scene && !c->batched && !c->band && c->scan_valid && !c->want_seg_line &&
                         device_plan == ((d->flags & TK_SCENE_SEGMENTS_FROM_DEVICE) != 0u) &&
                         (!device_plan || c->segment_needed) && d->path_count == c->path_count &&
                         d->line_count == c->line_count && d->path_count && d->paths;
        if (!can) {  // no scan to keep: a whole upload
            do_upload(c, *d);
            if (rescan_paths) *rescan_paths = d->path_count;
            return;
        }
        // The paths to rescan: the caller's (lines changed), the ones whose
        // records changed, and any still pending from an earlier delta.
        const std::vector<tk_path_record> old = c->h_paths;
        const uint64_t old_pool = c->pool_len, old_cap = c->host_segment_capacity, old_needed = c->segment_needed;
        std::vector<uint8_t> dirty(d->path_count, 0u);
        for (uint32_t k = 0; k < changed_count; ++k) {
            if (changed[k] >= d->path_count) invalid("changed path index out of range");
            dirty[changed[k]] = 1u;
        }
        for (uint32_t p : c->rescan) dirty[p] = 1u;
        for (uint32_t p = 0; p < d->path_count; ++p)
            if (std::memcmp(&old[p], &d->paths[p], sizeof(tk_path_record)) != 0) dirty[p] = 1u;
        // Device plans: every path keeps the segment slice the last scan
        // planned for it (the device records hold it), so the records go up
        // with those slices and only the replaced paths are counted again.
        tk_scene_desc dd = *d;
        std::vector<tk_path_record> planned;
        if (device_plan) {
            planned.resize(d->path_count);
            TK_CUDA(cudaMemcpyAsync(planned.data(), c->paths.ptr, d->path_count * sizeof(tk_path_record),
                                    cudaMemcpyDeviceToHost, c->stream));
            TK_CUDA(cudaStreamSynchronize(c->stream));
            for (uint32_t p = 0; p < d->path_count; ++p) {
                const uint32_t start = planned[p].segment_start, cap = planned[p].segment_capacity;
                planned[p] = d->paths[p];
                planned[p].segment_start = start;
                planned[p].segment_capacity = cap;
            }
            dd.paths = planned.data();
        }
        do_upload(c, dd, nullptr, &dirty);
        c->h_paths.assign(d->paths, d->paths + d->path_count);  // the caller's records, compared next time
        // the kept scan is valid only over the same pool and segment layout;
        // otherwise the next render scans everything
        c->rescan.clear();
        if (c->pool_len != old_pool || (!device_plan && c->host_segment_capacity != old_cap)) {
            if (rescan_paths) *rescan_paths = d->path_count;
            return;
        }
        if (device_plan) c->segment_needed = old_needed;  // the segment buffer as the last scan sized it
        for (uint32_t p = 0; p < d->path_count; ++p)
            if (dirty[p]) c->rescan.push_back(p);
        c->rescan_check = device_plan && !c->rescan.empty();
        c->scan_valid = true;
        if (rescan_paths) *rescan_paths = uint32_t(c->rescan.size());
    });
}

int32_t tk_render(tk_ctx* c) {
    return guarded(c, [&] {
        if (c->batched) do_batch_render(c);
        else if (c->band) do_render_band(c);
        else do_render(c);
    });
}

void tk_band_paths(const tk_path_record* in, uint32_t path_count, uint32_t tile_y0, uint32_t tile_y1,
                   tk_path_record* out) {
    uint32_t next = 0;
    for (uint32_t p = 0; p < path_count; ++p) {
        tk_path_record r = in[p];
        const uint32_t stride = r.tile_x1 > r.tile_x0 ? r.tile_x1 - r.tile_x0 : 0u;
        const uint32_t y0 = std::max(r.tile_y0, tile_y0), y1 = std::min(r.tile_y1, tile_y1);
        if (y0 >= y1 || stride == 0u) {
            r.tile_y0 = r.tile_y1 = tile_y0;
            r.data_len = 0u;
        } else {
            r.tile_y0 = y0;
            r.tile_y1 = y1;
            r.data_len = stride * (y1 - y0);
        }
        r.data_offset = next;
        next += r.data_len;
        r.segment_start = 0u;
        r.segment_capacity = 0u;
        out[p] = r;
    }
}

int32_t tk_set_band(tk_ctx* c, uint32_t tile_y0, uint32_t tile_y1) {
    return guarded(c, [&] {
        if (tile_y0 > tile_y1) invalid("band rows reversed");
        c->band = tile_y1 > tile_y0;
        c->band_y0 = c->band ? tile_y0 : 0u;
        c->band_y1 = c->band ? tile_y1 : 0u;
        c->have_scene = false;  // the next upload applies it
        c->rendered = false;
        c->history = false;
        c->scan_valid = false;
    });
}

int32_t tk_readback_rows(tk_ctx* c, uint32_t row0, uint32_t row1, uint32_t* rgba8, size_t pixel_count) {
    return guarded(c, [&] {
        if (!c->rendered) throw Fail{TK_E_STATE, "nothing rendered"};
        if (row0 > row1 || row1 > c->height) invalid("rows outside the image");
        const size_t n = size_t(c->width) * (row1 - row0);
        if (n && (!rgba8 || pixel_count < n)) invalid("readback buffer too small");
        if (n)
            TK_CUDA(cudaMemcpyAsync(rgba8, c->image.ptr + size_t(row0) * c->width, n * 4, cudaMemcpyDefault,
                                    c->stream));
        TK_CUDA(cudaStreamSynchronize(c->stream));
        check_error_word(c);
    });
}

int32_t tk_render_incremental(tk_ctx* c, const tk_damage* damage, float full_redraw_ratio,
                              tk_incremental_stats* stats) {
    return guarded(c, [&] {
        if (!damage) invalid("null damage");
        if (damage->rect_count && !damage->rects) invalid("null damage rects");
        if (!(full_redraw_ratio > 0.0f && full_redraw_ratio <= 1.0f)) invalid("full_redraw_ratio outside (0, 1]");
        if (c->batched) invalid("incremental rendering takes one uploaded scene, not a batch");
        if (!c->have_scene) throw Fail{TK_E_STATE, "no scene uploaded"};
        const uint32_t T = c->tw * c->th;
        tk_incremental_stats out{};
        out.total_tiles = T;
        uint32_t reason = TK_FULL_NONE;
        if (damage->full) reason = TK_FULL_REQUESTED;
        else if (!c->history || c->history_w != c->width || c->history_h != c->height || c->history_clear != c->clear)
            reason = TK_FULL_NO_HISTORY;
        else if (c->steps.size() != c->passes.size()) reason = TK_FULL_FILTERS;  // blur begin/end steps
        if (reason == TK_FULL_NONE) {
            // DamageTiles: every tile that meets a damage rectangle
            c->h_active.assign(T, 0u);
            for (uint32_t k = 0; k < damage->rect_count; ++k) {
                const int32_t* r = damage->rects + 4 * size_t(k);
                const int32_t x0 = std::max(r[0], 0), y0 = std::max(r[1], 0);
                const int32_t x1 = std::min(r[2], int32_t(c->width)), y1 = std::min(r[3], int32_t(c->height));
                if (x1 <= x0 || y1 <= y0) continue;
                const uint32_t tx0 = uint32_t(x0) / TK_TILE_SIZE, ty0 = uint32_t(y0) / TK_TILE_SIZE;
                const uint32_t tx1 = (uint32_t(x1) + TK_TILE_SIZE - 1u) / TK_TILE_SIZE;
                const uint32_t ty1 = (uint32_t(y1) + TK_TILE_SIZE - 1u) / TK_TILE_SIZE;
                for (uint32_t ty = ty0; ty < ty1; ++ty)
                    std::memset(c->h_active.data() + size_t(ty) * c->tw + tx0, 1, tx1 - tx0);
            }
            c->h_active_list.clear();
            for (uint32_t t = 0; t < T; ++t)
                if (c->h_active[t]) c->h_active_list.push_back(t);
            if (double(c->h_active_list.size()) >= double(full_redraw_ratio) * double(T)) reason = TK_FULL_THRESHOLD;
        }
        if (reason != TK_FULL_NONE) {
            c->last_scan_paths = 0;
            do_render(c);
            out.dirty_tiles = T;
            out.full_redraw = 1u;
        } else {
            out.dirty_tiles = uint32_t(c->h_active_list.size());
            // The uploaded scene's scan is reused when nothing was uploaded or
            // scanned since it (the reference reuses an unchanged scene's scan
            // history, src/native/runtime/program/scene_scan.rs:116-125).
            out.scan_reused = c->scan_valid && c->rescan.empty() ? 1u : 0u;
            c->last_scan_paths = 0;
            if (out.dirty_tiles) do_render_tiles(c, true);
            else c->rendered = true;  // nothing changed: the image is the frame
        }
        out.scanned_paths = c->last_scan_paths;
        out.reason = reason;
        if (stats) *stats = out;
    });
}

int32_t tk_readback(tk_ctx* c, uint32_t* rgba8, size_t pixel_count) {
    return guarded(c, [&] {
        if (!c->rendered) throw Fail{TK_E_STATE, "nothing rendered"};
        size_t n = size_t(c->width) * c->height;
        if (!rgba8 || pixel_count < n) throw Fail{TK_E_INVALID, "readback buffer too small"};
        TK_CUDA(cudaMemcpyAsync(rgba8, c->image.ptr, n * 4, cudaMemcpyDeviceToHost, c->stream));
        TK_CUDA(cudaStreamSynchronize(c->stream));
        check_error_word(c);
    });
}

int32_t tk_render_to_image(tk_ctx* c, const tk_scene_desc* d, uint32_t* rgba8, size_t pixel_count) {
    int32_t rc = tk_scene_upload(c, d);
    if (rc) return rc;
    rc = tk_render(c);
    if (rc) return rc;
    return tk_readback(c, rgba8, pixel_count);
}

int32_t tk_get_stats(tk_ctx* c, tk_stats* out) {
    return guarded(c, [&] {
        if (!out) throw Fail{TK_E_INVALID, "null stats"};
        std::memset(out, 0, sizeof(*out));
        out->lines = c->line_count;
        out->backdrop_len = c->pool_len;
        out->tile_draw_refs = c->tile_draw_refs;
        out->tiles = c->tw * c->th;
        out->passes = uint32_t(c->passes.size());
        bool device_plan = (c->flags & TK_SCENE_SEGMENTS_FROM_DEVICE) != 0u;
        if (c->rendered) {
            TK_CUDA(cudaStreamSynchronize(c->stream));
            if (device_plan) out->segments = c->segment_needed ? c->segment_needed - 1 : 0;
            else out->segments = c->host_segment_capacity;
            for (const Pass& p : c->passes) out->ptcl_records += p.ptcl_used;
            unsigned long long st[2] = {0, 0};
            TK_CUDA(cudaMemcpy(st, c->stats.ptr, sizeof(st), cudaMemcpyDeviceToHost));
            out->fill_particles = st[0];
            out->segment_visits = st[1];
        }
    });
}

namespace {

// Copies elements [first, first + count) of a debug stage buffer (count
// clipped to the buffer) and returns the buffer's element count.
uint64_t debug_read(tk_ctx* c, uint32_t stage, uint32_t index, uint64_t first, uint64_t count, void* dst) {
    if (!c->rendered) throw Fail{TK_E_STATE, "nothing rendered"};
    TK_CUDA(cudaStreamSynchronize(c->stream));
    const unsigned char* src = nullptr;
    uint64_t n = 0;     // elements
    size_t es = 4;      // bytes per element on the host side
    size_t dev_es = 0;  // bytes per element on the device when it differs
    std::vector<uint32_t> kinds;
    switch (stage) {
        case TK_STAGE_COUNTS: src = reinterpret_cast<const unsigned char*>(c->counts.ptr); n = c->pool_len; break;
        case TK_STAGE_BACKDROPS:
            src = reinterpret_cast<const unsigned char*>(c->backdrops.ptr);
            n = c->pool_len;
            break;
        case TK_STAGE_RANGES: src = reinterpret_cast<const unsigned char*>(c->ranges.ptr); n = c->pool_len; es = 8; break;
        case TK_STAGE_SEGMENTS: {
            // 32-byte device records -> 20-byte LineSegments
            bool device_plan = (c->flags & TK_SCENE_SEGMENTS_FROM_DEVICE) != 0u;
            n = device_plan ? (c->segment_needed ? c->segment_needed - 1 : 0) : c->host_segment_capacity;
            src = reinterpret_cast<const unsigned char*>(c->segments.ptr);
            es = sizeof(tk_line_segment);
            dev_es = sizeof(tk::SegmentRec);
            break;
        }
        case TK_STAGE_IMAGE: src = reinterpret_cast<const unsigned char*>(c->image.ptr); n = uint64_t(c->width) * c->height; break;
        case TK_STAGE_PATHS:
            src = reinterpret_cast<const unsigned char*>(c->paths.ptr);
            n = c->path_count;
            es = sizeof(tk_path_record);
            break;
        case TK_STAGE_LINES:
            src = reinterpret_cast<const unsigned char*>(c->lines.ptr);
            n = c->line_count;
            es = sizeof(tk_line);
            break;
        case TK_STAGE_PTCL:
        case TK_STAGE_TILES:
        case TK_STAGE_KINDS:
        case TK_STAGE_GLYPHS: {
            if (index >= c->passes.size()) throw Fail{TK_E_INVALID, "pass index out of range"};
            Pass& p = c->passes[index];
            uint32_t T = c->tw * c->th;
            if (stage == TK_STAGE_GLYPHS) {
                src = reinterpret_cast<const unsigned char*>(p.glyph_list.ptr);
                n = p.glyph_list.ptr ? p.glyph_used : 0;
            } else if (stage == TK_STAGE_PTCL) {
                src = reinterpret_cast<const unsigned char*>(p.ptcl.ptr);
                n = p.ptcl_used;
                es = sizeof(tk_ptcl_record);
            } else if (stage == TK_STAGE_TILES) {
                src = reinterpret_cast<const unsigned char*>(p.tiles.ptr);
                n = T;
                es = sizeof(tk_tile_record);
            } else {
                std::vector<tk_tile_record> tiles(T);
                TK_CUDA(cudaMemcpy(tiles.data(), p.tiles.ptr, T * sizeof(tk_tile_record), cudaMemcpyDeviceToHost));
                kinds.resize(T);
                for (uint32_t t = 0; t < T; ++t)
                    kinds[t] = tiles[t].ptcl_count ? TK_TILE_KIND_INTERPRETER : TK_TILE_KIND_EMPTY;
                n = T;
            }
            break;
        }
        default: throw Fail{TK_E_INVALID, "unknown stage"};
    }
    if (!dst || first >= n) return n;
    const uint64_t k = std::min(count, n - first);
    if (!k) return n;
    if (!kinds.empty()) {
        std::memcpy(dst, kinds.data() + first, k * 4);
    } else if (dev_es) {
        TK_CUDA(cudaMemcpy2D(dst, es, src + first * dev_es, dev_es, es, k, cudaMemcpyDeviceToHost));
    } else {
        TK_CUDA(cudaMemcpy(dst, src + first * es, k * es, cudaMemcpyDeviceToHost));
    }
    return n;
}

size_t debug_elem_bytes(uint32_t stage) {
    switch (stage) {
        case TK_STAGE_RANGES: return 8;
        case TK_STAGE_SEGMENTS: return sizeof(tk_line_segment);
        case TK_STAGE_PATHS: return sizeof(tk_path_record);
        case TK_STAGE_LINES: return sizeof(tk_line);
        case TK_STAGE_PTCL: return sizeof(tk_ptcl_record);
        case TK_STAGE_TILES: return sizeof(tk_tile_record);
        default: return 4;
    }
}

}  // namespace

int32_t tk_debug_readback(tk_ctx* c, uint32_t stage, uint32_t index, void* dst, size_t bytes, size_t* needed) {
    return guarded(c, [&] {
        const size_t es = debug_elem_bytes(stage);
        const uint64_t n = debug_read(c, stage, index, 0, bytes / es, dst);  // whole elements only
        if (needed) *needed = size_t(n * es);
    });
}

int32_t tk_debug_readback_range(tk_ctx* c, uint32_t stage, uint32_t index, uint64_t first, uint64_t count,
                                void* dst, uint64_t* total) {
    return guarded(c, [&] {
        const uint64_t n = debug_read(c, stage, index, first, count, dst);
        if (total) *total = n;
    });
}

int32_t tk_set_timing(tk_ctx* c, int32_t enabled) {
    return guarded(c, [&] { c->timing = enabled != 0; });
}

int32_t tk_get_stage_times(tk_ctx* c, float* ms, uint32_t count) {
    return guarded(c, [&] {
        if (!ms) invalid("null output");
        for (uint32_t i = 0; i < count; ++i) ms[i] = 0.0f;
        TK_CUDA(cudaStreamSynchronize(c->stream));
        for (auto& mk : c->marks) {
            float t = 0.0f;
            TK_CUDA(cudaEventElapsedTime(&t, mk.second.first, mk.second.second));
            if (uint32_t(mk.first) < count) ms[mk.first] += t;
        }
    });
}

int32_t tk_stage_scan_prefix(tk_ctx* c, const uint32_t* counts, uint64_t pool_len, const tk_path_record* paths,
                             uint32_t path_count, tk_segment_range* ranges, uint32_t* cursors, uint32_t* bumps) {
    return guarded(c, [&] {
        if ((pool_len && (!counts || !ranges || !cursors)) || (path_count && (!paths || !bumps)))
            invalid("null buffer");
        std::vector<tk::ScanItem> items;
        for (uint32_t p = 0; p < path_count; ++p) {
            const tk_path_record& r = paths[p];
            uint32_t stride = r.tile_x1 > r.tile_x0 ? r.tile_x1 - r.tile_x0 : 0u;
            uint32_t height = r.tile_y1 > r.tile_y0 ? r.tile_y1 - r.tile_y0 : 0u;
            if (uint64_t(stride) * height != r.data_len) invalid("data_len != bbox tiles");
            if (uint64_t(r.data_offset) + r.data_len > pool_len) invalid("path slice outside the pool");
            if (stride > tk::kScanItemElems) invalid("bbox wider than 4096 tiles");
            if (!r.data_len) continue;
            uint32_t rows_per = std::max<uint32_t>(1u, tk::kScanItemElems / stride);
            for (uint32_t row = 0; row < height; row += rows_per)
                items.push_back({p, row, std::min(rows_per, height - row), row == 0u ? 1u : 0u});
        }
        cudaStream_t st = c->stream;
        DBuf<uint32_t> d_counts, d_cursors, d_bumps, d_misc;
        DBuf<int32_t> d_bd;
        DBuf<tk_segment_range> d_ranges;
        DBuf<tk_path_record> d_paths;
        DBuf<tk::ScanItem> d_items;
        DBuf<unsigned long long> d_desc;
        upload(d_counts, counts, pool_len, st);
        upload(d_cursors, cursors, pool_len, st);
        upload(d_ranges, ranges, pool_len, st);
        upload(d_paths, paths, path_count, st);
        upload(d_items, items.data(), items.size(), st);
        d_bd.reserve(pool_len);
        TK_CUDA(cudaMemsetAsync(d_bd.ptr, 0, std::max<uint64_t>(pool_len, 1) * 4, st));
        d_bumps.reserve(path_count);
        d_misc.reserve(8);
        TK_CUDA(cudaMemsetAsync(d_misc.ptr, 0, 32, st));
        d_desc.reserve(items.size());
        tk::SceneView s{};
        s.paths = d_paths.ptr;
        s.path_count = path_count;
        s.counts = d_counts.ptr;
        s.backdrops = d_bd.ptr;
        s.ranges = d_ranges.ptr;
        s.cursors = d_cursors.ptr;
        s.pool_len = pool_len;
        s.error = d_misc.ptr;
        tk::launch_pool_scan(s, d_items.ptr, uint32_t(items.size()), d_desc.ptr, false, 0u, d_misc.ptr + 2, st);
        tk::launch_path_totals(s, d_bumps.ptr, false, d_misc.ptr + 2, st);
        TK_CUDA(cudaGetLastError());
        if (pool_len) {
            TK_CUDA(cudaMemcpyAsync(ranges, d_ranges.ptr, pool_len * 8, cudaMemcpyDeviceToHost, st));
            TK_CUDA(cudaMemcpyAsync(cursors, d_cursors.ptr, pool_len * 4, cudaMemcpyDeviceToHost, st));
        }
        if (path_count) TK_CUDA(cudaMemcpyAsync(bumps, d_bumps.ptr, path_count * 4, cudaMemcpyDeviceToHost, st));
        TK_CUDA(cudaStreamSynchronize(st));
        d_counts.release(); d_cursors.release(); d_bumps.release(); d_misc.release(); d_bd.release();
        d_ranges.release(); d_paths.release(); d_items.release(); d_desc.release();
    });
}

int32_t tk_stage_tile_prefix(tk_ctx* c, tk_tile_record* tiles, uint32_t tile_count, uint32_t poll_limit,
                             uint32_t withhold_first, uint32_t* total) {
    return guarded(c, [&] {
        if ((tile_count && !tiles) || !total) invalid("null buffer");
        if (withhold_first > 1u) invalid("withhold_first must be 0 or 1");
        cudaStream_t st = c->stream;
        DBuf<tk_tile_record> d_tiles;
        DBuf<uint32_t> d_misc;
        DBuf<unsigned long long> d_desc;
        upload(d_tiles, tiles, tile_count, st);
        d_misc.reserve(4);
        TK_CUDA(cudaMemsetAsync(d_misc.ptr, 0, 16, st));
        d_desc.reserve(tk::tile_prefix_blocks(tile_count) + 1u);
        tk::launch_tile_prefix_on(d_tiles.ptr, tile_count, d_desc.ptr, d_misc.ptr + 1, d_misc.ptr + 2, d_misc.ptr,
                                  poll_limit ? poll_limit : tk::kTilePrefixPollLimit, withhold_first, st);
        TK_CUDA(cudaGetLastError());
        uint32_t words[4] = {0, 0, 0, 0};
        TK_CUDA(cudaMemcpyAsync(words, d_misc.ptr, sizeof(words), cudaMemcpyDeviceToHost, st));
        if (tile_count)
            TK_CUDA(cudaMemcpyAsync(tiles, d_tiles.ptr, size_t(tile_count) * sizeof(tk_tile_record),
                                    cudaMemcpyDeviceToHost, st));
        TK_CUDA(cudaStreamSynchronize(st));
        d_tiles.release(); d_misc.release(); d_desc.release();
        *total = words[2];
        if (words[0] & tk::ERR_LOOKBACK_TIMEOUT)
            throw Fail{TK_E_TIMEOUT, "device error flags " + std::to_string(words[0]) +
                                         ": look-back wait gave up after " +
                                         std::to_string(poll_limit ? poll_limit : tk::kTilePrefixPollLimit) +
                                         " polls"};
    });
}

int32_t tk_stage_scan_count(tk_ctx* c, const tk_line* lines, uint64_t line_count, const tk_path_record* paths,
                            uint32_t path_count, int32_t* backdrops, uint32_t* counts, uint64_t pool_len) {
    return guarded(c, [&] {
        if ((line_count && !lines) || (path_count && !paths) || (pool_len && (!backdrops || !counts)))
            invalid("null buffer");
        for (uint32_t p = 0; p < path_count; ++p)
            if (uint64_t(paths[p].data_offset) + paths[p].data_len > pool_len) invalid("path slice outside the pool");
        cudaStream_t st = c->stream;
        DBuf<tk_line> d_lines;
        DBuf<tk_path_record> d_paths;
        DBuf<int32_t> d_bd;
        DBuf<uint32_t> d_counts;
        upload(d_lines, lines, line_count, st);
        upload(d_paths, paths, path_count, st);
        upload(d_bd, backdrops, pool_len, st);
        upload(d_counts, counts, pool_len, st);
        tk::SceneView s{};
        s.lines = d_lines.ptr;
        s.line_count = line_count;
        s.paths = d_paths.ptr;
        s.path_count = path_count;
        s.backdrops = d_bd.ptr;
        s.counts = d_counts.ptr;
        tk::launch_scan_count(s, st);
        TK_CUDA(cudaGetLastError());
        if (pool_len) {
            TK_CUDA(cudaMemcpyAsync(backdrops, d_bd.ptr, pool_len * 4, cudaMemcpyDeviceToHost, st));
            TK_CUDA(cudaMemcpyAsync(counts, d_counts.ptr, pool_len * 4, cudaMemcpyDeviceToHost, st));
        }
        TK_CUDA(cudaStreamSynchronize(st));
        d_lines.release(); d_paths.release(); d_bd.release(); d_counts.release();
    });
}

int32_t tk_stage_blur(tk_ctx* c, const uint32_t* src, uint32_t* dst, uint32_t width, uint32_t height,
                      const uint32_t region[4], const uint32_t source[4], float sigma, uint32_t axis) {
    return guarded(c, [&] {
        if (!src || !dst || !region || !source || width == 0 || height == 0) invalid("bad blur arguments");
        if (uint64_t(region[0]) + region[2] > width || uint64_t(region[1]) + region[3] > height)
            invalid("blur region outside the image");
        if (axis > 1u) invalid("bad axis");
        cudaStream_t st = c->stream;
        size_t n = size_t(width) * height;
        DBuf<uint32_t> d_src, d_dst;
        upload(d_src, src, n, st);
        upload(d_dst, dst, n, st);
        tk::BlurParams b{};
        b.width = width;
        b.height = height;
        std::memcpy(b.region, region, sizeof(b.region));
        bool sx = source[2] > source[0], sy = source[3] > source[1];
        b.bounds[0] = int32_t(sx ? source[0] : region[0]);
        b.bounds[1] = int32_t(sy ? source[1] : region[1]);
        b.bounds[2] = int32_t(sx ? source[2] : region[0] + region[2]);
        b.bounds[3] = int32_t(sy ? source[3] : region[1] + region[3]);
        b.sigma = sigma;
        b.axis = axis;
        tk::launch_blur(d_src.ptr, d_dst.ptr, b, st);
        TK_CUDA(cudaGetLastError());
        TK_CUDA(cudaMemcpyAsync(dst, d_dst.ptr, n * 4, cudaMemcpyDeviceToHost, st));
        TK_CUDA(cudaStreamSynchronize(st));
        d_src.release();
        d_dst.release();
    });
}

int32_t tk_pool_scan_noalloc(tk_ctx* c, const tk_path_record* paths, uint32_t path_count, const uint32_t* d_counts,
                             int32_t* d_backdrops, tk_segment_range* d_ranges, uint32_t* d_cursors, uint64_t pool_len,
                             uint32_t* d_bumps) {
    return guarded(c, [&] {
        if ((pool_len && (!d_counts || !d_backdrops || !d_ranges || !d_cursors)) || (path_count && (!paths || !d_bumps)))
            invalid("null buffer");
        if (path_count > TK_NOALLOC_MAX_PATHS)
            throw Fail{TK_E_CAPACITY, std::to_string(path_count) + " paths exceed the allocation-free limit of " +
                                          std::to_string(TK_NOALLOC_MAX_PATHS)};
        uint64_t n_items = 0;
        for (uint32_t p = 0; p < path_count; ++p) {
            const tk_path_record& r = paths[p];
            uint32_t stride = r.tile_x1 > r.tile_x0 ? r.tile_x1 - r.tile_x0 : 0u;
            uint32_t height = r.tile_y1 > r.tile_y0 ? r.tile_y1 - r.tile_y0 : 0u;
            if (uint64_t(stride) * height != r.data_len) invalid("data_len != bbox tiles");
            if (uint64_t(r.data_offset) + r.data_len > pool_len) invalid("path slice outside the pool");
            if (stride > tk::kScanItemElems) invalid("bbox wider than 4096 tiles");
            if (!r.data_len) continue;
            uint32_t rows_per = std::max<uint32_t>(1u, tk::kScanItemElems / stride);
            n_items += (height + rows_per - 1u) / rows_per;
        }
        if (n_items > TK_NOALLOC_MAX_SCAN_ITEMS)
            throw Fail{TK_E_CAPACITY, std::to_string(n_items) + " scan work items exceed the allocation-free limit of " +
                                          std::to_string(TK_NOALLOC_MAX_SCAN_ITEMS)};
        tk::NoAllocScratch sc{};
        TK_CUDA(tk::noalloc_scratch(c->device, &sc));
        cudaStream_t st = c->stream;
        TK_CUDA(cudaMemsetAsync(sc.words, 0, 4 * sizeof(uint32_t), st));
        if (path_count)
            TK_CUDA(cudaMemcpyAsync(sc.paths, paths, size_t(path_count) * sizeof(tk_path_record),
                                    cudaMemcpyHostToDevice, st));
        tk::launch_build_scan_items(sc.paths, path_count, sc.items, st);
        tk::SceneView s{};
        s.paths = sc.paths;
        s.path_count = path_count;
        s.counts = const_cast<uint32_t*>(d_counts);
        s.backdrops = d_backdrops;
        s.ranges = d_ranges;
        s.cursors = d_cursors;
        s.pool_len = pool_len;
        s.error = sc.words;
        tk::launch_pool_scan(s, sc.items, uint32_t(n_items), sc.desc, false, 0u, sc.words + 2, st);
        tk::launch_path_totals(s, d_bumps, false, sc.words + 2, st);
        TK_CUDA(cudaGetLastError());
        TK_CUDA(cudaStreamSynchronize(st));
    });
}

int32_t tk_diff_forward(tk_ctx* c, const tk_diff_scene* sc, const float* target, double* loss, float* image) {
    return guarded(c, [&] {
        if (!sc || !sc->points || !sc->colors || !target || !loss) invalid("null argument");
        if (sc->width == 0 || sc->height == 0 || sc->path_count == 0 || sc->cubics_per_path == 0)
            invalid("empty differentiable scene");
        if (!(sc->sigma >= 0.0f) || !std::isfinite(sc->sigma) || !(sc->tolerance > 0.0f))
            invalid("sigma must be >= 0 and tolerance > 0");
        DiffState& D = c->diff;
        D.ready = false;
        const uint32_t per = 1u + 3u * sc->cubics_per_path;
        // flattening with endpoint weights (paths on host threads)
        std::vector<tk_line>& lines = D.h_lines;
        std::vector<uint32_t>& ep_point = D.h_ep_point;
        std::vector<float>& ep_w = D.h_ep_w;
        tk_diff_flatten_all(sc, lines, ep_point, ep_w);
        const uint64_t nl = lines.size();
        // the same scene through the Canvas: blur group, one fill per path,
        // kept as Bezier elements and flattened on the device at upload
        std::unique_ptr<tk_canvas, void (*)(tk_canvas*)> cv(tk_canvas_new(sc->width, sc->height, 1.0f),
                                                           tk_canvas_free);
        tk_canvas_set_device_flatten(cv.get(), 1);
        if (sc->sigma > 0.0f) tk_canvas_push_blur_group(cv.get(), sc->sigma);
        D.colors.assign(sc->colors, sc->colors + 4ull * sc->path_count);
        std::vector<float4> colp(sc->path_count);
        for (uint32_t p = 0; p < sc->path_count; ++p) {
            const float* P = sc->points + size_t(2) * per * p;
            tk_path* path = tk_path_new();
            tk_path_move_to(path, P[0], P[1]);
            for (uint32_t k = 0; k < sc->cubics_per_path; ++k) {
                const float* q = P + 2 * (3 * k + 1);
                tk_path_cubic_to(path, q[0], q[1], q[2], q[3], q[4], q[5]);
            }
            tk_path_close(path);
            const float* col = sc->colors + 4 * p;
            tk_brush_desc b{};
            b.kind = TK_BRUSH_KIND_SOLID;
            std::memcpy(b.rgba, col, sizeof(b.rgba));
            tk_canvas_push_path(cv.get(), path, &b, nullptr, TK_FILL_NONZERO, double(sc->tolerance));
            tk_path_free(path);
            colp[p] = make_float4(col[0] * col[3], col[1] * col[3], col[2] * col[3], col[3]);
        }
        if (sc->sigma > 0.0f) tk_canvas_pop_layer(cv.get());
        tk_scene_desc d{};
        tk_flatten_desc fl{};
        if (tk_canvas_scene(cv.get(), &d) != TK_OK || tk_canvas_flatten_desc(cv.get(), &fl) != TK_OK)
            invalid("canvas compile failed");
        do_upload(c, d, &fl);
        // the device's lines must be the weighted flattening's, line for line
        {
            std::vector<tk_line>& dev = D.h_dev_lines;
            dev.resize(c->line_count);
            if (c->line_count)
                TK_CUDA(cudaMemcpyAsync(dev.data(), c->lines.ptr, c->line_count * sizeof(tk_line),
                                        cudaMemcpyDeviceToHost, c->stream));
            TK_CUDA(cudaStreamSynchronize(c->stream));
            if (c->line_count != nl || (nl && std::memcmp(dev.data(), lines.data(), nl * sizeof(tk_line)) != 0))
                throw Fail{TK_E_INVALID, "differentiable flattening differs from the canvas flattening"};
        }
        uint32_t pass = UINT32_MAX;
        for (const Step& s : c->steps)
            if (s.kind == STEP_PASS) {
                if (pass != UINT32_MAX) invalid("differentiable scenes have one target pass");
                pass = s.pass;
            }
        if (pass == UINT32_MAX) invalid("no draw pass");
        cudaStream_t st = c->stream;
        c->want_seg_line = true;  // sized by the scan (device segment plan)
        scan_phase(c);
        run_pass(c, c->passes[pass], nullptr, false);
        check_error_word(c);
        const uint64_t n = uint64_t(sc->width) * sc->height;
        upload(D.colp, colp.data(), colp.size(), st);
        upload(D.target, reinterpret_cast<const float4*>(target), n, st);
        upload(D.ep_point, ep_point.data(), ep_point.size(), st);
        upload(D.ep_w, ep_w.data(), ep_w.size(), st);
        D.layer.reserve(n);
        D.gI.reserve(n);
        D.sums.reserve(2);
        TK_CUDA(cudaMemsetAsync(D.sums.ptr, 0, 2 * sizeof(double), st));
        tk::SceneView s = view(c);
        tk::PassView v = pass_view(c, c->passes[pass]);
        tk::launch_diff_fine_fwd(s, v, D.colp.ptr, D.layer.ptr, st);
        const float4* B = D.layer.ptr;
        D.radius = 0;
        if (sc->sigma > 0.0f) {
            // taps and their sigma derivatives, r = ceil(3 sigma)
            const int32_t r = int32_t(std::ceil(3.0 * double(sc->sigma)));
            const double sg = double(sc->sigma);
            std::vector<double> e(2 * r + 1), de(2 * r + 1);
            double S = 0.0, dS = 0.0;
            for (int32_t k = -r; k <= r; ++k) {
                e[k + r] = std::exp(-double(k) * k / (2.0 * sg * sg));
                de[k + r] = e[k + r] * double(k) * k / (sg * sg * sg);
                S += e[k + r];
                dS += de[k + r];
            }
            std::vector<float> w(2 * r + 1), wd(2 * r + 1);
            for (int32_t k = 0; k <= 2 * r; ++k) {
                w[k] = float(e[k] / S);
                wd[k] = float((de[k] * S - e[k] * dS) / (S * S));
            }
            upload(D.taps, w.data(), w.size(), st);
            upload(D.dtaps, wd.data(), wd.size(), st);
            D.t1.reserve(n);
            D.blurred.reserve(n);
            tk::launch_diff_blur(D.layer.ptr, D.t1.ptr, D.taps.ptr, r, sc->width, sc->height, 0, st);
            tk::launch_diff_blur(D.t1.ptr, D.blurred.ptr, D.taps.ptr, r, sc->width, sc->height, 1, st);
            B = D.blurred.ptr;
            D.radius = r;
        }
        D.bg = make_float4(sc->background[0], sc->background[1], sc->background[2], sc->background[3]);
        if (image) D.d0.reserve(n);
        // the loss's pixel rows (all of them unless the objective is split by rows)
        const uint32_t r0 = sc->loss_row1 ? std::min(sc->loss_row0, sc->height) : 0u;
        const uint32_t r1 = sc->loss_row1 ? std::min(sc->loss_row1, sc->height) : sc->height;
        tk::launch_diff_composite(B, D.target.ptr, D.bg, n, uint64_t(r0) * sc->width, uint64_t(std::max(r0, r1)) * sc->width,
                                  image ? D.d0.ptr : nullptr, D.gI.ptr, D.sums.ptr, st);
        TK_CUDA(cudaGetLastError());
        check_error_word(c);
        TK_CUDA(cudaMemcpyAsync(loss, D.sums.ptr, sizeof(double), cudaMemcpyDeviceToHost, st));
        if (image) TK_CUDA(cudaMemcpyAsync(image, D.d0.ptr, n * sizeof(float4), cudaMemcpyDeviceToHost, st));
        TK_CUDA(cudaStreamSynchronize(st));
        D.width = sc->width;
        D.height = sc->height;
        D.paths = sc->path_count;
        D.points = per * sc->path_count;
        D.lines = nl;
        D.sigma = sc->sigma;
        D.pass = pass;
        D.ready = true;
    });
}

int32_t tk_diff_backward(tk_ctx* c, float* d_points, float* d_colors, float* d_sigma) {
    return guarded(c, [&] {
        DiffState& D = c->diff;
        if (!D.ready || !c->have_scene) throw Fail{TK_E_STATE, "no differentiable forward to differentiate"};
        cudaStream_t st = c->stream;
        const uint64_t n = uint64_t(D.width) * D.height;
        Pass& p = c->passes[D.pass];
        D.d0.reserve(n);
        D.d1.reserve(n);
        D.line_acc.reserve(D.lines);
        D.color_acc.reserve(5ull * c->draw_count);
        D.dpoints.reserve(2ull * D.points);
        D.scratch.reserve(std::max<uint64_t>(p.ptcl_used, 1) * 256);
        TK_CUDA(cudaMemsetAsync(D.sums.ptr + 1, 0, sizeof(double), st));
        TK_CUDA(cudaMemsetAsync(D.line_acc.ptr, 0, std::max<uint64_t>(D.lines, 1) * sizeof(float2), st));
        TK_CUDA(cudaMemsetAsync(D.color_acc.ptr, 0, 5ull * std::max(c->draw_count, 1u) * sizeof(float), st));
        TK_CUDA(cudaMemsetAsync(D.dpoints.ptr, 0, 2ull * D.points * sizeof(float), st));
        const float4* dL = nullptr;
        if (D.radius > 0) {
            // B = Gy(Gx L): dT1 = Gy^T dB (+ <dB, Gy' T1>), dL = Gx^T dT1 (+ <dT1, Gx' L>)
            tk::launch_diff_blur_bwd(D.gI.ptr, D.t1.ptr, D.d0.ptr, D.taps.ptr, D.dtaps.ptr, D.radius, D.width,
                                     D.height, 1, true, D.bg, D.sums.ptr + 1, st);
            tk::launch_diff_blur_bwd(D.d0.ptr, D.layer.ptr, D.d1.ptr, D.taps.ptr, D.dtaps.ptr, D.radius, D.width,
                                     D.height, 0, false, D.bg, D.sums.ptr + 1, st);
            dL = D.d1.ptr;
        } else {
            tk::launch_diff_composite_bwd(D.gI.ptr, D.bg, n, D.d0.ptr, st);
            dL = D.d0.ptr;
        }
        tk::SceneView s = view(c);
        tk::PassView v = pass_view(c, p);
        tk::launch_diff_fine_bwd(s, v, c->seg_line.ptr, D.colp.ptr, dL, D.scratch.ptr, D.line_acc.ptr,
                                 D.color_acc.ptr, st);
        tk::launch_diff_lines_to_points(c->lines.ptr, D.line_acc.ptr, D.ep_point.ptr, D.ep_w.ptr, D.lines,
                                        D.dpoints.ptr, st);
        TK_CUDA(cudaGetLastError());
        check_error_word(c);
        std::vector<float> cacc(5ull * c->draw_count);
        double dsig = 0.0;
        if (d_points)
            TK_CUDA(cudaMemcpyAsync(d_points, D.dpoints.ptr, 2ull * D.points * sizeof(float), cudaMemcpyDeviceToHost,
                                    st));
        if (!cacc.empty())
            TK_CUDA(cudaMemcpyAsync(cacc.data(), D.color_acc.ptr, cacc.size() * sizeof(float), cudaMemcpyDeviceToHost,
                                    st));
        TK_CUDA(cudaMemcpyAsync(&dsig, D.sums.ptr + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
        TK_CUDA(cudaStreamSynchronize(st));
        if (d_colors) {
            // colp = (r a, g a, b a, a): chain to the straight colour
            for (uint32_t i = 0; i < D.paths; ++i) {
                const float* col = D.colors.data() + 4 * i;
                const float* g = cacc.data() + 5 * i;
                d_colors[4 * i + 0] = g[0] * col[3];
                d_colors[4 * i + 1] = g[1] * col[3];
                d_colors[4 * i + 2] = g[2] * col[3];
                d_colors[4 * i + 3] = g[0] * col[0] + g[1] * col[1] + g[2] * col[2] + g[3] + g[4];
            }
        }
        if (d_sigma) *d_sigma = float(dsig);
    });
}

int32_t tk_scene_upload_flatten(tk_ctx* c, const tk_scene_desc* d, const tk_flatten_desc* fl) {
    return guarded(c, [&] {
        if (!d || !fl) invalid("null scene");
        do_upload(c, *d, fl);
    });
}

int32_t tk_batch_upload(tk_ctx* c, const tk_scene_desc* scenes, uint32_t scene_count) {
    return guarded(c, [&] { do_batch_upload(c, scenes, scene_count); });
}

int32_t tk_batch_render(tk_ctx* c) {
    return guarded(c, [&] { do_batch_render(c); });
}

int32_t tk_batch_info_get(tk_ctx* c, uint32_t scene, tk_batch_info* out) {
    return guarded(c, [&] {
        if (!c->batched) throw Fail{TK_E_STATE, "no batch uploaded"};
        if (!out || scene >= c->h_batch_info.size()) invalid("bad scene index");
        *out = c->h_batch_info[scene];
    });
}

int32_t tk_batch_readback(tk_ctx* c, uint32_t* rgba8, size_t pixel_count) {
    return guarded(c, [&] {
        if (!c->batched || !c->rendered) throw Fail{TK_E_STATE, "no batch rendered"};
        if (!rgba8 || pixel_count != c->total_pixels) invalid("pixel count does not match the batch");
        check_error_word(c);
        TK_CUDA(cudaMemcpyAsync(rgba8, c->image.ptr, pixel_count * 4, cudaMemcpyDeviceToHost, c->stream));
        TK_CUDA(cudaStreamSynchronize(c->stream));
    });
}

int32_t tk_autotune(tk_ctx* c, uint32_t iterations, tk_tune_result* out) {
    return guarded(c, [&] {
        if (!c->have_scene) throw Fail{TK_E_STATE, "no scene uploaded"};
        if (!out) invalid("null output");
        *out = tk_tune_result{};
        const uint32_t cand[4] = {512u, 1024u, 2048u, 4096u};
        const uint32_t iters = std::max<uint32_t>(iterations, 1u);
        cudaStream_t st = c->stream;
        cudaEvent_t e0, e1;
        TK_CUDA(cudaEventCreate(&e0));
        TK_CUDA(cudaEventCreate(&e1));
        const bool timing = c->timing;
        c->timing = false;
        auto frame = [&] {
            if (c->batched) do_batch_render(c);
            else do_render(c);
        };
        uint32_t best = c->scan_item_elems;
        float best_ms = 0.0f;
        try {
            for (uint32_t k = 0; k < 4; ++k) {
                c->scan_item_elems = cand[k];
                rebuild_items(c);
                drop_graph(c);
                frame();  // warm-up (and graph capture in batched mode)
                std::vector<float> ms;
                for (uint32_t i = 0; i < iters; ++i) {
                    TK_CUDA(cudaEventRecord(e0, st));
                    frame();
                    TK_CUDA(cudaEventRecord(e1, st));
                    TK_CUDA(cudaEventSynchronize(e1));
                    float t = 0.0f;
                    TK_CUDA(cudaEventElapsedTime(&t, e0, e1));
                    ms.push_back(t);
                }
                check_error_word(c);
                std::sort(ms.begin(), ms.end());
                const float med = ms[ms.size() / 2];
                out->candidate_elems[k] = cand[k];
                out->candidate_ms[k] = med;
                if (k == 0 || med < best_ms) {
                    best_ms = med;
                    best = cand[k];
                }
            }
        } catch (...) {
            c->timing = timing;
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        c->timing = timing;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        c->scan_item_elems = best;
        rebuild_items(c);
        drop_graph(c);
        out->scan_item_elems = best;
        out->tile_width = TK_TILE_SIZE;
        out->tile_height = TK_TILE_SIZE;
        out->candidates = 4;
    });
}

}  // extern "C"
