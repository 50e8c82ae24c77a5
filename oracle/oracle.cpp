// Oracle: CPU restatement of the reference's tile rasterization path.
// TEST INFRASTRUCTURE ONLY (see oracle.h). Built with -ffp-contract=off.
#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

namespace {

thread_local std::string g_error;

// ---------------------------------------------------------------------------
// f32 semantics of the reference shaders.
// ---------------------------------------------------------------------------
inline float fmin_(float a, float b) { return std::fmin(a, b); }
inline float fmax_(float a, float b) { return std::fmax(a, b); }
inline float clampf(float x, float lo, float hi) { return fmin_(fmax_(x, lo), hi); }
inline float mad(float a, float b, float c) { return std::fma(a, b, c); }
// HLSL round() is round-half-to-even (DXIL Round_ne).
inline float round_ne(float x) { return std::nearbyint(x); }
// float -> uint / int conversions saturate (NaN -> 0).
inline uint32_t f2u(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;
}
inline int32_t f2i(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return 0x7FFFFFFF;
    if (x <= -2147483648.0f) return (int32_t)0x80000000;
    return (int32_t)x;
}
inline float bits_f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint32_t f_bits(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

const float SCAN_EPSILON = 1.0e-6f;
const float TOP_TOUCH_EPSILON = 1.0e-12f;
const float TILE_CLIP_NUDGE = 1.0e-3f;
const float CHANNEL_SCALE = 1.0f / 255.0f;

// --- shared/pixel.hlsli:7-66 -------------------------------------------------
struct F4 { float r, g, b, a; };
inline uint32_t coverage_to_u8(float c) { return f2u(clampf(c, 0.0f, 1.0f) * 255.0f + 0.5f); }
inline uint32_t coverage_to_alpha(float v, uint32_t rule) {
    float alpha = fmin_(std::fabs(v), 1.0f);
    if (rule == 1u) alpha = std::fabs(v - 2.0f * round_ne(0.5f * v));
    return coverage_to_u8(alpha);
}
inline float signum_f32(float v) { return v < 0.0f ? -1.0f : 1.0f; }
inline uint32_t pack(uint32_t r, uint32_t g, uint32_t b, uint32_t a) { return r | (g << 8) | (b << 16) | (a << 24); }
inline uint32_t unorm_to_rgba8(F4 p) {
    return pack(f2u(clampf(p.r * 255.0f + 0.5f, 0.0f, 255.0f)), f2u(clampf(p.g * 255.0f + 0.5f, 0.0f, 255.0f)),
                f2u(clampf(p.b * 255.0f + 0.5f, 0.0f, 255.0f)), f2u(clampf(p.a * 255.0f + 0.5f, 0.0f, 255.0f)));
}
inline F4 rgba8_to_unorm(uint32_t p) {
    return {float(p & 255u) * CHANNEL_SCALE, float((p >> 8) & 255u) * CHANNEL_SCALE,
            float((p >> 16) & 255u) * CHANNEL_SCALE, float(p >> 24) * CHANNEL_SCALE};
}
inline uint32_t mul_div255(uint32_t a, uint32_t b) { uint32_t p = a * b + 128u; return (p + (p >> 8)) >> 8; }
inline uint32_t combine_alpha(uint32_t a, uint32_t b) { return mul_div255(a, b); }
inline uint32_t scale_premul_u8(uint32_t s, uint32_t f) {
    if (f == 0u) return 0u;
    if (f == 255u) return s;
    return pack(mul_div255(s & 255u, f), mul_div255((s >> 8) & 255u, f), mul_div255((s >> 16) & 255u, f),
                mul_div255(s >> 24, f));
}
inline F4 scale_premul_u8_to_unorm(uint32_t s, uint32_t f) {
    if (f == 0u || (s >> 24) == 0u) return {0, 0, 0, 0};
    float scale = float(f) * (1.0f / 65025.0f);
    return {float(s & 255u) * scale, float((s >> 8) & 255u) * scale, float((s >> 16) & 255u) * scale,
            float(s >> 24) * scale};
}
inline uint32_t src_over_premul_u8(uint32_t d, uint32_t s) {
    uint32_t a = s >> 24;
    if (a == 0u) return d;
    if (a == 255u) return s;
    uint32_t inv = 255u - a;
    return pack((s & 255u) + mul_div255(d & 255u, inv), ((s >> 8) & 255u) + mul_div255((d >> 8) & 255u, inv),
                ((s >> 16) & 255u) + mul_div255((d >> 16) & 255u, inv), a + mul_div255(d >> 24, inv));
}
inline F4 src_over_premul_unorm(F4 d, F4 s) {
    if (s.a <= 0.0f) return d;
    if (s.a >= 1.0f) return s;
    float k = 1.0f - s.a;
    return {s.r + d.r * k, s.g + d.g * k, s.b + d.b * k, s.a + d.a * k};
}
inline uint32_t lerp_premul_u8(uint32_t a, uint32_t b, float t) {
    uint32_t out = 0;
    for (int c = 0; c < 4; ++c) {
        float l = float((a >> (8 * c)) & 255u), r = float((b >> (8 * c)) & 255u);
        out |= f2u(clampf(mad(r - l, t, l) + 0.5f, 0.0f, 255.0f)) << (8 * c);
    }
    return out;
}
inline float rem_euclid_f32(float v, float m) { return mad(-std::floor(v / m), m, v); }
inline bool premul_u8_is_opaque(uint32_t p) { return (p >> 24) == 255u; }
// RGBA8 UNORM render-target texel conversions.
inline float unorm8_load(uint32_t k) { return float(k) / 255.0f; }
inline F4 texel_load(uint32_t p) {
    return {unorm8_load(p & 255u), unorm8_load((p >> 8) & 255u), unorm8_load((p >> 16) & 255u), unorm8_load(p >> 24)};
}
inline uint32_t unorm8_store(float x) { return (uint32_t)std::nearbyint(clampf(x, 0.0f, 1.0f) * 255.0f); }
inline uint32_t texel_store(F4 p) { return pack(unorm8_store(p.r), unorm8_store(p.g), unorm8_store(p.b), unorm8_store(p.a)); }

// ---------------------------------------------------------------------------
// Scan traversal (scan/geometry.hlsli:12-114).
// ---------------------------------------------------------------------------
struct Scan {
    uint32_t bx0, by0, bx1, by1;
    uint32_t data_offset;
    float qx0, qy0, qx1, qy1;  // sorted points (upper first)
    bool down;
    uint32_t count;
    float a, b, sign, x0, y0;
    uint32_t imin, imax;
    int32_t ymin, ymax;
};

inline bool is_tile_boundary_y(float v) { return std::fabs(v - std::floor(v)) <= TOP_TOUCH_EPSILON; }
inline int32_t ceil_tile_boundary_y(float v) {
    if (is_tile_boundary_y(v)) return f2i(std::floor(v));
    return f2i(std::ceil(v));
}
inline uint32_t span(float a, float b) {
    float hi = std::ceil(a);
    if (b > a) hi = std::ceil(b);
    float lo = std::floor(a);
    if (b < a) lo = std::floor(b);
    float v = hi - lo;
    if (v < 1.0f) v = 1.0f;
    return f2u(v);
}

bool scan_geometry(const tk_line& line, const tk_path_record* paths, uint32_t path_count, Scan& s) {
    s = Scan{};
    uint32_t pid = line.path_id;
    if (pid >= path_count) return false;
    const tk_path_record& p = paths[pid];
    s.bx0 = p.tile_x0; s.by0 = p.tile_y0; s.bx1 = p.tile_x1; s.by1 = p.tile_y1;
    s.data_offset = p.data_offset;
    if (s.bx1 - s.bx0 == 0u || s.by0 >= s.by1) return false;
    const tk_affine& t = p.transform;
    float p0x = t.a * line.p0[0] + t.c * line.p0[1] + t.e;
    float p0y = t.b * line.p0[0] + t.d * line.p0[1] + t.f;
    float p1x = t.a * line.p1[0] + t.c * line.p1[1] + t.e;
    float p1y = t.b * line.p1[0] + t.d * line.p1[1] + t.f;
    s.down = p1y >= p0y;
    if (s.down) { s.qx0 = p0x; s.qy0 = p0y; s.qx1 = p1x; s.qy1 = p1y; }
    else { s.qx0 = p1x; s.qy0 = p1y; s.qx1 = p0x; s.qy1 = p0y; }
    const float ts = 1.0f / float(TK_TILE_SIZE);
    float sx = s.qx0 * ts, sy = s.qy0 * ts, sz = s.qx1 * ts, sw = s.qy1 * ts;
    uint32_t count_x = span(sx, sz) - 1u;
    s.count = count_x + span(sy, sw);
    float dx = std::fabs(sz - sx);
    float dy = sw - sy;
    if (dx + dy == 0.0f || (dy == 0.0f && std::floor(sy) == sy)) return false;
    float rcp = 1.0f / (dx + dy);
    s.a = dx * rcp;
    bool positive = sz >= sx;
    s.sign = positive ? 1.0f : -1.0f;
    float xt0 = std::floor(sx * s.sign);
    float c = sx * s.sign - xt0;
    s.y0 = std::floor(sy);
    float ytop = s.y0 + 1.0f;
    if (sy == sw) ytop = std::ceil(sy);
    s.b = fmin_((dy * c + dx * (ytop - sy)) * rcp, 0.99999994f);
    float err = std::floor(s.a * (float(s.count) - 1.0f) + s.b) - float(count_x);
    if (err != 0.0f) {
        if (err > 0.0f) s.a -= 0.0000002f; else s.a += 0.0000002f;
    }
    s.x0 = positive ? xt0 * s.sign : xt0 * s.sign - 1.0f;
    float xmin = fmin_(sx, sz);
    if (sy >= float(s.by1) || sw <= float(s.by0) + TOP_TOUCH_EPSILON || xmin >= float(s.bx1)) return false;
    s.imin = 0u;
    if (sy < float(s.by0)) {
        float first = round_ne((float(s.by0) - s.y0 + s.b - s.a) / (1.0f - s.a)) - 1.0f;
        if (s.y0 + first - std::floor(s.a * first + s.b) < float(s.by0)) first += 1.0f;
        s.imin = f2u(first);
    }
    s.imax = s.count;
    if (sw > float(s.by1)) {
        float last = round_ne((float(s.by1) - s.y0 + s.b - s.a) / (1.0f - s.a)) - 1.0f;
        if (s.y0 + last - std::floor(s.a * last + s.b) < float(s.by1)) last += 1.0f;
        s.imax = f2u(last);
    }
    s.ymin = 0; s.ymax = 0;
    float xmax = fmax_(sx, sz);
    if (xmax < float(s.bx0)) {
        s.ymin = ceil_tile_boundary_y(sy);
        s.ymax = ceil_tile_boundary_y(sw);
        s.imax = s.imin;
    } else {
        float fudge = positive ? 0.0f : 1.0f;
        if (xmin < float(s.bx0)) {
            float cut = round_ne((s.sign * (float(s.bx0) - s.x0) - s.b + fudge) / s.a);
            if ((s.x0 + s.sign * std::floor(s.a * cut + s.b) < float(s.bx0)) == positive) cut += 1.0f;
            int32_t ynext = f2i(s.y0 + cut - std::floor(s.a * cut + s.b) + 1.0f);
            if (positive) {
                if (f2u(cut) > s.imin) {
                    float ystart = s.y0 + 1.0f;
                    if (is_tile_boundary_y(sy)) ystart = s.y0;
                    s.ymin = f2i(ystart); s.ymax = ynext; s.imin = f2u(cut);
                }
            } else if (f2u(cut) < s.imax) {
                s.ymin = ynext; s.ymax = ceil_tile_boundary_y(sw); s.imax = f2u(cut);
            }
        }
        if (xmax > float(s.bx1)) {
            float cut = round_ne((s.sign * (float(s.bx1) - s.x0) - s.b + fudge) / s.a);
            if ((s.x0 + s.sign * std::floor(s.a * cut + s.b) < float(s.bx1)) == positive) cut += 1.0f;
            if (positive) s.imax = std::min(s.imax, f2u(cut));
            else s.imin = std::max(s.imin, f2u(cut));
        }
    }
    s.imax = std::max(s.imin, s.imax);
    s.ymin = std::max(s.ymin, (int32_t)s.by0);
    s.ymax = std::min(s.ymax, (int32_t)s.by1);
    return true;
}
inline void scan_tile(const Scan& s, uint32_t i, float z, int32_t& tx, int32_t& ty) {
    tx = f2i(s.x0 + s.sign * z);
    ty = f2i(s.y0 + float(i) - z);
}
inline bool scan_tile_inside(const Scan& s, int32_t tx, int32_t ty) {
    return ty >= (int32_t)s.by0 && ty < (int32_t)s.by1 && tx >= (int32_t)s.bx0 && tx < (int32_t)s.bx1;
}
inline uint32_t scan_tile_offset(const Scan& s, int32_t tx, int32_t ty) {
    return s.data_offset + (uint32_t(ty) - s.by0) * (s.bx1 - s.bx0) + uint32_t(tx) - s.bx0;
}

// scan/count.hlsl:13-40 for one line.
void count_line(const tk_line& line, const tk_path_record* paths, uint32_t np, int32_t* backdrops,
                uint32_t* counts) {
    Scan s;
    if (!scan_geometry(line, paths, np, s)) return;
    int32_t delta = s.down ? -1 : 1;
    int32_t stride = int32_t(s.bx1 - s.bx0);
    for (int32_t y = s.ymin; y < s.ymax; ++y) {
        uint32_t local = uint32_t((y - int32_t(s.by0)) * stride);
        backdrops[s.data_offset + local] += delta;
    }
    float last_z = std::floor(s.a * (float(s.imin) - 1.0f) + s.b);
    for (uint32_t i = s.imin; i < s.imax; ++i) {
        float z = std::floor(s.a * float(i) + s.b);
        int32_t tx, ty;
        scan_tile(s, i, z, tx, ty);
        if (scan_tile_inside(s, tx, ty)) {
            bool top = last_z == z;
            if (i == 0u) top = std::fabs(s.y0 - s.qy0 * (1.0f / float(TK_TILE_SIZE))) <= SCAN_EPSILON;
            if (top && tx + 1 < int32_t(s.bx1)) {
                int32_t x = std::max(tx + 1, int32_t(s.bx0));
                uint32_t local = uint32_t((ty - int32_t(s.by0)) * stride + x - int32_t(s.bx0));
                backdrops[s.data_offset + local] += delta;
            }
            counts[scan_tile_offset(s, tx, ty)] += 1u;
        }
        last_z = z;
    }
}

// --- scan/clip.hlsli:10-75 -----------------------------------------------------
inline float x_at_y(const Scan& s, float y) { return mad(s.qx1 - s.qx0, (y - s.qy0) / (s.qy1 - s.qy0), s.qx0); }
inline float y_at_x(const Scan& s, float x) { return mad(s.qy1 - s.qy0, (x - s.qx0) / (s.qx1 - s.qx0), s.qy0); }
inline float clip_y_at_x(const Scan& s, float x, float tmin_y, float tmax_y) {
    float y = y_at_x(s, x);
    if (y <= tmin_y + SCAN_EPSILON) {
        float top_x = x_at_y(s, tmin_y);
        if (std::fabs(top_x - x) > TILE_CLIP_NUDGE) return tmin_y;
        return tmin_y + TILE_CLIP_NUDGE;
    }
    return clampf(y, tmin_y + TILE_CLIP_NUDGE, tmax_y);
}
tk_line_segment clipped_segment(const Scan& s, uint32_t sub, float z, int32_t tx, int32_t ty) {
    const float ts = float(TK_TILE_SIZE);
    float tminx = float(tx) * ts, tminy = float(ty) * ts;
    float tmaxx = tminx + ts, tmaxy = tminy + ts;
    float px = s.qx0, py = s.qy0, pz = s.qx1, pw = s.qy1;
    if (sub > 0u) {
        float prev = std::floor(s.a * (float(sub) - 1.0f) + s.b);
        if (z == prev) {
            float x = x_at_y(s, tminy);
            x = clampf(x, tminx + TILE_CLIP_NUDGE, tmaxx);
            px = x; py = tminy;
        } else {
            float xc = s.sign > 0.0f ? tminx : tmaxx;
            px = xc; py = clip_y_at_x(s, xc, tminy, tmaxy);
        }
    }
    if (sub < s.count - 1u) {
        float next = std::floor(s.a * (float(sub) + 1.0f) + s.b);
        if (z == next) {
            float x = x_at_y(s, tmaxy);
            x = clampf(x, tminx + TILE_CLIP_NUDGE, tmaxx);
            pz = x; pw = tmaxy;
        } else {
            float xc = s.sign > 0.0f ? tmaxx : tminx;
            pz = xc; pw = clip_y_at_x(s, xc, tminy, tmaxy);
        }
    }
    float edge = 1000000000.0f;
    float p0x = clampf(px - tminx, 0.0f, ts), p0y = clampf(py - tminy, 0.0f, ts);
    float p1x = clampf(pz - tminx, 0.0f, ts), p1y = clampf(pw - tminy, 0.0f, ts);
    if (p0x <= SCAN_EPSILON) p0x = 0.0f; else if (ts - p0x <= SCAN_EPSILON) p0x = ts;
    if (p0y <= SCAN_EPSILON) p0y = 0.0f; else if (ts - p0y <= SCAN_EPSILON) p0y = ts;
    if (p1x <= SCAN_EPSILON) p1x = 0.0f; else if (ts - p1x <= SCAN_EPSILON) p1x = ts;
    if (p1y <= SCAN_EPSILON) p1y = 0.0f; else if (ts - p1y <= SCAN_EPSILON) p1y = ts;
    if (p0x == 0.0f) {
        if (p1x == 0.0f) {
            p0x = SCAN_EPSILON;
            if (p0y == 0.0f) { p1x = SCAN_EPSILON; p1y = ts; }
            else { p1x = 2.0f * SCAN_EPSILON; p1y = p0y; }
        } else if (p0y == 0.0f) p0x = SCAN_EPSILON;
        else edge = p0y;
    } else if (p1x == 0.0f) {
        if (p1y == 0.0f) p1x = SCAN_EPSILON; else edge = p1y;
    }
    if (std::floor(p0x) == p0x && p0x != 0.0f) p0x -= SCAN_EPSILON;
    if (std::floor(p1x) == p1x && p1x != 0.0f) p1x -= SCAN_EPSILON;
    if (!s.down) { std::swap(p0x, p1x); std::swap(p0y, p1y); }
    return {p0x, p0y, p1x, p1y, edge};
}

// Canonical emit order: a path's lines in order, each line's DDA steps
// (i = imin ..) in order, each emitting step taking the next cursor of its
// tile. This is the sequential one of the reference's admissible atomic
// interleavings (scan/emit.hlsl:14-28).
void emit_path(const tk_line* lines, const tk_path_record* paths, uint32_t np, uint32_t pid, uint32_t* cursors,
               tk_line_segment* segments, uint64_t capacity) {
    const tk_path_record& p = paths[pid];
    for (uint32_t l = 0; l < p.line_count; ++l) {
        Scan s;
        if (!scan_geometry(lines[p.line_start + l], paths, np, s)) continue;
        for (uint32_t i = s.imin; i < s.imax; ++i) {
            float z = std::floor(s.a * float(i) + s.b);
            int32_t tx, ty;
            scan_tile(s, i, z, tx, ty);
            if (!scan_tile_inside(s, tx, ty)) continue;
            uint32_t dst = cursors[scan_tile_offset(s, tx, ty)]++;
            if (dst < capacity) segments[dst] = clipped_segment(s, i, z, tx, ty);
        }
    }
}

// --- shared/coverage.hlsli:7-51 -------------------------------------------------
struct Parts { float edge, dy, xmin, xmax; };
inline Parts segment_row_parts(const tk_line_segment& g, uint32_t y) {
    float delta_x = g.p1x - g.p0x, delta_y = g.p1y - g.p0y;
    float row_y = float(y), local_y = g.p0y - row_y;
    float y0 = clampf(local_y, 0.0f, 1.0f), y1 = clampf(g.p1y - row_y, 0.0f, 1.0f);
    float dy = y0 - y1;
    float row_edge = signum_f32(delta_x) * clampf(row_y - g.y_edge + 1.0f, 0.0f, 1.0f);
    if (dy == 0.0f) return {row_edge, dy, 0.0f, 0.0f};
    float slope = delta_x / delta_y;
    bool nearer_p0 = std::fabs(local_y - 0.5f) <= std::fabs(g.p1y - row_y - 0.5f);
    float anchor_x = nearer_p0 ? g.p0x : g.p1x;
    float anchor_y = nearer_p0 ? local_y : g.p1y - row_y;
    float sx0 = mad(y0 - anchor_y, slope, anchor_x);
    float sx1 = mad(y1 - anchor_y, slope, anchor_x);
    return {row_edge, dy, fmin_(sx0, sx1), fmax_(sx0, sx1)};
}
inline float segment_area_at(float xmin_abs, float xmax_abs, uint32_t x) {
    float xmin = xmin_abs - float(x), xmax = xmax_abs - float(x);
    float width = xmax - xmin;
    if (width == 0.0f) return clampf(1.0f - xmin, 0.0f, 1.0f);
    if (xmin >= 0.0f && xmax <= 1.0f) return mad(-0.5f, xmin + xmax, 1.0f);
    float left = clampf(xmin, 0.0f, 1.0f), right = clampf(xmax, 0.0f, 1.0f);
    float full = clampf(-xmin, 0.0f, width);
    return mad(right - left, mad(-0.5f, left + right, 1.0f), full) / width;
}
inline float fill_value(const tk_line_segment* segs, uint32_t start, uint32_t end, int32_t backdrop, uint32_t x,
                        uint32_t y) {
    float base = float(backdrop), running = 0.0f, partial = 0.0f;
    for (uint32_t i = start; i < end; ++i) {
        Parts q = segment_row_parts(segs[i], y);
        base += q.edge;
        if (q.dy != 0.0f) {
            int32_t full_start = std::min(std::max(f2i(std::ceil(q.xmax)), 0), int32_t(TK_TILE_SIZE));
            if (full_start < int32_t(TK_TILE_SIZE) && int32_t(x) >= full_start) running += q.dy;
            int32_t ps = std::min(std::max(f2i(std::floor(q.xmin)), 0), int32_t(TK_TILE_SIZE));
            int32_t pe = std::min(std::max(f2i(std::ceil(q.xmax)), 0), int32_t(TK_TILE_SIZE));
            if (int32_t(x) >= ps && int32_t(x) < pe) partial += segment_area_at(q.xmin, q.xmax, x) * q.dy;
        }
    }
    return base + running + partial;
}

// ---------------------------------------------------------------------------
// Brushes (shared/brush/*.hlsli, fine/draw.hlsli:16-21).
// ---------------------------------------------------------------------------
struct Paint {
    const uint32_t* words;
    uint64_t count;
    const tk_image_desc* images = nullptr;  // the scene's texture table
    uint32_t image_count = 0;
    uint32_t word(uint32_t base, uint32_t index) const {
        if (base < count) {
            if (index < count - base) return words[base + index];
        }
        return 0u;
    }
    float param(uint32_t base, uint32_t b, uint32_t i) const { return bits_f(word(base, b + i)); }
};
const float GRADIENT_FLOAT_EPSILON = 0.00000011920929f;
const float RADIAL_QUADRATIC_EPSILON = 0.000001f;
inline float apply_extend(float t, uint32_t extend) {
    if (extend == TK_EXTEND_REPEAT) return rem_euclid_f32(t, 1.0f);
    if (extend == TK_EXTEND_REFLECT) {
        float v = rem_euclid_f32(t, 2.0f);
        return v <= 1.0f ? v : 2.0f - v;
    }
    return clampf(t, 0.0f, 1.0f);
}
uint32_t sample_ramp(const Paint& P, uint32_t off, uint32_t len, float t, uint32_t extend) {
    if (len == 0u) return 0u;
    uint32_t last = len - 1u;
    float ext = apply_extend(t, extend);
    float pos = ext * float(last);
    uint32_t li = f2u(std::floor(pos)), ri = std::min(li + 1u, last);
    float frac = mad(ext, float(last), -float(li));
    uint32_t l = P.word(0u, off + li), r = P.word(0u, off + ri);
    if (frac <= GRADIENT_FLOAT_EPSILON || li == ri) return l;
    return lerp_premul_u8(l, r, frac);
}
uint32_t sample_linear(const Paint& P, float x, float y, uint32_t base, uint32_t extend, uint32_t off, uint32_t len) {
    float tx = mad(P.param(0, base, 4), x, mad(P.param(0, base, 6), y, P.param(0, base, 8)));
    float ty = mad(P.param(0, base, 5), x, mad(P.param(0, base, 7), y, P.param(0, base, 9)));
    float sx = P.param(0, base, 0), sy = P.param(0, base, 1), ex = P.param(0, base, 2), ey = P.param(0, base, 3);
    float dx = ex - sx, dy = ey - sy;
    float den = dx * dx + dy * dy, t = 0.0f;
    if (den > GRADIENT_FLOAT_EPSILON) t = mad(tx - sx, dx, (ty - sy) * dy) / den;
    return sample_ramp(P, off, len, t, extend);
}
uint32_t sample_radial(const Paint& P, float x, float y, uint32_t base, uint32_t extend, uint32_t off, uint32_t len) {
    float tx = mad(P.param(0, base, 6), x, mad(P.param(0, base, 8), y, P.param(0, base, 10)));
    float ty = mad(P.param(0, base, 7), x, mad(P.param(0, base, 9), y, P.param(0, base, 11)));
    float sx = P.param(0, base, 0), sy = P.param(0, base, 1), ex = P.param(0, base, 2), ey = P.param(0, base, 3);
    float sr = P.param(0, base, 4), er = P.param(0, base, 5);
    float qx = tx - sx, qy = ty - sy, dcx = ex - sx, dcy = ey - sy, dr = er - sr;
    float a = mad(dcx, dcx, mad(dcy, dcy, -dr * dr));
    float b = -2.0f * mad(qx, dcx, mad(qy, dcy, sr * dr));
    float c = mad(qx, qx, mad(qy, qy, -sr * sr));
    bool has_t = false;
    float t = 0.0f;
    if (std::fabs(a) <= RADIAL_QUADRATIC_EPSILON) {
        if (std::fabs(b) > RADIAL_QUADRATIC_EPSILON) {
            float cand = -c / b;
            if (mad(cand, dr, sr) >= 0.0f) { has_t = true; t = cand; }
        }
    } else {
        float disc = mad(b, b, -4.0f * a * c);
        if (disc >= 0.0f) {
            float root = std::sqrt(disc);
            float t0 = (-b - root) / (2.0f * a), t1 = (-b + root) / (2.0f * a);
            bool v0 = mad(t0, dr, sr) >= 0.0f, v1 = mad(t1, dr, sr) >= 0.0f;
            if (v0) { has_t = true; t = v1 ? fmax_(t0, t1) : t0; }
            else if (v1) { has_t = true; t = t1; }
        }
    }
    return has_t ? sample_ramp(P, off, len, t, extend) : 0u;
}
// --- shared/brush/pattern.hlsli:9-17, texture.hlsli:7-31, pattern_transform.hlsli:7-11 ---
uint32_t extend_coord_i32(int32_t value, uint32_t size, uint32_t extend) {
    if (size <= 1u) return 0u;
    if (extend == TK_EXTEND_REPEAT || extend == TK_EXTEND_REFLECT) {
        uint32_t period = size * (extend == TK_EXTEND_REFLECT ? 2u : 1u);
        // euclidean_remainder_i32 (shared/integer.hlsli:5-9)
        uint32_t magnitude = value < 0 ? 0u - uint32_t(value) : uint32_t(value);
        uint32_t remainder = magnitude % period;
        uint32_t coord = value < 0 && remainder != 0u ? period - remainder : remainder;
        return coord < size ? coord : period - coord - 1u;
    }
    return uint32_t(std::min(std::max(value, 0), int32_t(size) - 1));
}
float pattern_transform_component(float a, float b, float offset, float x, float y) {
    float by = b * y;
    float dot_product = mad(a, x, by) + mad(b, y, -by);
    return dot_product + offset;
}
uint32_t texel(const tk_image_desc& im, uint32_t col, uint32_t row) {
    return im.premul_rgba8[uint64_t(row) * im.width + col];
}
F4 lerp_unorm(F4 a, F4 b, float t) {
    return {mad(b.r - a.r, t, a.r), mad(b.g - a.g, t, a.g), mad(b.b - a.b, t, a.b), mad(b.a - a.a, t, a.a)};
}
// sample_resource_pattern_texture. The bilinear pad-extended form is the
// texture unit's filter there (SampleLevel, clamp-to-edge addressing), restated
// as the exact filter: texel centres at half-integers, f32 weights, one
// rounding to 8 bits.
uint32_t sample_pattern_texture(const tk_image_desc& im, float px, float py, uint32_t opacity, uint32_t extend,
                                uint32_t sampling) {
    const uint32_t w = im.width, h = im.height;
    uint32_t color;
    if (sampling == TK_PATTERN_BILINEAR && extend == TK_EXTEND_PAD) {
        float sx = clampf(px, 0.0f, float(w)) - 0.5f, sy = clampf(py, 0.0f, float(h)) - 0.5f;
        float bx = std::floor(sx), by = std::floor(sy), fx = sx - bx, fy = sy - by;
        int32_t ix = f2i(bx), iy = f2i(by);
        auto cl = [](int32_t v, uint32_t n) { return uint32_t(std::min(std::max(v, 0), int32_t(n) - 1)); };
        uint32_t x0 = cl(ix, w), x1 = cl(ix + 1, w), y0 = cl(iy, h), y1 = cl(iy + 1, h);
        F4 top = lerp_unorm(rgba8_to_unorm(texel(im, x0, y0)), rgba8_to_unorm(texel(im, x1, y0)), fx);
        F4 bot = lerp_unorm(rgba8_to_unorm(texel(im, x0, y1)), rgba8_to_unorm(texel(im, x1, y1)), fx);
        color = unorm_to_rgba8(lerp_unorm(top, bot, fy));
    } else if (sampling == TK_PATTERN_BILINEAR) {
        float sx = px - 0.5f, sy = py - 0.5f;
        float bx = std::floor(sx), by = std::floor(sy), fx = sx - bx, fy = sy - by;
        int32_t ix = f2i(bx), iy = f2i(by);
        int32_t jx = int32_t(uint32_t(ix) + 1u), jy = int32_t(uint32_t(iy) + 1u);
        uint32_t tl = texel(im, extend_coord_i32(ix, w, extend), extend_coord_i32(iy, h, extend));
        uint32_t tr = texel(im, extend_coord_i32(jx, w, extend), extend_coord_i32(iy, h, extend));
        uint32_t bl = texel(im, extend_coord_i32(ix, w, extend), extend_coord_i32(jy, h, extend));
        uint32_t br = texel(im, extend_coord_i32(jx, w, extend), extend_coord_i32(jy, h, extend));
        color = lerp_premul_u8(lerp_premul_u8(tl, tr, fx), lerp_premul_u8(bl, br, fx), fy);
    } else {
        color = texel(im, extend_coord_i32(f2i(std::floor(px)), w, extend),
                      extend_coord_i32(f2i(std::floor(py)), h, extend));
    }
    return scale_premul_u8(color, opacity);
}

uint32_t sample_draw_brush(const Paint& P, const tk_draw_record& d, float x, float y) {
    if (P.word(0u, d.brush_offset) == TK_BRUSH_SOLID) return P.word(0u, d.brush_offset + TK_BRUSH_COLOR_WORD);
    const tk_affine& m = d.inverse_transform;
    float lx = mad(m.a, x, mad(m.c, y, m.e));
    float ly = mad(m.b, x, mad(m.d, y, m.f));
    uint32_t db = d.brush_offset;
    uint32_t kind = P.word(0u, db), extend = P.word(0u, db + 1u);
    uint32_t payload = db + P.word(0u, db + 2u), len = P.word(0u, db + 3u);
    uint32_t base = db + TK_BRUSH_HEADER_WORDS;
    uint32_t color = P.word(0u, db + TK_BRUSH_COLOR_WORD);
    if (kind == TK_BRUSH_LINEAR) return sample_linear(P, lx, ly, base, extend, payload, len);
    if (kind == TK_BRUSH_RADIAL) return sample_radial(P, lx, ly, base, extend, payload, len);
    if (kind == 6u) return 0u;  // BRUSH_PATTERN
    if (kind != TK_BRUSH_PATTERN_RESOURCE) return color;  // other kinds are outside this path
    // sample_brush's texture-table branch (shared/brush/sample.hlsli:32-41)
    uint32_t placement = P.word(0u, db + 4u), w = P.word(0u, db + 5u), h = P.word(0u, db + 6u);
    if (w == 0u || h == 0u) return 0u;
    uint32_t index = placement & ~TK_BRUSH_TEXTURE_PLACEMENT_BIT;
    if (!(placement & TK_BRUSH_TEXTURE_PLACEMENT_BIT) || index >= P.image_count) return 0u;
    float tx = pattern_transform_component(P.param(0u, base, 0u), P.param(0u, base, 2u), P.param(0u, base, 4u), lx, ly) * float(w);
    float ty = pattern_transform_component(P.param(0u, base, 1u), P.param(0u, base, 3u), P.param(0u, base, 5u), lx, ly) * float(h);
    return sample_pattern_texture(P.images[index], tx, ty, P.word(0u, db + TK_BRUSH_IMAGE_ALPHA_WORD), extend,
                                  P.word(0u, db + 8u));
}


// ---------------------------------------------------------------------------
// SDF shapes (shared/sdf/{base,basic,line,coverage}.hlsli). `length` is
// sqrt(x*x + y*y) unfused; `mad` sites are fused as everywhere in this file.
// ---------------------------------------------------------------------------
struct SdfS { float dist, nx, ny; };

// shared/sdf/base.hlsli:7-12
float sdf_len(float x, float y) {
    float m = std::sqrt(x * x + y * y);
    if (m > 0.0f && std::isfinite(m)) return m;
    float axis = fmax_(std::fabs(x), std::fabs(y));
    if (axis == 0.0f) return 0.0f;
    float sx = x / axis, sy = y / axis;
    return axis * std::sqrt(sx * sx + sy * sy);
}
// shared/sdf/base.hlsli:14-23
void sdf_unit_or(float x, float y, float fx, float fy, float& ox, float& oy) {
    float m = std::sqrt(x * x + y * y);
    if (m > 0.0f && std::isfinite(m)) { ox = x / m; oy = y / m; return; }
    float axis = fmax_(std::fabs(x), std::fabs(y));
    if (axis == 0.0f) { ox = fx; oy = fy; return; }
    float sx = x / axis, sy = y / axis, l = std::sqrt(sx * sx + sy * sy);
    ox = sx / l;
    oy = sy / l;
}
// shared/sdf/basic.hlsli:6-19
SdfS sdf_rounded_box(float px, float py, float hx, float hy, float radius) {
    float qx = std::fabs(px) - hx + radius, qy = std::fabs(py) - hy + radius;
    float ox = fmax_(qx, 0.0f), oy = fmax_(qy, 0.0f);
    float ol = sdf_len(ox, oy);
    float dist = fmin_(fmax_(qx, qy), 0.0f) + ol - radius;
    float sgx = px >= 0.0f ? 1.0f : -1.0f, sgy = py >= 0.0f ? 1.0f : -1.0f;
    if (ol > 0.0f) return {dist, ox / ol * sgx, oy / ol * sgy};
    if (qx > qy) return {dist, sgx, 0.0f};
    return {dist, 0.0f, sgy};
}
// shared/sdf/basic.hlsli:21-25
SdfS sdf_line_rect(float axis, float normal, float x0, float x1, float hh) {
    float center = (x0 + x1) * 0.5f, hw = (x1 - x0) * 0.5f;
    return sdf_rounded_box(axis - center, normal, hw, hh, 0.0f);
}
// shared/sdf/basic.hlsli:27-32
SdfS sdf_circle(float x, float y, float cx, float cy, float radius) {
    float dx = x - cx, dy = y - cy;
    SdfS r;
    r.dist = sdf_len(dx, dy) - radius;
    sdf_unit_or(dx, dy, 1.0f, 0.0f, r.nx, r.ny);
    return r;
}
// shared/sdf/basic.hlsli:34-57
SdfS sdf_rect(float x, float y, float x0r, float y0r, float x1r, float y1r, float tl, float tr, float bl, float br) {
    float x0 = fmin_(x0r, x1r), y0 = fmin_(y0r, y1r), x1 = fmax_(x0r, x1r), y1 = fmax_(y0r, y1r);
    float cx = (x0 + x1) * 0.5f, cy = (y0 + y1) * 0.5f, hx = (x1 - x0) * 0.5f, hy = (y1 - y0) * 0.5f;
    float px = x - cx, py = y - cy;
    float radius = tl;
    if (px >= 0.0f) {
        radius = py <= 0.0f ? tr : br;
    } else if (py > 0.0f) {
        radius = bl;
    }
    return sdf_rounded_box(px, py, hx, hy, fmax_(fmin_(fmin_(radius, hx), hy), 0.0f));
}
// shared/sdf/line.hlsli:8-14, 41-76
SdfS sdf_line(float x, float y, float sx, float sy, float ex, float ey, float width, float cap) {
    float he = fmax_(width, 0.0f) * 0.5f;
    float dx = ex - sx, dy = ey - sy;
    float len = sdf_len(dx, dy);
    SdfS r{std::numeric_limits<float>::infinity(), 1.0f, 0.0f};
    if (len == 0.0f) {
        if (cap >= 0.5f) {
            if (cap > 1.5f) {
                float ax = x - sx, ay = y - sy;
                r.dist = sdf_len(ax, ay) - he;
                sdf_unit_or(ax, ay, 1.0f, 0.0f, r.nx, r.ny);
            } else {
                r = sdf_line_rect(x - sx, y - sy, -he, he, he);
            }
        }
        return r;
    }
    float ux = dx / len, uy = dy / len;
    float px = x - sx, py = y - sy;
    float axis = px * ux + py * uy;
    float normal = -px * uy + py * ux;
    if (cap < 0.5f) {
        r = sdf_line_rect(axis, normal, 0.0f, len, he);
    } else if (cap < 1.5f) {
        r = sdf_line_rect(axis, normal, -he, len + he, he);
    } else {
        float nearest = clampf(axis, 0.0f, len);
        float ax = axis - nearest;
        r.dist = sdf_len(ax, normal) - he;
        sdf_unit_or(ax, normal, 0.0f, 1.0f, r.nx, r.ny);
    }
    return {r.dist, r.nx * ux - r.ny * uy, r.nx * uy + r.ny * ux};
}
// shared/sdf/base.hlsli:39-52
float sdf_cov(const SdfS& s, const tk_affine& inv) {
    float gx = mad(inv.a, s.nx, inv.b * s.ny);
    float gy = mad(inv.c, s.nx, inv.d * s.ny);
    float fp = sdf_len(gx, gy);
    if (fp == 0.0f) return s.dist < 0.0f ? 1.0f : (s.dist > 0.0f ? 0.0f : 0.5f);
    return clampf(0.5f - s.dist / fp, 0.0f, 1.0f);
}
// The library evaluates the shadow falloff exp(x), x <= 0, in double as
// 2^k * e^r (k nearest to x / ln 2, e^r by its degree-12 Taylor polynomial in
// Horner form) with only exactly rounded multiplies and adds; restated so
// that the two agree bit for bit. Its distance to exp is checked in the tests.
float exp_nonpos(float x) {
    if (!(x <= 0.0f)) return x != x ? x : 1.0f;
    if (x < -104.0f) return 0.0f;
    const double ln2 = 0.69314718055994530942, inv_ln2 = 1.4426950408889634074;
    double xd = double(x);
    double k = std::floor(xd * inv_ln2 + 0.5);
    double r = xd - k * ln2;
    const double c[11] = {1.0 / 479001600.0, 1.0 / 39916800.0, 1.0 / 3628800.0, 1.0 / 362880.0, 1.0 / 40320.0,
                          1.0 / 5040.0,      1.0 / 720.0,       1.0 / 120.0,     1.0 / 24.0,     1.0 / 6.0,
                          0.5};
    double p = c[0];
    for (int n = 1; n < 11; ++n) p = p * r + c[n];
    p = p * r + 1.0;
    p = p * r + 1.0;
    int64_t bits = int64_t(1023 + int64_t(k)) << 52;
    double scale;
    std::memcpy(&scale, &bits, sizeof(scale));
    return float(p * scale);
}
// shared/sdf/base.hlsli:54-62
float sdf_shadow_cov(const SdfS& s, const tk_affine& inv, float expand, float intensity) {
    float ci = clampf(intensity, 0.0f, 1.0f);
    if (expand > 0.0f) return clampf(exp_nonpos(-fmax_(s.dist, 0.0f) / expand) * ci, 0.0f, 1.0f);
    return sdf_cov(s, inv) * ci;
}
// nearer_sdf_sample / farther_sdf_sample (shared/sdf/base.hlsli:25-37)
SdfS sdf_nearer(const SdfS& a, const SdfS& b) { return a.dist <= b.dist ? a : b; }
SdfS sdf_farther(const SdfS& a, const SdfS& b) { return a.dist >= b.dist ? a : b; }
// distance_to_segment_sdf_sample (shared/sdf/polygon.hlsli:7-26)
SdfS sdf_segment(float px, float py, float ax, float ay, float bx, float by, float fx, float fy) {
    float dx = bx - ax, dy = by - ay;
    float len2 = dx * dx + dy * dy;
    float nx = ax, ny = ay;
    if (len2 >= 1.175494351e-38f && std::isfinite(len2)) {
        float t = clampf(((px - ax) * dx + (py - ay) * dy) / len2, 0.0f, 1.0f);
        nx = ax + dx * t;
        ny = ay + dy * t;
    } else {
        float axis = fmax_(std::fabs(dx), std::fabs(dy));
        if (axis > 0.0f) {
            float sx = dx / axis, sy = dy / axis;
            float dot = sx * sx + sy * sy;
            float qx = sx / dot, qy = sy / dot;
            float t = clampf(((px - ax) * qx + (py - ay) * qy) / axis, 0.0f, 1.0f);
            nx = ax + dx * t;
            ny = ay + dy * t;
        }
    }
    SdfS r;
    r.dist = sdf_len(px - nx, py - ny);
    sdf_unit_or(px - nx, py - ny, fx, fy, r.nx, r.ny);
    return r;
}
// triangle_sdf_sample (shared/sdf/polygon.hlsli:32-85)
SdfS sdf_triangle(float x, float y, float ax, float ay, float bx, float by, float cx, float cy, float corner) {
    float abx = bx - ax, aby = by - ay, bcx = cx - bx, bcy = cy - by, cax = ax - cx, cay = ay - cy;
    float tb[2] = {bx - ax, by - ay}, tc[2] = {cx - ax, cy - ay}, tp[2] = {x - ax, y - ay};
    auto cross = [](float a0, float a1, float b0, float b1) { return a0 * b1 - a1 * b0; };
    float area = cross(tb[0], tb[1], tc[0], tc[1]);
    float lo[2] = {fmin_(fmin_(ax, bx), cx), fmin_(fmin_(ay, by), cy)};
    float hi[2] = {fmax_(fmax_(ax, bx), cx), fmax_(fmax_(ay, by), cy)};
    if (area == 0.0f || !std::isfinite(area)) {
        float span[2] = {hi[0] - lo[0], hi[1] - lo[1]};
        if (span[0] > 0.0f && span[1] > 0.0f) {
            for (int k = 0; k < 2; ++k) { tb[k] /= span[k]; tc[k] /= span[k]; tp[k] /= span[k]; }
            area = cross(tb[0], tb[1], tc[0], tc[1]);
        }
    }
    float o = area >= 0.0f ? 1.0f : -1.0f;
    float n[3][2];
    sdf_unit_or(aby * o, -abx * o, 1.0f, 0.0f, n[0][0], n[0][1]);
    sdf_unit_or(bcy * o, -bcx * o, 1.0f, 0.0f, n[1][0], n[1][1]);
    sdf_unit_or(cay * o, -cax * o, 1.0f, 0.0f, n[2][0], n[2][1]);
    SdfS r = sdf_nearer(sdf_segment(x, y, ax, ay, bx, by, n[0][0], n[0][1]),
                        sdf_segment(x, y, bx, by, cx, cy, n[1][0], n[1][1]));
    r = sdf_nearer(r, sdf_segment(x, y, cx, cy, ax, ay, n[2][0], n[2][1]));
    float side_ab = cross(tb[0], tb[1], tp[0], tp[1]) * o;
    float side_bc = cross(tc[0] - tb[0], tc[1] - tb[1], tp[0] - tb[0], tp[1] - tb[1]) * o;
    float side_ca = cross(-tc[0], -tc[1], tp[0] - tc[0], tp[1] - tc[1]) * o;
    if (area != 0.0f && x >= lo[0] && y >= lo[1] && x <= hi[0] && y <= hi[1] && side_ab >= 0.0f && side_bc >= 0.0f &&
        side_ca >= 0.0f)
        r = {-r.dist, -r.nx, -r.ny};
    return {r.dist - fmax_(corner, 0.0f), r.nx, r.ny};
}
// callout_sdf_sample (shared/sdf/polygon.hlsli:87-136)
SdfS sdf_callout(float x, float y, float x0r, float y0r, float x1r, float y1r, float body_radius, float tail_offset,
                 float tail_width, float tail_length, float tail_radius, float side, float visible) {
    float x0 = fmin_(x0r, x1r), y0 = fmin_(y0r, y1r), x1 = fmax_(x0r, x1r), y1 = fmax_(y0r, y1r);
    SdfS body = sdf_rect(x, y, x0, y0, x1, y1, body_radius, body_radius, body_radius, body_radius);
    if (visible < 0.5f) return body;
    bool vertical = side < 0.5f || (side >= 1.5f && side < 2.5f);
    float span = vertical ? x1 - x0 : y1 - y0;
    float width = fmin_(fmax_(tail_width, 0.0f), span);
    float half = width * 0.5f;
    float center = clampf(tail_offset, half, fmax_(span - half, half));
    float radius = clampf(tail_radius, 0.0f, fmin_(fmax_(half * 0.499f, 0.0f), fmax_(tail_length * 0.499f, 0.0f)));
    float sh = half - radius, sl = tail_length - radius;
    float a[2] = {x0 + center - sh, y0}, b[2] = {x0 + center + sh, y0}, c[2] = {x0 + center, y0 - sl};
    if (side >= 0.5f && side < 1.5f) {
        a[0] = x1; a[1] = y0 + center - sh; b[0] = x1; b[1] = y0 + center + sh; c[0] = x1 + sl; c[1] = y0 + center;
    } else if (side >= 1.5f && side < 2.5f) {
        a[0] = x0 + center - sh; a[1] = y1; b[0] = x0 + center + sh; b[1] = y1; c[0] = x0 + center; c[1] = y1 + sl;
    } else if (side >= 2.5f) {
        a[0] = x0; a[1] = y0 + center - sh; b[0] = x0; b[1] = y0 + center + sh; c[0] = x0 - sl; c[1] = y0 + center;
    }
    return sdf_nearer(body, sdf_triangle(x, y, a[0], a[1], b[0], b[1], c[0], c[1], radius));
}
// The library's sin, cos and atan2 for the arc and star kinds, in double with
// exactly rounded operations (Cody-Waite reduction by pi/2 with fdlibm's
// two-part constant and Taylor polynomials of degree 19 / 18; atan by
// reduction to |t| <= tan(pi/12) and its odd series to degree 27); restated so
// that the two agree bit for bit. Their distance to the C library is checked
// in the tests.
void lib_sincos(float a, float& s, float& c) {
    double x = double(a);
    if (!(std::fabs(x) < 1.0e9)) {
        s = c = std::numeric_limits<float>::quiet_NaN();
        return;
    }
    const double pio2_hi = 1.57079632673412561417e+00, pio2_lo = 6.07710050650619224932e-11;
    double k = std::floor(x * 0.63661977236758134308 + 0.5);
    double r = (x - k * pio2_hi) - k * pio2_lo, r2 = r * r;
    static const double sin_c[10] = {-1.0 / 121645100408832000.0, 1.0 / 355687428096000.0, -1.0 / 1307674368000.0,
                                     1.0 / 6227020800.0, -1.0 / 39916800.0, 1.0 / 362880.0, -1.0 / 5040.0,
                                     1.0 / 120.0, -1.0 / 6.0, 1.0};
    static const double cos_c[9] = {1.0 / 6402373705728000.0, -1.0 / 20922789888000.0, 1.0 / 87178291200.0,
                                    -1.0 / 479001600.0, 1.0 / 3628800.0, -1.0 / 40320.0, 1.0 / 720.0, -1.0 / 24.0,
                                    0.5};
    double ps = sin_c[0];
    for (int i = 1; i < 10; ++i) ps = ps * r2 + sin_c[i];
    double pc = cos_c[0];
    for (int i = 1; i < 9; ++i) pc = pc * r2 + cos_c[i];
    double sr = ps * r, cr = 1.0 - pc * r2;
    int q = int(std::fmod(k, 4.0) + 4.0) & 3;
    double vs[4] = {sr, cr, -sr, -cr}, vc[4] = {cr, -sr, -cr, sr};
    s = float(vs[q]);
    c = float(vc[q]);
}
float lib_atan2(float yf, float xf) {
    double y = double(yf), x = double(xf), ax = std::fabs(x), ay = std::fabs(y);
    bool swap = ay > ax;
    double z = swap ? ax / ay : ay / ax;
    const double sqrt3 = 1.73205080756887729353, pi6 = 0.52359877559829887308;
    const double pi2 = 1.57079632679489661923, pi = 3.14159265358979323846;
    bool reduce = z > 0.26794919243112270647;
    double t = reduce ? (z * sqrt3 - 1.0) / (z + sqrt3) : z, t2 = t * t;
    double p = 1.0 / 27.0;
    for (int n = 25; n >= 1; n -= 2) p = p * t2 * -1.0 + 1.0 / double(n);
    double a = p * t;
    if (reduce) a = pi6 + a;
    if (swap) a = pi2 - a;
    if (x < 0.0) a = pi - a;
    if (y < 0.0) a = -a;
    return float(a);
}
// arc.hlsli:10-16
bool arc_in_sweep(float angle, float start, float sweep) {
    const float tau = 6.2831855f;
    if (sweep >= 0.0f) return rem_euclid_f32(angle - start, tau) <= sweep;
    return rem_euclid_f32(start - angle, tau) <= -sweep;
}
// arc.hlsli:18-34
SdfS arc_cap_segment(float vx, float vy, float radius, float angle, float he, float sweep, bool end_cap) {
    float inner = fmax_(radius - he, 0.0f), outer = radius + he, si, co;
    lib_sincos(angle, si, co);
    float dir = sweep >= 0.0f ? 1.0f : -1.0f;
    float tx = -si * dir, ty = co * dir;
    return sdf_segment(vx, vy, inner * co, inner * si, outer * co, outer * si, end_cap ? tx : -tx, end_cap ? ty : -ty);
}
// arc.hlsli:36-41
SdfS arc_endpoint(float vx, float vy, float radius, float angle, float he) {
    float si, co;
    lib_sincos(angle, si, co);
    float dx = vx - radius * co, dy = vy - radius * si;
    SdfS r;
    r.dist = sdf_len(dx, dy) - he;
    sdf_unit_or(dx, dy, co, si, r.nx, r.ny);
    return r;
}
// arc.hlsli:66-85
SdfS arc_square_cap(float vx, float vy, float radius, float angle, float sweep, float x0, float x1, float he) {
    float dir = sweep < 0.0f ? -1.0f : 1.0f, si, co;
    lib_sincos(angle, si, co);
    float tx = -si * dir, ty = co * dir;
    float px = vx - radius * co, py = vy - radius * si;
    SdfS l = sdf_line_rect(px * tx + py * ty, -px * ty + py * tx, x0, x1, he);
    return {l.dist, l.nx * tx - l.ny * ty, l.nx * ty + l.ny * tx};
}
// arc_sdf_sample with arc_butt_sdf_sample (arc.hlsli:43-64, 87-123)
SdfS sdf_arc(float x, float y, float cx, float cy, float radius_raw, float width_raw, float start, float sweep,
             float cap) {
    float radius = fmax_(radius_raw, 0.0f), width = fmax_(width_raw, 0.0f);
    SdfS s{std::numeric_limits<float>::infinity(), 1.0f, 0.0f};
    if (!(radius > 0.0f && width > 0.0f && sweep != 0.0f)) return s;
    float vx = x - cx, vy = y - cy, len = sdf_len(vx, vy), he = width * 0.5f;
    if (std::fabs(sweep) >= 6.2831855f) {
        float nx, ny;
        sdf_unit_or(vx, vy, 1.0f, 0.0f, nx, ny);
        float sg = len >= radius ? 1.0f : -1.0f;
        return {std::fabs(len - radius) - he, nx * sg, ny * sg};
    }
    auto caps = [&]() {
        return sdf_nearer(arc_cap_segment(vx, vy, radius, start, he, sweep, false),
                          arc_cap_segment(vx, vy, radius, start + sweep, he, sweep, true));
    };
    if (len == 0.0f) {
        s = caps();
    } else {
        float angle = lib_atan2(vy, vx);
        if (arc_in_sweep(angle, start, sweep)) {
            float sg = len >= radius ? 1.0f : -1.0f;
            s = {std::fabs(len - radius) - he, vx / len * sg, vy / len * sg};
        } else {
            s = caps();
        }
    }
    if (cap > 1.5f) {
        s = sdf_nearer(sdf_nearer(s, arc_endpoint(vx, vy, radius, start, he)),
                       arc_endpoint(vx, vy, radius, start + sweep, he));
    } else if (cap >= 0.5f) {
        s = sdf_nearer(sdf_nearer(s, arc_square_cap(vx, vy, radius, start, sweep, -he, 0.0f, he)),
                       arc_square_cap(vx, vy, radius, start + sweep, sweep, 0.0f, he, he));
    }
    return s;
}
// star_vertex / star_sdf_sample (polygon.hlsli:158-206)
SdfS sdf_star(float x, float y, float cx, float cy, float outer, float inner, float corner, float rotation) {
    float sn, cs;
    lib_sincos(rotation, sn, cs);
    float rx = x - cx, ry = y - cy;
    float px = cs * rx + sn * ry, py = -sn * rx + cs * ry;
    auto vertex = [&](uint32_t i, float& vx, float& vy) {
        float r = (i & 1u) == 0u ? outer : inner, vs, vc;
        lib_sincos(float(i) * 0.62831855f, vs, vc);
        vx = vc * r;
        vy = vs * r;
    };
    SdfS nearest{std::numeric_limits<float>::infinity(), 1.0f, 0.0f};
    bool inside = false;
    float qx, qy;
    vertex(9u, qx, qy);
    for (uint32_t i = 0; i < 10u; ++i) {
        float ux, uy;
        vertex(i, ux, uy);
        float ex = ux - qx, ey = uy - qy, fx, fy;
        sdf_unit_or(ey, -ex, 1.0f, 0.0f, fx, fy);
        nearest = sdf_nearer(nearest, sdf_segment(px, py, qx, qy, ux, uy, fx, fy));
        if ((qy > py) != (uy > py)) {
            float fraction = (py - qy) / (uy - qy);
            float crossing = qx + fraction * (ux - qx);
            if (px < crossing) inside = !inside;
        }
        qx = ux;
        qy = uy;
    }
    if (inside) nearest = {-nearest.dist, -nearest.nx, -nearest.ny};
    return {nearest.dist - fmax_(corner, 0.0f), cs * nearest.nx - sn * nearest.ny, sn * nearest.nx + cs * nearest.ny};
}
// checkerboard_sdf_sample (shared/sdf/effects.hlsli:8-36)
SdfS sdf_checkerboard(float x, float y, float x0, float y0, float x1, float y1, float cell_raw) {
    float left = fmin_(x0, x1), top = fmin_(y0, y1), right = fmax_(x0, x1), bottom = fmax_(y0, y1);
    SdfS outer = sdf_rect(x, y, left, top, right, bottom, 0.0f, 0.0f, 0.0f, 0.0f);
    float cell = fmax_(cell_raw, 0.000001f);
    float cell_x = std::floor((x - left) / cell), cell_y = std::floor((y - top) / cell);
    float lx = rem_euclid_f32(x - left, cell), ly = rem_euclid_f32(y - top, cell);
    float e = lx, nx = 1.0f, ny = 0.0f;
    if (cell - lx < e) { e = cell - lx; nx = -1.0f; ny = 0.0f; }
    if (ly < e) { e = ly; nx = 0.0f; ny = 1.0f; }
    if (cell - ly < e) { e = cell - ly; nx = 0.0f; ny = -1.0f; }
    // (int(cell_x) + int(cell_y)) % 2 == 0, as two's complement parity
    bool filled = ((uint32_t(f2i(cell_x)) + uint32_t(f2i(cell_y))) & 1u) == 0u;
    return sdf_farther(outer, {filled ? -e : e, nx, ny});
}
// line_segment_sdf_sample (shared/sdf/line.hlsli:16-26)
SdfS sdf_line_segment(float axis, float normal, float start, float end, float he, float cap) {
    float nearest = clampf(axis, start, end);
    SdfS r;
    r.dist = sdf_len(axis - nearest, normal) - he;
    sdf_unit_or(axis - nearest, normal, 0.0f, 1.0f, r.nx, r.ny);
    if (cap < 0.5f) r = sdf_line_rect(axis, normal, start, end, he);
    else if (cap < 1.5f) r = sdf_line_rect(axis, normal, start - he, end + he, he);
    return r;
}
// dash_line_sdf_sample (shared/sdf/line.hlsli:28-39, 78-105)
SdfS sdf_dash_line(float x, float y, float sx, float sy, float ex, float ey, float width, float cap, float dash_raw,
                   float gap_raw, float offset_raw) {
    float dash = fmax_(dash_raw, 0.0f), gap = fmax_(gap_raw, 0.0f);
    SdfS r = sdf_line(x, y, sx, sy, ex, ey, width, cap);
    if (dash > 0.0f && gap > 0.0f) {
        float he = fmax_(width, 0.0f) * 0.5f;
        float dx = ex - sx, dy = ey - sy;
        float len = sdf_len(dx, dy);
        if (len > 0.0f) {
            float ux = dx / len, uy = dy / len, px = x - sx, py = y - sy;
            float axis = px * ux + py * uy;
            float normal = -px * uy + py * ux;
            float cycle = dash + gap;
            float offset = rem_euclid_f32(offset_raw, cycle);
            float base = std::floor((axis + offset) / cycle);
            auto seg = [&](float ix) {
                float s0 = ix * cycle - offset, s1 = s0 + dash;
                SdfS q{std::numeric_limits<float>::infinity(), 1.0f, 0.0f};
                if (s1 > 0.0f && s0 < len) {
                    float start = fmax_(s0, 0.0f), end = fmin_(s1, len);
                    if (end > start) q = sdf_line_segment(axis, normal, start, end, he, cap);
                }
                return q;
            };
            SdfS l = sdf_nearer(sdf_nearer(seg(base - 1.0f), seg(base)), seg(base + 1.0f));
            r = {l.dist, l.nx * ux - l.ny * uy, l.nx * uy + l.ny * ux};
        }
    }
    return r;
}
// sdf_coverage_from_blob (shared/sdf/coverage.hlsli:13-236) for the kinds the
// library accepts; others have no coverage.
float sdf_blob_coverage(const uint32_t* w, float x, float y, const tk_affine& inv) {
    auto f = [&](int i) { return bits_f(w[i]); };
    uint32_t kind = w[0];
    float x0 = f(1), y0 = f(2), x1 = f(3), y1 = f(4), r0 = f(5), r1 = f(6), r2 = f(7), r3 = f(8);
    float st = f(9), sr = f(10), sb = f(11), sl = f(12), ox = f(13), oy = f(14), ex = f(15), in = f(16);
    if (kind == TK_SDF_RECT) return sdf_cov(sdf_rect(x, y, x0, y0, x1, y1, r0, r1, r2, r3), inv);
    if (kind == TK_SDF_RECT_STROKE) {
        float ht = fmax_(st, 0.0f), hr = fmax_(sr, 0.0f), hb = fmax_(sb, 0.0f), hl = fmax_(sl, 0.0f);
        float rx0 = fmin_(x0, x1), ry0 = fmin_(y0, y1), rx1 = fmax_(x0, x1), ry1 = fmax_(y0, y1);
        float outer = sdf_cov(sdf_rect(x, y, rx0 - hl, ry0 - ht, rx1 + hr, ry1 + hb, r0 + fmax_(ht, hl),
                                       r1 + fmax_(ht, hr), r2 + fmax_(hb, hl), r3 + fmax_(hb, hr)),
                              inv);
        float ix0 = rx0 + hl, iy0 = ry0 + ht, ix1 = rx1 - hr, iy1 = ry1 - hb;
        float inner = 0.0f;
        if (ix0 < ix1 && iy0 < iy1)
            inner = sdf_cov(sdf_rect(x, y, ix0, iy0, ix1, iy1, fmax_(r0 - fmax_(ht, hl), 0.0f),
                                     fmax_(r1 - fmax_(ht, hr), 0.0f), fmax_(r2 - fmax_(hb, hl), 0.0f),
                                     fmax_(r3 - fmax_(hb, hr), 0.0f)),
                            inv);
        return clampf(outer - inner, 0.0f, 1.0f);
    }
    if (kind == TK_SDF_RECT_SHADOW)
        return sdf_shadow_cov(sdf_rect(x - ox, y - oy, x0, y0, x1, y1, r0, r1, r2, r3), inv, ex, in);
    if (kind == TK_SDF_CIRCLE) return sdf_cov(sdf_circle(x, y, x0, y0, x1), inv);
    if (kind == TK_SDF_CIRCLE_STROKE) {
        float he = fmax_(st, 0.0f), radius = fmax_(x1, 0.0f);
        float outer = sdf_cov(sdf_circle(x, y, x0, y0, radius + he), inv);
        float inner = radius > he ? sdf_cov(sdf_circle(x, y, x0, y0, radius - he), inv) : 0.0f;
        return clampf(outer - inner, 0.0f, 1.0f);
    }
    if (kind == TK_SDF_CIRCLE_SHADOW) return sdf_shadow_cov(sdf_circle(x - ox, y - oy, x0, y0, x1), inv, ex, in);
    if (kind == TK_SDF_LINE) return sdf_cov(sdf_line(x, y, x0, y0, x1, y1, r0, r1), inv);
    if (kind == TK_SDF_LINE_SHADOW)
        return sdf_shadow_cov(sdf_line(x - ox, y - oy, x0, y0, x1, y1, r0, r1), inv, ex, in);
    if (kind == TK_SDF_CANDLESTICK) {  // candlestick_sdf_coverage (shared/sdf/effects.hlsli:38-70)
        float cx = x0, high = y0, low = x1, top = y1, bottom = r0, body_w = r1, wick_w = r2;
        float wh = fmax_(wick_w, 1.0f) * 0.5f;
        float wick = sdf_cov(sdf_rect(x, y, cx - wh, fmin_(high, low), cx + wh, fmax_(high, low), 0, 0, 0, 0), inv);
        float bh = fmax_(body_w, 1.0f) * 0.5f;
        float by0 = fmin_(top, bottom), by1 = fmax_(top, bottom);
        if (by0 == by1) {
            by0 = by0 - 0.5f;
            by1 = by1 + 0.5f;
        }
        float body = sdf_cov(sdf_rect(x, y, cx - bh, by0, cx + bh, by1, 0, 0, 0, 0), inv);
        return fmax_(wick, body);
    }
    if (kind == TK_SDF_DASH_LINE) return sdf_cov(sdf_dash_line(x, y, x0, y0, x1, y1, r0, r1, r2, r3, st), inv);
    if (kind == TK_SDF_TRIANGLE) return sdf_cov(sdf_triangle(x, y, x0, y0, x1, y1, r0, r1, r2), inv);
    if (kind == TK_SDF_CHECKERBOARD) return sdf_cov(sdf_checkerboard(x, y, x0, y0, x1, y1, r0), inv);
    // callouts: words 9-12 tail radius, side, stroke half width, tail visible
    if (kind == TK_SDF_CALLOUT) return sdf_cov(sdf_callout(x, y, x0, y0, x1, y1, r0, r1, r2, r3, st, sr, sl), inv);
    if (kind == TK_SDF_CALLOUT_STROKE) {  // callout_stroke_sdf_sample (polygon.hlsli:138-156)
        SdfS c = sdf_callout(x, y, x0, y0, x1, y1, r0, r1, r2, r3, st, sr, sl);
        SdfS s{std::fabs(c.dist) - fmax_(sb, 0.0f), c.dist >= 0.0f ? c.nx : -c.nx, c.dist >= 0.0f ? c.ny : -c.ny};
        return sdf_cov(s, inv);
    }
    if (kind == TK_SDF_CALLOUT_SHADOW)
        return sdf_shadow_cov(sdf_callout(x - ox, y - oy, x0, y0, x1, y1, r0, r1, r2, r3, st, sr, sl), inv, ex, in);
    // arcs: centre, radius, width; start angle, sweep, cap
    if (kind == TK_SDF_ARC) return sdf_cov(sdf_arc(x, y, x0, y0, x1, y1, r0, r1, r2), inv);
    if (kind == TK_SDF_ARC_SHADOW) return sdf_shadow_cov(sdf_arc(x - ox, y - oy, x0, y0, x1, y1, r0, r1, r2), inv, ex, in);
    // stars: centre, outer and inner radius; corner radius, rotation; stroke half width
    if (kind == TK_SDF_STAR) return sdf_cov(sdf_star(x, y, x0, y0, x1, y1, r0, r1), inv);
    if (kind == TK_SDF_STAR_STROKE) {  // star_stroke_sdf_sample (polygon.hlsli:208-221)
        SdfS c = sdf_star(x, y, x0, y0, x1, y1, r0, r1);
        return sdf_cov({std::fabs(c.dist) - fmax_(st, 0.0f), c.dist >= 0.0f ? c.nx : -c.nx,
                        c.dist >= 0.0f ? c.ny : -c.ny},
                       inv);
    }
    return 0.0f;
}

// ---------------------------------------------------------------------------
// Scene state.
// ---------------------------------------------------------------------------
struct BatchStream {
    uint32_t batch;  // index into run's batch list
    uint32_t kind;   // kind | skip << 3
    std::vector<tk_ptcl_record> recs;  // reference stream including END
    // glyph indices of the stream's PTCL_GLYPH records, whose segment
    // ranges index this list (rebased onto the pass's glyph list on output)
    std::vector<uint32_t> glyphs;
};

struct Batch {
    uint32_t batch_id, layer_start, layer_end, pass;
    uint64_t total;  // PTCL records of this batch
};

template <class F>
void parallel_for(int threads, uint64_t n, F&& f) {
    if (threads <= 1 || n < 2) {
        for (uint64_t i = 0; i < n; ++i) f(i);
        return;
    }
    std::atomic<uint64_t> next{0};
    const uint64_t grain = std::max<uint64_t>(1, n / (uint64_t(threads) * 64));
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) {
        pool.emplace_back([&]() {
            for (;;) {
                uint64_t b = next.fetch_add(grain);
                if (b >= n) return;
                uint64_t e = std::min(n, b + grain);
                for (uint64_t i = b; i < e; ++i) f(i);
            }
        });
    }
    for (auto& th : pool) th.join();
}

struct PixelBox { uint32_t x0, y0, x1, y1; };

}  // namespace

struct or_scene {
    tk_scene_desc desc{};
    std::vector<tk_path_record> paths;
    std::vector<tk_draw_record> draws;
    std::vector<tk_layer_record> layers;
    std::vector<uint32_t> brush, batch_ids;
    std::vector<uint32_t> sdf, shadow;  // Canvas::sdf_blob, sdf_shadow_blob
    // the text blob
    std::vector<tk_glyph_run> glyph_runs;
    std::vector<tk_glyph> glyphs;
    std::vector<tk_glyph_image> glyph_images;
    std::vector<uint32_t> glyph_texels;
    uint32_t tw = 0, th = 0, T = 0;
    uint64_t B = 0, seg_capacity = 0;
    std::vector<int32_t> backdrops;
    std::vector<uint32_t> counts, cursors, bumps;
    std::vector<tk_segment_range> ranges;
    std::vector<tk_line_segment> segments;
    std::vector<std::vector<uint32_t>> bins;  // per tile draw indices, painter order
    std::vector<Batch> batches;
    // per pass: per tile, streams of the pass's batches touching the tile
    std::vector<std::vector<std::vector<BatchStream>>> pass_streams;
    std::vector<uint32_t> image;
    // coarse and fine cover the tile rows ty0 <= ty < ty1 with
    // (ty - ty0) % row_step == 0 (a band, or every row_step-th row)
    uint32_t ty0 = 0, ty1 = 0, row_step = 1;
    bool in_band(uint32_t ty) const { return ty >= ty0 && ty < ty1 && (ty - ty0) % row_step == 0u; }
    std::vector<uint32_t> band_tiles;  // the tiles of the rows in_band, row-major
    double times[7] = {0, 0, 0, 0, 0, 0, 0};
};

namespace {

using clk = std::chrono::steady_clock;
inline double since(clk::time_point t) { return std::chrono::duration<double>(clk::now() - t).count(); }

// --- shared/draw.hlsli:33-47 ------------------------------------------------------
inline uint32_t tile_min_(int32_t px, uint32_t lim) { return px > 0 ? std::min(uint32_t(px) / TK_TILE_SIZE, lim) : 0u; }
inline uint32_t tile_max_(int32_t px, uint32_t lim) {
    return px > 0 ? std::min((uint32_t(px) + TK_TILE_SIZE - 1u) / TK_TILE_SIZE, lim) : 0u;
}
inline bool draw_hits_tile(const tk_draw_record& d, uint32_t tx, uint32_t ty, uint32_t tw, uint32_t th) {
    uint32_t lx = tile_min_(d.pixel_bounds.x0, tw), ly = tile_min_(d.pixel_bounds.y0, th);
    uint32_t ux = tile_max_(d.pixel_bounds.x1, tw), uy = tile_max_(d.pixel_bounds.y1, th);
    return tx >= lx && ty >= ly && tx < ux && ty < uy;
}
inline uint32_t draw_backdrop(const or_scene& S, const tk_draw_record& d, uint32_t tx, uint32_t ty) {
    if (d.path_id == TK_INVALID_INDEX || d.tag > TK_DRAW_PATH_GLYPH || d.path_id >= S.paths.size() ||
        !draw_hits_tile(d, tx, ty, S.tw, S.th))
        return TK_INVALID_INDEX;
    const tk_path_record& p = S.paths[d.path_id];
    if (p.tile_x1 <= p.tile_x0 || tx < p.tile_x0 || ty < p.tile_y0 || tx >= p.tile_x1 || ty >= p.tile_y1)
        return TK_INVALID_INDEX;
    return p.data_offset + (ty - p.tile_y0) * (p.tile_x1 - p.tile_x0) + tx - p.tile_x0;
}

// --- coarse/classify.hlsli:11-33 ------------------------------------------------
inline bool has_sdf(const tk_draw_record& d);
bool sdf_clip_covers(const or_scene& S, const tk_draw_record& d, uint32_t tx, uint32_t ty);
uint32_t stack_wrapper_count(const or_scene& S, const Batch& b, uint32_t tx, uint32_t ty) {
    uint32_t count = 0;
    for (uint32_t i = b.layer_start; i < b.layer_end; ++i) {
        const tk_layer_record& L = S.layers[i];
        const tk_draw_record& d = S.draws[L.draw];
        if (has_sdf(d)) {  // SDF draws of layers are clips
            if (sdf_clip_covers(S, d, tx, ty)) continue;
            if (!draw_hits_tile(d, tx, ty, S.tw, S.th)) return TK_INVALID_INDEX;
            ++count;
            continue;
        }
        uint32_t bd = draw_backdrop(S, d, tx, ty);
        if (bd == TK_INVALID_INDEX) return TK_INVALID_INDEX;
        tk_segment_range r = S.ranges[bd];
        int32_t w = S.backdrops[bd];
        bool full = d.fill_rule == TK_FILL_EVEN_ODD ? (uint32_t(w) & 1u) != 0u : w != 0;
        if (L.tag == TK_LAYER_CLIP && r.start == r.end && full) continue;
        if (r.start == r.end && w == 0) return TK_INVALID_INDEX;
        ++count;
    }
    return count;
}
// coarse/emit_stack.hlsli:9-17
bool noop_stack_clip(const or_scene& S, const tk_layer_record& L, const tk_draw_record& d, uint32_t tx, uint32_t ty) {
    if (L.tag != TK_LAYER_CLIP) return false;
    if (has_sdf(d)) return sdf_clip_covers(S, d, tx, ty);
    uint32_t bd = draw_backdrop(S, d, tx, ty);
    tk_segment_range r = S.ranges[bd];
    uint32_t w = uint32_t(S.backdrops[bd]);
    return r.start == r.end && (d.fill_rule == TK_FILL_EVEN_ODD ? (w & 1u) != 0u : w != 0u);
}


// --- coarse/sdf_clip.hlsli:8-56 and coarse/paint.hlsli:13-40 -------------------
bool rounded_corner_covers(float px, float py, float cx, float cy, float ccx, float ccy, float radius, float inset) {
    bool in_square = radius > 0.0f && std::fabs(px - cx) < radius && std::fabs(py - cy) < radius;
    float inner = radius - inset;
    float dx = px - ccx, dy = py - ccy;
    return !in_square || (inner > 0.0f && dx * dx + dy * dy <= inner * inner);
}
bool rect_covers_tile(const float rect[4], const float radii_in[4], const tk_draw_record& d, uint32_t tx, uint32_t ty,
                      float inset) {
    float lx = fmin_(rect[0], rect[2]), ly = fmin_(rect[1], rect[3]);
    float ux = fmax_(rect[0], rect[2]), uy = fmax_(rect[1], rect[3]);
    float tlx = float(tx * TK_TILE_SIZE) + 0.5f - d.transform.e, tly = float(ty * TK_TILE_SIZE) + 0.5f - d.transform.f;
    float tux = tlx + float(TK_TILE_SIZE - 1u), tuy = tly + float(TK_TILE_SIZE - 1u);
    float sx = ux - lx, sy = uy - ly;
    float need = float(TK_TILE_SIZE - 1u) + 2.0f * inset;
    if (sx < need || sy < need || tlx < lx + inset || tly < ly + inset || tux > ux - inset || tuy > uy - inset)
        return false;
    float limit = fmin_(sx, sy) * 0.5f;
    for (int k = 0; k < 4; ++k)
        if (!(std::fabs(rect[k]) <= 65536.0f) || !(std::fabs(radii_in[k]) <= 65536.0f)) return false;
    if (!(std::fabs(d.transform.e) <= 65536.0f) || !(std::fabs(d.transform.f) <= 65536.0f)) return false;
    float q[4];
    for (int k = 0; k < 4; ++k) q[k] = fmin_(fmax_(radii_in[k], 0.0f), limit);
    return rounded_corner_covers(tlx, tly, lx, ly, lx + q[0], ly + q[0], q[0], inset) &&
           rounded_corner_covers(tux, tly, ux, ly, ux - q[1], ly + q[1], q[1], inset) &&
           rounded_corner_covers(tlx, tuy, lx, uy, lx + q[2], uy - q[2], q[2], inset) &&
           rounded_corner_covers(tux, tuy, ux, uy, ux - q[3], uy - q[3], q[3], inset);
}
inline bool identity_linear(const tk_draw_record& d) {
    return d.transform.a == 1.0f && d.transform.b == 0.0f && d.transform.c == 0.0f && d.transform.d == 1.0f;
}
inline bool has_sdf(const tk_draw_record& d) {
    return d.sdf_offset != TK_INVALID_INDEX || d.sdf_shadow_offset != TK_INVALID_INDEX;
}
bool sdf_clip_covers(const or_scene& S, const tk_draw_record& d, uint32_t tx, uint32_t ty) {
    if (d.sdf_offset == TK_INVALID_INDEX || d.sdf_shadow_offset != TK_INVALID_INDEX || d.sdf_len < 9u) return false;
    const uint32_t* w = S.sdf.data() + d.sdf_offset;
    if (w[0] != TK_SDF_RECT || !identity_linear(d)) return false;
    float rect[4], radii[4];
    for (int k = 0; k < 4; ++k) { rect[k] = bits_f(w[1 + k]); radii[k] = bits_f(w[5 + k]); }
    return rect_covers_tile(rect, radii, d, tx, ty, 0.5f);
}
bool sdf_stroke_empty(const or_scene& S, const tk_draw_record& d, uint32_t tx, uint32_t ty) {
    if (d.sdf_offset == TK_INVALID_INDEX || d.sdf_shadow_offset != TK_INVALID_INDEX || d.sdf_len < 13u ||
        !identity_linear(d))
        return false;
    const uint32_t* w = S.sdf.data() + d.sdf_offset;
    if (w[0] != TK_SDF_RECT_STROKE) return false;
    float rect[4], radii[4], stroke[4];
    for (int k = 0; k < 4; ++k) {
        rect[k] = bits_f(w[1 + k]);
        radii[k] = bits_f(w[5 + k]);
        stroke[k] = bits_f(w[9 + k]);
    }
    for (int k = 0; k < 4; ++k)
        if (!(std::fabs(rect[k]) <= 65536.0f) || !(std::fabs(radii[k]) <= 65536.0f) ||
            !(std::fabs(stroke[k]) <= 65536.0f))
            return false;
    float hw[4];
    for (int k = 0; k < 4; ++k) hw[k] = fmax_(stroke[k], 0.0f);  // top, right, bottom, left
    float lx = fmin_(rect[0], rect[2]), ly = fmin_(rect[1], rect[3]);
    float ux = fmax_(rect[0], rect[2]), uy = fmax_(rect[1], rect[3]);
    float inner[4] = {lx + hw[3], ly + hw[0], ux - hw[1], uy - hw[2]};
    if (inner[0] >= inner[2] || inner[1] >= inner[3]) return false;
    float corner[4] = {fmax_(hw[0], hw[3]), fmax_(hw[0], hw[1]), fmax_(hw[2], hw[3]), fmax_(hw[2], hw[1])};
    float r[4];
    for (int k = 0; k < 4; ++k) r[k] = fmax_(radii[k] - corner[k], 0.0f);
    return rect_covers_tile(inner, r, d, tx, ty, 1.0f);
}
bool nontransparent_solid(const or_scene& S, const tk_draw_record& d) {
    Paint P{S.brush.data(), S.brush.size(), S.desc.images, S.desc.image_count};
    return d.brush_offset != TK_INVALID_INDEX && P.word(0u, d.brush_offset) == TK_BRUSH_SOLID &&
           P.word(0u, d.brush_offset + TK_BRUSH_COLOR_WORD) != 0u;
}
bool solid_supported_sdf(const or_scene& S, const tk_draw_record& d) {
    if (!nontransparent_solid(S, d) || d.sdf_offset == TK_INVALID_INDEX || d.sdf_shadow_offset != TK_INVALID_INDEX ||
        d.sdf_len == 0u)
        return false;
    uint32_t kind = S.sdf[d.sdf_offset];
    return kind == TK_SDF_RECT || kind == 5u /* candlestick */ || kind == 14u /* checkerboard */;
}
// sdf_coverage_from_draw (fine/draw.hlsli:21-26)
float sdf_coverage_from_draw(const or_scene& S, const tk_draw_record& d, float x, float y) {
    const tk_affine& m = d.inverse_transform;
    float lx = mad(m.a, x, mad(m.c, y, m.e));
    float ly = mad(m.b, x, mad(m.d, y, m.f));
    if (d.sdf_offset != TK_INVALID_INDEX) return sdf_blob_coverage(S.sdf.data() + d.sdf_offset, lx, ly, m);
    if (d.sdf_shadow_offset != TK_INVALID_INDEX)
        return sdf_blob_coverage(S.shadow.data() + d.sdf_shadow_offset, lx, ly, m);
    return 0.0f;
}

struct Particle {
    bool valid = false;
    uint32_t tag = TK_PTCL_FILL, winding = 0, fill_rule = 0, seg0 = 0, seg1 = 0, color = 0;
    std::vector<uint32_t> glyphs;  // PTCL_GLYPH: the run's glyphs that meet the tile
};
// glyph_hits_tile over a run (coarse/text.hlsli:8-35): the glyphs whose
// image, a pixel wider each way, meets the tile under the draw transform
// (transformed_rect_hits_tile, shared/draw.hlsli:52-61).
void run_glyphs_in_tile(const or_scene& S, const tk_draw_record& d, uint32_t tx, uint32_t ty,
                        std::vector<uint32_t>& out) {
    const tk_glyph_run& run = S.glyph_runs[d.glyph_run_id];
    const tk_affine& t = d.transform;
    const float tlx = float(tx * TK_TILE_SIZE), tly = float(ty * TK_TILE_SIZE);
    for (uint32_t k = run.first; k < run.first + run.count; ++k) {
        const tk_glyph& g = S.glyphs[k];
        if (g.image == TK_INVALID_INDEX) continue;
        const tk_glyph_image& im = S.glyph_images[g.image];
        if (im.width == 0u || im.height == 0u) continue;
        const uint32_t lx = uint32_t(g.x) + uint32_t(im.left), ly = uint32_t(g.y) - uint32_t(im.top);
        const float x[2] = {float(int32_t(lx - 1u)), float(int32_t(lx + im.width + 1u))};
        const float y[2] = {float(int32_t(ly - 1u)), float(int32_t(ly + im.height + 1u))};
        float lox = 0, loy = 0, hix = 0, hiy = 0;
        // corners in the order rect.xy, rect.zy, rect.xw, rect.zw
        const int order[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
        float px[4], py[4];
        for (int c = 0; c < 4; ++c) {
            const float X = x[order[c][0]], Y = y[order[c][1]];
            px[c] = t.a * X + t.c * Y + t.e;
            py[c] = t.b * X + t.d * Y + t.f;
        }
        lox = fmin_(fmin_(px[0], px[1]), fmin_(px[2], px[3]));
        loy = fmin_(fmin_(py[0], py[1]), fmin_(py[2], py[3]));
        hix = fmax_(fmax_(px[0], px[1]), fmax_(px[2], px[3]));
        hiy = fmax_(fmax_(py[0], py[1]), fmax_(py[2], py[3]));
        if (lox < tlx + float(TK_TILE_SIZE) && loy < tly + float(TK_TILE_SIZE) && hix > tlx && hiy > tly)
            out.push_back(k);
    }
}
// coarse/emit_draw.hlsli:10-52 (path draws; coarse/paint.hlsli:14-21)
Particle draw_particle(const or_scene& S, const Batch& b, uint32_t di, uint32_t tx, uint32_t ty) {
    Particle r;
    if (di >= S.batch_ids.size() || S.batch_ids[di] != b.batch_id) return r;
    const tk_draw_record& d = S.draws[di];
    if (!S.glyph_runs.empty() && d.glyph_run_id != TK_INVALID_INDEX) {  // coarse/emit_draw.hlsli:15-22
        if (d.tag == TK_DRAW_BRUSH) {
            run_glyphs_in_tile(S, d, tx, ty, r.glyphs);
            r.valid = !r.glyphs.empty();
            r.tag = TK_PTCL_GLYPH;
            r.color = di;
        }
        return r;
    }
    if (has_sdf(d)) {  // coarse/emit_draw.hlsli:22-30
        if (d.tag == TK_DRAW_BRUSH && !sdf_stroke_empty(S, d, tx, ty)) {
            r.valid = true;
            Paint P{S.brush.data(), S.brush.size(), S.desc.images, S.desc.image_count};
            uint32_t color = nontransparent_solid(S, d) && sdf_clip_covers(S, d, tx, ty)
                                 ? P.word(0u, d.brush_offset + TK_BRUSH_COLOR_WORD)
                                 : 0u;
            // full_tile_image (coarse/paint.hlsli:30-34)
            const bool image = d.brush_offset != TK_INVALID_INDEX &&
                               P.word(0u, d.brush_offset) == TK_BRUSH_PATTERN_RESOURCE &&
                               P.word(0u, d.brush_offset + TK_BRUSH_IMAGE_ALPHA_WORD) == 255u;
            if (color != 0u) {
                r.tag = TK_PTCL_COLOR;
                r.color = color;
            } else if (image && sdf_clip_covers(S, d, tx, ty)) {
                r.tag = TK_PTCL_IMAGE;
                r.color = di;
            } else {
                r.tag = TK_PTCL_SDF;
                r.seg0 = di;
                r.color = di;
            }
        }
        return r;
    }
    uint32_t bd = draw_backdrop(S, d, tx, ty);
    if (bd == TK_INVALID_INDEX || (d.tag != TK_DRAW_BRUSH && d.tag != TK_DRAW_PATH_GLYPH && d.tag != TK_DRAW_CLIP))
        return r;
    tk_segment_range rg = S.ranges[bd];
    uint32_t w = uint32_t(S.backdrops[bd]);
    if (rg.start == rg.end && w == 0u) return r;
    r.valid = true;
    r.winding = w;
    r.fill_rule = d.fill_rule;
    r.seg0 = rg.start;
    r.seg1 = rg.end;
    Paint P{S.brush.data(), S.brush.size(), S.desc.images, S.desc.image_count};
    bool nontransparent_solid = d.brush_offset != TK_INVALID_INDEX && P.word(0u, d.brush_offset) == TK_BRUSH_SOLID &&
                                P.word(0u, d.brush_offset + TK_BRUSH_COLOR_WORD) != 0u;
    if (d.tag == TK_DRAW_CLIP) r.tag = TK_PTCL_BEGIN_CLIP;
    else if (d.tag == TK_DRAW_PATH_GLYPH) r.tag = TK_PTCL_PATH_GLYPH;
    else if (d.solid_rect != 0u && d.transform.b == 0.0f && d.transform.c == 0.0f && nontransparent_solid &&
             rg.start == rg.end)
        r.tag = TK_PTCL_COLOR;
    if (r.tag == TK_PTCL_COLOR) r.color = P.word(0u, d.brush_offset + TK_BRUSH_COLOR_WORD);
    else if (d.tag == TK_DRAW_BRUSH || d.tag == TK_DRAW_PATH_GLYPH) r.color = di;
    return r;
}

const uint32_t CHUNK_CLASS_COLOR = 1u, CHUNK_CLASS_SDF = 2u, CHUNK_CLASS_OTHER = 4u, CHUNK_CLASS_OCCLUDER = 8u;

// coarse/occlusion.hlsli:12-34 on one tile stream (records [0, end)).
uint32_t occluded_prefix(const std::vector<tk_ptcl_record>& recs, uint32_t end, uint32_t wrappers) {
    uint32_t start = 0;
    if (wrappers != 0u || end <= start || end - start <= 2u || end > recs.size()) return 0u;
    if (recs[end - 1u].tag != TK_PTCL_END) return 0u;
    uint32_t depth = 0;
    for (uint32_t cur = end - 1u; cur > start;) {
        const tk_ptcl_record& r = recs[--cur];
        uint32_t tag = r.tag;
        if (tag == TK_PTCL_END_CLIP || tag == TK_PTCL_END_OPACITY || tag == TK_PTCL_END_BLEND) ++depth;
        else if (tag == TK_PTCL_BEGIN_CLIP || tag == TK_PTCL_BEGIN_SDF_CLIP || tag == TK_PTCL_BEGIN_OPACITY ||
                 tag == TK_PTCL_BEGIN_BLEND) {
            if (depth == 0u) return 0u;
            --depth;
        } else if (tag == TK_PTCL_COLOR && depth == 0u && (r.color >> 24) == 255u) {
            return cur - start;
        }
    }
    return 0u;
}

// coarse_count_bins (coarse/count.hlsl:48-73) + coarse_emit_bins
// (coarse/emit.hlsl:82-142) for one (batch, tile); `first`/`last` bound the
// tile's candidate run for this batch. Returns false when the tile has no
// stream in this batch.
bool coarse_tile(const or_scene& S, const Batch& b, uint32_t bi, uint32_t tile, const uint32_t* cand, uint32_t n,
                 BatchStream& out) {
    uint32_t tx = tile % S.tw, ty = tile / S.tw;
    uint32_t wrappers = stack_wrapper_count(S, b, tx, ty);
    if (wrappers == TK_INVALID_INDEX) return false;
    uint32_t count = 0;
    for (uint32_t k = 0; k < n; ++k) count += draw_particle(S, b, cand[k], tx, ty).valid ? 1u : 0u;
    if (count == 0u) return false;
    count += wrappers * 2u + 1u;
    out.batch = bi;
    out.glyphs.clear();
    out.recs.assign(count, tk_ptcl_record{});
    uint32_t p = 0;
    uint32_t flags = wrappers != 0u ? CHUNK_CLASS_OTHER : 0u;
    for (uint32_t i = b.layer_start; i < b.layer_end; ++i) {  // emit_stack_begins
        const tk_layer_record& L = S.layers[i];
        const tk_draw_record& d = S.draws[L.draw];
        if (noop_stack_clip(S, L, d, tx, ty)) continue;
        if (has_sdf(d)) {
            out.recs[p++] = {TK_PTCL_BEGIN_SDF_CLIP, 0, 0u, 0u, 0u, L.draw};
            continue;
        }
        uint32_t bd = draw_backdrop(S, d, tx, ty);
        uint32_t tag = L.tag == TK_LAYER_OPACITY ? TK_PTCL_BEGIN_OPACITY
                       : (L.tag == TK_LAYER_BLEND ? TK_PTCL_BEGIN_BLEND : TK_PTCL_BEGIN_CLIP);
        out.recs[p++] = {tag, S.backdrops[bd], d.fill_rule, S.ranges[bd].start, S.ranges[bd].end, L.payload};
    }
    for (uint32_t k = 0; k < n; ++k) {
        Particle q = draw_particle(S, b, cand[k], tx, ty);
        if (!q.valid) continue;
        // particle_class_flags (coarse/paint.hlsli:35-40)
        if (q.tag == TK_PTCL_COLOR) flags |= CHUNK_CLASS_COLOR;
        else if (q.tag == TK_PTCL_IMAGE || (q.tag == TK_PTCL_SDF && solid_supported_sdf(S, S.draws[cand[k]])))
            flags |= CHUNK_CLASS_SDF;
        else flags |= CHUNK_CLASS_OTHER;
        if (wrappers == 0u && q.tag == TK_PTCL_COLOR && (q.color >> 24) == 255u && p > 0u) flags |= CHUNK_CLASS_OCCLUDER;
        if (q.tag == TK_PTCL_GLYPH) {
            q.seg0 = uint32_t(out.glyphs.size());
            out.glyphs.insert(out.glyphs.end(), q.glyphs.begin(), q.glyphs.end());
            q.seg1 = uint32_t(out.glyphs.size());
        }
        if (p < count) out.recs[p++] = {q.tag, int32_t(q.winding), q.fill_rule, q.seg0, q.seg1, q.color};
    }
    uint32_t q = p;
    for (uint32_t i = b.layer_end; i > b.layer_start;) {  // emit_stack_ends
        const tk_layer_record& L = S.layers[--i];
        const tk_draw_record& d = S.draws[L.draw];
        if (noop_stack_clip(S, L, d, tx, ty)) continue;
        uint32_t tag = L.tag == TK_LAYER_OPACITY ? TK_PTCL_END_OPACITY
                       : (L.tag == TK_LAYER_BLEND ? TK_PTCL_END_BLEND : TK_PTCL_END_CLIP);
        out.recs[q++] = {tag, 0, 0u, 0u, 0u, 0u};
    }
    out.recs[p + wrappers] = {TK_PTCL_END, 0, 0u, 0u, 0u, 0u};
    uint32_t skip = (flags & CHUNK_CLASS_OCCLUDER) ? occluded_prefix(out.recs, p + wrappers + 1u, wrappers) : 0u;
    uint32_t kind;  // coarse/tile_classification.hlsli:6-10
    if (flags & CHUNK_CLASS_OTHER) kind = TK_TILE_KIND_INTERPRETER;
    else if (flags & CHUNK_CLASS_SDF) kind = (flags & CHUNK_CLASS_COLOR) ? TK_TILE_KIND_MIXED : TK_TILE_KIND_SDF;
    else kind = (flags & CHUNK_CLASS_COLOR) ? TK_TILE_KIND_COLOR : TK_TILE_KIND_EMPTY;
    out.kind = kind | (skip << TK_TILE_PREFIX_SHIFT);
    return true;
}

// --- fine/text/{gamma,auto,basic}.hlsli: glyph outline compositing -----------
// The shaders' pow as exp(y ln x) in double with exactly rounded operations
// (ln m = 2 atanh((m - 1)/(m + 1)) by its odd series to s^21 after
// m = x / 2^e in [sqrt(1/2), sqrt(2)); exp by Cody-Waite reduction with
// fdlibm's two-part ln 2 and its Taylor polynomial to degree 16), the same
// steps as the library's, so that the two agree bit for bit; its distance to
// the C library's pow is checked in the tests. `lerp(a, b, t)` is
// a + t (b - a) and `dot` is (x x' + y y') + z z', each operation rounded.
float text_pow(float x, float y) {
    int e = 0;
    double m = std::frexp(double(x), &e);
    if (m < 0.70710678118654752440) {
        m *= 2.0;
        --e;
    }
    const double s = (m - 1.0) / (m + 1.0), s2 = s * s;
    static const double odd[11] = {1.0 / 21.0, 1.0 / 19.0, 1.0 / 17.0, 1.0 / 15.0, 1.0 / 13.0, 1.0 / 11.0,
                                   1.0 / 9.0,  1.0 / 7.0,  1.0 / 5.0,  1.0 / 3.0,  1.0};
    double p = odd[0];
    for (int k = 1; k < 11; ++k) p = p * s2 + odd[k];
    const double ln2_hi = 6.93147180369123816490e-01, ln2_lo = 1.90821492927058770002e-10;
    const double lnx = (double(e) * ln2_hi + 2.0 * s * p) + double(e) * ln2_lo;
    const double t = double(y) * lnx;
    const double k = std::nearbyint(t * 1.44269504088896338700);
    const double r = (t - k * ln2_hi) - k * ln2_lo;
    // 1/16!, 1/15!, ..., 1/2!, 1, 1
    static const double inv_fact[17] = {1.0 / 20922789888000.0, 1.0 / 1307674368000.0, 1.0 / 87178291200.0,
                                        1.0 / 6227020800.0, 1.0 / 479001600.0, 1.0 / 39916800.0, 1.0 / 3628800.0,
                                        1.0 / 362880.0, 1.0 / 40320.0, 1.0 / 5040.0, 1.0 / 720.0, 1.0 / 120.0,
                                        1.0 / 24.0, 1.0 / 6.0, 0.5, 1.0, 1.0};
    double q = inv_fact[0];
    for (int i = 1; i < 17; ++i) q = q * r + inv_fact[i];
    return float(std::ldexp(q, int(k)));
}
// gamma.hlsli:5-23
float srgb_to_linear(float value) {
    float v = clampf(value, 0.0f, 1.0f);
    float result = v / 12.92f;
    if (v > 0.04045f) result = text_pow((v + 0.055f) / 1.055f, 2.4f);
    return result;
}
float linear_to_srgb(float value) {
    float v = clampf(value, 0.0f, 1.0f);
    float result = v * 12.92f;
    if (v > 0.0031308f) result = 1.055f * text_pow(v, 1.0f / 2.4f) - 0.055f;
    return result;
}
// auto.hlsli:6-9, dotted with the luminance weights
float text_foreground_luma(uint32_t source) {
    float alpha = float(source >> 24);
    if (!(alpha > 0.0f)) return 0.0f;
    float r = clampf(float(source & 255u) / alpha, 0.0f, 1.0f);
    float g = clampf(float((source >> 8) & 255u) / alpha, 0.0f, 1.0f);
    float b = clampf(float((source >> 16) & 255u) / alpha, 0.0f, 1.0f);
    return (r * 0.2126f + g * 0.7152f) + b * 0.0722f;
}
// auto.hlsli:15-26
float text_correcting_coverage(uint32_t coverage, float foreground) {
    if (coverage == 0u || coverage == 255u) return float(coverage) * (1.0f / 255.0f);
    float raw = float(coverage) * (1.0f / 255.0f);
    float background = 1.0f - foreground;
    float bg_linear = srgb_to_linear(background);
    float enhanced = raw + raw * (1.0f - raw) * bg_linear;
    float difference = foreground - background;
    if (std::fabs(difference) < (1.0f / 256.0f)) return enhanced;
    float fg_linear = srgb_to_linear(foreground);
    float output = linear_to_srgb(bg_linear + enhanced * (fg_linear - bg_linear));
    return clampf((output - background) / difference, 0.0f, 1.0f);
}
// basic.hlsli:95-109 with the same coverage in the three channels
uint32_t src_over_subpixel_mask_f32(uint32_t destination, uint32_t source, float cr, float cg, float cb) {
    if ((source >> 24) == 0u || (cr == 0.0f && cg == 0.0f && cb == 0.0f)) return destination;
    if ((destination >> 24) != 255u) {
        float gray = (cr + cg + cb) / 3.0f;
        cr = cg = cb = gray;
    }
    float alpha = float(source >> 24) * (1.0f / 255.0f);
    float ar = alpha * cr, ag = alpha * cg, ab = alpha * cb;
    float r = float(source & 255u) * cr + float(destination & 255u) * (1.0f - ar);
    float g = float((source >> 8) & 255u) * cg + float((destination >> 8) & 255u) * (1.0f - ag);
    float b = float((source >> 16) & 255u) * cb + float((destination >> 16) & 255u) * (1.0f - ab);
    float maximum = fmax_(fmax_(ar, ag), ab);
    float a = maximum * 255.0f + float(destination >> 24) * (1.0f - maximum);
    return pack(f2u(r + 0.5f), f2u(g + 0.5f), f2u(b + 0.5f), f2u(a + 0.5f));
}
// auto.hlsli:28-33
uint32_t src_over_mask_linear_auto_u8(uint32_t destination, uint32_t source, uint32_t coverage) {
    if ((source >> 24) == 0u || coverage == 0u) return destination;
    float corrected = text_correcting_coverage(coverage, text_foreground_luma(source));
    return src_over_subpixel_mask_f32(destination, source, corrected, corrected, corrected);
}

// fine/text/auto.hlsli:6-9
void text_foreground(uint32_t source, float fg[3]) {
    float alpha = float(source >> 24);
    if (!(alpha > 0.0f)) {
        fg[0] = fg[1] = fg[2] = 0.0f;
        return;
    }
    for (int k = 0; k < 3; ++k) fg[k] = clampf(float((source >> (8 * k)) & 255u) / alpha, 0.0f, 1.0f);
}
// basic.hlsli:9-43
uint32_t src_over_subpixel_mask_u8(uint32_t dst, uint32_t src, uint32_t mask, uint32_t clip) {
    uint32_t sa = src >> 24;
    if (sa == 0u || clip == 0u) return dst;
    uint32_t m[3] = {combine_alpha(mask & 255u, clip), combine_alpha((mask >> 8) & 255u, clip),
                     combine_alpha((mask >> 16) & 255u, clip)};
    if ((dst >> 24) != 255u) {
        uint32_t gray = (m[0] + m[1] + m[2] + 1u) / 3u;
        m[0] = m[1] = m[2] = gray;
    }
    if (m[0] == 0u && m[1] == 0u && m[2] == 0u) return dst;
    uint32_t cov[3], out[3];
    for (int k = 0; k < 3; ++k) cov[k] = mul_div255(sa, m[k]);
    uint32_t ca = std::max(std::max(cov[0], cov[1]), cov[2]);
    for (int k = 0; k < 3; ++k)
        out[k] = mul_div255((src >> (8 * k)) & 255u, m[k]) + mul_div255((dst >> (8 * k)) & 255u, 255u - cov[k]);
    uint32_t a = ca + mul_div255((dst >> 24) & 255u, 255u - ca);
    return pack(out[0], out[1], out[2], a);
}
// fine/glyph.hlsli:17-53: texels, the bilinear sample (lerp as a + t (b - a))
// and the corrected sample
uint32_t glyph_texel(const or_scene& S, const tk_glyph_image& im, int32_t x, int32_t y) {
    if (x < 0 || y < 0 || x >= int32_t(im.width) || y >= int32_t(im.height)) return 0u;
    return S.glyph_texels[size_t(im.data_offset) + size_t(y) * im.width + size_t(x)];
}
inline F4 lerp4(F4 a, F4 b, float t) {
    return {a.r + t * (b.r - a.r), a.g + t * (b.g - a.g), a.b + t * (b.b - a.b), a.a + t * (b.a - a.a)};
}
uint32_t sample_glyph(const or_scene& S, const tk_glyph_image& im, float px, float py) {
    int32_t bx = f2i(std::floor(px)), by = f2i(std::floor(py));
    float fx = px - float(bx), fy = py - float(by);
    uint32_t a = glyph_texel(S, im, bx, by);
    if (fx == 0.0f && fy == 0.0f) return a;
    F4 top = lerp4(rgba8_to_unorm(a), rgba8_to_unorm(glyph_texel(S, im, bx + 1, by)), fx);
    F4 bottom = lerp4(rgba8_to_unorm(glyph_texel(S, im, bx, by + 1)), rgba8_to_unorm(glyph_texel(S, im, bx + 1, by + 1)),
                      fx);
    return unorm_to_rgba8(lerp4(top, bottom, fy));
}
void corrected_glyph_texel(uint32_t data, const float fg[3], bool lcd, float out[3]) {
    if (!lcd) {
        float alpha = text_correcting_coverage(data & 255u, (fg[0] * 0.2126f + fg[1] * 0.7152f) + fg[2] * 0.0722f);
        out[0] = out[1] = out[2] = alpha;
        return;
    }
    for (int k = 0; k < 3; ++k) out[k] = text_correcting_coverage((data >> (8 * k)) & 255u, fg[k]);
}
void sample_corrected_glyph(const or_scene& S, const tk_glyph_image& im, float px, float py, const float fg[3],
                            bool lcd, float out[3]) {
    int32_t bx = f2i(std::floor(px)), by = f2i(std::floor(py));
    float fx = px - float(bx), fy = py - float(by);
    float a[3], b[3], c[3], d[3];
    corrected_glyph_texel(glyph_texel(S, im, bx, by), fg, lcd, a);
    if (fx == 0.0f && fy == 0.0f) {
        for (int k = 0; k < 3; ++k) out[k] = a[k];
        return;
    }
    corrected_glyph_texel(glyph_texel(S, im, bx + 1, by), fg, lcd, b);
    corrected_glyph_texel(glyph_texel(S, im, bx, by + 1), fg, lcd, c);
    corrected_glyph_texel(glyph_texel(S, im, bx + 1, by + 1), fg, lcd, d);
    for (int k = 0; k < 3; ++k) {
        float top = a[k] + fx * (b[k] - a[k]);
        float bottom = c[k] + fx * (d[k] - c[k]);
        out[k] = top + fy * (bottom - top);
    }
}

// --- fine/interpreter.hlsli:21-219 (clip stack and opacity groups) ------------
struct Group { uint32_t kind; F4 parent; uint32_t parent_clip, layer_alpha, payload; };

// composite_glyphs_at (fine/glyph.hlsli:55-111)
F4 composite_glyphs_at(const or_scene& S, const Paint& P, F4 pixel, const uint32_t* list, uint32_t g0, uint32_t g1,
                       const tk_draw_record& d, uint32_t gx, uint32_t gy, uint32_t clip) {
    const tk_affine& m = d.inverse_transform;
    const float sx = float(gx) + 0.5f, sy = float(gy) + 0.5f;
    const float lx = mad(m.a, sx, mad(m.c, sy, m.e)) - 0.5f;
    const float ly = mad(m.b, sx, mad(m.d, sy, m.f)) - 0.5f;
    for (uint32_t g = g0; g < g1; ++g) {
        const tk_glyph& glyph = S.glyphs[list[g]];
        if (glyph.image == TK_INVALID_INDEX) continue;
        const tk_glyph_image& im = S.glyph_images[glyph.image];
        const int32_t x0 = int32_t(uint32_t(glyph.x) + uint32_t(im.left));
        const int32_t y0 = int32_t(uint32_t(glyph.y) - uint32_t(im.top));
        const float ux = lx - float(x0), uy = ly - float(y0);
        if (!(ux > -1.0f && uy > -1.0f && ux < float(int32_t(im.width)) && uy < float(int32_t(im.height)))) continue;
        const uint32_t content = im.content;
        if (content == TK_GLYPH_LINEAR_MASK || content == TK_GLYPH_LINEAR_SUBPIXEL_MASK) {
            const uint32_t color = sample_draw_brush(P, d, sx, sy);
            float fg[3], cov[3];
            text_foreground(color, fg);
            sample_corrected_glyph(S, im, ux, uy, fg, content == TK_GLYPH_LINEAR_SUBPIXEL_MASK, cov);
            const float k = float(clip) * (1.0f / 255.0f);
            pixel = rgba8_to_unorm(
                src_over_subpixel_mask_f32(unorm_to_rgba8(pixel), color, cov[0] * k, cov[1] * k, cov[2] * k));
        } else {
            const uint32_t data = sample_glyph(S, im, ux, uy);
            if (content == TK_GLYPH_MASK) {
                const uint32_t alpha = combine_alpha(data, clip);
                if (alpha != 0u)
                    pixel = src_over_premul_unorm(pixel, scale_premul_u8_to_unorm(sample_draw_brush(P, d, sx, sy), alpha));
            } else if (content == TK_GLYPH_COLOR) {
                pixel = src_over_premul_unorm(pixel, scale_premul_u8_to_unorm(data, clip));
            } else if (content == TK_GLYPH_LINEAR_COLOR) {
                pixel = rgba8_to_unorm(src_over_mask_linear_auto_u8(unorm_to_rgba8(pixel), data, clip));
            } else if (content == TK_GLYPH_SUBPIXEL_MASK) {
                pixel = rgba8_to_unorm(
                    src_over_subpixel_mask_u8(unorm_to_rgba8(pixel), sample_draw_brush(P, d, sx, sy), data, clip));
            }
        }
    }
    return pixel;
}

F4 interpret(const or_scene& S, const std::vector<tk_ptcl_record>& recs, uint32_t begin, uint32_t end, F4 pixel,
             uint32_t lx, uint32_t ly, uint32_t gx, uint32_t gy, const uint32_t* glyph_list = nullptr) {
    Paint P{S.brush.data(), S.brush.size(), S.desc.images, S.desc.image_count};
    uint32_t clip_mask = 255u;
    std::vector<uint32_t> clip_stack;
    std::vector<Group> groups;
    for (uint32_t ix = begin; ix < end; ++ix) {
        const tk_ptcl_record& r = recs[ix];
        uint32_t tag = r.tag;
        if (tag == TK_PTCL_END) break;
        if (tag == TK_PTCL_COLOR) {
            if (clip_mask != 0u) {
                if (clip_mask == 255u && premul_u8_is_opaque(r.color)) pixel = rgba8_to_unorm(r.color);
                else pixel = src_over_premul_unorm(pixel, scale_premul_u8_to_unorm(r.color, clip_mask));
            }
        } else if (tag == TK_PTCL_END_CLIP) {
            if (!clip_stack.empty()) { clip_mask = clip_stack.back(); clip_stack.pop_back(); }
            else clip_mask = 255u;
        } else if (tag == TK_PTCL_END_OPACITY || tag == TK_PTCL_END_BLEND) {
            if (!groups.empty()) {
                Group v = groups.back();
                groups.pop_back();
                if (v.kind == TK_PTCL_BEGIN_OPACITY) {
                    uint32_t alpha = combine_alpha(combine_alpha(v.layer_alpha, v.parent_clip), v.payload);
                    pixel = src_over_premul_unorm(v.parent, scale_premul_u8_to_unorm(unorm_to_rgba8(pixel), alpha));
                }
                // blend groups are outside this path (rejected at load)
            }
        } else if (tag == TK_PTCL_BEGIN_SDF_CLIP) {  // fine/interpreter.hlsli:131-150
            uint32_t parent = clip_mask, alpha = 0u;
            if (parent != 0u)
                alpha = coverage_to_u8(sdf_coverage_from_draw(S, S.draws[r.color], float(gx) + 0.5f, float(gy) + 0.5f));
            clip_stack.push_back(parent);
            clip_mask = combine_alpha(parent, alpha);
        } else if (tag == TK_PTCL_GLYPH) {  // fine/interpreter.hlsli:93-106
            const tk_draw_record& d = S.draws[r.color];
            const int32_t x = int32_t(gx), y = int32_t(gy);
            if (clip_mask != 0u && glyph_list && x >= d.pixel_bounds.x0 && y >= d.pixel_bounds.y0 &&
                x < d.pixel_bounds.x1 && y < d.pixel_bounds.y1)
                pixel = composite_glyphs_at(S, P, pixel, glyph_list, r.segment_start, r.segment_end, d, gx, gy,
                                            clip_mask);
        } else if (tag == TK_PTCL_IMAGE) {  // fine/interpreter.hlsli:65-69
            if (clip_mask != 0u) {
                uint32_t color = sample_draw_brush(P, S.draws[r.color], float(gx) + 0.5f, float(gy) + 0.5f);
                if (clip_mask == 255u && premul_u8_is_opaque(color)) pixel = rgba8_to_unorm(color);
                else pixel = src_over_premul_unorm(pixel, scale_premul_u8_to_unorm(color, clip_mask));
            }
        } else if (tag == TK_PTCL_SDF) {  // fine/interpreter.hlsli:70-84
            if (clip_mask != 0u) {
                const tk_draw_record& d = S.draws[r.color];
                float x = float(gx) + 0.5f, y = float(gy) + 0.5f;
                uint32_t alpha = combine_alpha(coverage_to_u8(sdf_coverage_from_draw(S, d, x, y)), clip_mask);
                if (alpha != 0u) {
                    uint32_t color = sample_draw_brush(P, d, x, y);
                    if (alpha == 255u && premul_u8_is_opaque(color)) pixel = rgba8_to_unorm(color);
                    else pixel = src_over_premul_unorm(pixel, scale_premul_u8_to_unorm(color, alpha));
                }
            }
        } else if (tag == TK_PTCL_FILL || tag == TK_PTCL_PATH_GLYPH || tag == TK_PTCL_BEGIN_CLIP ||
                   tag == TK_PTCL_BEGIN_OPACITY || tag == TK_PTCL_BEGIN_BLEND) {
            uint32_t alpha = coverage_to_alpha(
                fill_value(S.segments.data(), r.segment_start, r.segment_end, r.backdrop, lx, ly), r.fill_rule);
            if (tag == TK_PTCL_BEGIN_CLIP) {
                clip_stack.push_back(clip_mask);
                clip_mask = combine_alpha(clip_mask, alpha);
            } else if (tag == TK_PTCL_BEGIN_OPACITY || tag == TK_PTCL_BEGIN_BLEND) {
                // Parents beyond the two local slots are spilled as RGBA8
                // (fine/group.hlsli:21-36).
                F4 parent = groups.size() < 2 ? pixel : rgba8_to_unorm(unorm_to_rgba8(pixel));
                groups.push_back({tag, parent, clip_mask, alpha, r.color});
                pixel = {0, 0, 0, 0};
            } else {
                uint32_t masked = combine_alpha(alpha, clip_mask);
                if (masked != 0u) {
                    uint32_t color = sample_draw_brush(P, S.draws[r.color], float(gx) + 0.5f, float(gy) + 0.5f);
                    if (tag == TK_PTCL_PATH_GLYPH)  // interpreter.hlsli:205-206
                        pixel = rgba8_to_unorm(src_over_mask_linear_auto_u8(unorm_to_rgba8(pixel), color, masked));
                    else if (masked == 255u && premul_u8_is_opaque(color)) pixel = rgba8_to_unorm(color);
                    else pixel = src_over_premul_unorm(pixel, scale_premul_u8_to_unorm(color, masked));
                }
            }
        }
    }
    return pixel;
}
// fine/specialized.hlsli:19-45
F4 color_only(const std::vector<tk_ptcl_record>& recs, uint32_t begin, uint32_t end, F4 pixel) {
    for (uint32_t ix = begin; ix < end; ++ix) {
        const tk_ptcl_record& r = recs[ix];
        if (r.tag == TK_PTCL_END) break;
        if (premul_u8_is_opaque(r.color)) pixel = rgba8_to_unorm(r.color);
        else pixel = src_over_premul_unorm(pixel, rgba8_to_unorm(r.color));
    }
    return pixel;
}

// fine/specialized.hlsli:47-108 (SDF and MIXED tiles: colours and solid SDFs,
// no stacks; full-tile images are not produced on this path)
F4 analytic_solid(const or_scene& S, const std::vector<tk_ptcl_record>& recs, uint32_t begin, uint32_t end, F4 pixel,
                  uint32_t gx, uint32_t gy) {
    Paint P{S.brush.data(), S.brush.size(), S.desc.images, S.desc.image_count};
    float x = float(gx) + 0.5f, y = float(gy) + 0.5f;
    for (uint32_t ix = begin; ix < end; ++ix) {
        const tk_ptcl_record& r = recs[ix];
        if (r.tag == TK_PTCL_END) break;
        if (r.tag == TK_PTCL_COLOR) {
            if (premul_u8_is_opaque(r.color)) pixel = rgba8_to_unorm(r.color);
            else pixel = src_over_premul_unorm(pixel, rgba8_to_unorm(r.color));
        } else if (r.tag == TK_PTCL_IMAGE) {  // fine/specialized.hlsli:84-90
            uint32_t color = sample_draw_brush(P, S.draws[r.color], x, y);
            if (premul_u8_is_opaque(color)) pixel = rgba8_to_unorm(color);
            else pixel = src_over_premul_unorm(pixel, rgba8_to_unorm(color));
        } else {
            const tk_draw_record& d = S.draws[r.color];
            bool inside = int32_t(gx) >= d.pixel_bounds.x0 && int32_t(gy) >= d.pixel_bounds.y0 &&
                          int32_t(gx) < d.pixel_bounds.x1 && int32_t(gy) < d.pixel_bounds.y1;
            uint32_t alpha = coverage_to_u8(inside ? sdf_coverage_from_draw(S, d, x, y) : 0.0f);
            if (alpha != 0u) {
                uint32_t color = P.word(0u, d.brush_offset + TK_BRUSH_COLOR_WORD);
                if (alpha == 255u && premul_u8_is_opaque(color)) pixel = rgba8_to_unorm(color);
                else pixel = src_over_premul_unorm(pixel, scale_premul_u8_to_unorm(color, alpha));
            }
        }
    }
    return pixel;
}

// --- filter/blur*.hlsl -----------------------------------------------------------
inline void channels(uint32_t p, float c[4]) {
    c[0] = float(p & 255u); c[1] = float((p >> 8) & 255u); c[2] = float((p >> 16) & 255u); c[3] = float(p >> 24);
}
inline uint32_t pack_average(const float acc[4], float sum) {
    if (sum <= 0.0f) return 0u;
    float inv = 1.0f / sum;
    uint32_t o = 0;
    for (int c = 0; c < 4; ++c) o |= f2u(clampf(acc[c] * inv + 0.5f, 0.0f, 255.0f)) << (8 * c);
    return o;
}
inline int32_t blur_half_width(float sd) { return f2i(fmax_(std::ceil(sd * 3.0f), 1.0f)); }
inline bool inside_b(int32_t x, int32_t y, const int32_t b[4]) { return x >= b[0] && y >= b[1] && x < b[2] && y < b[3]; }

// filter/sample.hlsli:4-17 on an RGBA8 texture: texel loads are k/255.
F4 sample_premul(const uint32_t* src, uint32_t w, uint32_t h, float px, float py) {
    int32_t lastx = int32_t(w) - 1, lasty = int32_t(h) - 1;
    px = clampf(px, 0.0f, float(lastx));
    py = clampf(py, 0.0f, float(lasty));
    int32_t fx = f2i(std::floor(px)), fy = f2i(std::floor(py));
    int32_t nx = std::min(fx + 1, lastx), ny = std::min(fy + 1, lasty);
    float phx = px - float(fx), phy = py - float(fy);
    F4 a = texel_load(src[size_t(fy) * w + fx]), b = texel_load(src[size_t(fy) * w + nx]);
    F4 c = texel_load(src[size_t(ny) * w + fx]), d = texel_load(src[size_t(ny) * w + nx]);
    auto lerp = [](float u, float v, float t) { return mad(v - u, t, u); };
    F4 top{lerp(a.r, b.r, phx), lerp(a.g, b.g, phx), lerp(a.b, b.b, phx), lerp(a.a, b.a, phx)};
    F4 bot{lerp(c.r, d.r, phx), lerp(c.g, d.g, phx), lerp(c.b, d.b, phx), lerp(c.a, d.a, phx)};
    return {lerp(top.r, bot.r, phy), lerp(top.g, bot.g, phy), lerp(top.b, bot.b, phy), lerp(top.a, bot.a, phy)};
}

// filter/blur.hlsli:40-94 (global route, used for radius > 16).
uint32_t blur_pixel_global(const uint32_t* src, uint32_t w, uint32_t h, int32_t x, int32_t y, float sd,
                           const int32_t bounds[4], uint32_t axis, float weight0, float decay) {
    int32_t hw = blur_half_width(sd);
    int32_t ax = axis == 0u ? 1 : 0, ay = axis == 0u ? 0 : 1;
    bool interior = inside_b(x - ax * hw, y - ay * hw, bounds) && inside_b(x + ax * hw, y + ay * hw, bounds);
    float sum = 1.0f;
    uint32_t center = inside_b(x, y, bounds) ? src[size_t(y) * w + x] : 0u;
    float acc[4];
    channels(center, acc);
    float weight = weight0;
    float ratio = weight * decay;
    auto tap = [&](int32_t px, int32_t py, float wgt) {
        if (interior || inside_b(px, py, bounds)) {
            float c[4];
            channels(src[size_t(py) * w + px], c);
            for (int k = 0; k < 4; ++k) acc[k] = mad(c[k], wgt, acc[k]);
        }
    };
    auto pair_inside = [&](float off) {
        float fx = float(x) + float(ax) * off, fy = float(y) + float(ay) * off;
        float nx = fx + float(ax), ny = fy + float(ay);
        return fx >= float(bounds[0]) && fy >= float(bounds[1]) && nx < float(bounds[2]) && ny < float(bounds[3]);
    };
    auto pair = [&](float off, float wgt) {
        F4 s = sample_premul(src, w, h, float(x) + float(ax) * off, float(y) + float(ay) * off);
        float c[4] = {s.r * 255.0f, s.g * 255.0f, s.b * 255.0f, s.a * 255.0f};
        for (int k = 0; k < 4; ++k) acc[k] = mad(c[k], wgt, acc[k]);
    };
    for (int32_t d = 1; d <= hw; d += 2) {
        int32_t nd = d + 1;
        bool has_pair = nd <= hw;
        float next_weight = weight * ratio;
        float pw = weight + (has_pair ? next_weight : 0.0f);
        sum += 2.0f * pw;
        if (has_pair && (interior || pair_inside(float(d)))) {
            pair(float(d) + next_weight / pw, pw);
        } else {
            tap(x + ax * d, y + ay * d, weight);
            if (has_pair) tap(x + ax * nd, y + ay * nd, next_weight);
        }
        if (has_pair && (interior || pair_inside(-float(nd)))) {
            pair(-(float(d) + next_weight / pw), pw);
        } else {
            tap(x - ax * d, y - ay * d, weight);
            if (has_pair) tap(x - ax * nd, y - ay * nd, next_weight);
        }
        float next_ratio = ratio * decay;
        weight = next_weight * next_ratio;
        ratio = next_ratio * decay;
    }
    return pack_average(acc, sum);
}

void blur_pass(const uint32_t* src, uint32_t* dst, uint32_t w, uint32_t h, const uint32_t region[4],
               const uint32_t source[4], float amount, uint32_t axis, int threads) {
    float sd = fmax_(amount, 0.0f);
    int32_t bounds[4];
    bool sx = source[2] > source[0], sy = source[3] > source[1];
    bounds[0] = int32_t(sx ? source[0] : region[0]);
    bounds[1] = int32_t(sy ? source[1] : region[1]);
    bounds[2] = int32_t(sx ? source[2] : region[0] + region[2]);
    bounds[3] = int32_t(sy ? source[3] : region[1] + region[3]);
    // region = x0, y0, width, height
    uint32_t rx1 = std::min(region[0] + region[2], w), ry1 = std::min(region[1] + region[3], h);
    float sigma = fmax_(sd, 0.0001f);
    float two = 2.0f * sigma * sigma;
    float weight0 = std::exp(-1.0f / two), decay = std::exp(-2.0f / two);
    int32_t hw = blur_half_width(sd);
    parallel_for(threads, ry1 > region[1] ? ry1 - region[1] : 0, [&](uint64_t row) {
        int32_t y = int32_t(region[1] + row);
        for (int32_t x = int32_t(region[0]); x < int32_t(rx1); ++x) {
            uint32_t out;
            if (sd <= 0.0f) {
                out = src[size_t(y) * w + x];
            } else if (hw > int32_t(TK_SHARED_BLUR_MAX_RADIUS)) {
                out = blur_pixel_global(src, w, h, x, y, sd, bounds, axis, weight0, decay);
            } else {  // filter/blur_shared.hlsl:39-73
                auto at = [&](int32_t px, int32_t py) -> uint32_t {
                    return inside_b(px, py, bounds) ? src[size_t(py) * w + px] : 0u;
                };
                int32_t ax = axis == 0u ? 1 : 0, ay = axis == 0u ? 0 : 1;
                float acc[4];
                channels(at(x, y), acc);
                float sum = 1.0f, weight = weight0, ratio = weight0 * decay;
                for (int32_t d = 1; d <= hw; ++d) {
                    sum += 2.0f * weight;
                    float c[4];
                    channels(at(x + ax * d, y + ay * d), c);
                    for (int k = 0; k < 4; ++k) acc[k] = mad(c[k], weight, acc[k]);
                    channels(at(x - ax * d, y - ay * d), c);
                    for (int k = 0; k < 4; ++k) acc[k] = mad(c[k], weight, acc[k]);
                    weight = weight * ratio;
                    ratio = ratio * decay;
                }
                out = pack_average(acc, sum);
            }
            dst[size_t(y) * w + x] = out;
        }
    });
}

// --- filter/resample.hlsli: reduced-resolution blur (BlurSampling factor > 1) ---
// filter_downsample_pixel for every low texel of `low_rect`: the cell's centre
// texel (filter 0) or its byte average rounded half up (filter 1).
// --- filter/color.hlsli:7-76, filter/basic.hlsl:49-56 ------------------------
// The filter layer chain: colour filters and the colour matrix on the stored
// RGBA8 word (mad fused, every other product and sum rounded on its own), and
// the whole-pixel offset, each over the layer's bounds
// (render/filter_program/effects.rs:3-268).
inline float svg_luminance(float r, float g, float b) { return (0.2126f * r + 0.7152f * g) + 0.0722f * b; }

uint32_t filter_color_pixel(uint32_t pixel, uint32_t kind, float amount) {
    if ((kind == TK_FILTER_INVERT || kind == TK_FILTER_SEPIA) && (pixel >> 24) != 0u) {
        const float cr = float(pixel & 255u), cg = float((pixel >> 8) & 255u), cb = float((pixel >> 16) & 255u);
        const float alpha = float(pixel >> 24);
        float mr = alpha - cr, mg = alpha - cg, mb = alpha - cb;
        if (kind == TK_FILTER_SEPIA) {
            mr = mad(0.393f, cr, mad(0.769f, cg, 0.189f * cb));
            mg = mad(0.349f, cr, mad(0.686f, cg, 0.168f * cb));
            mb = mad(0.272f, cr, mad(0.534f, cg, 0.131f * cb));
        }
        const float t = clampf(amount, 0.0f, 1.0f);
        return pack(f2u(clampf(mad(mr - cr, t, cr), 0.0f, alpha) + 0.5f),
                    f2u(clampf(mad(mg - cg, t, cg), 0.0f, alpha) + 0.5f),
                    f2u(clampf(mad(mb - cb, t, cb), 0.0f, alpha) + 0.5f), pixel >> 24);
    }
    F4 c = rgba8_to_unorm(pixel);
    if (kind == TK_FILTER_OPACITY) {
        const float a = clampf(amount, 0.0f, 1.0f);
        c = {c.r * a, c.g * a, c.b * a, c.a * a};
    } else if (c.a > 0.0f) {
        float r = c.r / c.a, g = c.g / c.a, b = c.b / c.a;
        if (kind == TK_FILTER_BRIGHTNESS) {
            r = r * amount;
            g = g * amount;
            b = b * amount;
        } else if (kind == TK_FILTER_CONTRAST) {
            r = (r - 0.5f) * amount + 0.5f;
            g = (g - 0.5f) * amount + 0.5f;
            b = (b - 0.5f) * amount + 0.5f;
        } else if (kind == TK_FILTER_GRAYSCALE) {
            const float l = svg_luminance(r, g, b), t = clampf(amount, 0.0f, 1.0f);
            r = mad(l - r, t, r);
            g = mad(l - g, t, g);
            b = mad(l - b, t, b);
        } else if (kind == TK_FILTER_HUE_ROTATE) {
            float si, co;
            lib_sincos(amount * 0.017453292f, si, co);
            const float nr = ((0.213f + co * 0.787f) - si * 0.213f) * r + ((0.715f - co * 0.715f) - si * 0.715f) * g +
                             ((0.072f - co * 0.072f) + si * 0.928f) * b;
            const float ng = ((0.213f - co * 0.213f) + si * 0.143f) * r + ((0.715f + co * 0.285f) + si * 0.140f) * g +
                             ((0.072f - co * 0.072f) - si * 0.283f) * b;
            const float nb = ((0.213f - co * 0.213f) - si * 0.787f) * r + ((0.715f - co * 0.715f) + si * 0.715f) * g +
                             ((0.072f + co * 0.928f) + si * 0.072f) * b;
            r = nr;
            g = ng;
            b = nb;
        } else if (kind == TK_FILTER_SATURATE) {
            const float l = svg_luminance(r, g, b);
            r = l + (r - l) * amount;
            g = l + (g - l) * amount;
            b = l + (b - l) * amount;
        }
        c = {clampf(r, 0.0f, 1.0f) * c.a, clampf(g, 0.0f, 1.0f) * c.a, clampf(b, 0.0f, 1.0f) * c.a, c.a};
    }
    return pack(f2u(clampf(c.r, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(c.g, 0.0f, 1.0f) * 255.0f + 0.5f),
                f2u(clampf(c.b, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(c.a, 0.0f, 1.0f) * 255.0f + 0.5f));
}

inline float filter_dot4(const float* a, float x, float y, float z, float w) {
    return mad(a[0], x, mad(a[1], y, mad(a[2], z, a[3] * w)));
}

uint32_t filter_color_matrix_pixel(const float* m, uint32_t pixel) {
    const float alpha = float(pixel >> 24);
    const float cr = float(pixel & 255u), cg = float((pixel >> 8) & 255u), cb = float((pixel >> 16) & 255u);
    float sr = 0.0f, sg = 0.0f, sb = 0.0f;
    if ((pixel >> 24) == 255u) {
        sr = cr;
        sg = cg;
        sb = cb;
    } else if (alpha > 0.0f) {
        const float k = 255.0f / alpha;
        sr = cr * k;
        sg = cg * k;
        sb = cb * k;
    }
    const float out_a = std::floor(clampf(filter_dot4(m + 15, sr, sg, sb, alpha) + m[19] * 255.0f, 0.0f, 255.0f) + 0.5f);
    float rr, rg, rb;
    if (alpha > 0.0f) {
        const float sw = alpha * alpha * CHANNEL_SCALE;
        const float mr = mad(m[4], alpha, filter_dot4(m + 0, cr, cg, cb, sw));
        const float mg = mad(m[9], alpha, filter_dot4(m + 5, cr, cg, cb, sw));
        const float mb = mad(m[14], alpha, filter_dot4(m + 10, cr, cg, cb, sw));
        const float scale = out_a == alpha ? 1.0f : out_a / alpha;
        rr = mr >= alpha ? out_a : clampf(mr, 0.0f, alpha) * scale;
        rg = mg >= alpha ? out_a : clampf(mg, 0.0f, alpha) * scale;
        rb = mb >= alpha ? out_a : clampf(mb, 0.0f, alpha) * scale;
    } else {
        rr = clampf(m[4], 0.0f, 1.0f) * out_a;
        rg = clampf(m[9], 0.0f, 1.0f) * out_a;
        rb = clampf(m[14], 0.0f, 1.0f) * out_a;
    }
    return pack(f2u(clampf(rr, 0.0f, 255.0f) + 0.5f), f2u(clampf(rg, 0.0f, 255.0f) + 0.5f),
                f2u(clampf(rb, 0.0f, 255.0f) + 0.5f), f2u(clampf(out_a, 0.0f, 255.0f) + 0.5f));
}

// filter_morphology_pixel (filter/morphology.hlsli:8-27) over bounds b,
// whose lines are the surface's, along x (horizontal) or y.
void morphology_pass(const uint32_t* src, uint32_t* dst, uint32_t width, const int32_t b[4], uint32_t radius,
                     bool dilate, bool horizontal) {
    const uint32_t w = uint32_t(b[2] - b[0]), h = uint32_t(b[3] - b[1]), len = horizontal ? w : h;
    for (uint32_t ly = 0; ly < h; ++ly)
        for (uint32_t lx = 0; lx < w; ++lx) {
            const size_t o = size_t(uint32_t(b[1]) + ly) * width + uint32_t(b[0]) + lx;
            const uint32_t pos = horizontal ? lx : ly;
            if (!dilate && (pos < radius || pos + radius >= len)) {
                dst[o] = 0u;
                continue;
            }
            float v[4];
            for (float& x : v) x = dilate ? 0.0f : 1.0f;
            const uint32_t start = pos > radius ? pos - radius : 0u, end = std::min(len - 1u, pos + radius);
            for (uint32_t sp = start; sp <= end; ++sp) {
                const size_t so = horizontal ? size_t(uint32_t(b[1]) + ly) * width + uint32_t(b[0]) + sp
                                             : size_t(uint32_t(b[1]) + sp) * width + uint32_t(b[0]) + lx;
                const uint32_t p = src[so], al = p >> 24;
                const float s[4] = {al == 0u ? 0.0f : float(p & 255u) / float(al),
                                    al == 0u ? 0.0f : float((p >> 8) & 255u) / float(al),
                                    al == 0u ? 0.0f : float((p >> 16) & 255u) / float(al), float(al) / 255.0f};
                for (int c = 0; c < 4; ++c) v[c] = dilate ? fmax_(v[c], s[c]) : fmin_(v[c], s[c]);
            }
            dst[o] = pack(f2u(clampf(v[0] * v[3], 0.0f, 1.0f) * 255.0f + 0.5f),
                          f2u(clampf(v[1] * v[3], 0.0f, 1.0f) * 255.0f + 0.5f),
                          f2u(clampf(v[2] * v[3], 0.0f, 1.0f) * 255.0f + 0.5f),
                          f2u(clampf(v[3], 0.0f, 1.0f) * 255.0f + 0.5f));
        }
}

// filter_transfer_pixel (filter/transfer.hlsli:5-19)
inline uint32_t straight_index(uint32_t premul, uint32_t alpha) {
    return alpha == 0u ? 0u : std::min((premul * 255u + alpha / 2u) / alpha, 255u);
}
uint32_t filter_transfer_pixel(const uint32_t* t, uint32_t pixel) {
    const uint32_t alpha = pixel >> 24;
    const float r = float(t[straight_index(pixel & 255u, alpha)]) * CHANNEL_SCALE;
    const float g = float(t[256u + straight_index((pixel >> 8) & 255u, alpha)]) * CHANNEL_SCALE;
    const float bl = float(t[512u + straight_index((pixel >> 16) & 255u, alpha)]) * CHANNEL_SCALE;
    const float a = float(t[768u + alpha]) * CHANNEL_SCALE;
    return pack(f2u(clampf(r * a, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(g * a, 0.0f, 1.0f) * 255.0f + 0.5f),
                f2u(clampf(bl * a, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(a, 0.0f, 1.0f) * 255.0f + 0.5f));
}

// filter_convolve_pixel (filter/convolve.hlsli:9-98) over bounds b
inline int32_t conv_wrap(int32_t c, int32_t origin, int32_t len) {
    const int32_t r = (c - origin) % len;
    return origin + (r < 0 ? r + len : r);
}
inline float conv_scale_24(float v) {
    const uint32_t bits = f_bits(v), mag = bits & 0x7fffffffu, e = mag >> 23;
    if (e == 0u) {
        const float s = float(mag) * bits_f(0x01000000u);
        return (bits & 0x80000000u) ? -s : s;
    }
    if (e >= 231u) return bits_f((bits & 0x80000000u) | 0x7f800000u);
    return bits_f(bits + (24u << 23));
}
inline float conv_unscale_24(float v) {
    const uint32_t bits = f_bits(v), e = (bits & 0x7fffffffu) >> 23;
    if (e <= 24u) return 0.0f;
    return bits_f(bits - (24u << 23));
}
void convolve_pass(const uint32_t* src, uint32_t* dst, uint32_t width, const int32_t b[4], const tk_filter& k,
                   const float* kernel) {
    const uint32_t dmag = f_bits(k.divisor) & 0x7fffffffu;
    for (int32_t y = b[1]; y < b[3]; ++y)
        for (int32_t x = b[0]; x < b[2]; ++x) {
            const size_t o = size_t(y) * width + size_t(x);
            const uint32_t center = src[o];
            if (k.columns == 0u || k.rows == 0u || dmag == 0u) {
                dst[o] = center;
                continue;
            }
            float s[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            for (uint32_t ky = 0; ky < k.rows; ++ky)
                for (uint32_t kx = 0; kx < k.columns; ++kx) {
                    const float wt = kernel[(k.rows - 1u - ky) * k.columns + (k.columns - 1u - kx)];
                    int32_t px = x + int32_t(kx) - int32_t(k.target_x), py = y + int32_t(ky) - int32_t(k.target_y);
                    uint32_t p = 0u;
                    if (k.edge_mode == TK_CONVOLVE_EDGE_DUPLICATE) {
                        px = std::min(std::max(px, b[0]), b[2] - 1);
                        py = std::min(std::max(py, b[1]), b[3] - 1);
                        p = src[size_t(py) * width + size_t(px)];
                    } else if (k.edge_mode == TK_CONVOLVE_EDGE_WRAP) {
                        px = conv_wrap(px, b[0], b[2] - b[0]);
                        py = conv_wrap(py, b[1], b[3] - b[1]);
                        p = src[size_t(py) * width + size_t(px)];
                    } else if (px >= b[0] && py >= b[1] && px < b[2] && py < b[3]) {
                        p = src[size_t(py) * width + size_t(px)];
                    }
                    const uint32_t al = p >> 24;
                    F4 v = rgba8_to_unorm(p);
                    if (k.preserve_alpha) {
                        v.r = al == 0u ? 0.0f : v.r / v.a;
                        v.g = al == 0u ? 0.0f : v.g / v.a;
                        v.b = al == 0u ? 0.0f : v.b / v.a;
                    }
                    v.a = float(al);
                    s[0] = mad(v.r, wt, s[0]);
                    s[1] = mad(v.g, wt, s[1]);
                    s[2] = mad(v.b, wt, s[2]);
                    s[3] = mad(v.a, wt, s[3]);
                }
            float q[3], qa;
            if (dmag < 0x00800000u) {
                float sd = float(dmag) * bits_f(0x01000000u);
                if (f_bits(k.divisor) & 0x80000000u) sd = -sd;
                for (int c = 0; c < 3; ++c) q[c] = conv_scale_24(s[c]) / sd;
                qa = conv_scale_24(s[3]) / (sd * 255.0f);
            } else if (dmag > 0x7e800000u) {
                const float inv = 1.0f / conv_unscale_24(k.divisor);
                for (int c = 0; c < 3; ++c) q[c] = conv_unscale_24(s[c]) * inv;
                qa = conv_unscale_24(s[3]) * inv * CHANNEL_SCALE;
            } else {
                const float rc = 1.0f / k.divisor;
                for (int c = 0; c < 3; ++c) q[c] = s[c] * rc;
                qa = (s[3] * rc) * CHANNEL_SCALE;
            }
            const float ua = k.preserve_alpha ? float(center >> 24) * CHANNEL_SCALE : qa + k.bias;
            const float a = clampf(ua, 0.0f, 1.0f);
            const float bb = k.bias * ua;
            float c3[3];
            for (int c = 0; c < 3; ++c) {
                const float v = q[c] + bb;
                c3[c] = k.preserve_alpha ? clampf(v, 0.0f, 1.0f) * a : clampf(v, 0.0f, a);
            }
            dst[o] = pack(f2u(clampf(c3[0], 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(c3[1], 0.0f, 1.0f) * 255.0f + 0.5f),
                          f2u(clampf(c3[2], 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(a, 0.0f, 1.0f) * 255.0f + 0.5f));
        }
}

void filter_chain(uint32_t* surface, uint32_t width, const int32_t b[4], const tk_filter* chain, uint32_t count,
                  const uint32_t* tables = nullptr) {
    if (b[2] <= b[0] || b[3] <= b[1]) return;
    for (uint32_t k = 0; k < count; ++k) {
        const tk_filter& f = chain[k];
        if (f.kind == TK_FILTER_BLUR) {  // apply_blur at full resolution (blur.rs:194-244)
            const float sx = fmax_(f.std_dev, 0.0f), sy = fmax_(f.amount, 0.0f);
            if (sx <= 0.0f && sy <= 0.0f) continue;
            std::vector<uint32_t> temp(size_t(width) * size_t(b[3]), 0u);
            const uint32_t region[4] = {uint32_t(b[0]), uint32_t(b[1]), uint32_t(b[2] - b[0]), uint32_t(b[3] - b[1])};
            const uint32_t none[4] = {0, 0, 0, 0};
            const uint32_t h = uint32_t(b[3]);
            blur_pass(surface, temp.data(), width, h, region, none, sx > 0.0f ? sx : sy, sx > 0.0f ? 0u : 1u, 1);
            if (sx > 0.0f && sy > 0.0f) {
                blur_pass(temp.data(), surface, width, h, region, none, sy, 1, 1);
            } else {
                for (int32_t y = b[1]; y < b[3]; ++y)
                    for (int32_t x = b[0]; x < b[2]; ++x) surface[size_t(y) * width + x] = temp[size_t(y) * width + x];
            }
        } else if (f.kind == TK_FILTER_CONVOLVE) {  // into a scratch copy, then back (effects.rs:115-133)
            std::vector<uint32_t> temp(size_t(width) * size_t(b[3]), 0u);
            float* kernel = nullptr;
            std::vector<float> kv(size_t(f.columns) * f.rows);
            for (size_t t = 0; t < kv.size(); ++t) kv[t] = bits_f(tables[f.color + t]);
            kernel = kv.data();
            convolve_pass(surface, temp.data(), width, b, f, kernel);
            for (int32_t y = b[1]; y < b[3]; ++y)
                for (int32_t x = b[0]; x < b[2]; ++x) surface[size_t(y) * width + x] = temp[size_t(y) * width + x];
        } else if (f.kind == TK_FILTER_FLOOD) {  // filter_flood_region (filter/brush.hlsl:19-26)
            for (int32_t y = b[1]; y < b[3]; ++y)
                for (int32_t x = b[0]; x < b[2]; ++x) surface[size_t(y) * width + x] = f.color;
        } else if (f.kind == TK_FILTER_DROP_SHADOW) {
            // shadow.rs:3-52: the alpha mask at the offset, the blur, the tinted
            // shadow under the source (filter/basic.hlsl:58-66, filter/brush.hlsl:27-36)
            std::vector<uint32_t> mask(size_t(width) * size_t(b[3]), 0u), temp(mask.size(), 0u);
            for (int32_t y = b[1]; y < b[3]; ++y)
                for (int32_t x = b[0]; x < b[2]; ++x) {
                    const uint32_t a = surface[size_t(y) * width + x] >> 24;
                    if (a == 0u) continue;
                    const int64_t tx = int64_t(x) + f.dx, ty = int64_t(y) + f.dy;
                    if (tx >= b[0] && ty >= b[1] && tx < b[2] && ty < b[3]) mask[size_t(ty) * width + size_t(tx)] = a * 0x01010101u;
                }
            if (f.std_dev > 0.0f) {
                const uint32_t region[4] = {uint32_t(b[0]), uint32_t(b[1]), uint32_t(b[2] - b[0]), uint32_t(b[3] - b[1])};
                const uint32_t none[4] = {0, 0, 0, 0};
                const uint32_t h = uint32_t(b[3]);
                blur_pass(mask.data(), temp.data(), width, h, region, none, f.std_dev, 0, 1);
                blur_pass(temp.data(), mask.data(), width, h, region, none, f.std_dev, 1, 1);
            }
            for (int32_t y = b[1]; y < b[3]; ++y)
                for (int32_t x = b[0]; x < b[2]; ++x) {
                    uint32_t& p = surface[size_t(y) * width + x];
                    p = src_over_premul_u8(scale_premul_u8(f.color, mask[size_t(y) * width + x] >> 24), p);
                }
        } else if (f.kind == TK_FILTER_ERODE || f.kind == TK_FILTER_DILATE) {
            // effects.rs:169-221: nothing for zero radii; an erosion whose
            // doubled radius reaches the surface size clears it; else x, then y
            if (f.dx == 0 && f.dy == 0) continue;
            const uint32_t sw = uint32_t(b[2] - b[0]), sh = uint32_t(b[3] - b[1]);
            const uint32_t rx = uint32_t(f.dx), ry = uint32_t(f.dy);
            const bool dilate = f.kind == TK_FILTER_DILATE;
            if (!dilate && (uint64_t(rx) * 2 >= sw || uint64_t(ry) * 2 >= sh)) {
                for (int32_t y = b[1]; y < b[3]; ++y)
                    for (int32_t x = b[0]; x < b[2]; ++x) surface[size_t(y) * width + x] = 0u;
                continue;
            }
            std::vector<uint32_t> temp(size_t(width) * size_t(b[3]), 0u);
            morphology_pass(surface, temp.data(), width, b, std::min(rx, sw - 1u), dilate, true);
            morphology_pass(temp.data(), surface, width, b, std::min(ry, sh - 1u), dilate, false);
        } else if (f.kind == TK_FILTER_OFFSET) {
            if (f.dx == 0 && f.dy == 0) continue;
            std::vector<uint32_t> temp(size_t(b[2] - b[0]) * size_t(b[3] - b[1]));
            for (int32_t y = b[1]; y < b[3]; ++y)
                for (int32_t x = b[0]; x < b[2]; ++x) {
                    const int64_t sx = int64_t(x) - f.dx, sy = int64_t(y) - f.dy;
                    uint32_t p = 0u;
                    if (sx >= b[0] && sy >= b[1] && sx < b[2] && sy < b[3]) p = surface[size_t(sy) * width + size_t(sx)];
                    temp[size_t(y - b[1]) * size_t(b[2] - b[0]) + size_t(x - b[0])] = p;
                }
            for (int32_t y = b[1]; y < b[3]; ++y)
                for (int32_t x = b[0]; x < b[2]; ++x)
                    surface[size_t(y) * width + x] = temp[size_t(y - b[1]) * size_t(b[2] - b[0]) + size_t(x - b[0])];
        } else {
            for (int32_t y = b[1]; y < b[3]; ++y)
                for (int32_t x = b[0]; x < b[2]; ++x) {
                    uint32_t& p = surface[size_t(y) * width + x];
                    p = f.kind == TK_FILTER_COLOR_MATRIX ? filter_color_matrix_pixel(f.matrix, p)
                        : f.kind == TK_FILTER_COMPONENT_TRANSFER
                            ? filter_transfer_pixel(tables + f.color, p)
                            : filter_color_pixel(p, f.kind, f.amount);
                }
        }
    }
}

// --- filter/progressive.hlsl and progressive/{mod,pyramid}.rs -------------------
// The progressive blur: a pyramid of RGBA8 levels (each the previous one
// convolved with a paired Gaussian kernel along x then y and decimated by its
// step), then per pixel the smoothstep standard deviation of the gradient,
// interpolated between the two levels that bracket its variance (a 7-tap
// kernel for sigma <= 1). Level samples are explicit bilinear lerps
// (a + t (b - a)) with transparent texels outside a level.
struct ProgLevel {
    uint32_t w, h;
    float scale, variance;
    uint32_t step;
    std::vector<float> offset, weight;  // paired kernel
};
// levels() and gaussian_kernel() (pyramid.rs:17-90) in f32, the host's
// expf / powf / sqrtf
std::vector<ProgLevel> prog_levels(uint32_t w, uint32_t h, float sigma, uint32_t quality) {
    const float octave_steps = quality == TK_PROGRESSIVE_HIGH ? 3.0f : 2.0f;
    const float min_sigma = quality == TK_PROGRESSIVE_HIGH ? 2.0f : 1.5f;
    const float support = quality == TK_PROGRESSIVE_HIGH ? 4.0f : 3.0f;
    std::vector<ProgLevel> levels{{w, h, 1.0f, 0.0f, 1u, {}, {}}};
    if (sigma <= 1.0f) return levels;
    float raw_variance = 0.0f, target_sigma = 1.0f;
    while (levels.back().variance < sigma * sigma) {
        if (levels.size() > 64) throw std::runtime_error("progressive blur level count overflow");
        const ProgLevel prev = levels.back();
        const uint32_t step = target_sigma >= min_sigma * prev.scale * 2.0f ? 2u : 1u;
        const float scale = prev.scale * float(step);
        const float reconstruction = scale == 1.0f ? 0.0f : (2.0f * scale * scale + 1.0f) / 12.0f;
        const float incremental =
            std::sqrt((target_sigma * target_sigma - reconstruction - raw_variance) / (prev.scale * prev.scale));
        const int32_t radius = int32_t(std::ceil(incremental * support));
        const float center = float(step - 1u) * 0.5f;
        std::vector<float> xs, ws;
        for (int32_t x = -radius; x < radius + int32_t(step); ++x) {
            const float d = (float(x) - center) / incremental;
            xs.push_back(float(x));
            ws.push_back(std::exp(-0.5f * (d * d)));
        }
        float total = 0.0f;
        for (float v : ws) total += v;
        float variance = 0.0f;
        for (size_t k = 0; k < ws.size(); ++k) {
            ws[k] /= total;
            const float d = xs[k] - center;
            variance += ws[k] * (d * d);
        }
        ProgLevel L{(prev.w + step - 1u) / step, (prev.h + step - 1u) / step, scale, 0.0f, step, {}, {}};
        for (size_t k = 0; k < ws.size(); k += 2) {
            float weight = ws[k], moment = xs[k] * ws[k];
            if (k + 1 < ws.size()) {
                weight += ws[k + 1];
                moment += xs[k + 1] * ws[k + 1];
            }
            L.offset.push_back(moment / weight);
            L.weight.push_back(weight);
        }
        raw_variance += variance * prev.scale * prev.scale;
        L.variance = raw_variance + reconstruction;
        levels.push_back(std::move(L));
        target_sigma *= std::pow(2.0f, 1.0f / octave_steps);
    }
    if (levels.size() > 64) throw std::runtime_error("progressive blur level count overflow");
    return levels;
}
inline F4 prog_fetch(const std::vector<uint32_t>& img, uint32_t w, uint32_t h, int32_t x, int32_t y) {
    if (x < 0 || y < 0 || x >= int32_t(w) || y >= int32_t(h)) return {0, 0, 0, 0};
    return texel_load(img[size_t(y) * w + size_t(x)]);
}
inline F4 lerp_f4(F4 a, F4 b, float t) {
    return {a.r + t * (b.r - a.r), a.g + t * (b.g - a.g), a.b + t * (b.b - a.b), a.a + t * (b.a - a.a)};
}
F4 prog_bilinear(const std::vector<uint32_t>& img, uint32_t w, uint32_t h, float px, float py) {
    const float bx = std::floor(px), by = std::floor(py);
    const int32_t ix = f2i(bx), iy = f2i(by);
    const float fx = px - bx, fy = py - by;
    return lerp_f4(lerp_f4(prog_fetch(img, w, h, ix, iy), prog_fetch(img, w, h, ix + 1, iy), fx),
                   lerp_f4(prog_fetch(img, w, h, ix, iy + 1), prog_fetch(img, w, h, ix + 1, iy + 1), fx), fy);
}
void progressive_blur(uint32_t* surface, uint32_t width, const int32_t rect[4], const tk_progressive_blur& blur) {
    const uint32_t w = uint32_t(rect[2] - rect[0]), h = uint32_t(rect[3] - rect[1]);
    const std::vector<ProgLevel> plan = prog_levels(w, h, blur.max_std_dev, blur.quality);
    std::vector<std::vector<uint32_t>> img(plan.size());
    img[0].resize(size_t(w) * h);
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x)
            img[0][size_t(y) * w + x] = surface[size_t(rect[1] + int32_t(y)) * width + size_t(rect[0]) + x];
    for (size_t i = 1; i < plan.size(); ++i) {  // progressive_blur_reduce along x, then y
        const ProgLevel& L = plan[i];
        const ProgLevel& P = plan[i - 1];
        auto reduce = [&](const std::vector<uint32_t>& src, uint32_t sw, uint32_t sh, std::vector<uint32_t>& dst,
                          uint32_t dw, uint32_t dh, uint32_t axis) {
            dst.assign(size_t(dw) * dh, 0u);
            for (uint32_t y = 0; y < dh; ++y)
                for (uint32_t x = 0; x < dw; ++x) {
                    float cx = float(x), cy = float(y);
                    if (axis == 0u) cx *= float(L.step);
                    else cy *= float(L.step);
                    F4 c{0, 0, 0, 0};
                    for (size_t k = 0; k < L.offset.size(); ++k) {
                        float px = cx, py = cy;
                        if (axis == 0u) px += L.offset[k];
                        else py += L.offset[k];
                        const F4 sv = prog_bilinear(src, sw, sh, px, py);
                        const float wt = L.weight[k];
                        c = {c.r + wt * sv.r, c.g + wt * sv.g, c.b + wt * sv.b, c.a + wt * sv.a};
                    }
                    dst[size_t(y) * dw + x] = texel_store(c);
                }
        };
        std::vector<uint32_t> scratch;
        reduce(img[i - 1], P.w, P.h, scratch, L.w, P.h, 0u);
        reduce(scratch, L.w, P.h, img[i], L.w, L.h, 1u);
    }
    auto sample_level = [&](size_t i, float px, float py) {
        const ProgLevel& L = plan[i];
        return prog_bilinear(img[i], L.w, L.h, px / L.scale - 0.5f, py / L.scale - 0.5f);
    };
    for (uint32_t y = uint32_t(rect[1]); y < uint32_t(rect[3]); ++y)  // progressive_blur_resolve
        for (uint32_t x = uint32_t(rect[0]); x < uint32_t(rect[2]); ++x) {
            float t = 1.0f;
            if (!(blur.dir_x == 0.0f && blur.dir_y == 0.0f))
                t = clampf(((float(x) + 0.5f) - blur.start_x) * blur.dir_x +
                               ((float(y) + 0.5f) - blur.start_y) * blur.dir_y,
                           0.0f, 1.0f);
            const float sigma = blur.max_std_dev * t * t * (3.0f - 2.0f * t);
            if (sigma < 0.125f) continue;
            const float px = float(x - uint32_t(rect[0])) + 0.5f, py = float(y - uint32_t(rect[1])) + 0.5f;
            F4 out;
            if (sigma <= 1.0f) {  // shallow_blur (progressive.hlsl:68-95)
                float wts[7], total = 0.0f;
                for (int k = 0; k < 7; ++k) {
                    const float d = float(k - 3);
                    wts[k] = exp_nonpos(-0.5f * d * d / (sigma * sigma));
                    total += wts[k];
                }
                float off[4], comb[4];
                for (int k = 0; k < 4; ++k) {
                    const int first = 2 * k;
                    const float second = first + 1 < 7 ? wts[first + 1] : 0.0f;
                    comb[k] = wts[first] + second;
                    off[k] = float(first - 3) + (comb[k] > 0.0f ? second / comb[k] : 0.0f);
                }
                F4 c{0, 0, 0, 0};
                for (int j = 0; j < 4; ++j)
                    for (int k = 0; k < 4; ++k) {
                        const float wt = comb[k] * comb[j];
                        const F4 sv = sample_level(0, px + off[k], py + off[j]);
                        c = {c.r + wt * sv.r, c.g + wt * sv.g, c.b + wt * sv.b, c.a + wt * sv.a};
                    }
                const float tt = total * total;
                out = {c.r / tt, c.g / tt, c.b / tt, c.a / tt};
            } else {
                const float variance = sigma * sigma;
                size_t upper = 1;
                while (upper + 1 < plan.size() && plan[upper].variance < variance) ++upper;
                const float lo = plan[upper - 1].variance, hi = plan[upper].variance;
                const float weight = clampf((variance - lo) / (hi - lo), 0.0f, 1.0f);
                out = lerp_f4(sample_level(upper - 1, px, py), sample_level(upper, px, py), weight);
            }
            surface[size_t(y) * width + x] = texel_store(out);
        }
}

void downsample_region(const uint32_t* src, uint32_t* low, uint32_t width, const int32_t rect[4],
                       const int32_t low_rect[4], uint32_t factor, uint32_t filter) {
    const uint32_t x0 = uint32_t(rect[0]), y0 = uint32_t(rect[1]), x1 = uint32_t(rect[2]), y1 = uint32_t(rect[3]);
    for (uint32_t ly = uint32_t(low_rect[1]); ly < uint32_t(low_rect[3]); ++ly)
        for (uint32_t lx = uint32_t(low_rect[0]); lx < uint32_t(low_rect[2]); ++lx) {
            const uint32_t bx = std::max(lx * factor, x0), by = std::max(ly * factor, y0);
            const uint32_t ex = std::min((lx + 1u) * factor, x1), ey = std::min((ly + 1u) * factor, y1);
            uint32_t out = 0u;
            if (bx < ex && by < ey) {
                if (filter == 0u) {
                    const uint32_t px = std::min(std::max((bx + ex - 1u) / 2u, x0), x1 - 1u);
                    const uint32_t py = std::min(std::max((by + ey - 1u) / 2u, y0), y1 - 1u);
                    out = src[size_t(py) * width + px];
                } else {
                    float sum[4] = {0, 0, 0, 0};
                    for (uint32_t sy = by; sy < ey; ++sy)
                        for (uint32_t sx = bx; sx < ex; ++sx) {
                            const uint32_t p = src[size_t(sy) * width + sx];
                            for (int c = 0; c < 4; ++c) sum[c] += float((p >> (8 * c)) & 255u);
                        }
                    const float inv = 1.0f / float((ex - bx) * (ey - by));
                    uint32_t b[4];
                    for (int c = 0; c < 4; ++c) b[c] = f2u(clampf(mad(sum[c], inv, 0.5f), 0.0f, 255.0f));
                    out = pack(b[0], b[1], b[2], b[3]);
                }
            }
            low[size_t(ly) * width + lx] = out;
        }
}
// filter_upsample_pixel for every texel of `rect`: the nearest low texel
// (filter 0) or the bilinear sample stored by pack_premul_rgba8 (filter 1).
void upsample_region(const uint32_t* low, uint32_t* dst, uint32_t width, uint32_t height, const int32_t rect[4],
                     const int32_t low_rect[4], uint32_t factor, uint32_t filter) {
    const float f = float(std::max(factor, 1u));
    for (uint32_t y = uint32_t(rect[1]); y < uint32_t(rect[3]); ++y)
        for (uint32_t x = uint32_t(rect[0]); x < uint32_t(rect[2]); ++x) {
            const float px = clampf((float(x) + 0.5f) / f - 0.5f, float(low_rect[0]), float(uint32_t(low_rect[2]) - 1u));
            const float py = clampf((float(y) + 0.5f) / f - 0.5f, float(low_rect[1]), float(uint32_t(low_rect[3]) - 1u));
            uint32_t out;
            if (filter == 0u) {
                out = low[size_t(f2i(round_ne(py))) * width + uint32_t(f2i(round_ne(px)))];
            } else {
                const F4 p = sample_premul(low, width, height, px, py);
                out = pack(f2u(clampf(p.r, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(p.g, 0.0f, 1.0f) * 255.0f + 0.5f),
                           f2u(clampf(p.b, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(p.a, 0.0f, 1.0f) * 255.0f + 0.5f));
            }
            dst[size_t(y) * width + x] = out;
        }
}

// ---------------------------------------------------------------------------
// Frame driver.
// ---------------------------------------------------------------------------
void fine_pass(or_scene& S, uint32_t pass, std::vector<uint32_t>& target, int threads) {
    auto& streams = S.pass_streams[pass];
    parallel_for(threads, S.band_tiles.size(), [&](uint64_t bt) {
        const uint32_t tile = S.band_tiles[bt];
        uint32_t ty = tile / S.tw, tx = tile % S.tw;
        const auto& list = streams[tile];
        if (list.empty()) return;  // EMPTY in every batch: target unchanged
        for (uint32_t ly = 0; ly < TK_TILE_SIZE; ++ly) {
            uint32_t gy = ty * TK_TILE_SIZE + ly;
            if (gy >= S.desc.height) break;
            for (uint32_t lx = 0; lx < TK_TILE_SIZE; ++lx) {
                uint32_t gx = tx * TK_TILE_SIZE + lx;
                if (gx >= S.desc.width) break;
                uint32_t& texel = target[size_t(gy) * S.desc.width + gx];
                for (const BatchStream& bs : list) {  // one reference fine dispatch per batch
                    F4 pixel = texel_load(texel);     // fine_initial_pixel with load_target
                    uint32_t kind = bs.kind & TK_TILE_KIND_MASK;
                    uint32_t begin = bs.kind >> TK_TILE_PREFIX_SHIFT;
                    uint32_t end = uint32_t(bs.recs.size());
                    if (kind == TK_TILE_KIND_INTERPRETER)
                        pixel = interpret(S, bs.recs, begin, end, pixel, lx, ly, gx, gy, bs.glyphs.data());
                    else if (kind == TK_TILE_KIND_COLOR) pixel = color_only(bs.recs, begin, end, pixel);
                    else if (kind == TK_TILE_KIND_SDF || kind == TK_TILE_KIND_MIXED)
                        pixel = analytic_solid(S, bs.recs, begin, end, pixel, gx, gy);
                    texel = texel_store(pixel);
                }
            }
        }
    });
}

// Scan (count, prefix + cumsum, emit) over every line and the tile bins of
// every draw: the frame's work that does not depend on the tile rows drawn.
void scan_scene(or_scene& S, int threads) {
    const tk_scene_desc& D = S.desc;
    S.tw = (D.width + TK_TILE_SIZE - 1) / TK_TILE_SIZE;
    S.th = (D.height + TK_TILE_SIZE - 1) / TK_TILE_SIZE;
    S.T = S.tw * S.th;
    uint32_t np = uint32_t(S.paths.size());
    for (const auto& p : S.paths) {
        S.B = std::max<uint64_t>(S.B, uint64_t(p.data_offset) + p.data_len);
        S.seg_capacity = std::max<uint64_t>(S.seg_capacity, uint64_t(p.segment_start) + p.segment_capacity);
    }
    S.backdrops.assign(S.B, 0);
    S.counts.assign(S.B, 0u);
    S.ranges.assign(S.B, tk_segment_range{0, 0});
    S.cursors.assign(S.B, 0u);
    S.bumps.assign(np, 0u);

    // scan_count: per path (disjoint slices), lines in order.
    auto t0 = clk::now();
    parallel_for(threads, np, [&](uint64_t pid) {
        const tk_path_record& p = S.paths[pid];
        for (uint32_t l = 0; l < p.line_count; ++l)
            count_line(D.lines[p.line_start + l], S.paths.data(), np, S.backdrops.data(), S.counts.data());
    });
    S.times[0] = since(t0);

    // Device segment plan (TK_SCENE_SEGMENTS_FROM_DEVICE, the library's
    // chained pool scan): capacities are the scanned totals and segment
    // slices follow each other from 0 in path order.
    if (D.flags & TK_SCENE_SEGMENTS_FROM_DEVICE) {
        uint64_t next = 0;
        for (tk_path_record& p : S.paths) {
            uint32_t total = 0;
            for (uint32_t k = 0; k < p.data_len; ++k) total += S.counts[p.data_offset + k];
            p.segment_start = uint32_t(next);
            p.segment_capacity = total;
            next += total;
        }
        S.seg_capacity = next;
    }

    // prefix (scan_prefix_chunks + offsets) and row cumsum (cumsum.hlsl).
    t0 = clk::now();
    parallel_for(threads, np, [&](uint64_t pid) {
        const tk_path_record& p = S.paths[pid];
        uint32_t next = p.segment_start;
        for (uint32_t k = 0; k < p.data_len; ++k) {
            uint32_t t = p.data_offset + k;
            uint32_t c = S.counts[t];
            S.ranges[t] = {next, next + c};
            S.cursors[t] = next;
            next += c;
        }
        S.bumps[pid] = next - p.segment_start;
        uint32_t stride = p.tile_x1 > p.tile_x0 ? p.tile_x1 - p.tile_x0 : 0u;
        if (stride == 0u) return;
        for (uint32_t row = 0; row * stride < p.data_len; ++row) {
            int32_t acc = 0;
            for (uint32_t k = 0; k < stride; ++k) {
                int32_t& v = S.backdrops[p.data_offset + row * stride + k];
                acc = int32_t(uint32_t(acc) + uint32_t(v));
                v = acc;
            }
        }
    });
    S.times[1] = since(t0);

    // scan_emit in canonical order.
    t0 = clk::now();
    S.segments.assign(S.seg_capacity, tk_line_segment{0, 0, 0, 0, 0});
    parallel_for(threads, np, [&](uint64_t pid) {
        emit_path(D.lines, S.paths.data(), np, uint32_t(pid), S.cursors.data(), S.segments.data(), S.seg_capacity);
    });
    S.times[2] = since(t0);

    // Tile bins (tile_bins/build.rs:54-77).
    t0 = clk::now();
    S.bins.assign(S.T, {});
    for (uint32_t k = 0; k < D.draw_order_count; ++k) {
        uint32_t di = D.draw_order[k];
        const tk_pixel_bounds& pb = S.draws[di].pixel_bounds;
        uint32_t x0 = std::min(uint32_t(std::max(pb.x0, 0)) / TK_TILE_SIZE, S.tw);
        uint32_t y0 = std::min(uint32_t(std::max(pb.y0, 0)) / TK_TILE_SIZE, S.th);
        uint32_t x1 = std::min((uint32_t(std::max(pb.x1, 0)) + TK_TILE_SIZE - 1) / TK_TILE_SIZE, S.tw);
        uint32_t y1 = std::min((uint32_t(std::max(pb.y1, 0)) + TK_TILE_SIZE - 1) / TK_TILE_SIZE, S.th);
        for (uint32_t y = y0; y < y1; ++y)
            for (uint32_t x = x0; x < x1; ++x) S.bins[size_t(y) * S.tw + x].push_back(di);
    }
    S.times[3] = since(t0);
}

// Coarse and fine of every target pass, and the blur layers, over the tile
// rows of S.in_band (the rows outside keep the clear colour).
void raster_scene(or_scene& S, int threads) {
    const tk_scene_desc& D = S.desc;
    if (S.ty1 == 0 || S.ty1 > S.th) S.ty1 = S.th;
    if (S.row_step == 0u) S.row_step = 1u;
    S.batches.clear();
    S.pass_streams.clear();
    S.times[4] = S.times[5] = S.times[6] = 0.0;
    S.band_tiles.clear();
    for (uint32_t ty = 0; ty < S.th; ++ty)
        if (S.in_band(ty))
            for (uint32_t tx = 0; tx < S.tw; ++tx) S.band_tiles.push_back(ty * S.tw + tx);
    // Walk ops: batches, passes, blur layers.
    std::vector<uint32_t> main_target(size_t(D.width) * D.height, D.clear_color);
    struct Surface {
        std::vector<uint32_t> img;
        float sigma;
        int32_t bounds[4];
        uint32_t sampling;
        bool progressive = false;
        tk_progressive_blur prog{};
        bool filter = false;  // a filter layer: its chain
        std::vector<tk_filter> chain;
    };
    std::vector<Surface> surfaces;
    auto current = [&]() -> std::vector<uint32_t>& { return surfaces.empty() ? main_target : surfaces.back().img; };
    bool pass_open = false;
    std::vector<uint32_t> pass_batches;
    auto flush_pass = [&]() {
        if (!pass_open) return;
        pass_open = false;
        uint32_t pass = uint32_t(S.pass_streams.size());
        S.pass_streams.emplace_back(S.T);
        auto& streams = S.pass_streams.back();
        auto tc = clk::now();
        // Batch ids grow along the draw order and along the pass's batches in
        // compiled plans, so each tile's candidates of one batch are one
        // painter-order run that a single walk finds (the reference's
        // per-batch bins); other plans search the whole candidate list.
        bool sorted = true;
        for (size_t k = 1; k < pass_batches.size(); ++k)
            sorted = sorted && S.batches[pass_batches[k - 1]].batch_id < S.batches[pass_batches[k]].batch_id;
        for (uint32_t k = 1; k < D.draw_order_count && sorted; ++k)
            sorted = S.batch_ids[D.draw_order[k - 1]] <= S.batch_ids[D.draw_order[k]];
        parallel_for(threads, S.band_tiles.size(), [&](uint64_t bt) {
            const uint32_t tile = S.band_tiles[bt];
            const auto& cand = S.bins[tile];
            uint32_t walk = 0;
            for (uint32_t bi : pass_batches) {
                const Batch& b = S.batches[bi];
                // Candidates of one batch form a contiguous painter-order run.
                uint32_t first = 0, n = 0;
                if (sorted) {
                    while (walk < cand.size() && S.batch_ids[cand[walk]] < b.batch_id) ++walk;
                    first = walk;
                    while (walk < cand.size() && S.batch_ids[cand[walk]] == b.batch_id) ++walk;
                    n = walk - first;
                } else {
                    for (uint32_t k = 0; k < cand.size(); ++k) {
                        if (S.batch_ids[cand[k]] == b.batch_id) {
                            if (n == 0) first = k;
                            ++n;
                        }
                    }
                }
                BatchStream bs;
                if (b.layer_end > b.layer_start || n > 0) {
                    // Non-contiguous runs cannot occur for compiled plans; fall back to the full list.
                    bool contiguous = n == 0 || (first + n <= cand.size() && S.batch_ids[cand[first + n - 1]] == b.batch_id);
                    bool ok = contiguous ? coarse_tile(S, b, bi, uint32_t(tile), cand.data() + first, n, bs)
                                         : coarse_tile(S, b, bi, uint32_t(tile), cand.data(), uint32_t(cand.size()), bs);
                    if (ok) streams[tile].push_back(std::move(bs));
                }
            }
        });
        for (uint32_t bi : pass_batches) {
            uint64_t total = 0;
            for (uint32_t t = 0; t < S.T; ++t)
                for (const auto& bs : streams[t]) if (bs.batch == bi) total += bs.recs.size();
            S.batches[bi].total = total;
        }
        S.times[4] += since(tc);
        tc = clk::now();
        fine_pass(S, pass, current(), threads);
        S.times[5] += since(tc);
        pass_batches.clear();
    };
    for (uint32_t oi = 0; oi < D.op_count; ++oi) {
        const tk_op& op = D.ops[oi];
        if (op.kind == TK_OP_DRAW_BATCH) {
            if (!pass_open) pass_open = true;
            uint32_t bi = uint32_t(S.batches.size());
            S.batches.push_back({op.batch_id, op.layer_start, op.layer_end, uint32_t(S.pass_streams.size()), 0});
            pass_batches.push_back(bi);
        } else if (op.kind == TK_OP_BLUR_BEGIN) {
            flush_pass();
            Surface s;
            s.img.assign(size_t(D.width) * D.height, 0u);
            s.sigma = op.sigma;
            std::memcpy(s.bounds, op.bounds, sizeof(s.bounds));
            s.sampling = (op.batch_id & 255u) > 1u ? op.batch_id : 0u;  // BlurSampling word
            surfaces.push_back(std::move(s));
        } else if (op.kind == TK_OP_PROGRESSIVE_BEGIN) {
            flush_pass();
            if (op.batch_id >= D.progressive_count) throw std::runtime_error("progressive blur out of range");
            Surface s;
            s.img.assign(size_t(D.width) * D.height, 0u);
            s.sigma = op.sigma;
            std::memcpy(s.bounds, op.bounds, sizeof(s.bounds));
            s.sampling = 0u;
            s.progressive = true;
            s.prog = D.progressive_blurs[op.batch_id];
            surfaces.push_back(std::move(s));
        } else if (op.kind == TK_OP_FILTER_BEGIN) {
            flush_pass();
            if (op.batch_id >= D.filter_layer_count) throw std::runtime_error("filter layer out of range");
            const tk_filter_layer& L = D.filter_layers[op.batch_id];
            if (uint64_t(L.first) + L.count > D.filter_count) throw std::runtime_error("filter chain out of range");
            Surface s;
            s.img.assign(size_t(D.width) * D.height, 0u);
            s.sigma = 0.0f;
            // output bounds: the surface clipped to the canvas (filter.rs:510-527)
            s.bounds[0] = std::max(L.surface[0], 0);
            s.bounds[1] = std::max(L.surface[1], 0);
            s.bounds[2] = std::min(L.surface[2], int32_t(D.width));
            s.bounds[3] = std::min(L.surface[3], int32_t(D.height));
            s.sampling = 0u;
            s.filter = true;
            s.chain.assign(D.filters + L.first, D.filters + L.first + L.count);
            for (const tk_filter& f : s.chain)
                if ((f.kind == TK_FILTER_COMPONENT_TRANSFER &&
                     uint64_t(f.color) + TK_TRANSFER_TABLE_WORDS > D.filter_word_count) ||
                    (f.kind == TK_FILTER_CONVOLVE && uint64_t(f.color) + uint64_t(f.columns) * f.rows > D.filter_word_count))
                    throw std::runtime_error("filter words out of range");
            surfaces.push_back(std::move(s));
        } else if (op.kind == TK_OP_BLUR_END) {
            flush_pass();
            if (surfaces.empty()) throw std::runtime_error("unbalanced BLUR_END");
            Surface s = std::move(surfaces.back());
            surfaces.pop_back();
            auto tb = clk::now();
            // Output bounds (op.bounds) and the surface they read from: the
            // output outset by the blur radius, clipped to the canvas
            // (shared/layer/filter.rs:510-531,599-601).
            int32_t bx0 = std::max(s.bounds[0], 0), by0 = std::max(s.bounds[1], 0);
            int32_t bx1 = std::min(s.bounds[2], int32_t(D.width)), by1 = std::min(s.bounds[3], int32_t(D.height));
            int32_t rad = int32_t(std::ceil(fmax_(s.sigma, 0.0f) * 3.0f));
            int32_t sx0 = std::max(s.bounds[0] - rad, 0), sy0 = std::max(s.bounds[1] - rad, 0);
            int32_t sx1 = std::min(s.bounds[2] + rad, int32_t(D.width));
            int32_t sy1 = std::min(s.bounds[3] + rad, int32_t(D.height));
            if (s.filter) {
                const int32_t rect[4] = {bx0, by0, bx1, by1};
                filter_chain(s.img.data(), D.width, rect, s.chain.data(), uint32_t(s.chain.size()), D.filter_words);
            } else if (s.progressive) {
                if (bx1 > bx0 && by1 > by0 && s.prog.max_std_dev > 0.0f) {
                    const int32_t rect[4] = {bx0, by0, bx1, by1};
                    progressive_blur(s.img.data(), D.width, rect, s.prog);
                }
            } else if (s.sampling != 0u && bx1 > bx0 && by1 > by0 && s.sigma > 0.0f) {
                // BlurSampling factor > 1 (render/filter_program/blur.rs:24-73): reduce
                // the output bounds, blur at sigma / factor, restore
                const uint32_t factor = s.sampling & 255u;
                const int32_t f = int32_t(factor);
                auto fdiv = [](int32_t v, int32_t d) { return v >= 0 ? v / d : -((-v + d - 1) / d); };
                const int32_t rect[4] = {bx0, by0, bx1, by1};
                const int32_t lr[4] = {fdiv(bx0, f), fdiv(by0, f), -fdiv(-bx1, f), -fdiv(-by1, f)};
                std::vector<uint32_t> low(s.img.size(), 0u), temp(s.img.size(), 0u);
                downsample_region(s.img.data(), low.data(), D.width, rect, lr, factor, (s.sampling >> 8) & 255u);
                uint32_t region[4] = {uint32_t(lr[0]), uint32_t(lr[1]), uint32_t(lr[2] - lr[0]), uint32_t(lr[3] - lr[1])};
                uint32_t none[4] = {0, 0, 0, 0};
                const float low_sigma = s.sigma / float(factor);
                blur_pass(low.data(), temp.data(), D.width, D.height, region, none, low_sigma, 0, threads);
                blur_pass(temp.data(), low.data(), D.width, D.height, region, none, low_sigma, 1, threads);
                upsample_region(low.data(), s.img.data(), D.width, D.height, rect, lr, factor, (s.sampling >> 16) & 255u);
            } else if (bx1 > bx0 && by1 > by0 && s.sigma > 0.0f) {
                uint32_t region[4] = {uint32_t(sx0), uint32_t(sy0), uint32_t(sx1 - sx0), uint32_t(sy1 - sy0)};
                uint32_t none[4] = {0, 0, 0, 0};
                std::vector<uint32_t> temp(s.img.size(), 0u);
                blur_pass(s.img.data(), temp.data(), D.width, D.height, region, none, s.sigma, 0, threads);
                blur_pass(temp.data(), s.img.data(), D.width, D.height, region, none, s.sigma, 1, threads);
            }
            std::vector<uint32_t>& dst = current();
            for (int32_t y = by0; y < by1; ++y)
                for (int32_t x = bx0; x < bx1; ++x) {
                    size_t i = size_t(y) * D.width + x;
                    dst[i] = src_over_premul_u8(dst[i], scale_premul_u8(s.img[i], 255u));
                }
            S.times[6] += since(tb);
        }
    }
    flush_pass();
    if (!surfaces.empty()) throw std::runtime_error("unbalanced BLUR_BEGIN");
    S.image = std::move(main_target);
}

}  // namespace

extern "C" {

const char* or_error(void) { return g_error.c_str(); }

}  // extern "C"

namespace {
void copy_text(or_scene& S, const tk_scene_desc* d) {
    S.glyph_runs.assign(d->glyph_runs, d->glyph_runs + d->glyph_run_count);
    S.glyphs.assign(d->glyphs, d->glyphs + d->glyph_count);
    S.glyph_images.assign(d->glyph_images, d->glyph_images + d->glyph_image_count);
    S.glyph_texels.assign(d->glyph_texels, d->glyph_texels + d->glyph_texel_count);
}
}  // namespace

extern "C" {

int32_t or_run(const tk_scene_desc* d, int32_t threads, uint32_t tile_y0, uint32_t tile_y1, or_scene** out) {
    *out = nullptr;
    try {
        auto* S = new or_scene();
        S->desc = *d;
        S->paths.assign(d->paths, d->paths + d->path_count);
        S->draws.assign(d->draws, d->draws + d->draw_count);
        S->layers.assign(d->layers, d->layers + d->layer_count);
        S->brush.assign(d->brush_blob, d->brush_blob + d->brush_word_count);
        S->sdf.assign(d->sdf_blob, d->sdf_blob + d->sdf_word_count);
        S->shadow.assign(d->sdf_shadow_blob, d->sdf_shadow_blob + d->sdf_shadow_word_count);
        S->batch_ids.assign(d->draw_batch_ids, d->draw_batch_ids + d->draw_count);
        copy_text(*S, d);
        S->ty0 = tile_y0;
        S->ty1 = tile_y1;
        scan_scene(*S, threads < 1 ? 1 : threads);
        raster_scene(*S, threads < 1 ? 1 : threads);
        *out = S;
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

int32_t or_prepare(const tk_scene_desc* d, int32_t threads, or_scene** out) {
    *out = nullptr;
    try {
        auto* S = new or_scene();
        S->desc = *d;
        S->paths.assign(d->paths, d->paths + d->path_count);
        S->draws.assign(d->draws, d->draws + d->draw_count);
        S->layers.assign(d->layers, d->layers + d->layer_count);
        S->brush.assign(d->brush_blob, d->brush_blob + d->brush_word_count);
        S->sdf.assign(d->sdf_blob, d->sdf_blob + d->sdf_word_count);
        S->shadow.assign(d->sdf_shadow_blob, d->sdf_shadow_blob + d->sdf_shadow_word_count);
        S->batch_ids.assign(d->draw_batch_ids, d->draw_batch_ids + d->draw_count);
        copy_text(*S, d);
        scan_scene(*S, threads < 1 ? 1 : threads);
        *out = S;
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

int32_t or_raster(or_scene* S, int32_t threads, uint32_t tile_y0, uint32_t tile_y1, uint32_t row_step) {
    try {
        S->ty0 = tile_y0;
        S->ty1 = tile_y1;
        S->row_step = row_step ? row_step : 1u;
        raster_scene(*S, threads < 1 ? 1 : threads);
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

void or_free(or_scene* s) { delete s; }
uint32_t or_batch_count(const or_scene* s) { return uint32_t(s->batches.size()); }
uint32_t or_pass_count(const or_scene* s) { return uint32_t(s->pass_streams.size()); }
void or_stage_times(const or_scene* s, double out[7]) { std::memcpy(out, s->times, sizeof(s->times)); }

static size_t copy_out(const void* src, size_t need, void* dst, size_t bytes) {
    if (dst) std::memcpy(dst, src, std::min(need, bytes));
    return need;
}

size_t or_get(const or_scene* s, uint32_t what, uint32_t index, void* dst, size_t bytes) {
    switch (what) {
        case OR_COUNTS: return copy_out(s->counts.data(), s->counts.size() * 4, dst, bytes);
        case OR_BACKDROPS: return copy_out(s->backdrops.data(), s->backdrops.size() * 4, dst, bytes);
        case OR_RANGES: return copy_out(s->ranges.data(), s->ranges.size() * 8, dst, bytes);
        case OR_SEGMENTS: return copy_out(s->segments.data(), s->segments.size() * sizeof(tk_line_segment), dst, bytes);
        case OR_IMAGE: return copy_out(s->image.data(), s->image.size() * 4, dst, bytes);
        case OR_PATHS: return copy_out(s->paths.data(), s->paths.size() * sizeof(tk_path_record), dst, bytes);
        case OR_BUMPS: return copy_out(s->bumps.data(), s->bumps.size() * 4, dst, bytes);
        case OR_BATCH_PTCL:
        case OR_BATCH_TILES:
        case OR_BATCH_KINDS: {
            if (index >= s->batches.size()) return 0;
            const Batch& b = s->batches[index];
            const auto& streams = s->pass_streams[b.pass];
            std::vector<tk_ptcl_record> ptcl;
            std::vector<tk_tile_record> tiles(s->T, tk_tile_record{0, 0, 0, 0, 0, 0});
            std::vector<uint32_t> kinds(s->T, TK_TILE_KIND_EMPTY);
            uint32_t next = 0;
            for (uint32_t t = 0; t < s->T; ++t) {
                const BatchStream* found = nullptr;
                for (const auto& bs : streams[t]) if (bs.batch == index) found = &bs;
                uint32_t n = found ? uint32_t(found->recs.size()) : 0u;
                tiles[t] = {n, next, next + n, 0, 0, 0};
                if (found) {
                    ptcl.insert(ptcl.end(), found->recs.begin(), found->recs.end());
                    kinds[t] = found->kind;
                }
                next += n;
            }
            if (what == OR_BATCH_PTCL) return copy_out(ptcl.data(), ptcl.size() * sizeof(tk_ptcl_record), dst, bytes);
            if (what == OR_BATCH_TILES) return copy_out(tiles.data(), tiles.size() * sizeof(tk_tile_record), dst, bytes);
            return copy_out(kinds.data(), kinds.size() * 4, dst, bytes);
        }
        case OR_PASS_PTCL:
        case OR_PASS_TILES:
        case OR_PASS_KINDS:
        case OR_PASS_GLYPHS: {
            // Merged layout: per tile, for each batch with a stream:
            // BATCH_BEGIN{segment_start=batch_id, segment_end=n-1, color=kind}
            // followed by the batch's records without END; then one END.
            if (index >= s->pass_streams.size()) return 0;
            const auto& streams = s->pass_streams[index];
            std::vector<tk_ptcl_record> ptcl;
            std::vector<tk_tile_record> tiles(s->T, tk_tile_record{0, 0, 0, 0, 0, 0});
            std::vector<uint32_t> kinds(s->T, TK_TILE_KIND_EMPTY);
            std::vector<uint32_t> glyphs;  // the pass's glyph list: tile after tile, stream after stream
            uint32_t next = 0;
            for (uint32_t t = 0; t < s->T; ++t) {
                uint32_t n = 0;
                const uint32_t g0 = uint32_t(glyphs.size());
                for (const auto& bs : streams[t]) {
                    uint32_t m = uint32_t(bs.recs.size());
                    ptcl.push_back({TK_PTCL_BATCH_BEGIN, 0, 0u, s->batches[bs.batch].batch_id, m - 1u, bs.kind});
                    const size_t first = ptcl.size();
                    ptcl.insert(ptcl.end(), bs.recs.begin(), bs.recs.end() - 1);
                    const uint32_t base = uint32_t(glyphs.size());
                    for (size_t k = first; k < ptcl.size(); ++k)
                        if (ptcl[k].tag == TK_PTCL_GLYPH) {
                            ptcl[k].segment_start += base;
                            ptcl[k].segment_end += base;
                        }
                    glyphs.insert(glyphs.end(), bs.glyphs.begin(), bs.glyphs.end());
                    n += m;
                }
                if (n) {
                    ptcl.push_back({TK_PTCL_END, 0, 0u, 0u, 0u, 0u});
                    n += 1;
                    kinds[t] = TK_TILE_KIND_INTERPRETER;
                }
                const uint32_t gn = uint32_t(glyphs.size()) - g0;
                tiles[t] = {n, next, next + n, gn, s->glyph_runs.empty() ? 0u : g0, s->glyph_runs.empty() ? 0u : g0 + gn};
                next += n;
            }
            if (what == OR_PASS_GLYPHS) return copy_out(glyphs.data(), glyphs.size() * 4, dst, bytes);
            if (what == OR_PASS_PTCL) return copy_out(ptcl.data(), ptcl.size() * sizeof(tk_ptcl_record), dst, bytes);
            if (what == OR_PASS_TILES) return copy_out(tiles.data(), tiles.size() * sizeof(tk_tile_record), dst, bytes);
            return copy_out(kinds.data(), kinds.size() * 4, dst, bytes);
        }
        default: return 0;
    }
}

uint64_t or_get_range(const or_scene* s, uint32_t what, uint64_t first, uint64_t count, void* dst) {
    const unsigned char* src = nullptr;
    uint64_t n = 0;
    size_t es = 4;
    switch (what) {
        case OR_COUNTS: src = reinterpret_cast<const unsigned char*>(s->counts.data()); n = s->counts.size(); break;
        case OR_BACKDROPS:
            src = reinterpret_cast<const unsigned char*>(s->backdrops.data());
            n = s->backdrops.size();
            break;
        case OR_RANGES: src = reinterpret_cast<const unsigned char*>(s->ranges.data()); n = s->ranges.size(); es = 8; break;
        case OR_SEGMENTS:
            src = reinterpret_cast<const unsigned char*>(s->segments.data());
            n = s->segments.size();
            es = sizeof(tk_line_segment);
            break;
        case OR_IMAGE: src = reinterpret_cast<const unsigned char*>(s->image.data()); n = s->image.size(); break;
        case OR_BUMPS: src = reinterpret_cast<const unsigned char*>(s->bumps.data()); n = s->bumps.size(); break;
        default: return 0;
    }
    if (dst && first < n) std::memcpy(dst, src + first * es, std::min(count, n - first) * es);
    return n;
}

uint32_t or_line_scanned_tile_count(const tk_line* line, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1) {
    // src/shared/scan_line.rs:37-143 (Rust f32::round rounds half away from zero).
    const float ts = 1.0f / float(TK_TILE_SIZE);
    const float* p0 = line->p0;
    const float* p1 = line->p1;
    bool is_down = p1[1] >= p0[1];
    const float* a0 = is_down ? p0 : p1;
    const float* a1 = is_down ? p1 : p0;
    float s0x = a0[0] * ts, s0y = a0[1] * ts, s1x = a1[0] * ts, s1y = a1[1] * ts;
    auto span_r = [](float a, float b) {
        float hi = std::ceil(fmax_(a, b)), lo = std::floor(fmin_(a, b));
        return f2u(fmax_(hi - lo, 1.0f));
    };
    uint32_t count_x = span_r(s0x, s1x) - 1u;
    uint32_t count = count_x + span_r(s0y, s1y);
    float dx = std::fabs(s1x - s0x), dy = s1y - s0y;
    if (dx + dy == 0.0f) return 0;
    if (dy == 0.0f && std::floor(s0y) == s0y) return 0;
    float idxdy = 1.0f / (dx + dy);
    float a = dx * idxdy;
    bool pos = s1x >= s0x;
    float sign = pos ? 1.0f : -1.0f;
    float xt0 = std::floor(s0x * sign);
    float c = s0x * sign - xt0;
    float y0f = std::floor(s0y);
    float ytop = s0y == s1y ? std::ceil(s0y) : y0f + 1.0f;
    float b = fmin_((dy * c + dx * (ytop - s0y)) * idxdy, 0.99999994f);
    float err = std::floor(a * (float(count) - 1.0f) + b) - float(count_x);
    if (err != 0.0f) a -= std::copysign(2e-7f, err);
    float x0f = xt0 * sign + (pos ? 0.0f : -1.0f);
    float xmin = fmin_(s0x, s1x);
    if (s0y >= float(y1) || s1y <= float(y0) + TOP_TOUCH_EPSILON || xmin >= float(x1)) return 0;
    uint32_t imin = 0, imax = count;
    if (s0y < float(y0)) {
        float f = std::round((float(y0) - y0f + b - a) / (1.0f - a)) - 1.0f;
        if (y0f + f - std::floor(a * f + b) < float(y0)) f += 1.0f;
        imin = f2u(f);
    }
    if (s1y > float(y1)) {
        float f = std::round((float(y1) - y0f + b - a) / (1.0f - a)) - 1.0f;
        if (y0f + f - std::floor(a * f + b) < float(y1)) f += 1.0f;
        imax = f2u(f);
    }
    if (fmax_(s0x, s1x) < float(x0)) {
        imax = imin;
    } else {
        float fudge = pos ? 0.0f : 1.0f;
        if (xmin < float(x0)) {
            float f = std::round((sign * (float(x0) - x0f) - b + fudge) / a);
            if ((x0f + sign * std::floor(a * f + b) < float(x0)) == pos) f += 1.0f;
            if (pos) { if (f2u(f) > imin) imin = f2u(f); }
            else if (f2u(f) < imax) imax = f2u(f);
        }
        if (fmax_(s0x, s1x) > float(x1)) {
            float f = std::round((sign * (float(x1) - x0f) - b + fudge) / a);
            if ((x0f + sign * std::floor(a * f + b) < float(x1)) == pos) f += 1.0f;
            if (pos) imax = std::min(imax, f2u(f)); else imin = std::max(imin, f2u(f));
        }
    }
    imax = std::max(imin, imax);
    uint32_t n = 0;
    for (uint32_t i = imin; i < imax; ++i) {
        float z = std::floor(a * float(i) + b);
        int32_t y = f2i(y0f + float(i) - z);
        int32_t x = f2i(x0f + sign * z);
        n += (y >= int32_t(y0) && y < int32_t(y1) && x >= int32_t(x0) && x < int32_t(x1)) ? 1u : 0u;
    }
    return n;
}

void or_scan_count(const tk_line* lines, uint64_t line_count, const tk_path_record* paths, uint32_t path_count,
                   int32_t* backdrops, uint32_t* counts) {
    for (uint64_t l = 0; l < line_count; ++l) count_line(lines[l], paths, path_count, backdrops, counts);
}

void or_scan_prefix(const uint32_t* counts, const tk_path_record* paths, uint32_t path_count,
                    tk_segment_range* ranges, uint32_t* cursors, uint32_t* bumps) {
    for (uint32_t pid = 0; pid < path_count; ++pid) {
        const tk_path_record& p = paths[pid];
        uint32_t next = p.segment_start;
        for (uint32_t k = 0; k < p.data_len; ++k) {
            uint32_t t = p.data_offset + k;
            ranges[t] = {next, next + counts[t]};
            cursors[t] = next;
            next += counts[t];
        }
        bumps[pid] = next - p.segment_start;
    }
}

void or_blur_pass(const uint32_t* src, uint32_t* dst, uint32_t width, uint32_t height, const uint32_t region[4],
                  const uint32_t source[4], float sigma, uint32_t axis) {
    blur_pass(src, dst, width, height, region, source, sigma, axis, 1);
}

float or_fill_value(const tk_line_segment* segments, uint32_t count, int32_t backdrop, uint32_t x, uint32_t y) {
    return fill_value(segments, 0, count, backdrop, x, y);
}

float or_sdf_coverage(const uint32_t* record, float x, float y, const tk_affine* inv) {
    return sdf_blob_coverage(record, x, y, *inv);
}
float or_exp_nonpos(float x) { return exp_nonpos(x); }
void or_sincos(float x, float* s, float* c) { lib_sincos(x, *s, *c); }
float or_atan2(float y, float x) { return lib_atan2(y, x); }
float or_text_pow(float x, float y) { return text_pow(x, y); }
void or_filter_chain(uint32_t* surface, uint32_t width, const int32_t rect[4], const tk_filter* chain, uint32_t count,
                     const uint32_t* tables) {
    filter_chain(surface, width, rect, chain, count, tables);
}
int32_t or_progressive_blur(uint32_t* surface, uint32_t width, uint32_t height, const int32_t rect[4],
                            const tk_progressive_blur* blur) {
    try {
        const int32_t r[4] = {std::max(rect[0], 0), std::max(rect[1], 0), std::min(rect[2], int32_t(width)),
                              std::min(rect[3], int32_t(height))};
        if (r[2] > r[0] && r[3] > r[1] && blur->max_std_dev > 0.0f) progressive_blur(surface, width, r, *blur);
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}
uint32_t or_progressive_levels(uint32_t w, uint32_t h, float sigma, uint32_t quality, float* out, uint32_t cap) {
    const std::vector<ProgLevel> plan = prog_levels(w, h, sigma, quality);
    for (uint32_t i = 0; i < plan.size() && i < cap; ++i) {
        const ProgLevel& L = plan[i];
        const float center = float(L.step - 1u) * 0.5f;
        float sum = 0.0f, radius = 0.0f;
        for (size_t k = 0; k < L.weight.size(); ++k) {
            sum += L.weight[k];
            radius = std::max(radius, std::ceil(std::fabs(L.offset[k] - center)) + 1.0f);
        }
        const float v[7] = {float(L.w), float(L.h), L.scale, L.variance, float(L.step), sum, radius};
        std::memcpy(out + 7 * i, v, sizeof(v));
    }
    return uint32_t(plan.size());
}
uint32_t or_glyph_over(uint32_t destination, uint32_t source, uint32_t coverage) {
    return src_over_mask_linear_auto_u8(destination, source, coverage);
}

// Fine-only oracle (src/native/runtime/tests/coarse_count/rect_pixels.rs:3-13):
// every draw interpreted as a PTCL_SDF particle in every tile, in draw-record
// order, from the clear colour, with no coarse stage, so an incorrect
// full-tile proof, hollow-stroke proof or occlusion skip changes pixels.
int32_t or_interpret_particles(const tk_scene_desc* d, const tk_ptcl_record* particles, uint32_t count,
                               uint32_t* image);
// Fine-only oracle for path draws, the method of rect_pixels.rs:3-13 applied
// to fills: after the scan (count, prefix + cumsum, emit), every batch's
// stream in every tile is its whole layer stack (BEGIN_CLIP / BEGIN_OPACITY
// with the layer path's segment range and cumsum backdrop in the tile, or
// BEGIN_SDF_CLIP), then every draw of the batch in painter order (FILL with
// the tile's segment range and backdrop, or SDF), then the reversed ends.
// Outside a path's bbox the range is empty and the backdrop 0. No tile bins,
// no particle elision, no stack-wrapper elision, no colour promotion and no
// occlusion skip: an error in any coarse decision changes pixels. Each batch
// loads and stores the RGBA8 target, as the reference's per-batch fine
// dispatch does. Scenes with blur layers are rejected.
int32_t or_interpret_path_draws(const tk_scene_desc* d, int32_t threads, uint32_t* image) {
    try {
        or_scene S;
        S.desc = *d;
        S.paths.assign(d->paths, d->paths + d->path_count);
        S.draws.assign(d->draws, d->draws + d->draw_count);
        S.layers.assign(d->layers, d->layers + d->layer_count);
        S.brush.assign(d->brush_blob, d->brush_blob + d->brush_word_count);
        S.sdf.assign(d->sdf_blob, d->sdf_blob + d->sdf_word_count);
        S.shadow.assign(d->sdf_shadow_blob, d->sdf_shadow_blob + d->sdf_shadow_word_count);
        S.batch_ids.assign(d->draw_batch_ids, d->draw_batch_ids + d->draw_count);
        copy_text(S, d);
        threads = threads < 1 ? 1 : threads;
        scan_scene(S, threads);
        const uint32_t W = d->width, H = d->height;
        for (size_t i = 0; i < size_t(W) * H; ++i) image[i] = d->clear_color;
        auto range_in_tile = [&](const tk_draw_record& dr, uint32_t tx, uint32_t ty, int32_t& w, uint32_t& s0,
                                 uint32_t& s1) {
            const uint32_t bd = draw_backdrop(S, dr, tx, ty);
            if (bd == TK_INVALID_INDEX) { w = 0; s0 = s1 = 0u; return; }
            w = S.backdrops[bd];
            s0 = S.ranges[bd].start;
            s1 = S.ranges[bd].end;
        };
        for (uint32_t oi = 0; oi < d->op_count; ++oi) {
            const tk_op& op = d->ops[oi];
            if (op.kind != TK_OP_DRAW_BATCH) throw std::runtime_error("fine-only path oracle: blur layers unsupported");
            std::vector<uint32_t> draws;
            for (uint32_t k = 0; k < d->draw_order_count; ++k)
                if (S.batch_ids[d->draw_order[k]] == op.batch_id) draws.push_back(d->draw_order[k]);
            parallel_for(threads, S.T, [&](uint64_t tile) {
                const uint32_t tx = uint32_t(tile) % S.tw, ty = uint32_t(tile) / S.tw;
                std::vector<tk_ptcl_record> recs;
                int32_t w;
                uint32_t s0, s1;
                for (uint32_t i = op.layer_start; i < op.layer_end; ++i) {
                    const tk_layer_record& L = S.layers[i];
                    const tk_draw_record& dr = S.draws[L.draw];
                    if (has_sdf(dr)) {
                        recs.push_back({TK_PTCL_BEGIN_SDF_CLIP, 0, 0u, 0u, 0u, L.draw});
                        continue;
                    }
                    range_in_tile(dr, tx, ty, w, s0, s1);
                    const uint32_t tag = L.tag == TK_LAYER_OPACITY ? TK_PTCL_BEGIN_OPACITY : TK_PTCL_BEGIN_CLIP;
                    recs.push_back({tag, w, dr.fill_rule, s0, s1, L.payload});
                }
                std::vector<uint32_t> glyphs;  // every glyph of every run, in every tile
                for (uint32_t di : draws) {
                    const tk_draw_record& dr = S.draws[di];
                    if (!S.glyph_runs.empty() && dr.glyph_run_id != TK_INVALID_INDEX) {
                        const tk_glyph_run& run = S.glyph_runs[dr.glyph_run_id];
                        const uint32_t g0 = uint32_t(glyphs.size());
                        for (uint32_t k = run.first; k < run.first + run.count; ++k) glyphs.push_back(k);
                        recs.push_back({TK_PTCL_GLYPH, 0, 0u, g0, uint32_t(glyphs.size()), di});
                        continue;
                    }
                    if (has_sdf(dr)) {
                        recs.push_back({TK_PTCL_SDF, 0, 0u, di, 0u, di});
                        continue;
                    }
                    range_in_tile(dr, tx, ty, w, s0, s1);
                    recs.push_back({dr.tag == TK_DRAW_PATH_GLYPH ? TK_PTCL_PATH_GLYPH : TK_PTCL_FILL, w, dr.fill_rule,
                                    s0, s1, di});
                }
                for (uint32_t i = op.layer_end; i > op.layer_start;) {
                    const tk_layer_record& L = S.layers[--i];
                    recs.push_back({L.tag == TK_LAYER_OPACITY ? TK_PTCL_END_OPACITY : TK_PTCL_END_CLIP, 0, 0u, 0u, 0u,
                                    0u});
                }
                recs.push_back({TK_PTCL_END, 0, 0u, 0u, 0u, 0u});
                const uint32_t n = uint32_t(recs.size());
                for (uint32_t ly = 0; ly < TK_TILE_SIZE; ++ly) {
                    const uint32_t gy = ty * TK_TILE_SIZE + ly;
                    if (gy >= H) break;
                    for (uint32_t lx = 0; lx < TK_TILE_SIZE; ++lx) {
                        const uint32_t gx = tx * TK_TILE_SIZE + lx;
                        if (gx >= W) break;
                        uint32_t& texel = image[size_t(gy) * W + gx];
                        texel = texel_store(interpret(S, recs, 0u, n, texel_load(texel), lx, ly, gx, gy, glyphs.data()));
                    }
                }
            });
        }
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

int32_t or_interpret_sdf_draws(const tk_scene_desc* d, uint32_t* image) {
    std::vector<tk_ptcl_record> recs;
    for (uint32_t k = 0; k < d->draw_count; ++k) recs.push_back({TK_PTCL_SDF, 0, 0u, 0u, 0u, k});
    return or_interpret_particles(d, recs.data(), uint32_t(recs.size()), image);
}
// The fine-only oracle with a given particle stream for every tile
// (interpret_particles, src/native/runtime/tests/coarse_count/rect_pixels.rs:15-110).
int32_t or_interpret_particles(const tk_scene_desc* d, const tk_ptcl_record* particles, uint32_t count,
                               uint32_t* image) {
    try {
        or_scene S;
        S.desc = *d;
        S.draws.assign(d->draws, d->draws + d->draw_count);
        S.brush.assign(d->brush_blob, d->brush_blob + d->brush_word_count);
        S.sdf.assign(d->sdf_blob, d->sdf_blob + d->sdf_word_count);
        S.shadow.assign(d->sdf_shadow_blob, d->sdf_shadow_blob + d->sdf_shadow_word_count);
        std::vector<tk_ptcl_record> recs(particles, particles + count);
        recs.push_back({TK_PTCL_END, 0, 0u, 0u, 0u, 0u});
        const uint32_t n = uint32_t(recs.size());
        parallel_for(8, d->height, [&](uint64_t y) {
            for (uint32_t x = 0; x < d->width; ++x) {
                F4 pixel = rgba8_to_unorm(d->clear_color);  // fine_initial_pixel without load_target
                pixel = interpret(S, recs, 0u, n, pixel, x % TK_TILE_SIZE, uint32_t(y) % TK_TILE_SIZE, x,
                                  uint32_t(y));
                image[y * d->width + x] = texel_store(pixel);
            }
        });
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

}  // extern "C"
