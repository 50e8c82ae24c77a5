// Device arithmetic of the tile rasterization path (sm_100a).
//
// Compiled with -fmad=false: every multiply-add below is either an explicit
// __fmaf_rn (where the reference shader writes `mad`) or an unfused multiply
// followed by an add, so results are IEEE f32 and reproducible.
// HLSL `round` is round-half-to-even (rintf); float->int conversions
// saturate (__float2uint_rz / __float2int_rz).
#pragma once
#include <cstdint>

#include "../../include/tileink.h"

namespace tkd {

constexpr float SCAN_EPSILON = 1.0e-6f;
constexpr float TOP_TOUCH_EPSILON = 1.0e-12f;
constexpr float TILE_CLIP_NUDGE = 1.0e-3f;
constexpr float CHANNEL_SCALE = 1.0f / 255.0f;
constexpr float GRADIENT_FLOAT_EPSILON = 0.00000011920929f;
constexpr float RADIAL_QUADRATIC_EPSILON = 0.000001f;

__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float mad(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ uint32_t f2u(float x) { return __float2uint_rz(x); }
__device__ __forceinline__ int32_t f2i(float x) { return __float2int_rz(x); }

// --- shared/pixel.hlsli:7-66 -------------------------------------------------
__device__ __forceinline__ uint32_t pack4(uint32_t r, uint32_t g, uint32_t b, uint32_t a) {
    return r | (g << 8) | (b << 16) | (a << 24);
}
__device__ __forceinline__ uint32_t coverage_to_u8(float c) { return f2u(clampf(c, 0.0f, 1.0f) * 255.0f + 0.5f); }
__device__ __forceinline__ uint32_t coverage_to_alpha(float v, uint32_t rule) {
    float alpha = fminf(fabsf(v), 1.0f);
    if (rule == 1u) alpha = fabsf(v - 2.0f * rintf(0.5f * v));
    return coverage_to_u8(alpha);
}
__device__ __forceinline__ float signum_f32(float v) { return v < 0.0f ? -1.0f : 1.0f; }
__device__ __forceinline__ uint32_t mul_div255(uint32_t a, uint32_t b) {
    uint32_t p = a * b + 128u;
    return (p + (p >> 8)) >> 8;
}
__device__ __forceinline__ uint32_t combine_alpha(uint32_t a, uint32_t b) { return mul_div255(a, b); }
__device__ __forceinline__ uint32_t scale_premul_u8(uint32_t s, uint32_t f) {
    if (f == 0u) return 0u;
    if (f == 255u) return s;
    return pack4(mul_div255(s & 255u, f), mul_div255((s >> 8) & 255u, f), mul_div255((s >> 16) & 255u, f),
                 mul_div255(s >> 24, f));
}
__device__ __forceinline__ uint32_t src_over_premul_u8(uint32_t d, uint32_t s) {
    uint32_t a = s >> 24;
    if (a == 0u) return d;
    if (a == 255u) return s;
    uint32_t inv = 255u - a;
    return pack4((s & 255u) + mul_div255(d & 255u, inv), ((s >> 8) & 255u) + mul_div255((d >> 8) & 255u, inv),
                 ((s >> 16) & 255u) + mul_div255((d >> 16) & 255u, inv), a + mul_div255(d >> 24, inv));
}
__device__ __forceinline__ float4 rgba8_to_unorm(uint32_t p) {
    return make_float4(float(p & 255u) * CHANNEL_SCALE, float((p >> 8) & 255u) * CHANNEL_SCALE,
                       float((p >> 16) & 255u) * CHANNEL_SCALE, float(p >> 24) * CHANNEL_SCALE);
}
__device__ __forceinline__ uint32_t unorm_to_rgba8(float4 p) {
    return pack4(f2u(clampf(p.x * 255.0f + 0.5f, 0.0f, 255.0f)), f2u(clampf(p.y * 255.0f + 0.5f, 0.0f, 255.0f)),
                 f2u(clampf(p.z * 255.0f + 0.5f, 0.0f, 255.0f)), f2u(clampf(p.w * 255.0f + 0.5f, 0.0f, 255.0f)));
}
__device__ __forceinline__ float4 scale_premul_u8_to_unorm(uint32_t s, uint32_t f) {
    if (f == 0u || (s >> 24) == 0u) return make_float4(0.f, 0.f, 0.f, 0.f);
    float scale = float(f) * (1.0f / 65025.0f);
    return make_float4(float(s & 255u) * scale, float((s >> 8) & 255u) * scale, float((s >> 16) & 255u) * scale,
                       float(s >> 24) * scale);
}
__device__ __forceinline__ float4 src_over_premul_unorm(float4 d, float4 s) {
    if (s.w <= 0.0f) return d;
    if (s.w >= 1.0f) return s;
    float k = 1.0f - s.w;
    return make_float4(s.x + d.x * k, s.y + d.y * k, s.z + d.z * k, s.w + d.w * k);
}
__device__ __forceinline__ uint32_t lerp_premul_u8(uint32_t a, uint32_t b, float t) {
    uint32_t out = 0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float l = float((a >> (8 * c)) & 255u), r = float((b >> (8 * c)) & 255u);
        out |= f2u(clampf(mad(r - l, t, l) + 0.5f, 0.0f, 255.0f)) << (8 * c);
    }
    return out;
}
__device__ __forceinline__ float rem_euclid_f32(float v, float m) { return mad(-floorf(v / m), m, v); }
__device__ __forceinline__ bool premul_u8_is_opaque(uint32_t p) { return (p >> 24) == 255u; }
// RGBA8 UNORM render-target texels: loads are k/255, stores round to nearest even.
__device__ __forceinline__ float4 texel_load(uint32_t p) {
    return make_float4(float(p & 255u) / 255.0f, float((p >> 8) & 255u) / 255.0f, float((p >> 16) & 255u) / 255.0f,
                       float(p >> 24) / 255.0f);
}
__device__ __forceinline__ uint32_t unorm8_store(float x) { return __float2uint_rn(clampf(x, 0.0f, 1.0f) * 255.0f); }
__device__ __forceinline__ uint32_t texel_store(float4 p) {
    return pack4(unorm8_store(p.x), unorm8_store(p.y), unorm8_store(p.z), unorm8_store(p.w));
}

// --- scan/geometry.hlsli:12-114 ---------------------------------------------------
struct Scan {
    uint32_t bx0, by0, bx1, by1;
    uint32_t data_offset;
    float qx0, qy0, qx1, qy1;
    bool down;
    uint32_t count;
    float a, b, sign, x0, y0;
    uint32_t imin, imax;
    int32_t ymin, ymax;
};
__device__ __forceinline__ bool is_tile_boundary_y(float v) { return fabsf(v - floorf(v)) <= TOP_TOUCH_EPSILON; }
__device__ __forceinline__ int32_t ceil_tile_boundary_y(float v) {
    return is_tile_boundary_y(v) ? f2i(floorf(v)) : f2i(ceilf(v));
}
__device__ __forceinline__ uint32_t span(float a, float b) {
    float hi = ceilf(a);
    if (b > a) hi = ceilf(b);
    float lo = floorf(a);
    if (b < a) lo = floorf(b);
    float v = hi - lo;
    if (v < 1.0f) v = 1.0f;
    return f2u(v);
}
// `p` holds the path record words (76 B) already loaded.
__device__ __forceinline__ bool scan_geometry(const tk_line& line, const tk_path_record& p, Scan& s) {
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
    float dx = fabsf(sz - sx);
    float dy = sw - sy;
    if (dx + dy == 0.0f || (dy == 0.0f && floorf(sy) == sy)) return false;
    float rcp = 1.0f / (dx + dy);
    s.a = dx * rcp;
    bool positive = sz >= sx;
    s.sign = positive ? 1.0f : -1.0f;
    float xt0 = floorf(sx * s.sign);
    float c = sx * s.sign - xt0;
    s.y0 = floorf(sy);
    float ytop = s.y0 + 1.0f;
    if (sy == sw) ytop = ceilf(sy);
    s.b = fminf((dy * c + dx * (ytop - sy)) * rcp, 0.99999994f);
    float err = floorf(s.a * (float(s.count) - 1.0f) + s.b) - float(count_x);
    if (err != 0.0f) {
        if (err > 0.0f) s.a -= 0.0000002f;
        else s.a += 0.0000002f;
    }
    s.x0 = positive ? xt0 * s.sign : xt0 * s.sign - 1.0f;
    float xmin = fminf(sx, sz);
    if (sy >= float(s.by1) || sw <= float(s.by0) + TOP_TOUCH_EPSILON || xmin >= float(s.bx1)) return false;
    s.imin = 0u;
    if (sy < float(s.by0)) {
        float first = rintf((float(s.by0) - s.y0 + s.b - s.a) / (1.0f - s.a)) - 1.0f;
        if (s.y0 + first - floorf(s.a * first + s.b) < float(s.by0)) first += 1.0f;
        s.imin = f2u(first);
    }
    s.imax = s.count;
    if (sw > float(s.by1)) {
        float last = rintf((float(s.by1) - s.y0 + s.b - s.a) / (1.0f - s.a)) - 1.0f;
        if (s.y0 + last - floorf(s.a * last + s.b) < float(s.by1)) last += 1.0f;
        s.imax = f2u(last);
    }
    s.ymin = 0;
    s.ymax = 0;
    float xmax = fmaxf(sx, sz);
    if (xmax < float(s.bx0)) {
        s.ymin = ceil_tile_boundary_y(sy);
        s.ymax = ceil_tile_boundary_y(sw);
        s.imax = s.imin;
    } else {
        float fudge = positive ? 0.0f : 1.0f;
        if (xmin < float(s.bx0)) {
            float cut = rintf((s.sign * (float(s.bx0) - s.x0) - s.b + fudge) / s.a);
            if ((s.x0 + s.sign * floorf(s.a * cut + s.b) < float(s.bx0)) == positive) cut += 1.0f;
            int32_t ynext = f2i(s.y0 + cut - floorf(s.a * cut + s.b) + 1.0f);
            if (positive) {
                if (f2u(cut) > s.imin) {
                    float ystart = s.y0 + 1.0f;
                    if (is_tile_boundary_y(sy)) ystart = s.y0;
                    s.ymin = f2i(ystart);
                    s.ymax = ynext;
                    s.imin = f2u(cut);
                }
            } else if (f2u(cut) < s.imax) {
                s.ymin = ynext;
                s.ymax = ceil_tile_boundary_y(sw);
                s.imax = f2u(cut);
            }
        }
        if (xmax > float(s.bx1)) {
            float cut = rintf((s.sign * (float(s.bx1) - s.x0) - s.b + fudge) / s.a);
            if ((s.x0 + s.sign * floorf(s.a * cut + s.b) < float(s.bx1)) == positive) cut += 1.0f;
            if (positive) s.imax = min(s.imax, f2u(cut));
            else s.imin = max(s.imin, f2u(cut));
        }
    }
    s.imax = max(s.imin, s.imax);
    s.ymin = max(s.ymin, int32_t(s.by0));
    s.ymax = min(s.ymax, int32_t(s.by1));
    return true;
}
__device__ __forceinline__ void scan_tile(const Scan& s, uint32_t i, float z, int32_t& tx, int32_t& ty) {
    tx = f2i(s.x0 + s.sign * z);
    ty = f2i(s.y0 + float(i) - z);
}
__device__ __forceinline__ bool scan_tile_inside(const Scan& s, int32_t tx, int32_t ty) {
    return ty >= int32_t(s.by0) && ty < int32_t(s.by1) && tx >= int32_t(s.bx0) && tx < int32_t(s.bx1);
}
__device__ __forceinline__ uint32_t scan_tile_offset(const Scan& s, int32_t tx, int32_t ty) {
    return s.data_offset + (uint32_t(ty) - s.by0) * (s.bx1 - s.bx0) + uint32_t(tx) - s.bx0;
}

// --- scan/clip.hlsli:10-75 ---------------------------------------------------------
__device__ __forceinline__ float x_at_y(const Scan& s, float y) {
    return mad(s.qx1 - s.qx0, (y - s.qy0) / (s.qy1 - s.qy0), s.qx0);
}
__device__ __forceinline__ float y_at_x(const Scan& s, float x) {
    return mad(s.qy1 - s.qy0, (x - s.qx0) / (s.qx1 - s.qx0), s.qy0);
}
__device__ __forceinline__ float clip_y_at_x(const Scan& s, float x, float tmin_y, float tmax_y) {
    float y = y_at_x(s, x);
    if (y <= tmin_y + SCAN_EPSILON) {
        float top_x = x_at_y(s, tmin_y);
        if (fabsf(top_x - x) > TILE_CLIP_NUDGE) return tmin_y;
        return tmin_y + TILE_CLIP_NUDGE;
    }
    return clampf(y, tmin_y + TILE_CLIP_NUDGE, tmax_y);
}
__device__ __forceinline__ tk_line_segment clipped_segment(const Scan& s, uint32_t sub, float z, int32_t tx,
                                                           int32_t ty) {
    const float ts = float(TK_TILE_SIZE);
    float tminx = float(tx) * ts, tminy = float(ty) * ts;
    float tmaxx = tminx + ts, tmaxy = tminy + ts;
    float px = s.qx0, py = s.qy0, pz = s.qx1, pw = s.qy1;
    if (sub > 0u) {
        float prev = floorf(s.a * (float(sub) - 1.0f) + s.b);
        if (z == prev) {
            px = clampf(x_at_y(s, tminy), tminx + TILE_CLIP_NUDGE, tmaxx);
            py = tminy;
        } else {
            float xc = s.sign > 0.0f ? tminx : tmaxx;
            px = xc;
            py = clip_y_at_x(s, xc, tminy, tmaxy);
        }
    }
    if (sub < s.count - 1u) {
        float next = floorf(s.a * (float(sub) + 1.0f) + s.b);
        if (z == next) {
            pz = clampf(x_at_y(s, tmaxy), tminx + TILE_CLIP_NUDGE, tmaxx);
            pw = tmaxy;
        } else {
            float xc = s.sign > 0.0f ? tmaxx : tminx;
            pz = xc;
            pw = clip_y_at_x(s, xc, tminy, tmaxy);
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
        } else if (p0y == 0.0f) {
            p0x = SCAN_EPSILON;
        } else {
            edge = p0y;
        }
    } else if (p1x == 0.0f) {
        if (p1y == 0.0f) p1x = SCAN_EPSILON;
        else edge = p1y;
    }
    if (floorf(p0x) == p0x && p0x != 0.0f) p0x -= SCAN_EPSILON;
    if (floorf(p1x) == p1x && p1x != 0.0f) p1x -= SCAN_EPSILON;
    tk_line_segment out;
    if (s.down) out = {p0x, p0y, p1x, p1y, edge};
    else out = {p1x, p1y, p0x, p0y, edge};
    return out;
}

// --- shared/coverage.hlsli:7-33 ---------------------------------------------------
struct RowParts {
    float edge, dy, xmin, xmax;
};
__device__ __forceinline__ RowParts segment_row_parts(float p0x, float p0y, float p1x, float p1y, float y_edge,
                                                      uint32_t y) {
    float delta_x = p1x - p0x, delta_y = p1y - p0y;
    float row_y = float(y), local_y = p0y - row_y;
    float y0 = clampf(local_y, 0.0f, 1.0f), y1 = clampf(p1y - row_y, 0.0f, 1.0f);
    float dy = y0 - y1;
    float row_edge = signum_f32(delta_x) * clampf(row_y - y_edge + 1.0f, 0.0f, 1.0f);
    if (dy == 0.0f) return {row_edge, dy, 0.0f, 0.0f};
    float slope = delta_x / delta_y;
    bool nearer_p0 = fabsf(local_y - 0.5f) <= fabsf(p1y - row_y - 0.5f);
    float anchor_x = nearer_p0 ? p0x : p1x;
    float anchor_y = nearer_p0 ? local_y : p1y - row_y;
    float sx0 = mad(y0 - anchor_y, slope, anchor_x);
    float sx1 = mad(y1 - anchor_y, slope, anchor_x);
    return {row_edge, dy, fminf(sx0, sx1), fmaxf(sx0, sx1)};
}
__device__ __forceinline__ float segment_area_at(float xmin_abs, float xmax_abs, uint32_t x) {
    float xmin = xmin_abs - float(x), xmax = xmax_abs - float(x);
    float width = xmax - xmin;
    if (width == 0.0f) return clampf(1.0f - xmin, 0.0f, 1.0f);
    if (xmin >= 0.0f && xmax <= 1.0f) return mad(-0.5f, xmin + xmax, 1.0f);
    float left = clampf(xmin, 0.0f, 1.0f), right = clampf(xmax, 0.0f, 1.0f);
    float full = clampf(-xmin, 0.0f, width);
    return mad(right - left, mad(-0.5f, left + right, 1.0f), full) / width;
}

// --- shared/brush/*.hlsli ------------------------------------------------------------
struct Paint {
    const uint32_t* __restrict__ words;
    uint64_t count;
    const uint32_t* __restrict__ texels = nullptr;  // the scene's images (PaintInfo gives each one's first texel)
    __device__ __forceinline__ uint32_t word(uint32_t index) const { return index < count ? __ldg(words + index) : 0u; }
    __device__ __forceinline__ float param(uint32_t base, uint32_t i) const { return __uint_as_float(word(base + i)); }
};
__device__ __forceinline__ float apply_extend(float t, uint32_t extend) {
    if (extend == TK_EXTEND_REPEAT) return rem_euclid_f32(t, 1.0f);
    if (extend == TK_EXTEND_REFLECT) {
        float v = rem_euclid_f32(t, 2.0f);
        return v <= 1.0f ? v : 2.0f - v;
    }
    return clampf(t, 0.0f, 1.0f);
}
__device__ __forceinline__ uint32_t sample_ramp(const Paint& P, uint32_t off, uint32_t len, float t, uint32_t extend) {
    if (len == 0u) return 0u;
    uint32_t last = len - 1u;
    float ext = apply_extend(t, extend);
    float pos = ext * float(last);
    uint32_t li = f2u(floorf(pos)), ri = min(li + 1u, last);
    float frac = mad(ext, float(last), -float(li));
    uint32_t l = P.word(off + li), r = P.word(off + ri);
    if (frac <= GRADIENT_FLOAT_EPSILON || li == ri) return l;
    return lerp_premul_u8(l, r, frac);
}
static __device__ __noinline__ uint32_t sample_gradient(const Paint& P, uint32_t db, float x, float y) {
    uint32_t kind = P.word(db), extend = P.word(db + 1u);
    uint32_t payload = db + P.word(db + 2u), len = P.word(db + 3u);
    uint32_t base = db + TK_BRUSH_HEADER_WORDS;
    if (kind == TK_BRUSH_LINEAR) {
        float tx = mad(P.param(base, 4), x, mad(P.param(base, 6), y, P.param(base, 8)));
        float ty = mad(P.param(base, 5), x, mad(P.param(base, 7), y, P.param(base, 9)));
        float sx = P.param(base, 0), sy = P.param(base, 1), ex = P.param(base, 2), ey = P.param(base, 3);
        float dx = ex - sx, dy = ey - sy;
        float den = dx * dx + dy * dy, t = 0.0f;
        if (den > GRADIENT_FLOAT_EPSILON) t = mad(tx - sx, dx, (ty - sy) * dy) / den;
        return sample_ramp(P, payload, len, t, extend);
    }
    if (kind == TK_BRUSH_RADIAL) {
        float tx = mad(P.param(base, 6), x, mad(P.param(base, 8), y, P.param(base, 10)));
        float ty = mad(P.param(base, 7), x, mad(P.param(base, 9), y, P.param(base, 11)));
        float sx = P.param(base, 0), sy = P.param(base, 1), ex = P.param(base, 2), ey = P.param(base, 3);
        float sr = P.param(base, 4), er = P.param(base, 5);
        float qx = tx - sx, qy = ty - sy, dcx = ex - sx, dcy = ey - sy, dr = er - sr;
        float a = mad(dcx, dcx, mad(dcy, dcy, -dr * dr));
        float b = -2.0f * mad(qx, dcx, mad(qy, dcy, sr * dr));
        float c = mad(qx, qx, mad(qy, qy, -sr * sr));
        bool has_t = false;
        float t = 0.0f;
        if (fabsf(a) <= RADIAL_QUADRATIC_EPSILON) {
            if (fabsf(b) > RADIAL_QUADRATIC_EPSILON) {
                float cand = -c / b;
                if (mad(cand, dr, sr) >= 0.0f) { has_t = true; t = cand; }
            }
        } else {
            float disc = mad(b, b, -4.0f * a * c);
            if (disc >= 0.0f) {
                float root = sqrtf(disc);
                float t0 = (-b - root) / (2.0f * a), t1 = (-b + root) / (2.0f * a);
                bool v0 = mad(t0, dr, sr) >= 0.0f, v1 = mad(t1, dr, sr) >= 0.0f;
                if (v0) { has_t = true; t = v1 ? fmaxf(t0, t1) : t0; }
                else if (v1) { has_t = true; t = t1; }
            }
        }
        return has_t ? sample_ramp(P, payload, len, t, extend) : 0u;
    }
    if (kind == 6u) return 0u;  // BRUSH_PATTERN
    return P.word(db + TK_BRUSH_COLOR_WORD);
}

}  // namespace tkd
