// Host scan-line planner (src/shared/scan_line.rs:17-151). Arithmetic is
// Rust f32: no contraction, `round` rounds half away from zero, `as u32` and
// `as i32` saturate.
#include "planner.h"

#include <algorithm>
#include <cmath>

namespace {

inline uint32_t sat_u32(float v) {
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967296.0f) return 0xFFFFFFFFu;
    return uint32_t(v);
}
inline int32_t sat_i32(float v) {
    if (v != v) return 0;
    if (v >= 2147483648.0f) return 0x7FFFFFFF;
    if (v <= -2147483648.0f) return int32_t(0x80000000);
    return int32_t(v);
}
inline uint32_t span_tiles(float a, float b) {
    float hi = std::ceil(std::max(a, b));
    float lo = std::floor(std::min(a, b));
    return sat_u32(std::max(hi - lo, 1.0f));
}

}  // namespace

extern "C" uint32_t tk_plan_line_tile_count(const tk_line* line, uint32_t bx0, uint32_t by0, uint32_t bx1,
                                            uint32_t by1) {
    const float scale = 1.0f / float(TK_TILE_SIZE);
    bool down = line->p1[1] >= line->p0[1];
    const float* u = down ? line->p0 : line->p1;
    const float* w = down ? line->p1 : line->p0;
    float ax = u[0] * scale, ay = u[1] * scale, bx = w[0] * scale, by = w[1] * scale;
    uint32_t count_x = span_tiles(ax, bx) - 1u;
    uint32_t count = count_x + span_tiles(ay, by);
    float dx = std::fabs(bx - ax), dy = by - ay;
    if (dx + dy == 0.0f) return 0u;
    if (dy == 0.0f && std::floor(ay) == ay) return 0u;
    float inv = 1.0f / (dx + dy);
    float a = dx * inv;
    bool positive = bx >= ax;
    float sign = positive ? 1.0f : -1.0f;
    float xt0 = std::floor(ax * sign);
    float c = ax * sign - xt0;
    float y0 = std::floor(ay);
    float ytop = ay == by ? std::ceil(ay) : y0 + 1.0f;
    float b = std::min((dy * c + dx * (ytop - ay)) * inv, 0.99999994f);
    float robust = std::floor(a * (float(count) - 1.0f) + b) - float(count_x);
    if (robust != 0.0f) a -= std::copysign(2e-7f, robust);
    float x0 = xt0 * sign + (positive ? 0.0f : -1.0f);
    float xmin = std::min(ax, bx), xmax = std::max(ax, bx);
    if (ay >= float(by1) || by <= float(by0) + 1.0e-12f || xmin >= float(bx1)) return 0u;
    uint32_t imin = 0u, imax = count;
    if (ay < float(by0)) {
        float f = std::round((float(by0) - y0 + b - a) / (1.0f - a)) - 1.0f;
        if (y0 + f - std::floor(a * f + b) < float(by0)) f += 1.0f;
        imin = sat_u32(f);
    }
    if (by > float(by1)) {
        float f = std::round((float(by1) - y0 + b - a) / (1.0f - a)) - 1.0f;
        if (y0 + f - std::floor(a * f + b) < float(by1)) f += 1.0f;
        imax = sat_u32(f);
    }
    if (xmax < float(bx0)) {
        imax = imin;
    } else {
        float fudge = positive ? 0.0f : 1.0f;
        if (xmin < float(bx0)) {
            float f = std::round((sign * (float(bx0) - x0) - b + fudge) / a);
            if ((x0 + sign * std::floor(a * f + b) < float(bx0)) == positive) f += 1.0f;
            if (positive) {
                if (sat_u32(f) > imin) imin = sat_u32(f);
            } else if (sat_u32(f) < imax) {
                imax = sat_u32(f);
            }
        }
        if (xmax > float(bx1)) {
            float f = std::round((sign * (float(bx1) - x0) - b + fudge) / a);
            if ((x0 + sign * std::floor(a * f + b) < float(bx1)) == positive) f += 1.0f;
            if (positive) imax = std::min(imax, sat_u32(f));
            else imin = std::max(imin, sat_u32(f));
        }
    }
    imax = std::max(imin, imax);
    uint32_t visited = 0u;
    for (uint32_t i = imin; i < imax; ++i) {
        float z = std::floor(a * float(i) + b);
        int32_t y = sat_i32(y0 + float(i) - z);
        int32_t x = sat_i32(x0 + sign * z);
        visited += (y >= int32_t(by0) && y < int32_t(by1) && x >= int32_t(bx0) && x < int32_t(bx1)) ? 1u : 0u;
    }
    return visited;
}
