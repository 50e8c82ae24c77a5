// Analytic SDF shapes: the distance samples, their pixel coverage, and the
// coarse-stage tile proofs (full-tile colour, hollow stroke interiors).
//
// Follows shared/sdf/{base,basic,line,coverage}.hlsli and
// coarse/sdf_clip.hlsli of the reference. Every operation is an IEEE
// single-precision add, multiply, divide or square root (no contraction: the
// library is built with -fmad=false) or an explicit fused multiply-add where
// the reference writes `mad`, so a host restatement with the same operation
// order gives identical bits. Shadow falloff uses sdf_exp_nonpos below
// instead of the device exp for the same reason.
#pragma once
#include <math.h>
#include <stdint.h>

#include "../../include/tileink.h"
#include "device.cuh"

namespace tkd {

struct SdfSample {
    float d, nx, ny;
};

// sdf_length (shared/sdf/base.hlsli:7-12): the plain length, rescaled by the
// larger axis only when the squared length leaves the float range.
__device__ __forceinline__ float sdf_length(float x, float y) {
    const float m = sqrtf(x * x + y * y);
    if (m > 0.0f && isfinite(m)) return m;
    const float axis = fmaxf(fabsf(x), fabsf(y));
    if (axis == 0.0f) return 0.0f;
    const float sx = x / axis, sy = y / axis;
    return axis * sqrtf(sx * sx + sy * sy);
}

// normalized_or (shared/sdf/base.hlsli:14-23).
__device__ __forceinline__ void normalized_or(float x, float y, float fx, float fy, float& ox, float& oy) {
    const float m = sqrtf(x * x + y * y);
    if (m > 0.0f && isfinite(m)) {
        ox = x / m;
        oy = y / m;
        return;
    }
    const float axis = fmaxf(fabsf(x), fabsf(y));
    if (axis == 0.0f) {
        ox = fx;
        oy = fy;
        return;
    }
    const float sx = x / axis, sy = y / axis;
    const float l = sqrtf(sx * sx + sy * sy);
    ox = sx / l;
    oy = sy / l;
}

// rounded_box_sdf_sample (shared/sdf/basic.hlsli:6-19).
__device__ __forceinline__ SdfSample rounded_box(float px, float py, float hx, float hy, float radius) {
    const float qx = fabsf(px) - hx + radius, qy = fabsf(py) - hy + radius;
    const float ox = fmaxf(qx, 0.0f), oy = fmaxf(qy, 0.0f);
    const float ol = sdf_length(ox, oy);
    const float d = fminf(fmaxf(qx, qy), 0.0f) + ol - radius;
    const float sx = px >= 0.0f ? 1.0f : -1.0f, sy = py >= 0.0f ? 1.0f : -1.0f;
    if (ol > 0.0f) return SdfSample{d, ox / ol * sx, oy / ol * sy};
    if (qx > qy) return SdfSample{d, sx, 0.0f};
    return SdfSample{d, 0.0f, sy};
}

// local_line_rect_sample (shared/sdf/basic.hlsli:21-25).
__device__ __forceinline__ SdfSample line_rect(float axis, float normal, float x0, float x1, float half_height) {
    const float center = (x0 + x1) * 0.5f, half_width = (x1 - x0) * 0.5f;
    return rounded_box(axis - center, normal, half_width, half_height, 0.0f);
}

// circle_sdf_sample (shared/sdf/basic.hlsli:27-32).
__device__ __forceinline__ SdfSample circle_sample(float x, float y, float cx, float cy, float radius) {
    const float dx = x - cx, dy = y - cy;
    SdfSample s;
    s.d = sdf_length(dx, dy) - radius;
    normalized_or(dx, dy, 1.0f, 0.0f, s.nx, s.ny);
    return s;
}

// rect_sdf_sample (shared/sdf/basic.hlsli:34-57): the corner radius of the
// quadrant the point is in, clamped to the half extents.
__device__ __forceinline__ SdfSample rect_sample(float x, float y, float x0r, float y0r, float x1r, float y1r, float tl,
                                                 float tr, float bl, float br) {
    const float x0 = fminf(x0r, x1r), y0 = fminf(y0r, y1r), x1 = fmaxf(x0r, x1r), y1 = fmaxf(y0r, y1r);
    const float cx = (x0 + x1) * 0.5f, cy = (y0 + y1) * 0.5f;
    const float hx = (x1 - x0) * 0.5f, hy = (y1 - y0) * 0.5f;
    const float px = x - cx, py = y - cy;
    float radius = tl;
    if (px >= 0.0f) radius = py <= 0.0f ? tr : br;
    else if (py > 0.0f) radius = bl;
    const float r = fmaxf(fminf(fminf(radius, hx), hy), 0.0f);
    return rounded_box(px, py, hx, hy, r);
}

// line_sdf_sample (shared/sdf/line.hlsli:8-76): butt (cap 0), square (1) or
// round (2) ends; the normal is rotated back from the line frame.
__device__ __forceinline__ SdfSample line_sample(float x, float y, float sx, float sy, float ex, float ey, float width,
                                                 float cap) {
    const float he = fmaxf(width, 0.0f) * 0.5f;
    const float dx = ex - sx, dy = ey - sy;
    const float len = sdf_length(dx, dy);
    SdfSample s{__int_as_float(0x7f800000), 1.0f, 0.0f};
    if (len == 0.0f) {
        if (cap >= 0.5f) {
            if (cap > 1.5f) {
                const float px = x - sx, py = y - sy;
                s.d = sdf_length(px, py) - he;
                normalized_or(px, py, 1.0f, 0.0f, s.nx, s.ny);
            } else {
                s = line_rect(x - sx, y - sy, -he, he, he);
            }
        }
        return s;
    }
    const float ux = dx / len, uy = dy / len;
    const float px = x - sx, py = y - sy;
    const float axis = px * ux + py * uy;
    const float normal = -px * uy + py * ux;
    if (cap < 0.5f) {
        s = line_rect(axis, normal, 0.0f, len, he);
    } else if (cap < 1.5f) {
        s = line_rect(axis, normal, -he, len + he, he);
    } else {
        const float nearest = fminf(fmaxf(axis, 0.0f), len);
        const float ax = axis - nearest;
        s.d = sdf_length(ax, normal) - he;
        normalized_or(ax, normal, 0.0f, 1.0f, s.nx, s.ny);
    }
    return SdfSample{s.d, s.nx * ux - s.ny * uy, s.nx * uy + s.ny * ux};
}

// sdf_coverage_from_dist / sdf_coverage_from_sample
// (shared/sdf/base.hlsli:39-52): the distance in device pixels is the local
// distance over the length of the inverse transform applied to the normal.
__device__ __forceinline__ float coverage_from_sample(const SdfSample& s, const tk_affine& inv) {
    const float gx = __fmaf_rn(inv.a, s.nx, inv.b * s.ny);
    const float gy = __fmaf_rn(inv.c, s.nx, inv.d * s.ny);
    const float footprint = sdf_length(gx, gy);
    if (footprint == 0.0f) return s.d < 0.0f ? 1.0f : (s.d > 0.0f ? 0.0f : 0.5f);
    return fminf(fmaxf(0.5f - s.d / footprint, 0.0f), 1.0f);
}

// exp(x) for x <= 0 (positive x is not used and gives 1): evaluated in double
// as 2^k * e^r with k the nearest integer to x / ln 2 (|r| <= ln 2 / 2 plus
// rounding), e^r by its Taylor polynomial of degree 12 in Horner form
// (truncation below 2e-16), 2^k assembled from its exponent bits. Only
// exactly rounded double multiplies and adds are used, so host and device
// agree bit for bit; the float result is within half an ulp of exp(x) over the
// tested range.
__device__ __forceinline__ float sdf_exp_nonpos(float x) {
    if (!(x <= 0.0f)) return x != x ? x : 1.0f;
    if (x < -104.0f) return 0.0f;
    const double ln2 = 0.69314718055994530942, inv_ln2 = 1.4426950408889634074;
    const double xd = double(x);
    const double k = floor(xd * inv_ln2 + 0.5);
    const double r = xd - k * ln2;
    // 1/n! for n = 12 .. 2
    const double c[11] = {1.0 / 479001600.0, 1.0 / 39916800.0, 1.0 / 3628800.0, 1.0 / 362880.0, 1.0 / 40320.0,
                          1.0 / 5040.0,      1.0 / 720.0,       1.0 / 120.0,     1.0 / 24.0,     1.0 / 6.0,
                          0.5};
    double p = c[0];
#pragma unroll
    for (int n = 1; n < 11; ++n) p = p * r + c[n];
    p = p * r + 1.0;
    p = p * r + 1.0;
    const double scale = __longlong_as_double((long long)(1023 + (long long)k) << 52);
    return float(p * scale);
}

// sdf_shadow_coverage_from_sample (shared/sdf/base.hlsli:54-62).
__device__ __forceinline__ float shadow_coverage(const SdfSample& s, const tk_affine& inv, float expand,
                                                 float intensity) {
    const float ci = fminf(fmaxf(intensity, 0.0f), 1.0f);
    if (expand > 0.0f) return fminf(fmaxf(sdf_exp_nonpos(-fmaxf(s.d, 0.0f) / expand) * ci, 0.0f), 1.0f);
    return coverage_from_sample(s, inv) * ci;
}

__device__ __forceinline__ float sdf_word_f(const uint32_t* w, uint32_t i) { return __uint_as_float(__ldg(w + i)); }

__device__ __forceinline__ SdfSample nearer(const SdfSample& a, const SdfSample& b) { return a.d <= b.d ? a : b; }
__device__ __forceinline__ SdfSample farther(const SdfSample& a, const SdfSample& b) { return a.d >= b.d ? a : b; }

// distance_to_segment_sdf_sample (shared/sdf/polygon.hlsli:7-26): unsigned
// distance to segment a-b, `f` the normal where the point is on it.
__device__ __forceinline__ SdfSample segment_sample(float px, float py, float ax, float ay, float bx, float by, float fx,
                                                    float fy) {
    const float dx = bx - ax, dy = by - ay;
    const float len2 = dx * dx + dy * dy;
    float nx = ax, ny = ay;
    if (len2 >= 1.175494351e-38f && isfinite(len2)) {
        const float t = fminf(fmaxf(((px - ax) * dx + (py - ay) * dy) / len2, 0.0f), 1.0f);
        nx = ax + dx * t;
        ny = ay + dy * t;
    } else {
        const float axis = fmaxf(fabsf(dx), fabsf(dy));
        if (axis > 0.0f) {
            const float sx = dx / axis, sy = dy / axis;
            const float dd = sx * sx + sy * sy;
            const float qx = sx / dd, qy = sy / dd;
            const float t = fminf(fmaxf(((px - ax) * qx + (py - ay) * qy) / axis, 0.0f), 1.0f);
            nx = ax + dx * t;
            ny = ay + dy * t;
        }
    }
    const float ex = px - nx, ey = py - ny;
    SdfSample s;
    s.d = sdf_length(ex, ey);
    normalized_or(ex, ey, fx, fy, s.nx, s.ny);
    return s;
}

// triangle_sdf_sample (shared/sdf/polygon.hlsli:32-85): the nearest edge,
// negated inside, less the corner radius. 
__device__ __forceinline__ SdfSample triangle_sample(float x, float y, float ax, float ay, float bx, float by,
                                                         float cx, float cy, float corner) {
    float tbx = bx - ax, tby = by - ay, tcx = cx - ax, tcy = cy - ay, tpx = x - ax, tpy = y - ay;
    float area = tbx * tcy - tby * tcx;
    const float lox = fminf(fminf(ax, bx), cx), loy = fminf(fminf(ay, by), cy);
    const float hix = fmaxf(fmaxf(ax, bx), cx), hiy = fmaxf(fmaxf(ay, by), cy);
    if (area == 0.0f || !isfinite(area)) {
        const float spx = hix - lox, spy = hiy - loy;
        if (spx > 0.0f && spy > 0.0f) {
            tbx /= spx; tby /= spy; tcx /= spx; tcy /= spy; tpx /= spx; tpy /= spy;
            area = tbx * tcy - tby * tcx;
        }
    }
    const float o = area >= 0.0f ? 1.0f : -1.0f;
    float n0x, n0y, n1x, n1y, n2x, n2y;
    normalized_or((by - ay) * o, -(bx - ax) * o, 1.0f, 0.0f, n0x, n0y);
    normalized_or((cy - by) * o, -(cx - bx) * o, 1.0f, 0.0f, n1x, n1y);
    normalized_or((ay - cy) * o, -(ax - cx) * o, 1.0f, 0.0f, n2x, n2y);
    SdfSample s = nearer(segment_sample(x, y, ax, ay, bx, by, n0x, n0y), segment_sample(x, y, bx, by, cx, cy, n1x, n1y));
    s = nearer(s, segment_sample(x, y, cx, cy, ax, ay, n2x, n2y));
    const float side_ab = (tbx * tpy - tby * tpx) * o;
    const float side_bc = ((tcx - tbx) * (tpy - tby) - (tcy - tby) * (tpx - tbx)) * o;
    const float side_ca = ((-tcx) * (tpy - tcy) - (-tcy) * (tpx - tcx)) * o;
    if (area != 0.0f && x >= lox && y >= loy && x <= hix && y <= hiy && side_ab >= 0.0f && side_bc >= 0.0f &&
        side_ca >= 0.0f)
        s = SdfSample{-s.d, -s.nx, -s.ny};
    return SdfSample{s.d - fmaxf(corner, 0.0f), s.nx, s.ny};
}

// ---------------------------------------------------------------------------
// Trigonometry for the arc and star kinds, evaluated in double with exactly
// rounded operations only, so host and device agree bit for bit (the float
// results are within half an ulp of sin, cos and atan2 over the tested
// ranges).
//   sin, cos: x = k pi/2 + r (Cody-Waite reduction with fdlibm's two-part
//   pi/2, exact products for |k| < 2^20), sin r and cos r by their Taylor
//   polynomials of degree 19 and 18 (|r| <= pi/4), the quadrant from k mod 4.
//   atan2: the angle of the smaller over the larger coordinate in [0, 1],
//   reduced by atan z = pi/6 + atan((z sqrt3 - 1)/(z + sqrt3)) above
//   tan(pi/12), the odd series to degree 27, then placed in its quadrant.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void sdf_sincos(float a, float& s, float& c) {
    const double x = double(a);
    if (!(fabs(x) < 1.0e9)) {
        s = c = __int_as_float(0x7fc00000);
        return;
    }
    const double pio2_hi = 1.57079632673412561417e+00, pio2_lo = 6.07710050650619224932e-11;
    const double k = floor(x * 0.63661977236758134308 + 0.5);
    const double r = (x - k * pio2_hi) - k * pio2_lo;
    const double r2 = r * r;
    // sin r = r (1 - r^2/3! + ... - r^18/19!), cos r = 1 - r^2/2! + ... + r^18/18!
    double ps = -1.0 / 121645100408832000.0;
    ps = ps * r2 + 1.0 / 355687428096000.0;
    ps = ps * r2 - 1.0 / 1307674368000.0;
    ps = ps * r2 + 1.0 / 6227020800.0;
    ps = ps * r2 - 1.0 / 39916800.0;
    ps = ps * r2 + 1.0 / 362880.0;
    ps = ps * r2 - 1.0 / 5040.0;
    ps = ps * r2 + 1.0 / 120.0;
    ps = ps * r2 - 1.0 / 6.0;
    ps = ps * r2 + 1.0;
    const double sr = ps * r;
    double pc = 1.0 / 6402373705728000.0;
    pc = pc * r2 - 1.0 / 20922789888000.0;
    pc = pc * r2 + 1.0 / 87178291200.0;
    pc = pc * r2 - 1.0 / 479001600.0;
    pc = pc * r2 + 1.0 / 3628800.0;
    pc = pc * r2 - 1.0 / 40320.0;
    pc = pc * r2 + 1.0 / 720.0;
    pc = pc * r2 - 1.0 / 24.0;
    pc = pc * r2 + 0.5;
    const double cr = 1.0 - pc * r2;
    const int q = int(fmod(k, 4.0) + 4.0) & 3;
    const double ss = q == 0 ? sr : (q == 1 ? cr : (q == 2 ? -sr : -cr));
    const double cc = q == 0 ? cr : (q == 1 ? -sr : (q == 2 ? -cr : sr));
    s = float(ss);
    c = float(cc);
}

__device__ __forceinline__ float sdf_atan2(float yf, float xf) {
    const double y = double(yf), x = double(xf);
    const double ax = fabs(x), ay = fabs(y);
    const bool swap = ay > ax;
    const double z = swap ? ax / ay : ay / ax;  // in [0, 1]; NaN for 0/0 and inf/inf
    const double sqrt3 = 1.73205080756887729353, pi6 = 0.52359877559829887308;
    const double pi2 = 1.57079632679489661923, pi = 3.14159265358979323846;
    const bool reduce = z > 0.26794919243112270647;
    const double t = reduce ? (z * sqrt3 - 1.0) / (z + sqrt3) : z;
    const double t2 = t * t;
    double p = 1.0 / 27.0;
    p = p * t2 * -1.0 + 1.0 / 25.0;
    p = p * t2 * -1.0 + 1.0 / 23.0;
    p = p * t2 * -1.0 + 1.0 / 21.0;
    p = p * t2 * -1.0 + 1.0 / 19.0;
    p = p * t2 * -1.0 + 1.0 / 17.0;
    p = p * t2 * -1.0 + 1.0 / 15.0;
    p = p * t2 * -1.0 + 1.0 / 13.0;
    p = p * t2 * -1.0 + 1.0 / 11.0;
    p = p * t2 * -1.0 + 1.0 / 9.0;
    p = p * t2 * -1.0 + 1.0 / 7.0;
    p = p * t2 * -1.0 + 1.0 / 5.0;
    p = p * t2 * -1.0 + 1.0 / 3.0;
    p = p * t2 * -1.0 + 1.0;
    double a = p * t;
    if (reduce) a = pi6 + a;
    if (swap) a = pi2 - a;
    if (x < 0.0) a = pi - a;
    if (y < 0.0) a = -a;
    return float(a);
}

// arc_angle_in_sweep (shared/sdf/arc.hlsli:10-16)
__device__ __forceinline__ bool arc_in_sweep(float angle, float start, float sweep) {
    const float tau = 6.2831855f;
    if (sweep >= 0.0f) return rem_euclid_f32(angle - start, tau) <= sweep;
    return rem_euclid_f32(start - angle, tau) <= -sweep;
}

// arc_cap_segment_sdf_sample (arc.hlsli:18-34)
__device__ __forceinline__ SdfSample arc_cap_segment(float vx, float vy, float radius, float angle, float he,
                                                     float sweep, bool end_cap) {
    const float inner = fmaxf(radius - he, 0.0f), outer = radius + he;
    float si, co;
    sdf_sincos(angle, si, co);
    const float dir = sweep >= 0.0f ? 1.0f : -1.0f;
    const float tx = -si * dir, ty = co * dir;
    return segment_sample(vx, vy, inner * co, inner * si, outer * co, outer * si, end_cap ? tx : -tx,
                          end_cap ? ty : -ty);
}

// arc_endpoint_sdf_sample (arc.hlsli:36-41)
__device__ __forceinline__ SdfSample arc_endpoint(float vx, float vy, float radius, float angle, float he) {
    float si, co;
    sdf_sincos(angle, si, co);
    const float dx = vx - radius * co, dy = vy - radius * si;
    SdfSample s;
    s.d = sdf_length(dx, dy) - he;
    normalized_or(dx, dy, co, si, s.nx, s.ny);
    return s;
}

// arc_square_cap_sdf_sample (arc.hlsli:66-85)
__device__ __forceinline__ SdfSample arc_square_cap(float vx, float vy, float radius, float angle, float sweep,
                                                    float x0, float x1, float he) {
    const float dir = sweep < 0.0f ? -1.0f : 1.0f;
    float si, co;
    sdf_sincos(angle, si, co);
    const float tx = -si * dir, ty = co * dir;
    const float px = vx - radius * co, py = vy - radius * si;
    const float lx = px * tx + py * ty, ly = -px * ty + py * tx;
    const SdfSample l = line_rect(lx, ly, x0, x1, he);
    return SdfSample{l.d, l.nx * tx - l.ny * ty, l.nx * ty + l.ny * tx};
}

// arc_sdf_sample (arc.hlsli:43-64, 87-123): a ring sector with butt, square or
// round ends.
__device__ __forceinline__ SdfSample arc_sample(float x, float y, float cx, float cy, float radius_raw,
                                                float width_raw, float start, float sweep, float cap) {
    const float radius = fmaxf(radius_raw, 0.0f), width = fmaxf(width_raw, 0.0f);
    SdfSample s{__int_as_float(0x7f800000), 1.0f, 0.0f};
    if (!(radius > 0.0f && width > 0.0f && sweep != 0.0f)) return s;
    const float vx = x - cx, vy = y - cy;
    const float len = sdf_length(vx, vy);
    const float he = width * 0.5f;
    if (fabsf(sweep) >= 6.2831855f) {
        float nx, ny;
        normalized_or(vx, vy, 1.0f, 0.0f, nx, ny);
        const float sg = len >= radius ? 1.0f : -1.0f;
        return SdfSample{fabsf(len - radius) - he, nx * sg, ny * sg};
    }
    // arc_butt_sdf_sample (arc.hlsli:43-64)
    bool on_ring = false;
    if (len != 0.0f) {
        const float angle = sdf_atan2(vy, vx);
        if (arc_in_sweep(angle, start, sweep)) {
            const float sg = len >= radius ? 1.0f : -1.0f;
            s = SdfSample{fabsf(len - radius) - he, vx / len * sg, vy / len * sg};
            on_ring = true;
        }
    }
    if (!on_ring)
        s = nearer(arc_cap_segment(vx, vy, radius, start, he, sweep, false),
                   arc_cap_segment(vx, vy, radius, start + sweep, he, sweep, true));
    if (cap > 1.5f) {
        s = nearer(nearer(s, arc_endpoint(vx, vy, radius, start, he)), arc_endpoint(vx, vy, radius, start + sweep, he));
    } else if (cap >= 0.5f) {
        s = nearer(nearer(s, arc_square_cap(vx, vy, radius, start, sweep, -he, 0.0f, he)),
                   arc_square_cap(vx, vy, radius, start + sweep, sweep, 0.0f, he, he));
    }
    return s;
}

// cos and sin of the star vertex angles i pi/5 (star_vertex's float(i) *
// 0.6283185307179586), i = 0..9, by sdf_sincos: written by fine's
// k_star_table before the kernels that read them, so that star pixels need
// one sincos (the rotation) instead of eleven.
static __device__ float2 g_star_dir[10];

// star_sdf_sample (shared/sdf/polygon.hlsli:158-206): a five-point star, its
// ten vertices alternating outer and inner radius every pi/5, rotated.
__device__ __forceinline__ SdfSample star_sample(float x, float y, float cx, float cy, float outer, float inner,
                                                 float corner, float rotation) {
    float sn, cs;
    sdf_sincos(rotation, sn, cs);
    const float rx = x - cx, ry = y - cy;
    const float px = cs * rx + sn * ry, py = -sn * rx + cs * ry;
    SdfSample nearest{__int_as_float(0x7f800000), 1.0f, 0.0f};
    bool inside = false;
    auto vertex = [&](uint32_t i, float& vx, float& vy) {  // star_vertex
        const float r = (i & 1u) == 0u ? outer : inner;
        const float2 dir = g_star_dir[i];  // (cos, sin) of float(i) * 0.62831855f
        vx = dir.x * r;
        vy = dir.y * r;
    };
    float qx, qy;
    vertex(9u, qx, qy);
    for (uint32_t i = 0; i < 10u; ++i) {
        float ux, uy;
        vertex(i, ux, uy);
        const float ex = ux - qx, ey = uy - qy;
        float fx, fy;
        normalized_or(ey, -ex, 1.0f, 0.0f, fx, fy);
        nearest = nearer(nearest, segment_sample(px, py, qx, qy, ux, uy, fx, fy));
        if ((qy > py) != (uy > py)) {
            const float fraction = (py - qy) / (uy - qy);
            const float crossing = qx + fraction * (ux - qx);
            if (px < crossing) inside = !inside;
        }
        qx = ux;
        qy = uy;
    }
    if (inside) nearest = SdfSample{-nearest.d, -nearest.nx, -nearest.ny};
    const float d = nearest.d - fmaxf(corner, 0.0f);
    return SdfSample{d, cs * nearest.nx - sn * nearest.ny, sn * nearest.nx + cs * nearest.ny};
}

// callout_sdf_sample (shared/sdf/polygon.hlsli:87-136): a rounded body and,
// unless hidden, a rounded triangular tail on side 0 top, 1 right, 2 bottom
// or 3 left, nearest of the two.
__device__ __forceinline__ SdfSample callout_sample(float x, float y, float x0r, float y0r, float x1r, float y1r,
                                                    float body_radius, float tail_offset, float tail_width,
                                                    float tail_length, float tail_radius, float side, float visible) {
    const float x0 = fminf(x0r, x1r), y0 = fminf(y0r, y1r), x1 = fmaxf(x0r, x1r), y1 = fmaxf(y0r, y1r);
    const SdfSample body = rect_sample(x, y, x0, y0, x1, y1, body_radius, body_radius, body_radius, body_radius);
    if (visible < 0.5f) return body;
    const bool vertical = side < 0.5f || (side >= 1.5f && side < 2.5f);
    const float span = vertical ? x1 - x0 : y1 - y0;
    const float width = fminf(fmaxf(tail_width, 0.0f), span);
    const float hw = width * 0.5f;
    const float center = fminf(fmaxf(tail_offset, hw), fmaxf(span - hw, hw));
    const float radius =
        fminf(fmaxf(tail_radius, 0.0f), fminf(fmaxf(hw * 0.499f, 0.0f), fmaxf(tail_length * 0.499f, 0.0f)));
    const float shw = hw - radius, sl = tail_length - radius;
    float ax = x0 + center - shw, ay = y0, bx = x0 + center + shw, by = y0, cx = x0 + center, cy = y0 - sl;
    if (side >= 0.5f && side < 1.5f) {
        ax = x1; ay = y0 + center - shw; bx = x1; by = y0 + center + shw; cx = x1 + sl; cy = y0 + center;
    } else if (side >= 1.5f && side < 2.5f) {
        ax = x0 + center - shw; ay = y1; bx = x0 + center + shw; by = y1; cx = x0 + center; cy = y1 + sl;
    } else if (side >= 2.5f) {
        ax = x0; ay = y0 + center - shw; bx = x0; by = y0 + center + shw; cx = x0 - sl; cy = y0 + center;
    }
    return nearer(body, triangle_sample(x, y, ax, ay, bx, by, cx, cy, radius));
}

// checkerboard_sdf_sample (shared/sdf/effects.hlsli:8-36): the cells of even
// parity, inside the rectangle. 
__device__ __forceinline__ SdfSample checkerboard_sample(float x, float y, float x0, float y0, float x1, float y1,
                                                             float cell_raw) {
    const float left = fminf(x0, x1), top = fminf(y0, y1), right = fmaxf(x0, x1), bottom = fmaxf(y0, y1);
    const SdfSample outer = rect_sample(x, y, left, top, right, bottom, 0.0f, 0.0f, 0.0f, 0.0f);
    const float cell = fmaxf(cell_raw, 0.000001f);
    const float cell_x = floorf((x - left) / cell), cell_y = floorf((y - top) / cell);
    const float lx = rem_euclid_f32(x - left, cell), ly = rem_euclid_f32(y - top, cell);
    float e = lx, nx = 1.0f, ny = 0.0f;
    if (cell - lx < e) { e = cell - lx; nx = -1.0f; ny = 0.0f; }
    if (ly < e) { e = ly; nx = 0.0f; ny = 1.0f; }
    if (cell - ly < e) { e = cell - ly; nx = 0.0f; ny = -1.0f; }
    const bool filled = ((uint32_t(f2i(cell_x)) + uint32_t(f2i(cell_y))) & 1u) == 0u;
    return farther(outer, SdfSample{filled ? -e : e, nx, ny});
}

// line_segment_sdf_sample (shared/sdf/line.hlsli:16-26) in the line's frame.
__device__ __forceinline__ SdfSample dash_segment(float axis, float normal, float start, float end, float he, float cap) {
    if (cap < 0.5f) return line_rect(axis, normal, start, end, he);
    if (cap < 1.5f) return line_rect(axis, normal, start - he, end + he, he);
    const float nearest = fminf(fmaxf(axis, start), end);
    const float dx = axis - nearest;
    SdfSample s;
    s.d = sdf_length(dx, normal) - he;
    normalized_or(dx, normal, 0.0f, 1.0f, s.nx, s.ny);
    return s;
}

// The dashes of dash_line_sdf_sample (shared/sdf/line.hlsli:28-39, 78-105):
// the nearest of the dashes before, under and after the point along the
// line; `s` (the plain line's sample) when there are no gaps.
__device__ __forceinline__ SdfSample dash_sample(SdfSample s, float x, float y, float sx, float sy, float ex,
                                                     float ey, float width, float cap, float dash_raw, float gap_raw,
                                                     float offset_raw) {
    const float dash = fmaxf(dash_raw, 0.0f), gap = fmaxf(gap_raw, 0.0f);
    if (!(dash > 0.0f && gap > 0.0f)) return s;
    const float he = fmaxf(width, 0.0f) * 0.5f;
    const float dx = ex - sx, dy = ey - sy;
    const float len = sdf_length(dx, dy);
    if (!(len > 0.0f)) return s;
    const float ux = dx / len, uy = dy / len;
    const float px = x - sx, py = y - sy;
    const float axis = px * ux + py * uy;
    const float normal = -px * uy + py * ux;
    const float cycle = dash + gap;
    const float offset = rem_euclid_f32(offset_raw, cycle);
    const float base = floorf((axis + offset) / cycle);
    // dash_line_segment_sample for dash index ix
    auto dash_at = [&](float ix) {
        const float dash_start = ix * cycle - offset, dash_end = dash_start + dash;
        SdfSample d{__int_as_float(0x7f800000), 1.0f, 0.0f};
        if (dash_end > 0.0f && dash_start < len) {
            const float start = fmaxf(dash_start, 0.0f), end = fminf(dash_end, len);
            if (end > start) d = dash_segment(axis, normal, start, end, he, cap);
        }
        return d;
    };
    const SdfSample l = nearer(nearer(dash_at(base - 1.0f), dash_at(base)), dash_at(base + 1.0f));
    return SdfSample{l.d, l.nx * ux - l.ny * uy, l.nx * uy + l.ny * ux};
}

// sdf_coverage_from_blob (shared/sdf/coverage.hlsli:13-236) for the record at
// `w` (TK_SDF_RECORD_WORDS words), sampled at local point (x, y). The kinds
// share one copy of each sampler: a shape (rect, circle or line) sampled in
// one pass, or two for strokes (outer minus inner coverage), with shadows
// shifted by their offset and weighted by their falloff. The operations and
// their order per kind are those of the reference's per-kind branches; the
// sharing only keeps the code small enough for the instruction cache.
//
// EXT adds the candlestick, dash line, triangle, checkerboard and callout
// kinds; their
// code costs the other kinds 18% and more of fine time (registers and
// instruction cache), so scenes without them use the instance without.
template <bool EXT>
__device__ __forceinline__ float sdf_coverage(const uint32_t* w, float x, float y, const tk_affine& inv) {
    const uint32_t kind = __ldg(w);
    const bool candle = EXT && kind == TK_SDF_CANDLESTICK;
    const bool rect = kind == TK_SDF_RECT || kind == TK_SDF_RECT_STROKE || kind == TK_SDF_RECT_SHADOW || candle;
    const bool circle = kind == TK_SDF_CIRCLE || kind == TK_SDF_CIRCLE_STROKE || kind == TK_SDF_CIRCLE_SHADOW;
    const bool dashed = EXT && kind == TK_SDF_DASH_LINE;
    const bool line = kind == TK_SDF_LINE || kind == TK_SDF_LINE_SHADOW || dashed;
    const bool triangle = EXT && kind == TK_SDF_TRIANGLE, checker = EXT && kind == TK_SDF_CHECKERBOARD;
    const bool callout = EXT && (kind == TK_SDF_CALLOUT || kind == TK_SDF_CALLOUT_STROKE || kind == TK_SDF_CALLOUT_SHADOW);
    const bool arc = EXT && (kind == TK_SDF_ARC || kind == TK_SDF_ARC_SHADOW);
    const bool star = EXT && (kind == TK_SDF_STAR || kind == TK_SDF_STAR_STROKE);
    if (!(rect || circle || line || triangle || checker || callout || arc || star)) return 0.0f;
    const bool shadow = kind == TK_SDF_RECT_SHADOW || kind == TK_SDF_CIRCLE_SHADOW || kind == TK_SDF_LINE_SHADOW ||
                        (EXT && (kind == TK_SDF_CALLOUT_SHADOW || kind == TK_SDF_ARC_SHADOW));
    const bool stroke = kind == TK_SDF_RECT_STROKE || kind == TK_SDF_CIRCLE_STROKE;
    const float x0 = sdf_word_f(w, 1), y0 = sdf_word_f(w, 2), x1 = sdf_word_f(w, 3), y1 = sdf_word_f(w, 4);
    const float r0 = sdf_word_f(w, 5), r1 = sdf_word_f(w, 6), r2 = sdf_word_f(w, 7), r3 = sdf_word_f(w, 8);
    float px = x, py = y, expand = 0.0f, intensity = 0.0f;
    if (shadow) {
        px = x - sdf_word_f(w, 13);
        py = y - sdf_word_f(w, 14);
        expand = sdf_word_f(w, 15);
        intensity = sdf_word_f(w, 16);
    }
    // pass 0: the shape (a stroke's outer edge); pass 1: a stroke's inner edge
    float o[8] = {x0, y0, x1, y1, r0, r1, r2, r3}, in[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool inner = false;
    if (kind == TK_SDF_RECT_STROKE) {
        const float ht = fmaxf(sdf_word_f(w, 9), 0.0f), hr = fmaxf(sdf_word_f(w, 10), 0.0f);
        const float hb = fmaxf(sdf_word_f(w, 11), 0.0f), hl = fmaxf(sdf_word_f(w, 12), 0.0f);
        const float rx0 = fminf(x0, x1), ry0 = fminf(y0, y1), rx1 = fmaxf(x0, x1), ry1 = fmaxf(y0, y1);
        const float c0 = fmaxf(ht, hl), c1 = fmaxf(ht, hr), c2 = fmaxf(hb, hl), c3 = fmaxf(hb, hr);
        o[0] = rx0 - hl; o[1] = ry0 - ht; o[2] = rx1 + hr; o[3] = ry1 + hb;
        o[4] = r0 + c0; o[5] = r1 + c1; o[6] = r2 + c2; o[7] = r3 + c3;
        in[0] = rx0 + hl; in[1] = ry0 + ht; in[2] = rx1 - hr; in[3] = ry1 - hb;
        in[4] = fmaxf(r0 - c0, 0.0f); in[5] = fmaxf(r1 - c1, 0.0f);
        in[6] = fmaxf(r2 - c2, 0.0f); in[7] = fmaxf(r3 - c3, 0.0f);
        inner = in[0] < in[2] && in[1] < in[3];
    } else if (kind == TK_SDF_CIRCLE_STROKE) {
        const float he = fmaxf(sdf_word_f(w, 9), 0.0f), radius = fmaxf(x1, 0.0f);
        o[2] = radius + he;
        in[0] = x0; in[1] = y0; in[2] = radius - he;
        inner = radius > he;
    } else if (candle) {
        // candlestick_sdf_coverage (shared/sdf/effects.hlsli:38-70): the wick and
        // the body, max of their coverages; words: centre x, high y, low y,
        // body top y, body bottom y, body width, wick width
        const float cx = x0, wh = fmaxf(r2, 1.0f) * 0.5f, bh = fmaxf(r1, 1.0f) * 0.5f;
        o[0] = cx - wh; o[1] = fminf(y0, x1); o[2] = cx + wh; o[3] = fmaxf(y0, x1);
        float by0 = fminf(y1, r0), by1 = fmaxf(y1, r0);
        if (by0 == by1) {
            by0 = by0 - 0.5f;
            by1 = by1 + 0.5f;
        }
        in[0] = cx - bh; in[1] = by0; in[2] = cx + bh; in[3] = by1;
        o[4] = o[5] = o[6] = o[7] = 0.0f;
        inner = true;
    }
    float cov[2] = {0.0f, 0.0f};
    for (int pass = 0; pass < (inner ? 2 : 1); ++pass) {
        float q[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) q[k] = pass ? in[k] : o[k];
        SdfSample s{0.0f, 1.0f, 0.0f};
        if (rect) {
            s = rect_sample(px, py, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7]);
        } else if (circle) {
            s = circle_sample(px, py, q[0], q[1], q[2]);
        } else if (line) {
            s = line_sample(px, py, q[0], q[1], q[2], q[3], q[4], q[5]);
            if (dashed)
                s = dash_sample(s, px, py, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], sdf_word_f(w, 9));
        } else if (triangle) {
            s = triangle_sample(px, py, q[0], q[1], q[2], q[3], q[4], q[5], q[6]);
        } else if (checker) {
            s = checkerboard_sample(px, py, q[0], q[1], q[2], q[3], q[4]);
        } else if (callout) {
            // words 9-12: tail radius, side, stroke half width, tail visible
            s = callout_sample(px, py, q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], sdf_word_f(w, 9),
                               sdf_word_f(w, 10), sdf_word_f(w, 12));
            if (kind == TK_SDF_CALLOUT_STROKE)  // callout_stroke_sdf_sample (polygon.hlsli:138-156)
                s = s.d >= 0.0f ? SdfSample{fabsf(s.d) - fmaxf(sdf_word_f(w, 11), 0.0f), s.nx, s.ny}
                                : SdfSample{fabsf(s.d) - fmaxf(sdf_word_f(w, 11), 0.0f), -s.nx, -s.ny};
        } else if (arc) {
            // words: centre, radius, width; start angle, sweep, cap
            s = arc_sample(px, py, q[0], q[1], q[2], q[3], q[4], q[5], q[6]);
        } else if (star) {
            // words: centre, outer and inner radius; corner radius, rotation; stroke half width
            s = star_sample(px, py, q[0], q[1], q[2], q[3], q[4], q[5]);
            if (kind == TK_SDF_STAR_STROKE)  // star_stroke_sdf_sample (polygon.hlsli:208-221)
                s = s.d >= 0.0f ? SdfSample{fabsf(s.d) - fmaxf(sdf_word_f(w, 9), 0.0f), s.nx, s.ny}
                                : SdfSample{fabsf(s.d) - fmaxf(sdf_word_f(w, 9), 0.0f), -s.nx, -s.ny};
        }
        cov[pass] = shadow ? shadow_coverage(s, inv, expand, intensity) : coverage_from_sample(s, inv);
    }
    if (candle) return fmaxf(cov[0], cov[1]);
    return stroke ? fminf(fmaxf(cov[0] - cov[1], 0.0f), 1.0f) : cov[0];
}

// ---------------------------------------------------------------------------
// Coarse tile proofs (coarse/sdf_clip.hlsli:8-56). `tx, ty` is the tile and
// (ex, ey) the draw's translation.
// ---------------------------------------------------------------------------
constexpr float kFullTileSdfInset = 0.5f;

__device__ __forceinline__ bool rounded_corner_covers(float px, float py, float cx, float cy, float ccx, float ccy,
                                                      float radius, float inset) {
    const bool in_square = radius > 0.0f && fabsf(px - cx) < radius && fabsf(py - cy) < radius;
    const float inner = radius - inset;
    const float dx = px - ccx, dy = py - ccy;
    return !in_square || (inner > 0.0f && dx * dx + dy * dy <= inner * inner);
}

// rect_covers_tile: every pixel centre of the tile lies at least `inset`
// inside the (rounded) rectangle.
__device__ __forceinline__ bool rect_covers_tile(float rx0, float ry0, float rx1, float ry1, float q0, float q1,
                                                 float q2, float q3, float ex, float ey, uint32_t tx, uint32_t ty,
                                                 float inset) {
    const float lx = fminf(rx0, rx1), ly = fminf(ry0, ry1), ux = fmaxf(rx0, rx1), uy = fmaxf(ry0, ry1);
    const float tlx = float(tx * TK_TILE_SIZE) + 0.5f - ex, tly = float(ty * TK_TILE_SIZE) + 0.5f - ey;
    const float tux = tlx + float(TK_TILE_SIZE - 1u), tuy = tly + float(TK_TILE_SIZE - 1u);
    const float sx = ux - lx, sy = uy - ly;
    const float need = float(TK_TILE_SIZE - 1u) + 2.0f * inset;
    if (sx < need || sy < need || tlx < lx + inset || tly < ly + inset || tux > ux - inset || tuy > uy - inset)
        return false;
    const float limit = fminf(sx, sy) * 0.5f;
    const float big = 65536.0f;
    if (!(fabsf(rx0) <= big && fabsf(ry0) <= big && fabsf(rx1) <= big && fabsf(ry1) <= big)) return false;
    if (!(fabsf(q0) <= big && fabsf(q1) <= big && fabsf(q2) <= big && fabsf(q3) <= big)) return false;
    if (!(fabsf(ex) <= big && fabsf(ey) <= big)) return false;
    q0 = fminf(fmaxf(q0, 0.0f), limit);
    q1 = fminf(fmaxf(q1, 0.0f), limit);
    q2 = fminf(fmaxf(q2, 0.0f), limit);
    q3 = fminf(fmaxf(q3, 0.0f), limit);
    return rounded_corner_covers(tlx, tly, lx, ly, lx + q0, ly + q0, q0, inset) &&
           rounded_corner_covers(tux, tly, ux, ly, ux - q1, ly + q1, q1, inset) &&
           rounded_corner_covers(tlx, tuy, lx, uy, lx + q2, uy - q2, q2, inset) &&
           rounded_corner_covers(tux, tuy, ux, uy, ux - q3, uy - q3, q3, inset);
}

// sdf_clip_covers for a RECT record `w` (identity linear part checked by the
// caller): the rectangle covers the whole tile.
__device__ __forceinline__ bool sdf_rect_covers(const uint32_t* w, float ex, float ey, uint32_t tx, uint32_t ty) {
    return rect_covers_tile(sdf_word_f(w, 1), sdf_word_f(w, 2), sdf_word_f(w, 3), sdf_word_f(w, 4), sdf_word_f(w, 5),
                            sdf_word_f(w, 6), sdf_word_f(w, 7), sdf_word_f(w, 8), ex, ey, tx, ty,
                            kFullTileSdfInset);
}

// sdf_stroke_empty for a RECT_STROKE record: the tile lies inside the
// stroke's hole, at least one pixel from its inner edge.
__device__ __forceinline__ bool sdf_stroke_empty(const uint32_t* w, float ex, float ey, uint32_t tx, uint32_t ty) {
    const float x0 = sdf_word_f(w, 1), y0 = sdf_word_f(w, 2), x1 = sdf_word_f(w, 3), y1 = sdf_word_f(w, 4);
    const float r0 = sdf_word_f(w, 5), r1 = sdf_word_f(w, 6), r2 = sdf_word_f(w, 7), r3 = sdf_word_f(w, 8);
    const float s0 = sdf_word_f(w, 9), s1 = sdf_word_f(w, 10), s2 = sdf_word_f(w, 11), s3 = sdf_word_f(w, 12);
    const float big = 65536.0f;
    if (!(fabsf(x0) <= big && fabsf(y0) <= big && fabsf(x1) <= big && fabsf(y1) <= big)) return false;
    if (!(fabsf(r0) <= big && fabsf(r1) <= big && fabsf(r2) <= big && fabsf(r3) <= big)) return false;
    if (!(fabsf(s0) <= big && fabsf(s1) <= big && fabsf(s2) <= big && fabsf(s3) <= big)) return false;
    const float ht = fmaxf(s0, 0.0f), hr = fmaxf(s1, 0.0f), hb = fmaxf(s2, 0.0f), hl = fmaxf(s3, 0.0f);
    const float lx = fminf(x0, x1), ly = fminf(y0, y1), ux = fmaxf(x0, x1), uy = fmaxf(y0, y1);
    const float ix0 = lx + hl, iy0 = ly + ht, ix1 = ux - hr, iy1 = uy - hb;
    if (ix0 >= ix1 || iy0 >= iy1) return false;
    const float c0 = fmaxf(ht, hl), c1 = fmaxf(ht, hr), c2 = fmaxf(hb, hl), c3 = fmaxf(hb, hr);
    return rect_covers_tile(ix0, iy0, ix1, iy1, fmaxf(r0 - c0, 0.0f), fmaxf(r1 - c1, 0.0f), fmaxf(r2 - c2, 0.0f),
                            fmaxf(r3 - c3, 0.0f), ex, ey, tx, ty, 1.0f);
}

}  // namespace tkd
