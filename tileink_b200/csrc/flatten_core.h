// Bezier flattening shared by the host Canvas (canvas.cpp) and the device
// flattener (flatten.cu). Both compile this same source with IEEE double
// arithmetic and no contraction (-ffp-contract=off on the host, -fmad=false on
// the device), and it calls only correctly rounded operations (+ - * /,
// sqrt, floor, ceil), so host and device emit bit-identical points.
//
// Quadratics use the parabola-integral subdivision of R. Levien, "Flattening
// quadratic Beziers" (2019): map the quadratic onto y = x^2, use closed-form
// approximations of the arc-length-like integral and its inverse to place n
// points with equal error. Cubics are first split into m quadratics with the
// cubic-to-quadratic error bound sqrt(3)/36 * |p3 - 3p2 + 3p1 - p0| / m^3.
#pragma once
#include <math.h>

#include "../../include/tileink.h"

#ifdef __CUDACC__
#define TK_HD __host__ __device__
#else
#define TK_HD
#endif

namespace tkf {

struct alignas(16) Pt {
    double x, y;
};
TK_HD inline Pt operator+(Pt a, Pt b) { return {a.x + b.x, a.y + b.y}; }
TK_HD inline Pt operator-(Pt a, Pt b) { return {a.x - b.x, a.y - b.y}; }
TK_HD inline Pt operator*(Pt a, double s) { return {a.x * s, a.y * s}; }
TK_HD inline const Pt& val(const Pt& p) { return p; }

constexpr int kMaxSubdivisions = 1 << 16;

// max(1, ceil(v)) capped at `cap`; 1 for v <= 1 or NaN.
TK_HD inline int count_of(double v, int cap) {
    if (!(v > 1.0)) return 1;
    if (v >= double(cap)) return cap;
    return int(::ceil(v));
}

// The smallest m >= 1 with m^3 >= v, capped: an exact integer cube root, so the
// result does not depend on how a math library rounds cbrt.
TK_HD inline int ceil_cbrt(double v, int cap) {
    if (!(v > 1.0)) return 1;
    if (v >= double(cap) * double(cap) * double(cap)) return cap;
    double m = ::ceil(::cbrt(v));
    while (m > 1.0 && (m - 1.0) * (m - 1.0) * (m - 1.0) >= v) m -= 1.0;
    while (m * m * m < v) m += 1.0;
    return int(m);
}

TK_HD inline double approx_integral(double x) {
    const double d = 0.67;
    return x / (1.0 - d + ::sqrt(::sqrt(d * d * d * d + 0.25 * x * x)));
}
TK_HD inline double approx_inv_integral(double x) {
    const double b = 0.39;
    return x * (1.0 - b + ::sqrt(b * b + 0.25 * x * x));
}
template <class P>
TK_HD inline P quad_eval(P p0, P p1, P p2, double t) {
    double mt = 1.0 - t;
    return p0 * (mt * mt) + p1 * (2.0 * mt * t) + p2 * (t * t);
}
template <class P, class Emit>
TK_HD void flatten_quad(P q0, P q1, P q2, double tol, Emit&& emit) {
    const Pt &p0 = val(q0), &p1 = val(q1), &p2 = val(q2);
    double ddx = 2.0 * p1.x - p0.x - p2.x, ddy = 2.0 * p1.y - p0.y - p2.y;
    double u0 = (p1.x - p0.x) * ddx + (p1.y - p0.y) * ddy;
    double u2 = (p2.x - p1.x) * ddx + (p2.y - p1.y) * ddy;
    double cross = (p2.x - p0.x) * ddy - (p2.y - p0.y) * ddx;
    double dd = ::sqrt(ddx * ddx + ddy * ddy);
    if (dd < 1e-12) {
        emit(q2);
        return;
    }
    double x0 = u0 / cross, x2 = u2 / cross;
    double scale = ::fabs(cross) / (dd * ::fabs(x2 - x0));
    if (!(isfinite(x0) && isfinite(x2) && isfinite(scale)) || ::fabs(cross) < 1e-12 * dd * dd) {
        // Nearly collinear control points: uniform steps with the chord bound
        // |B''| h^2 / 8 = |dd| h^2 / 4 <= tol.
        int n = count_of(::sqrt(dd / (4.0 * tol)), kMaxSubdivisions);
        for (int i = 1; i < n; ++i) emit(quad_eval(q0, q1, q2, double(i) / n));
        emit(q2);
        return;
    }
    double a0 = approx_integral(x0), a2 = approx_integral(x2);
    double count = 0.5 * ::fabs(a2 - a0) * ::sqrt(scale / tol);
    int n = count_of(count, kMaxSubdivisions);
    double v0 = approx_inv_integral(a0), v2 = approx_inv_integral(a2);
    for (int i = 1; i < n; ++i) {
        double v = approx_inv_integral(a0 + (a2 - a0) * double(i) / n);
        double t = (v - v0) / (v2 - v0);
        emit(quad_eval(q0, q1, q2, t));
    }
    emit(q2);
}
template <class P>
TK_HD inline P cubic_eval(const P c[4], double t) {
    double mt = 1.0 - t;
    return c[0] * (mt * mt * mt) + c[1] * (3.0 * mt * mt * t) + c[2] * (3.0 * mt * t * t) + c[3] * (t * t * t);
}
template <class P>
TK_HD inline P cubic_deriv(const P c[4], double t) {
    double mt = 1.0 - t;
    return (c[1] - c[0]) * (3.0 * mt * mt) + (c[2] - c[1]) * (6.0 * mt * t) + (c[3] - c[2]) * (3.0 * t * t);
}
template <class P, class Emit>
TK_HD void flatten_cubic(const P c[4], double tol, Emit&& emit) {
    const double quad_share = 0.1;
    const Pt &c0 = val(c[0]), &c1 = val(c[1]), &c2 = val(c[2]), &c3 = val(c[3]);
    Pt third{c3.x - 3.0 * c2.x + 3.0 * c1.x - c0.x, c3.y - 3.0 * c2.y + 3.0 * c1.y - c0.y};
    double err = ::sqrt(3.0) / 36.0 * ::sqrt(third.x * third.x + third.y * third.y);
    int m = ceil_cbrt(err / (quad_share * tol), kMaxSubdivisions);
    for (int j = 0; j < m; ++j) {
        double t0 = double(j) / m, t1 = double(j + 1) / m, h = (t1 - t0) / 3.0;
        P q0 = cubic_eval(c, t0), q3 = cubic_eval(c, t1);
        P q1 = q0 + cubic_deriv(c, t0) * h, q2 = q3 - cubic_deriv(c, t1) * h;
        P ctrl = ((q1 + q2) * 3.0 - q0 - q3) * 0.25;
        if (j == m - 1) q3 = c[3];
        flatten_quad(q0, ctrl, q3, (1.0 - quad_share) * tol, emit);
    }
}

// PathFlatten::flatten's edge filter (src/shared/path_flatten.rs:20-82): an
// edge is kept when its squared length exceeds 1e-24.
TK_HD inline bool keep_edge(Pt a, Pt b) {
    double dx = a.x - b.x, dy = a.y - b.y;
    return dx * dx + dy * dy > 1.0e-12 * 1.0e-12;
}

// The points one element contributes to its contour, its start point
// excluded: a move's point, a line's end, or the flattened curve.
template <class Emit>
TK_HD void element_points(const tk_flatten_el& e, Emit& emit) {
    const Pt from{e.p[0][0], e.p[0][1]};
    if (e.verb == TK_EL_MOVE) {
        emit(from);
    } else if (e.verb == TK_EL_LINE) {
        emit(Pt{e.p[1][0], e.p[1][1]});
    } else if (e.verb == TK_EL_QUAD) {
        flatten_quad(from, Pt{e.p[1][0], e.p[1][1]}, Pt{e.p[2][0], e.p[2][1]}, e.tolerance, emit);
    } else if (e.verb == TK_EL_CUBIC) {
        const Pt c[4] = {from, Pt{e.p[1][0], e.p[1][1]}, Pt{e.p[2][0], e.p[2][1]}, Pt{e.p[3][0], e.p[3][1]}};
        flatten_cubic(c, e.tolerance, emit);
    }
}

}  // namespace tkf
