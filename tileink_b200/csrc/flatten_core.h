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
// One quadratic's flattening plan: n points (n >= 1), the last of them the
// end point. mode 0: the end point only (degenerate); 1: uniform steps in t
// (nearly collinear control points); 2: the integral parametrisation.
struct QuadPlan {
    int n, mode;
    double a0, a2, v0, v2;
};
TK_HD inline QuadPlan plan_quad(const Pt& p0, const Pt& p1, const Pt& p2, double tol) {
    QuadPlan q{1, 0, 0.0, 0.0, 0.0, 0.0};
    double ddx = 2.0 * p1.x - p0.x - p2.x, ddy = 2.0 * p1.y - p0.y - p2.y;
    double u0 = (p1.x - p0.x) * ddx + (p1.y - p0.y) * ddy;
    double u2 = (p2.x - p1.x) * ddx + (p2.y - p1.y) * ddy;
    double cross = (p2.x - p0.x) * ddy - (p2.y - p0.y) * ddx;
    double dd = ::sqrt(ddx * ddx + ddy * ddy);
    if (dd < 1e-12) return q;
    double x0 = u0 / cross, x2 = u2 / cross;
    double scale = ::fabs(cross) / (dd * ::fabs(x2 - x0));
    if (!(isfinite(x0) && isfinite(x2) && isfinite(scale)) || ::fabs(cross) < 1e-12 * dd * dd) {
        // Nearly collinear control points: uniform steps with the chord bound
        // |B''| h^2 / 8 = |dd| h^2 / 4 <= tol.
        q.mode = 1;
        q.n = count_of(::sqrt(dd / (4.0 * tol)), kMaxSubdivisions);
        return q;
    }
    q.mode = 2;
    q.a0 = approx_integral(x0);
    q.a2 = approx_integral(x2);
    double count = 0.5 * ::fabs(q.a2 - q.a0) * ::sqrt(scale / tol);
    q.n = count_of(count, kMaxSubdivisions);
    q.v0 = approx_inv_integral(q.a0);
    q.v2 = approx_inv_integral(q.a2);
    return q;
}
// The curve parameter of point i (1 <= i < n) of a plan of mode 1 or 2.
TK_HD inline double quad_param(const QuadPlan& q, int i) {
    if (q.mode == 1) return double(i) / q.n;
    double v = approx_inv_integral(q.a0 + (q.a2 - q.a0) * double(i) / q.n);
    return (v - q.v0) / (q.v2 - q.v0);
}
template <class P, class Emit>
TK_HD void flatten_quad(P q0, P q1, P q2, double tol, Emit&& emit) {
    const QuadPlan q = plan_quad(val(q0), val(q1), val(q2), tol);
    for (int i = 1; i < q.n; ++i) emit(quad_eval(q0, q1, q2, quad_param(q, i)));
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
constexpr double kQuadShare = 0.1;  // share of the tolerance spent on the cubic-to-quadratic split

// Number of quadratics a cubic is split into.
TK_HD inline int cubic_quad_count(const Pt& c0, const Pt& c1, const Pt& c2, const Pt& c3, double tol) {
    Pt third{c3.x - 3.0 * c2.x + 3.0 * c1.x - c0.x, c3.y - 3.0 * c2.y + 3.0 * c1.y - c0.y};
    double err = ::sqrt(3.0) / 36.0 * ::sqrt(third.x * third.x + third.y * third.y);
    return ceil_cbrt(err / (kQuadShare * tol), kMaxSubdivisions);
}
template <class P>
struct SubQuad {
    P q0, ctrl, q3;
};
// Quadratic j of the m a cubic is split into (the last one ends exactly at
// the cubic's end point); flattened with tolerance (1 - kQuadShare) tol.
template <class P>
TK_HD inline SubQuad<P> cubic_sub_quad(const P c[4], int j, int m) {
    double t0 = double(j) / m, t1 = double(j + 1) / m, h = (t1 - t0) / 3.0;
    P q0 = cubic_eval(c, t0), q3 = cubic_eval(c, t1);
    P q1 = q0 + cubic_deriv(c, t0) * h, q2 = q3 - cubic_deriv(c, t1) * h;
    P ctrl = ((q1 + q2) * 3.0 - q0 - q3) * 0.25;
    if (j == m - 1) q3 = c[3];
    return SubQuad<P>{q0, ctrl, q3};
}
template <class P, class Emit>
TK_HD void flatten_cubic(const P c[4], double tol, Emit&& emit) {
    const int m = cubic_quad_count(val(c[0]), val(c[1]), val(c[2]), val(c[3]), tol);
    for (int j = 0; j < m; ++j) {
        const SubQuad<P> s = cubic_sub_quad(c, j, m);
        flatten_quad(s.q0, s.ctrl, s.q3, (1.0 - kQuadShare) * tol, emit);
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
