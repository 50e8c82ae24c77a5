// Warp-cooperative flattening of one element: the 32 lanes of a warp produce
// the element's points in order, 32 at a time, instead of one thread walking
// them all. The points are those of tkf::element_points (flatten_core.h),
// computed by the same functions on the same values, so they are bit for bit
// the host flattener's:
//   * a move gives its point, a line its end point;
//   * a quadratic is planned once (tkf::plan_quad) and its point i is
//     quad_eval at quad_param(plan, i), the last one the end point;
//   * a cubic is split into m quadratics (tkf::cubic_sub_quad), which lanes
//     plan 32 at a time; a lane then finds the quadratic of its point by a
//     binary search over the warp's inclusive point counts and takes that
//     quadratic's plan from its lane.
// Each round hands the sink 32 lanes' (valid, point) with the valid lanes a
// prefix of the warp, in the order the sequential flattener emits them.
#pragma once
#include "flatten_core.h"

namespace tk {

struct WarpQuad {
    tkf::Pt q0, q1, q2;
    tkf::QuadPlan plan;
};

__device__ inline double shfl_d(double v, uint32_t src) { return __shfl_sync(0xffffffffu, v, int(src)); }
__device__ inline tkf::Pt shfl_pt(const tkf::Pt& p, uint32_t src) { return {shfl_d(p.x, src), shfl_d(p.y, src)}; }

__device__ inline WarpQuad shfl_quad(const WarpQuad& q, uint32_t src) {
    WarpQuad r;
    r.q0 = shfl_pt(q.q0, src);
    r.q1 = shfl_pt(q.q1, src);
    r.q2 = shfl_pt(q.q2, src);
    r.plan.n = __shfl_sync(0xffffffffu, q.plan.n, int(src));
    r.plan.mode = __shfl_sync(0xffffffffu, q.plan.mode, int(src));
    r.plan.a0 = shfl_d(q.plan.a0, src);
    r.plan.a2 = shfl_d(q.plan.a2, src);
    r.plan.v0 = shfl_d(q.plan.v0, src);
    r.plan.v2 = shfl_d(q.plan.v2, src);
    return r;
}

// Point i (1 <= i <= n) of a planned quadratic.
__device__ inline tkf::Pt quad_point(const WarpQuad& q, int i) {
    if (i >= q.plan.n) return q.q2;
    return tkf::quad_eval(q.q0, q.q1, q.q2, tkf::quad_param(q.plan, i));
}

// The points of quadratics held by lanes 0..k-1 (lane j: quadratic j of the
// group, `mine`), in order.
template <class Sink>
__device__ void warp_quads(const WarpQuad& mine, uint32_t k, uint32_t lane, Sink& sink) {
    const uint32_t n = lane < k ? uint32_t(mine.plan.n) : 0u;
    uint32_t incl = n;  // inclusive point counts over the group's quadratics
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= uint32_t(d)) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    for (uint32_t g0 = 0; g0 < total; g0 += 32u) {
        const uint32_t g = g0 + lane;
        const bool valid = g < total;
        // the quadratic j of point g: the first with incl[j] > g
        uint32_t j = 0;
#pragma unroll
        for (uint32_t step = 16; step; step >>= 1) {
            const uint32_t probe = __shfl_sync(0xffffffffu, incl, int(j + step - 1u));
            if (probe <= g) j += step;
        }
        const WarpQuad q = shfl_quad(mine, valid ? j : 0u);
        const uint32_t before = __shfl_sync(0xffffffffu, incl - n, int(valid ? j : 0u));
        tkf::Pt p{0.0, 0.0};
        if (valid) p = quad_point(q, int(g - before) + 1);
        sink(valid, p, min(32u, total - g0));
    }
}

// All points of element e (verb and coordinates already checked).
template <class Sink>
__device__ void warp_element_points(const tk_flatten_el& e, uint32_t lane, Sink& sink) {
    using tkf::Pt;
    const Pt c[4] = {Pt{e.p[0][0], e.p[0][1]}, Pt{e.p[1][0], e.p[1][1]}, Pt{e.p[2][0], e.p[2][1]},
                     Pt{e.p[3][0], e.p[3][1]}};
    if (e.verb == TK_EL_MOVE || e.verb == TK_EL_LINE) {
        sink(lane == 0u, e.verb == TK_EL_MOVE ? c[0] : c[1], 1u);
        return;
    }
    if (e.verb == TK_EL_QUAD) {
        WarpQuad q{c[0], c[1], c[2], tkf::plan_quad(c[0], c[1], c[2], e.tolerance)};
        warp_quads(q, 1u, lane, sink);
        return;
    }
    const int m = tkf::cubic_quad_count(c[0], c[1], c[2], c[3], e.tolerance);
    const double tol = (1.0 - tkf::kQuadShare) * e.tolerance;
    for (int j0 = 0; j0 < m; j0 += 32) {
        const int j = j0 + int(lane);
        WarpQuad q{};
        if (j < m) {
            const tkf::SubQuad<Pt> s = tkf::cubic_sub_quad(c, j, m);
            q = WarpQuad{s.q0, s.ctrl, s.q3, tkf::plan_quad(s.q0, s.ctrl, s.q3, tol)};
        }
        warp_quads(q, uint32_t(min(32, m - j0)), lane, sink);
    }
}

}  // namespace tk
