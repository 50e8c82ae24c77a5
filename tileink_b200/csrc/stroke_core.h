// Stroking with round joins and round caps, shared by the host Canvas
// (canvas.cpp) and the device stroker (stroke.cu). Both compile this source
// with IEEE double arithmetic and no contraction, and it calls only correctly
// rounded operations (+ - * /, sqrt, fmax), so both produce the same outline
// lines bit for bit.
//
// Contract (kurbo::stroke with Join::Round and Cap::Round, the stroking step of
// src/canvas/primitives/paths.rs:24-48): the centerline is flattened
// (flatten_core.h); each segment is offset by +-h (h = width / 2); outer joins
// get circular arcs, inner joins pivot through the centerline vertex, open
// ends get semicircular caps and a polyline of one point gets a disc. The
// outline loops are filled with the nonzero rule.
//
// Centerlines. A polyline starts at a move_to (or, for a drawing element after
// a close or before any move_to, at the current point), collects the
// flattened points of its elements, drops each point within 1e-9 of the last
// point kept, and on close drops a last point within 1e-9 of its first.
//
// Outline loops. A closed polyline of n >= 3 points gives two loops (its left
// offset forwards and backwards); any other polyline of n >= 1 points gives
// one. A loop is a cycle of units. A unit belongs to one vertex c with incoming
// direction din: it is the offset edge (c_prev + L(din) h -> c + L(din) h)
// followed by the vertex's join towards the outgoing direction (or its cap,
// at an open end), and it ends at c + L(dout) h, where the next unit's offset
// edge starts, bit for bit. So every unit's lines are known from its own
// vertex and its two neighbours, and the units of a loop can be generated in
// parallel. L(d) = (-d.y, d.x) is the left normal.
//
// Arcs are built without trigonometry: an arc of at most a quarter turn is
// split into 2^k equal pieces by bisecting unit vectors (u_mid =
// normalize(u_lo + u_hi)), with the smallest k (at most 12) whose piece keeps
// the chord's sagitta within tol: cos(angle / 2^(k+1)) >= 1 - tol / r. Arcs of
// more than a quarter turn are split at a quarter turn first.
//
// Lines. Outline points are mapped to device pixels by the affine transform
// (x' = t0 x + t2 y + t4, y' = t1 x + t3 y + t5) and every edge of squared
// device length above 1e-24 becomes a line (PathFlatten::flatten's filter,
// src/shared/path_flatten.rs:20-82).
#pragma once
#include "flatten_core.h"

namespace tkf {

constexpr double kPointEps2 = 1e-18;  // points closer than 1e-9 are the same point
constexpr int kMaxArcLevels = 12;     // at most 4096 pieces per quarter turn

TK_HD inline bool distinct(Pt a, Pt b) {
    const double dx = a.x - b.x, dy = a.y - b.y;
    return dx * dx + dy * dy > kPointEps2;
}
TK_HD inline Pt normalize(Pt a) {
    const double l = ::sqrt(a.x * a.x + a.y * a.y);
    return {a.x / l, a.y / l};
}
TK_HD inline Pt left_normal(Pt d) { return {-d.y, d.x}; }
TK_HD inline double dot(Pt a, Pt b) { return a.x * b.x + a.y * b.y; }
TK_HD inline double cross(Pt a, Pt b) { return a.x * b.y - a.y * b.x; }

// Arc from unit vector u0 to u1 (dot(u0, u1) >= 0) around c with radius r:
// emits the end points of its pieces in order, the last one c + u1 * r.
template <class Emit>
TK_HD void arc_short(Pt c, double r, Pt u0, Pt u1, double tol, Emit& emit) {
    const double target = r > tol ? 1.0 - tol / r : -2.0;
    int k = 0;
    for (Pt v = u1;;) {  // v: the end of the first piece at level k
        const double half = ::sqrt(::fmax(0.0, (1.0 + dot(u0, v)) * 0.5));
        if (half >= target || k >= kMaxArcLevels) break;
        v = normalize(u0 + v);
        ++k;
    }
    // In-order walk of the bisection tree: hi[] holds the right ends still to
    // reach, lo the last point reached.
    Pt hi[kMaxArcLevels + 1];
    int level[kMaxArcLevels + 1];
    int sp = 0;
    hi[0] = u1;
    level[0] = 0;
    Pt lo = u0;
    while (sp >= 0) {
        if (level[sp] == k) {
            lo = hi[sp--];
            emit(c + lo * r);
            continue;
        }
        const Pt mid = normalize(lo + hi[sp]);
        const int l = ++level[sp];
        ++sp;
        hi[sp] = mid;
        level[sp] = l;
    }
}

// Clockwise arc (turning right, y up) from u0 to u1 of at most a half turn.
template <class Emit>
TK_HD void arc_cw(Pt c, double r, Pt u0, Pt u1, double tol, Emit& emit) {
    if (dot(u0, u1) >= 0.0) {
        arc_short(c, r, u0, u1, tol, emit);
        return;
    }
    const Pt m{u0.y, -u0.x};  // u0 turned a quarter clockwise
    arc_short(c, r, u0, m, tol, emit);
    arc_short(c, r, m, u1, tol, emit);
}

// The join at vertex c from direction din to dout on the left offset: an arc
// around c when the path turns right (the left side is outside), else the
// pivot c -> c + L(dout) h.
template <class Emit>
TK_HD void join(Pt c, Pt din, Pt dout, double h, double tol, Emit& emit) {
    const Pt nin = left_normal(din), nout = left_normal(dout);
    if (cross(din, dout) < 0.0) {
        arc_cw(c, h, nin, nout, tol, emit);
    } else {
        emit(c);
        emit(c + nout * h);
    }
}

TK_HD inline uint32_t outline_loops(uint32_t n, bool closed) {
    if (n == 0u) return 0u;
    return (closed && n >= 3u) ? 2u : 1u;
}
TK_HD inline uint32_t outline_units(uint32_t n, bool closed) {
    if (closed && n >= 3u) return n;
    return n >= 2u ? 2u * (n - 1u) : n;
}

// Unit u of loop `loop` of the polyline v[0..n): emit() gets the unit's start
// (the previous unit's end) first, then its points; consecutive emitted points
// are the unit's edges.
template <class V, class Emit>
TK_HD void outline_unit(const V& v, uint32_t n, bool closed, uint32_t loop, uint32_t u, double h, double tol,
                        Emit& emit) {
    if (n == 1u) {  // a dot: the disc, counterclockwise from +x
        const Pt c = v[0];
        const Pt q[5] = {{1.0, 0.0}, {0.0, 1.0}, {-1.0, 0.0}, {0.0, -1.0}, {1.0, 0.0}};
        emit(c + q[0] * h);
        for (int s = 0; s < 4; ++s) arc_short(c, h, q[s], q[s + 1], tol, emit);
        return;
    }
    if (closed && n >= 3u) {  // loop 1 walks the polyline backwards
        auto at = [&](uint32_t i) -> Pt {
            i %= n;
            return loop ? v[n - 1u - i] : v[i];
        };
        const Pt cp = at(u + n - 1u), c = at(u), cn = at(u + 1u);
        const Pt din = normalize(c - cp);
        const Pt nin = left_normal(din);
        emit(cp + nin * h);
        emit(c + nin * h);
        join(c, din, normalize(cn - c), h, tol, emit);
        return;
    }
    // Open: units 0..n-2 are vertices 1..n-1 walking forwards (the last one
    // the end cap), units n-1..2n-3 vertices n-2..0 walking backwards (the
    // last one the start cap).
    const bool back = u >= n - 1u;
    const uint32_t j = back ? u - (n - 1u) + 1u : u + 1u;
    auto at = [&](uint32_t i) -> Pt { return back ? v[n - 1u - i] : v[i]; };
    const Pt cp = at(j - 1u), c = at(j);
    const Pt din = normalize(c - cp);
    const Pt nin = left_normal(din);
    emit(cp + nin * h);
    emit(c + nin * h);
    if (j + 1u < n) join(c, din, normalize(at(j + 1u) - c), h, tol, emit);
    else arc_cw(c, h, nin, nin * -1.0, tol, emit);
}

struct Affine {
    double t[6];
    TK_HD Pt operator()(Pt p) const { return {t[0] * p.x + t[2] * p.y + t[4], t[1] * p.x + t[3] * p.y + t[5]}; }
};

// Consecutive emitted points -> device-space edges kept by keep_edge.
template <class Line>
struct EdgeChain {
    Affine xf;
    Line& line;
    bool has = false;
    Pt last{0.0, 0.0};
    TK_HD void operator()(Pt p) {
        const Pt q = xf(p);
        if (has && keep_edge(last, q)) line(last, q);
        last = q;
        has = true;
    }
};

// Centerline cleanup of one polyline whose raw points are v[0..raw): keeps
// each point farther than 1e-9 from the last point kept (compacting in
// place), then for a closed polyline drops a last point within 1e-9 of the
// first. Returns the number of points kept.
template <class V>
TK_HD uint32_t dedupe_polyline(V& v, uint32_t raw, bool closed) {
    if (raw == 0u) return 0u;
    uint32_t n = 1u;
    Pt back = v[0];
    for (uint32_t i = 1; i < raw; ++i) {
        const Pt p = v[i];
        if (distinct(p, back)) {
            v[n++] = p;
            back = p;
        }
    }
    if (closed && n > 1u && !distinct(v[0], back)) --n;
    return n;
}

// Largest stretch |M x| / |x| of the transform's linear part (its largest
// singular value): the outline lies within h of the centerline in local
// units, so within h * stretch of it in device pixels.
TK_HD inline double max_stretch(const double t[6]) {
    const double s = t[0] * t[0] + t[1] * t[1] + t[2] * t[2] + t[3] * t[3];
    const double det = t[0] * t[3] - t[1] * t[2];
    return ::sqrt(0.5 * (s + ::sqrt(::fmax(0.0, s * s - 4.0 * det * det))));
}

}  // namespace tkf
