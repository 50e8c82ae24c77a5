// Device stroking (the stroking step of Canvas::push_stroke,
// src/canvas/primitives/paths.rs:24-48, kurbo::stroke with round joins and
// caps, moved onto the GPU). The arithmetic is stroke_core.h and
// flatten_core.h, shared with the host Canvas, so the outline lines are
// bit-identical to the host stroker's.
//
// 1. Centerline points: one thread per element writes its points (a move's
//    point, a line's end, a flattened curve) at its scanned offset.
// 2. Centerline cleanup: one thread per polyline drops repeated points in
//    place (a sequential rule, but only a compare per point).
// 3. Outline: one warp per polyline; lanes take the outline's units (one
//    vertex's offset edge plus its join or cap each), which depend only on
//    the vertex and its neighbours. Lines are counted, scanned over the
//    polylines, then written 32 units at a time at warp-scanned offsets, in
//    the host stroker's order.
#include <cuda_runtime.h>

#include "flatten_core.h"
#include "kernels.h"
#include "stroke_core.h"

namespace tk {
namespace {

using tkf::Pt;

constexpr uint32_t kStrokeThreads = 128;

// Stroke elements the device accepts: a move, line, quadratic or cubic with
// tolerance >= 1e-3 and finite coordinates within 1e6 (bounding one thread's
// flattening work); anything else is flagged and contributes no points.
__device__ bool stroke_element_ok(const tk_flatten_el& e) {
    if (e.verb < TK_EL_LINE || e.verb > TK_EL_MOVE) return false;
    if (!(e.tolerance >= 1e-3) || !isfinite(e.tolerance)) return false;
    const uint32_t pts = e.verb == TK_EL_MOVE ? 1u : e.verb + 1u;
    for (uint32_t k = 0; k < pts; ++k)
        if (!(fabs(e.p[k][0]) <= 1e6) || !(fabs(e.p[k][1]) <= 1e6)) return false;
    return true;
}

struct CountPoints {
    uint32_t n = 0;
    __device__ void operator()(Pt) { ++n; }
};

struct WritePoints {
    Pt* out;
    uint64_t at, end;
    uint32_t* error;
    __device__ void operator()(Pt p) {
        if (at < end) out[at] = p;
        else atomicOr(error, ERR_SEGMENT_OVERFLOW);
        ++at;
    }
};

__global__ void k_stroke_count(const tk_flatten_el* __restrict__ els, uint64_t n, uint32_t* counts,
                               unsigned long long* total64, uint32_t* error) {
    unsigned long long sum = 0;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const tk_flatten_el e = els[i];
        CountPoints c;
        if (stroke_element_ok(e)) tkf::element_points(e, c);
        else atomicOr(error, ERR_UNSUPPORTED);
        counts[i] = c.n;
        sum += c.n;
    }
    if (sum) atomicAdd(total64, sum);
}

__global__ void k_stroke_points(const tk_flatten_el* __restrict__ els, uint64_t n, const uint32_t* __restrict__ offsets,
                                Pt* pts, uint64_t cap, uint32_t* error) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const tk_flatten_el e = els[i];
        WritePoints w{pts, offsets[i], cap, error};
        if (stroke_element_ok(e)) tkf::element_points(e, w);
    }
}

// Raw point range of polyline `pl`: [offsets[element0], offsets[element0 + count]).
__device__ inline void raw_range(const tk_stroke_polyline& P, const uint32_t* offsets, uint64_t n_els,
                                 uint32_t total, uint32_t& a, uint32_t& b) {
    a = offsets[P.element0];
    const uint64_t e1 = uint64_t(P.element0) + P.element_count;
    b = e1 < n_els ? offsets[e1] : total;
}

__global__ void k_stroke_polylines(const tk_stroke_polyline* __restrict__ polys, uint32_t npl,
                                   const tk_flatten_el* __restrict__ els, uint64_t n_els,
                                   const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ total, Pt* pts,
                                   uint32_t* poly_n, uint32_t* error) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npl) return;
    const tk_stroke_polyline P = polys[i];
    bool ok = els[P.element0].verb == TK_EL_MOVE;
    for (uint32_t e = P.element0; e < P.element0 + P.element_count; ++e)  // the elements carry their polyline
        ok = ok && els[e].path == i;
    if (!ok) {
        atomicOr(error, ERR_LINE_PATH_MISMATCH);
        poly_n[i] = 0u;
        return;
    }
    uint32_t a, b;
    raw_range(P, offsets, n_els, *total, a, b);
    Pt* v = pts + a;
    poly_n[i] = tkf::dedupe_polyline(v, b - a, P.closed != 0u);
}

struct CountLines {
    uint32_t n = 0;
    __device__ void operator()(Pt, Pt) { ++n; }
};

struct WriteLines {
    tk_line* out;
    uint64_t at, end;
    uint32_t path;
    uint32_t* error;
    __device__ void operator()(Pt a, Pt b) {
        if (at < end) out[at] = tk_line{path, 0.0f, {float(a.x), float(a.y)}, {float(b.x), float(b.y)}};
        else atomicOr(error, ERR_SEGMENT_OVERFLOW);
        ++at;
    }
};

struct PolyView {
    const Pt* v;
    uint32_t n, loops, units;
    bool closed;
    double h, tol;
    tkf::Affine xf;
    uint32_t path;
};

__device__ inline PolyView poly_view(uint32_t pl, const tk_stroke_polyline* polys, const tk_stroke_desc* strokes,
                                     const uint32_t* offsets, const Pt* pts, const uint32_t* poly_n) {
    const tk_stroke_polyline P = polys[pl];
    const tk_stroke_desc& S = strokes[P.stroke];
    PolyView q;
    q.v = pts + offsets[P.element0];
    q.n = poly_n[pl];
    q.closed = P.closed != 0u;
    q.loops = tkf::outline_loops(q.n, q.closed);
    q.units = tkf::outline_units(q.n, q.closed);
    q.h = S.half_width;
    q.tol = S.tolerance;
    for (int k = 0; k < 6; ++k) q.xf.t[k] = S.transform[k];
    q.path = S.path;
    return q;
}

__device__ inline uint32_t unit_lines(const PolyView& q, uint32_t loop, uint32_t u) {
    CountLines c;
    tkf::EdgeChain<CountLines> ch{q.xf, c};
    tkf::outline_unit(q.v, q.n, q.closed, loop, u, q.h, q.tol, ch);
    return c.n;
}

__global__ void __launch_bounds__(kStrokeThreads) k_outline_count(const tk_stroke_polyline* __restrict__ polys,
                                                                  uint32_t npl, const tk_stroke_desc* __restrict__ strokes,
                                                                  const uint32_t* __restrict__ offsets,
                                                                  const Pt* __restrict__ pts,
                                                                  const uint32_t* __restrict__ poly_n,
                                                                  uint32_t* poly_lines, unsigned long long* total64,
                                                                  uint32_t* error) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t pl = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); pl < npl; pl += warps) {
        const PolyView q = poly_view(pl, polys, strokes, offsets, pts, poly_n);
        unsigned long long cnt = 0;
        for (uint32_t loop = 0; loop < q.loops; ++loop)
            for (uint32_t u = lane; u < q.units; u += 32u) cnt += unit_lines(q, loop, u);
#pragma unroll
        for (int d = 16; d; d >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, d);
        if (lane == 0) {
            if (cnt > 0xFFFFFFFFull) atomicOr(error, ERR_SEGMENT_OVERFLOW);
            poly_lines[pl] = uint32_t(cnt);
            if (cnt) atomicAdd(total64, cnt);
        }
    }
}

__global__ void __launch_bounds__(kStrokeThreads) k_outline_emit(const tk_stroke_polyline* __restrict__ polys,
                                                                 uint32_t npl, const tk_stroke_desc* __restrict__ strokes,
                                                                 const uint32_t* __restrict__ offsets,
                                                                 const Pt* __restrict__ pts,
                                                                 const uint32_t* __restrict__ poly_n,
                                                                 const uint32_t* __restrict__ line_off, tk_line* lines,
                                                                 uint64_t line_base, uint64_t line_end, uint32_t* error) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t pl = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); pl < npl; pl += warps) {
        const PolyView q = poly_view(pl, polys, strokes, offsets, pts, poly_n);
        uint64_t at = line_base + line_off[pl];
        for (uint32_t loop = 0; loop < q.loops; ++loop) {
            for (uint32_t u0 = 0; u0 < q.units; u0 += 32u) {
                const uint32_t u = u0 + lane;
                const uint32_t c = u < q.units ? unit_lines(q, loop, u) : 0u;
                uint32_t incl = c;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
                    if (lane >= uint32_t(d)) incl += y;
                }
                if (u < q.units && c) {
                    WriteLines w{lines, at + incl - c, line_end, q.path, error};
                    tkf::EdgeChain<WriteLines> ch{q.xf, w};
                    tkf::outline_unit(q.v, q.n, q.closed, loop, u, q.h, q.tol, ch);
                }
                at += __shfl_sync(0xffffffffu, incl, 31);
            }
        }
    }
}

// Line ranges of the stroked paths: their polylines' lines, contiguous.
__global__ void k_stroke_paths(const tk_stroke_desc* __restrict__ strokes, uint32_t n_strokes, uint32_t npl,
                               const uint32_t* __restrict__ line_off, const uint32_t* __restrict__ line_total,
                               tk_path_record* paths, uint32_t line_base) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_strokes) return;
    const tk_stroke_desc S = strokes[s];
    uint32_t a = 0, b = 0;
    if (S.polyline_count) {
        a = line_off[S.polyline0];
        const uint32_t p1 = S.polyline0 + S.polyline_count;
        b = p1 < npl ? line_off[p1] : *line_total;
    }
    paths[S.path].line_start = line_base + a;
    paths[S.path].line_count = b - a;
}

unsigned grid_for(uint64_t n, unsigned per_block) {
    const uint64_t g = (n + per_block - 1) / per_block;
    return unsigned(g < 148ull * 16 ? (g ? g : 1) : 148ull * 16);
}

}  // namespace

void launch_stroke_count(const tk_flatten_el* els, uint64_t n, uint32_t* counts, uint32_t* block_sums,
                         uint32_t* total, unsigned long long* total64, uint32_t* error, cudaStream_t st) {
    if (n) k_stroke_count<<<grid_for(n, 128), 128, 0, st>>>(els, n, counts, total64, error);
    launch_exclusive_scan(counts, n, block_sums, total, st);
}

void launch_stroke_outline_count(const StrokeView& v, uint32_t* block_sums, uint32_t* line_total,
                                 unsigned long long* line_total64, cudaStream_t st) {
    if (v.n_els) k_stroke_points<<<grid_for(v.n_els, 128), 128, 0, st>>>(v.els, v.n_els, v.offsets, v.pts, v.pt_cap,
                                                                         v.error);
    if (v.npl) {
        k_stroke_polylines<<<(v.npl + 127) / 128, 128, 0, st>>>(v.polys, v.npl, v.els, v.n_els, v.offsets,
                                                                 v.pt_total, v.pts, v.poly_n, v.error);
        k_outline_count<<<grid_for(uint64_t(v.npl) * 32, kStrokeThreads), kStrokeThreads, 0, st>>>(
            v.polys, v.npl, v.strokes, v.offsets, v.pts, v.poly_n, v.line_off, line_total64, v.error);
    }
    launch_exclusive_scan(v.line_off, v.npl, block_sums, line_total, st);
}

void launch_stroke_emit(const StrokeView& v, const uint32_t* line_total, tk_path_record* paths, tk_line* lines,
                        uint64_t line_base, uint64_t line_end, cudaStream_t st) {
    if (v.npl)
        k_outline_emit<<<grid_for(uint64_t(v.npl) * 32, kStrokeThreads), kStrokeThreads, 0, st>>>(
            v.polys, v.npl, v.strokes, v.offsets, v.pts, v.poly_n, v.line_off, lines, line_base, line_end, v.error);
    if (v.n_strokes)
        k_stroke_paths<<<(v.n_strokes + 127) / 128, 128, 0, st>>>(v.strokes, v.n_strokes, v.npl, v.line_off,
                                                                   line_total, paths, uint32_t(line_base));
}

}  // namespace tk
