// Device stroking (the stroking step of Canvas::push_stroke,
// src/canvas/primitives/paths.rs:24-48, kurbo::stroke with round joins and
// caps, moved onto the GPU). The arithmetic is stroke_core.h and
// flatten_core.h, shared with the host Canvas, so the outline lines are
// bit-identical to the host stroker's.
//
// 1. Centerline points: one thread per element counts its points from the
//    quadratics' plans alone; one warp per element writes them (a move's
//    point, a line's end, a flattened curve; warp_flatten.cuh) at its
//    scanned offset, 32 consecutive points per store round.
// 2. Centerline cleanup: one warp per polyline drops repeated points in
//    place. The rule is sequential (a point is compared with the last point
//    kept), so a warp takes 32 points at once only when each is distinct
//    from its predecessor and the first from the last point kept, which
//    keeps all of them; a group holding a repeat is walked by one lane.
// 3. Outline: one warp per polyline; lanes take the outline's units (one
//    vertex's offset edge plus its join or cap each), which depend only on
//    the vertex and its neighbours. The count pass keeps each unit's line
//    count (slot 2 x the polyline's first raw point + loop x units + unit:
//    a polyline of r raw points has at most 2r unit slots); the counts are
//    scanned over the polylines, and the emit pass writes 32 units at a time
//    at warp-scanned offsets, in the host stroker's order, through a
//    per-warp shared-memory stage so that the stores to the line buffer are
//    whole contiguous runs.
#include <cuda_runtime.h>

#include "flatten_core.h"
#include "kernels.h"
#include "stroke_core.h"
#include "warp_flatten.cuh"

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

struct WarpWritePoints {
    Pt* out;
    uint64_t at, end;
    uint32_t lane;
    uint32_t* error;
    __device__ void operator()(bool valid, Pt p, uint32_t k) {
        if (valid) {
            if (at + lane < end) out[at + lane] = p;
            else atomicOr(error, ERR_SEGMENT_OVERFLOW);
        }
        at += k;
    }
};

// Points of one element, on one thread: a move or line gives one; a curve's
// count is the sum of its quadratics' plans, which needs no point evaluated.
__device__ uint32_t element_point_count(const tk_flatten_el& e) {
    const Pt c[4] = {Pt{e.p[0][0], e.p[0][1]}, Pt{e.p[1][0], e.p[1][1]}, Pt{e.p[2][0], e.p[2][1]},
                     Pt{e.p[3][0], e.p[3][1]}};
    if (e.verb == TK_EL_MOVE || e.verb == TK_EL_LINE) return 1u;
    if (e.verb == TK_EL_QUAD) return uint32_t(tkf::plan_quad(c[0], c[1], c[2], e.tolerance).n);
    const int m = tkf::cubic_quad_count(c[0], c[1], c[2], c[3], e.tolerance);
    const double tol = (1.0 - tkf::kQuadShare) * e.tolerance;
    uint32_t n = 0;
    for (int j = 0; j < m; ++j) {
        const tkf::SubQuad<Pt> s = tkf::cubic_sub_quad(c, j, m);
        n += uint32_t(tkf::plan_quad(s.q0, s.ctrl, s.q3, tol).n);
    }
    return n;
}

__global__ void __launch_bounds__(kStrokeThreads)
    k_stroke_count(const tk_flatten_el* __restrict__ els, uint64_t n, uint32_t* counts, unsigned long long* total64,
                   uint32_t* error) {
    unsigned long long sum = 0;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const tk_flatten_el e = els[i];
        uint32_t c = 0;
        if (stroke_element_ok(e)) c = element_point_count(e);
        else atomicOr(error, ERR_UNSUPPORTED);
        counts[i] = c;
        sum += c;
    }
    if (sum) atomicAdd(total64, sum);
}

__global__ void __launch_bounds__(kStrokeThreads)
    k_stroke_points(const tk_flatten_el* __restrict__ els, uint64_t n, const uint32_t* __restrict__ offsets, Pt* pts,
                    uint64_t cap, uint32_t* error) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
        const tk_flatten_el e = els[i];
        WarpWritePoints w{pts, offsets[i], cap, lane, error};
        if (stroke_element_ok(e)) warp_element_points(e, lane, w);
    }
}

// Raw point range of polyline `pl`: [offsets[element0], offsets[element0 + count]).
__device__ inline void raw_range(const tk_stroke_polyline& P, const uint32_t* offsets, uint64_t n_els,
                                 uint32_t total, uint32_t& a, uint32_t& b) {
    a = offsets[P.element0];
    const uint64_t e1 = uint64_t(P.element0) + P.element_count;
    b = e1 < n_els ? offsets[e1] : total;
}

__global__ void __launch_bounds__(kStrokeThreads)
    k_stroke_polylines(const tk_stroke_polyline* __restrict__ polys, uint32_t npl,
                       const tk_flatten_el* __restrict__ els, uint64_t n_els, const uint32_t* __restrict__ offsets,
                       const uint32_t* __restrict__ total, Pt* pts, uint32_t* poly_n, uint32_t* error) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < npl; i += warps) {
        const tk_stroke_polyline P = polys[i];
        bool ok = true;  // the elements carry their polyline; the first is a move
        for (uint32_t e = P.element0 + lane; e < P.element0 + P.element_count; e += 32u)
            ok = ok && els[e].path == i && (e != P.element0 || els[e].verb == TK_EL_MOVE);
        if (!__all_sync(0xffffffffu, ok)) {
            if (lane == 0) {
                atomicOr(error, ERR_LINE_PATH_MISMATCH);
                poly_n[i] = 0u;
            }
            continue;
        }
        uint32_t a, b;
        raw_range(P, offsets, n_els, *total, a, b);
        Pt* v = pts + a;
        const uint32_t raw = b - a;
        if (raw == 0u) {
            if (lane == 0) poly_n[i] = 0u;
            continue;
        }
        uint32_t n = 1u;
        Pt back = v[0];
        for (uint32_t i0 = 1; i0 < raw; i0 += 32u) {
            const uint32_t k = i0 + lane;
            const bool in = k < raw;
            const Pt p = in ? v[k] : back;
            Pt prev{__shfl_up_sync(0xffffffffu, p.x, 1), __shfl_up_sync(0xffffffffu, p.y, 1)};
            if (lane == 0) prev = back;
            const unsigned keep_all = __ballot_sync(0xffffffffu, !in || tkf::distinct(p, prev));
            __syncwarp();
            if (keep_all == 0xffffffffu) {  // every point of the group is kept
                if (in) v[n + lane] = p;
                const uint32_t m = min(32u, raw - i0);
                back = Pt{__shfl_sync(0xffffffffu, p.x, m - 1u), __shfl_sync(0xffffffffu, p.y, m - 1u)};
                n += m;
            } else {  // a repeat: the sequential rule, on one lane
                if (lane == 0) {
                    const uint32_t end = min(raw, i0 + 32u);
                    for (uint32_t q = i0; q < end; ++q) {
                        const Pt r = v[q];
                        if (tkf::distinct(r, back)) {
                            v[n++] = r;
                            back = r;
                        }
                    }
                }
                n = __shfl_sync(0xffffffffu, n, 0);
                back = Pt{__shfl_sync(0xffffffffu, back.x, 0), __shfl_sync(0xffffffffu, back.y, 0)};
            }
            __syncwarp();
        }
        if (P.closed != 0u && n > 1u && !tkf::distinct(v[0], back)) --n;
        if (lane == 0) poly_n[i] = n;
    }
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
                                                                  uint32_t* poly_lines, uint32_t* unit_lines_out,
                                                                  unsigned long long* total64, uint32_t* error) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t pl = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); pl < npl; pl += warps) {
        const PolyView q = poly_view(pl, polys, strokes, offsets, pts, poly_n);
        uint32_t* slots = unit_lines_out + 2ull * offsets[polys[pl].element0];
        unsigned long long cnt = 0;
        for (uint32_t loop = 0; loop < q.loops; ++loop)
            for (uint32_t u = lane; u < q.units; u += 32u) {
                const uint32_t c = unit_lines(q, loop, u);
                slots[loop * q.units + u] = c;
                cnt += c;
            }
#pragma unroll
        for (int d = 16; d; d >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, d);
        if (lane == 0) {
            if (cnt > 0xFFFFFFFFull) atomicOr(error, ERR_SEGMENT_OVERFLOW);
            poly_lines[pl] = uint32_t(cnt);
            if (cnt) atomicAdd(total64, cnt);
        }
    }
}

// Lines into a warp's shared-memory stage (positions relative to the group's
// first line).
struct StageLines {
    tk_line* out;
    uint32_t at, end;  // this unit's slots: [at, end)
    uint32_t path;
    __device__ void operator()(Pt a, Pt b) {
        if (at < end) out[at] = tk_line{path, 0.0f, {float(a.x), float(a.y)}, {float(b.x), float(b.y)}};
        ++at;
    }
};

constexpr uint32_t kStageLines = 256;  // per warp: 6 KB

__global__ void __launch_bounds__(kStrokeThreads) k_outline_emit(const tk_stroke_polyline* __restrict__ polys,
                                                                 uint32_t npl, const tk_stroke_desc* __restrict__ strokes,
                                                                 const uint32_t* __restrict__ offsets,
                                                                 const Pt* __restrict__ pts,
                                                                 const uint32_t* __restrict__ poly_n,
                                                                 const uint32_t* __restrict__ line_off,
                                                                 const uint32_t* __restrict__ unit_lines_in,
                                                                 tk_line* lines, uint64_t line_base, uint64_t line_end,
                                                                 uint32_t* error) {
    __shared__ __align__(16) tk_line s_stage[kStrokeThreads / 32][kStageLines];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    tk_line* stage = s_stage[warp];
    for (uint32_t pl = blockIdx.x * (blockDim.x >> 5) + warp; pl < npl; pl += warps) {
        const PolyView q = poly_view(pl, polys, strokes, offsets, pts, poly_n);
        const uint32_t* slots = unit_lines_in + 2ull * offsets[polys[pl].element0];
        uint64_t at = line_base + line_off[pl];
        for (uint32_t loop = 0; loop < q.loops; ++loop) {
            for (uint32_t u0 = 0; u0 < q.units; u0 += 32u) {
                const uint32_t u = u0 + lane;
                const uint32_t c = u < q.units ? slots[loop * q.units + u] : 0u;
                uint32_t incl = c;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
                    if (lane >= uint32_t(d)) incl += y;
                }
                const uint32_t group = __shfl_sync(0xffffffffu, incl, 31);
                if (group <= kStageLines && at + group <= line_end) {
                    // staged: the group's lines are one contiguous run
                    if (c) {
                        StageLines w{stage, incl - c, incl, q.path};
                        tkf::EdgeChain<StageLines> ch{q.xf, w};
                        tkf::outline_unit(q.v, q.n, q.closed, loop, u, q.h, q.tol, ch);
                    }
                    __syncwarp();
                    // 8-byte words of the run, lane-strided (tk_line is 24 bytes, 8-aligned)
                    const uint2* src = reinterpret_cast<const uint2*>(stage);
                    uint2* dst = reinterpret_cast<uint2*>(lines + at);
                    for (uint32_t k = lane; k < group * 3u; k += 32u) dst[k] = src[k];
                    __syncwarp();
                } else if (u < q.units && c) {
                    WriteLines w{lines, at + incl - c, line_end, q.path, error};
                    tkf::EdgeChain<WriteLines> ch{q.xf, w};
                    tkf::outline_unit(q.v, q.n, q.closed, loop, u, q.h, q.tol, ch);
                }
                at += group;
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
    if (n) k_stroke_count<<<grid_for(n, kStrokeThreads), kStrokeThreads, 0, st>>>(els, n, counts, total64, error);
    launch_exclusive_scan(counts, n, block_sums, total, st);
}

void launch_stroke_outline_count(const StrokeView& v, uint32_t* block_sums, uint32_t* line_total,
                                 unsigned long long* line_total64, cudaStream_t st) {
    if (v.n_els)
        k_stroke_points<<<grid_for(v.n_els * 32, kStrokeThreads), kStrokeThreads, 0, st>>>(v.els, v.n_els, v.offsets,
                                                                                          v.pts, v.pt_cap, v.error);
    if (v.npl) {
        k_stroke_polylines<<<grid_for(uint64_t(v.npl) * 32, kStrokeThreads), kStrokeThreads, 0, st>>>(
            v.polys, v.npl, v.els, v.n_els, v.offsets, v.pt_total, v.pts, v.poly_n, v.error);
        k_outline_count<<<grid_for(uint64_t(v.npl) * 32, kStrokeThreads), kStrokeThreads, 0, st>>>(
            v.polys, v.npl, v.strokes, v.offsets, v.pts, v.poly_n, v.line_off, v.unit_lines, line_total64, v.error);
    }
    launch_exclusive_scan(v.line_off, v.npl, block_sums, line_total, st);
}

void launch_stroke_emit(const StrokeView& v, const uint32_t* line_total, tk_path_record* paths, tk_line* lines,
                        uint64_t line_base, uint64_t line_end, cudaStream_t st) {
    if (v.npl)
        k_outline_emit<<<grid_for(uint64_t(v.npl) * 32, kStrokeThreads), kStrokeThreads, 0, st>>>(
            v.polys, v.npl, v.strokes, v.offsets, v.pts, v.poly_n, v.line_off, v.unit_lines, lines, line_base,
            line_end, v.error);
    if (v.n_strokes)
        k_stroke_paths<<<(v.n_strokes + 127) / 128, 128, 0, st>>>(v.strokes, v.n_strokes, v.npl, v.line_off,
                                                                   line_total, paths, uint32_t(line_base));
}

}  // namespace tk
