// Device flattening (the Canvas::push_path flattening step,
// src/shared/path_flatten.rs:20-82, moved onto the GPU): Bezier elements to
// lines with the count / scan / emit pattern. One warp emits one element
// (a line, quadratic or cubic with its start point) 32 points at a time
// (warp_flatten.cuh); the host has already resolved move_to / close into
// explicit elements, so elements are independent. The arithmetic is
// flatten_core.h, shared with the host, so the lines are bit-identical to the
// host Canvas's. An element's lines are its kept edges (tkf::keep_edge from
// each point's predecessor), ranked within each round by ballot, so a round
// stores consecutive lines from consecutive lanes. The count pass, which
// stores nothing, runs one element per thread.
#include <cuda_runtime.h>

#include "flatten_core.h"
#include "kernels.h"
#include "warp_flatten.cuh"

namespace tk {
namespace {

using tkf::Pt;

constexpr uint32_t kFlattenThreads = 128;

// The previous point of each lane's point: the lane before it, or for lane 0
// the last point of the previous round.
__device__ inline Pt prev_point(const Pt& p, const Pt& last, uint32_t lane) {
    Pt q{__shfl_up_sync(0xffffffffu, p.x, 1), __shfl_up_sync(0xffffffffu, p.y, 1)};
    return lane == 0u ? last : q;
}

// The count pass walks each element on one thread (tkf::element_points):
// counting needs no stores, and a thread per element keeps more elements in
// flight than a warp per element.
struct CountEmit {
    Pt prev;
    uint32_t n;
    __device__ void operator()(Pt p) {
        if (tkf::keep_edge(prev, p)) ++n;
        prev = p;
    }
};

struct WarpWriteEdges {
    Pt last;
    tk_line* out;
    uint64_t at, end;
    uint32_t path, lane;
    uint32_t* error;
    __device__ void operator()(bool valid, Pt p, uint32_t k) {
        const Pt prev = prev_point(p, last, lane);
        const bool keep = valid && tkf::keep_edge(prev, p);
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const uint64_t q = at + __popc(mask & ((1u << lane) - 1u));
            if (q < end) out[q] = tk_line{path, 0.0f, {float(prev.x), float(prev.y)}, {float(p.x), float(p.y)}};
            else atomicOr(error, ERR_SEGMENT_OVERFLOW);
        }
        at += __popc(mask);
        last = shfl_pt(p, k - 1u);
    }
};

// Elements the flattener accepts: a known verb, tolerance >= 1e-3 px and
// finite coordinates within 1e6 px. These bounds bound one thread's work
// (about 1e6 points for the worst element); anything else is flagged and
// produces no lines.
__device__ bool element_ok(const tk_flatten_el& e) {
    if (e.verb < TK_EL_LINE || e.verb > TK_EL_CUBIC) return false;
    if (!(e.tolerance >= 1e-3) || !isfinite(e.tolerance)) return false;
    for (uint32_t k = 0; k <= e.verb; ++k)
        if (!(fabs(e.p[k][0]) <= 1e6) || !(fabs(e.p[k][1]) <= 1e6)) return false;
    return true;
}

__global__ void __launch_bounds__(kFlattenThreads)
    k_flatten_count(const tk_flatten_el* __restrict__ els, uint64_t n, uint32_t* counts, uint32_t* error) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const tk_flatten_el e = els[i];
        CountEmit c{Pt{e.p[0][0], e.p[0][1]}, 0u};
        if (element_ok(e)) tkf::element_points(e, c);
        else atomicOr(error, ERR_UNSUPPORTED);
        counts[i] = c.n;
    }
}

constexpr int kScanBlock = 1024;

// Exclusive scan of `v` (n values) in place, 1024 per block; block totals go
// to `sums`.
__global__ void __launch_bounds__(kScanBlock) k_scan_local(uint32_t* v, uint64_t n, uint32_t* sums) {
    __shared__ uint32_t s_w[32];
    const uint64_t i = blockIdx.x * uint64_t(kScanBlock) + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t x = i < n ? v[i] : 0u;
    uint32_t incl = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= uint32_t(d)) incl += y;
    }
    if (lane == 31u) s_w[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = s_w[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= uint32_t(d)) w += y;
        }
        s_w[lane] = w;
    }
    __syncthreads();
    if (i < n) v[i] = (warp ? s_w[warp - 1] : 0u) + incl - x;
    if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = s_w[31];
}

// Block offsets: exclusive scan of the block totals by one block, looping.
__global__ void __launch_bounds__(kScanBlock) k_scan_sums(uint32_t* sums, uint32_t blocks, uint32_t* total) {
    __shared__ uint32_t s_w[32];
    __shared__ uint32_t s_run;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_run = 0u;
    __syncthreads();
    for (uint32_t b0 = 0; b0 < blocks; b0 += kScanBlock) {
        const uint32_t b = b0 + threadIdx.x;
        const uint32_t x = b < blocks ? sums[b] : 0u;
        uint32_t incl = x;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= uint32_t(d)) incl += y;
        }
        if (lane == 31u) s_w[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = s_w[lane];
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
                if (lane >= uint32_t(d)) w += y;
            }
            s_w[lane] = w;
        }
        __syncthreads();
        const uint32_t run = s_run;
        if (b < blocks) sums[b] = run + (warp ? s_w[warp - 1] : 0u) + incl - x;
        __syncthreads();
        if (threadIdx.x == 0) s_run = run + s_w[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = s_run;
}

__global__ void k_scan_add(uint32_t* v, uint64_t n, const uint32_t* sums) {
    const uint64_t i = blockIdx.x * uint64_t(kScanBlock) + threadIdx.x;
    if (i < n) v[i] += sums[blockIdx.x];
}

// Line ranges of the device-flattened paths: lines [line_base + offset of the
// first element, + the elements' lines).
__global__ void k_flatten_paths(tk_path_record* paths, uint32_t path_count, const uint32_t* __restrict__ path_els,
                                const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ total,
                                uint64_t n_els, uint32_t line_base, const tk_flatten_el* __restrict__ els,
                                uint32_t* error) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= path_count) return;
    const uint32_t e0 = path_els[2 * p], ne = path_els[2 * p + 1];
    if (ne == 0u) return;
    for (uint32_t e = e0; e < e0 + ne; ++e)  // the path's elements carry its index
        if (els[e].path != p) atomicOr(error, ERR_LINE_PATH_MISMATCH);
    const uint32_t a = offsets[e0];
    const uint32_t b = uint64_t(e0) + ne < n_els ? offsets[e0 + ne] : *total;
    paths[p].line_start = line_base + a;
    paths[p].line_count = b - a;
}

__global__ void __launch_bounds__(kFlattenThreads)
    k_flatten_emit(const tk_flatten_el* __restrict__ els, uint64_t n, const uint32_t* __restrict__ offsets,
                   tk_line* lines, uint64_t line_base, uint64_t line_end, uint32_t* error) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
        const tk_flatten_el e = els[i];
        WarpWriteEdges w{Pt{e.p[0][0], e.p[0][1]}, lines, line_base + offsets[i], line_end, e.path, lane, error};
        if (element_ok(e)) warp_element_points(e, lane, w);
    }
}

}  // namespace

void launch_exclusive_scan(uint32_t* v, uint64_t n, uint32_t* block_sums, uint32_t* total, cudaStream_t st) {
    if (n == 0) {
        cudaMemsetAsync(total, 0, sizeof(uint32_t), st);
        return;
    }
    const uint32_t blocks = uint32_t((n + kScanBlock - 1) / kScanBlock);
    k_scan_local<<<blocks, kScanBlock, 0, st>>>(v, n, block_sums);
    k_scan_sums<<<1, kScanBlock, 0, st>>>(block_sums, blocks, total);
    k_scan_add<<<blocks, kScanBlock, 0, st>>>(v, n, block_sums);
}

void launch_flatten_count(const tk_flatten_el* els, uint64_t n, uint32_t* counts, uint32_t* block_sums,
                          uint32_t* total, uint32_t* error, cudaStream_t st) {
    if (n) k_flatten_count<<<148 * 16, kFlattenThreads, 0, st>>>(els, n, counts, error);
    launch_exclusive_scan(counts, n, block_sums, total, st);
}

void launch_flatten_emit(const tk_flatten_el* els, uint64_t n, const uint32_t* offsets, const uint32_t* total,
                         tk_path_record* paths, uint32_t path_count, const uint32_t* path_els, tk_line* lines,
                         uint64_t line_base, uint64_t line_end, uint32_t* error, cudaStream_t st) {
    if (path_count) k_flatten_paths<<<(path_count + 255) / 256, 256, 0, st>>>(paths, path_count, path_els, offsets,
                                                                             total, n, uint32_t(line_base), els, error);
    if (n) k_flatten_emit<<<148 * 16, kFlattenThreads, 0, st>>>(els, n, offsets, lines, line_base, line_end, error);
}

size_t flatten_block_sums(uint64_t n) { return size_t((n + kScanBlock - 1) / kScanBlock) + 1; }

}  // namespace tk
