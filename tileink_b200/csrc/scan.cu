// Scan stage: tile segment counts, pool prefix + backdrop cumsum, emit.
//
// scan_count  (scan/count.hlsl:13-40): one thread per line, atomics into the
//             path's backdrop slice. Counts and backdrop deltas are sums, so
//             their order does not matter.
// pool scan   (scan/prefix_chunks.hlsl, chunk_offsets.hlsl,
//             apply_chunk_offsets.hlsl, cumsum.hlsl): work items of whole bbox
//             rows. Pass 1 sums each item's counts (one CTA per item), pass 2
//             scans the item sums in one CTA (chained per path, or over the
//             whole pool when segment starts are planned on the device), pass 3
//             writes each item's ranges and cursors from its prefix and does
//             the row-wise backdrop cumsum as a segmented scan in the same
//             CTA. No CTA waits on another.
// scan_emit   (scan/emit.hlsl:14-28, scan/clip.hlsli:10-75): one warp per
//             path; lanes take 32 consecutive lines, DDA step r is the outer
//             loop and lanes rank their slots with __match_any_sync, giving a
//             fixed segment order inside every tile.
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.h"

namespace tk {
namespace {

using namespace tkd;

__device__ __forceinline__ tk_line load_line(const tk_line* lines, uint64_t i) {
    const uint2* w = reinterpret_cast<const uint2*>(lines + i);
    uint2 a = __ldg(w), b = __ldg(w + 1), c = __ldg(w + 2);
    tk_line l;
    l.path_id = a.x;
    l.pad = __uint_as_float(a.y);
    l.p0[0] = __uint_as_float(b.x);
    l.p0[1] = __uint_as_float(b.y);
    l.p1[0] = __uint_as_float(c.x);
    l.p1[1] = __uint_as_float(c.y);
    return l;
}
__device__ __forceinline__ tk_path_record load_path(const tk_path_record* paths, uint32_t i) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(paths + i);
    tk_path_record p;
    uint32_t* o = reinterpret_cast<uint32_t*>(&p);
#pragma unroll
    for (int k = 0; k < 19; ++k) o[k] = w[k];
    return p;
}

// scan/count.hlsl:13-40 for one line: backdrop deltas and tile counts.
__device__ __forceinline__ void count_line(const tk_line& line, const tk_path_record* __restrict__ paths,
                                           int32_t* backdrops, uint32_t* counts) {
    tk_path_record p = load_path(paths, line.path_id);
    Scan s;
    if (!scan_geometry(line, p, s)) return;
    int32_t delta = s.down ? -1 : 1;
    int32_t stride = int32_t(s.bx1 - s.bx0);
    for (int32_t y = s.ymin; y < s.ymax; ++y) {
        uint32_t local = uint32_t((y - int32_t(s.by0)) * stride);
        atomicAdd(backdrops + s.data_offset + local, delta);
    }
    float last_z = floorf(s.a * (float(s.imin) - 1.0f) + s.b);
    for (uint32_t i = s.imin; i < s.imax; ++i) {
        float z = floorf(s.a * float(i) + s.b);
        int32_t tx, ty;
        scan_tile(s, i, z, tx, ty);
        if (scan_tile_inside(s, tx, ty)) {
            bool top = last_z == z;
            if (i == 0u) top = fabsf(s.y0 - s.qy0 * (1.0f / float(TK_TILE_SIZE))) <= SCAN_EPSILON;
            if (top && tx + 1 < int32_t(s.bx1)) {
                int32_t x = max(tx + 1, int32_t(s.bx0));
                uint32_t local = uint32_t((ty - int32_t(s.by0)) * stride + x - int32_t(s.bx0));
                atomicAdd(backdrops + s.data_offset + local, delta);
            }
            atomicAdd(counts + scan_tile_offset(s, tx, ty), 1u);
        }
        last_z = z;
    }
}

__global__ void k_scan_count(const tk_line* __restrict__ lines, uint64_t line_count,
                             const tk_path_record* __restrict__ paths, uint32_t path_count, int32_t* backdrops,
                             uint32_t* counts) {
    for (uint64_t li = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; li < line_count;
         li += uint64_t(gridDim.x) * blockDim.x) {
        tk_line line = load_line(lines, li);
        if (line.path_id >= path_count) continue;
        count_line(line, paths, backdrops, counts);
    }
}

// The selected paths only (a partial rescan): one CTA per listed path clears
// its backdrop and count slices, then counts its lines.
__global__ void k_scan_count_paths(const tk_line* __restrict__ lines, const tk_path_record* __restrict__ paths,
                                   uint32_t path_count, const uint32_t* __restrict__ list, int32_t* backdrops,
                                   uint32_t* counts) {
    const uint32_t pid = list[blockIdx.x];
    const tk_path_record p = load_path(paths, pid);
    for (uint32_t k = threadIdx.x; k < p.data_len; k += blockDim.x) {
        backdrops[p.data_offset + k] = 0;
        counts[p.data_offset + k] = 0u;
    }
    __syncthreads();
    for (uint32_t l = threadIdx.x; l < p.line_count; l += blockDim.x) {
        tk_line line = load_line(lines, uint64_t(p.line_start) + l);
        if (line.path_id != pid || pid >= path_count) continue;  // the emit pass reports mismatches
        count_line(line, paths, backdrops, counts);
    }
}

// ---------------------------------------------------------------------------
// Pool scan.
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanPerThread = kScanItemElems / kScanThreads;  // 16

// Inclusive warp scan of (flag, value) pairs under the segmented operator
// (f1, v1) + (f2, v2) = (f1 | f2, f2 ? v2 : v1 + v2).
__device__ __forceinline__ void warp_seg_scan(uint32_t& f, uint32_t& v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t pf = __shfl_up_sync(0xffffffffu, f, o), pv = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) {
            v = f ? v : pv + v;
            f |= pf;
        }
    }
}

// Block-wide exclusive segmented scan of per-thread aggregates.
__device__ __forceinline__ void block_seg_exclusive(uint32_t f, uint32_t v, uint32_t& ef, uint32_t& ev,
                                                    uint32_t* sf, uint32_t* sv, uint32_t& tot) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl_f = f, incl_v = v;
    warp_seg_scan(incl_f, incl_v);
    if (lane == 31) { sf[warp] = incl_f; sv[warp] = incl_v; }
    __syncthreads();
    if (warp == 0) {
        uint32_t wf = lane < kScanThreads / 32 ? sf[lane] : 0u, wv = lane < kScanThreads / 32 ? sv[lane] : 0u;
        warp_seg_scan(wf, wv);
        if (lane < kScanThreads / 32) { sf[lane + 8] = wf; sv[lane + 8] = wv; }  // inclusive warp prefixes
    }
    __syncthreads();
    // exclusive within warp
    uint32_t xf = __shfl_up_sync(0xffffffffu, incl_f, 1), xv = __shfl_up_sync(0xffffffffu, incl_v, 1);
    if (lane == 0) { xf = 0u; xv = 0u; }
    // combine with the previous warps' inclusive prefix
    uint32_t pf = warp ? sf[8 + warp - 1] : 0u, pv = warp ? sv[8 + warp - 1] : 0u;
    ef = pf | xf;
    ev = xf ? xv : pv + xv;
    tot = sv[8 + kScanThreads / 32 - 1];
}

// Element range of work item k: [e0, e0 + n) of the pool, rows of `stride`.
struct ItemSpan {
    uint64_t e0;
    uint32_t n, stride;
};
__device__ __forceinline__ ItemSpan item_span(const ScanItem& it, const tk_path_record* paths) {
    const tk_path_record& p = paths[it.path];
    const uint32_t stride = p.tile_x1 - p.tile_x0;
    return {uint64_t(p.data_offset) + uint64_t(it.row0) * stride, it.rows * stride, stride};
}

// Pass 1: the segment count of every work item (its sum of tile counts).
__global__ void __launch_bounds__(kScanThreads)
    k_item_sums(const ScanItem* __restrict__ items, const tk_path_record* __restrict__ paths,
                const uint32_t* __restrict__ counts, uint32_t* item_words) {
    __shared__ uint32_t s_w[kScanThreads / 32];
    const uint32_t k = blockIdx.x, tid = threadIdx.x;
    const ItemSpan sp = item_span(items[k], paths);
    uint32_t v[kScanPerThread];
#pragma unroll
    for (int j = 0; j < kScanPerThread; ++j) {
        const uint32_t i = tid + uint32_t(j) * kScanThreads;
        v[j] = i < sp.n ? counts[sp.e0 + i] : 0u;
    }
    uint32_t sum = 0u;
#pragma unroll
    for (int j = 0; j < kScanPerThread; ++j) sum += v[j];
    sum = __reduce_add_sync(0xffffffffu, sum);
    if ((tid & 31u) == 0u) s_w[tid >> 5] = sum;
    __syncthreads();
    if (tid == 0) {
        uint32_t t = 0u;
        for (int w = 0; w < kScanThreads / 32; ++w) t += s_w[w];
        item_words[2u * k] = t;
    }
}

// Pass 2 (one CTA): item prefixes, a segmented exclusive scan of the item
// sums in item order (u32, wrapping). A chain starts at item 0 with
// device_base when the segment slices are planned on the device, else at
// every path's first item with the path's segment_start. `total` receives the
// last item's prefix + sum.
constexpr uint32_t kPrefixThreads = 1024;
__global__ void __launch_bounds__(kPrefixThreads)
    k_item_prefix(const ScanItem* __restrict__ items, uint32_t n_items, const tk_path_record* __restrict__ paths,
                  uint32_t* item_words, int device_plan, uint32_t device_base, uint32_t* total) {
    __shared__ uint32_t s_f[kPrefixThreads / 32], s_v[kPrefixThreads / 32];
    __shared__ uint32_t s_carry;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    if (tid == 0) s_carry = 0u;
    __syncthreads();
    for (uint32_t k0 = 0; k0 < n_items; k0 += kPrefixThreads) {
        const uint32_t k = k0 + tid;
        uint32_t f = 0u, v = 0u, agg = 0u;
        if (k < n_items) {
            const ScanItem it = items[k];
            agg = item_words[2u * k];
            const bool head = device_plan ? k == 0u : it.first != 0u;
            f = head ? 1u : 0u;
            v = head ? (device_plan ? device_base : paths[it.path].segment_start) + agg : agg;
        }
        // inclusive segmented scan: warps, then the warp totals
        warp_seg_scan(f, v);
        if (lane == 31u) {
            s_f[warp] = f;
            s_v[warp] = v;
        }
        __syncthreads();
        if (warp == 0) {
            uint32_t wf = s_f[lane], wv = s_v[lane];
            warp_seg_scan(wf, wv);
            s_f[lane] = wf;
            s_v[lane] = wv;
        }
        __syncthreads();
        if (warp > 0 && !f) v += s_v[warp - 1];
        const uint32_t fw = f | (warp > 0 ? s_f[warp - 1] : 0u);
        if (!fw) v += s_carry;  // no chain head at or before k within this block
        if (k < n_items) {
            item_words[2u * k + 1u] = v - agg;  // exclusive prefix
            if (k + 1u == n_items) *total = v;
        }
        __syncthreads();
        if (tid == kPrefixThreads - 1u) s_carry = v;
        __syncthreads();
    }
}

__device__ __forceinline__ uint32_t pad16(uint32_t i) { return i + (i >> 4); }

// Pass 3: per work item the exclusive prefix of the tile counts (segment
// ranges and cursors, starting at the item's prefix) and the row-wise backdrop
// cumsum.
__global__ void __launch_bounds__(kScanThreads)
    k_pool_scan(const ScanItem* __restrict__ items, tk_path_record* paths, uint32_t* counts, int32_t* backdrops,
                tk_segment_range* ranges, uint32_t* cursors, const uint32_t* __restrict__ item_words) {
    // element i lives at pad(i) = i + i / 16, so that thread t's run of 16
    // elements starts at 17 t and a warp's sequential walk meets 32 banks
    __shared__ uint32_t s_cnt[kScanItemElems + kScanItemElems / 16];
    __shared__ int32_t s_bd[kScanItemElems + kScanItemElems / 16];
    __shared__ uint32_t s_f[24], s_v[24];
    const int tid = threadIdx.x;
    const uint32_t k = blockIdx.x;
    const ScanItem it = items[k];
    const tk_path_record& p = paths[it.path];
    const uint32_t stride = p.tile_x1 - p.tile_x0;
    const uint32_t n = it.rows * stride;
    const uint64_t e0 = uint64_t(p.data_offset) + uint64_t(it.row0) * stride;
    // coalesced loads, eight of a thread's in flight before the first is used
#pragma unroll
    for (int j0 = 0; j0 < kScanPerThread; j0 += 8) {
        uint32_t vc[8];
        int32_t vb[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t i = tid + uint32_t(j0 + j) * kScanThreads;
            vc[j] = i < n ? counts[e0 + i] : 0u;
            vb[j] = i < n ? backdrops[e0 + i] : 0;
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint32_t i = tid + uint32_t(j0 + j) * kScanThreads;
            if (i < n) {
                s_cnt[pad16(i)] = vc[j];
                s_bd[pad16(i)] = vb[j];
            }
        }
    }
    __syncthreads();
    // thread-local sums over elements [tid*16, tid*16+16); rows start at
    // multiples of stride, the first at or after lo found with one division
    // (n == 0 when stride == 0, and then no element is visited)
    const uint32_t lo = tid * kScanPerThread;
    const uint32_t row_start0 = stride ? (lo + stride - 1u) / stride * stride : 0u;
    uint32_t csum = 0u, bf = 0u, bsum = 0u;
    uint32_t row_start = row_start0;
#pragma unroll
    for (int j = 0; j < kScanPerThread; ++j) {
        uint32_t i = lo + j;
        if (i < n) {
            csum += s_cnt[pad16(i)];
            if (i == row_start) {
                bf = 1u;
                bsum = 0u;
                row_start += stride;
            }
            bsum += uint32_t(s_bd[pad16(i)]);
        }
    }
    // counts: plain exclusive scan (flags 0)
    uint32_t ef, ecount, agg;
    block_seg_exclusive(0u, csum, ef, ecount, s_f, s_v, agg);
    __syncthreads();
    uint32_t bef, bexcl, btot;
    block_seg_exclusive(bf, bsum, bef, bexcl, s_f, s_v, btot);
    (void)btot;
    (void)ef;
    const uint32_t prefix = item_words[2u * k + 1u];
    uint32_t run = prefix + ecount;
    uint32_t brun = bexcl;
    row_start = row_start0;
#pragma unroll
    for (int j = 0; j < kScanPerThread; ++j) {
        uint32_t i = lo + j;
        if (i < n) {
            uint32_t c = s_cnt[pad16(i)];
            s_cnt[pad16(i)] = run;  // exclusive start
            run += c;
            if (i == row_start) {
                brun = 0u;
                row_start += stride;
            }
            brun += uint32_t(s_bd[pad16(i)]);
            s_bd[pad16(i)] = int32_t(brun);
        }
    }
    __syncthreads();
    for (uint32_t i = tid; i < n; i += kScanThreads) {
        uint32_t start = s_cnt[pad16(i)];
        uint32_t end = (i + 1 < n) ? s_cnt[pad16(i + 1)] : prefix + agg;
        ranges[e0 + i] = tk_segment_range{start, end};
        cursors[e0 + i] = start;
        backdrops[e0 + i] = s_bd[pad16(i)];
    }
}

__global__ void k_path_totals(tk_path_record* paths, uint32_t path_count, const tk_segment_range* ranges,
                              uint64_t pool_end, uint32_t* bumps, int device_plan, const uint32_t* total) {
    uint32_t pid = blockIdx.x * blockDim.x + threadIdx.x;
    if (pid >= path_count) return;
    tk_path_record& p = paths[pid];
    uint32_t start, count;
    if (p.data_len > 0u) {
        start = ranges[p.data_offset].start;
        count = ranges[p.data_offset + p.data_len - 1u].end - start;
    } else {
        start = uint64_t(p.data_offset) < pool_end ? ranges[p.data_offset].start : *total;
        count = 0u;
    }
    bumps[pid] = count;
    if (device_plan) {
        p.segment_start = start;
        p.segment_capacity = count;
    }
}

// scan_emit (scan/emit.hlsl:14-28) in canonical order: a path's lines in
// order, each line's DDA steps in order, every emitting step taking the next
// cursor of its tile. Warps take paths from a queue, longest first (the line
// counts are heavy-tailed and a path is one warp's sequential work). Per group
// of 32 lines the warp computes each line's scan geometry, then walks the
// group's (line, step) pairs 32 at a time, so that lanes do not idle on the
// group's longest line; pairs that fall in the same tile in one round are
// ranked by lane, which keeps the canonical order.
constexpr int kEmitThreads = 256;

__global__ void __launch_bounds__(kEmitThreads, 4)
    k_scan_emit(const tk_line* __restrict__ lines, const tk_path_record* __restrict__ paths, uint32_t path_count,
                uint32_t* cursors, SegmentRec* segments, uint64_t capacity, uint32_t* error, uint32_t* seg_line,
                const uint32_t* __restrict__ order, uint32_t* ticket) {
    __shared__ Scan s_scan[kEmitThreads / 32][32];
    __shared__ uint32_t s_first[kEmitThreads / 32][33];  // exclusive prefix of the lines' step counts
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t lt_mask = (1u << lane) - 1u;
    Scan* sc = s_scan[warp];
    uint32_t* first = s_first[warp];
    for (;;) {
        uint32_t k = 0;
        if (lane == 0) k = atomicAdd(ticket, 1u);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= path_count) break;
        const uint32_t pid = order ? __ldg(order + k) : k;
        const tk_path_record p = load_path(paths, pid);
        for (uint32_t g = 0; g < p.line_count; g += 32u) {
            const uint32_t l = g + lane;
            Scan s;
            bool ok = false;
            if (l < p.line_count) {
                tk_line line = load_line(lines, uint64_t(p.line_start) + l);
                if (line.path_id != pid) atomicOr(error, ERR_LINE_PATH_MISMATCH);
                else ok = scan_geometry(line, p, s);
            }
            const uint32_t n = ok ? s.imax - s.imin : 0u;
            uint32_t incl = n;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= uint32_t(o)) incl += v;
            }
            const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
            __syncwarp();  // the previous group's readers are done with sc / first
            if (n) sc[lane] = s;
            first[lane] = incl - n;
            if (lane == 31) first[32] = total;
            __syncwarp();
            for (uint32_t base = 0; base < total; base += 32u) {
                const uint32_t j = base + lane;
                bool emitting = false;
                uint32_t off = 0xFFFFFFFFu, i = 0, L = 0;
                float z = 0.0f;
                int32_t tx = 0, ty = 0;
                if (j < total) {
                    // the line whose steps hold pair j: the last lane with first <= j
                    uint32_t lo = 0, hi = 32;
                    while (hi - lo > 1u) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (first[mid] <= j) lo = mid;
                        else hi = mid;
                    }
                    L = lo;
                    const Scan& sl = sc[L];
                    i = sl.imin + (j - first[L]);
                    z = floorf(sl.a * float(i) + sl.b);
                    scan_tile(sl, i, z, tx, ty);
                    if (scan_tile_inside(sl, tx, ty)) {
                        emitting = true;
                        off = scan_tile_offset(sl, tx, ty);
                    }
                }
                // A path's cursors are read and written by its warp alone;
                // __syncwarp orders the lanes' accesses, so they can be plain
                // (L1-cached) loads and stores. The cursor load is issued
                // first and the clipped segment computed while it is in flight.
                const uint32_t group = __match_any_sync(0xffffffffu, off);
                uint32_t cbase = 0;
                if (emitting) cbase = cursors[off];
                tk_line_segment seg{};
                float slope = 0.0f;
                if (emitting) {
                    seg = clipped_segment(sc[L], i, z, tx, ty);
                    const float delta_y = seg.p1y - seg.p0y;
                    slope = delta_y != 0.0f ? (seg.p1x - seg.p0x) / delta_y : 0.0f;
                }
                __syncwarp();
                if (emitting) {
                    const uint32_t leader = __ffs(group) - 1u;
                    if (lane == leader) cursors[off] = cbase + __popc(group);
                    const uint32_t slot = cbase + __popc(group & lt_mask);
                    if (slot < capacity) {
                        float4* dst = reinterpret_cast<float4*>(segments + slot);
                        dst[0] = make_float4(seg.p0x, seg.p0y, seg.p1x, seg.p1y);
                        dst[1] = make_float4(seg.y_edge, slope, 0.0f, 0.0f);
                        if (seg_line) seg_line[slot] = p.line_start + g + L;
                    } else {
                        atomicOr(error, ERR_SEGMENT_OVERFLOW);
                    }
                }
                __syncwarp();
            }
        }
    }
}

// The listed paths' counted segment totals (bumps) against the segment
// slices they were planned (segment_capacity): any difference sets *changed.
__global__ void k_check_path_totals(const tk_path_record* __restrict__ paths, const uint32_t* __restrict__ bumps,
                                    const uint32_t* __restrict__ list, uint32_t n, uint32_t* changed) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t p = __ldg(list + k);
    if (__ldg(bumps + p) != paths[p].segment_capacity) atomicOr(changed, 1u);
}

inline unsigned grid_for(uint64_t n, unsigned block, unsigned cap) {
    uint64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return unsigned(g);
}

}  // namespace

void launch_scan_count(const SceneView& s, cudaStream_t st) {
    if (s.line_count == 0) return;
    k_scan_count<<<grid_for(s.line_count, 256, 148 * 64), 256, 0, st>>>(s.lines, s.line_count, s.paths, s.path_count,
                                                                       s.backdrops, s.counts);
}

void launch_pool_scan(const SceneView& s, const ScanItem* items, uint32_t n_items, unsigned long long* item_scratch,
                      bool device_plan, uint32_t device_base, uint32_t* total, cudaStream_t st) {
    cudaMemsetAsync(total, 0, sizeof(uint32_t), st);
    if (n_items == 0) return;
    uint32_t* words = reinterpret_cast<uint32_t*>(item_scratch);  // per item: sum, prefix
    k_item_sums<<<n_items, kScanThreads, 0, st>>>(items, s.paths, s.counts, words);
    k_item_prefix<<<1, kPrefixThreads, 0, st>>>(items, n_items, s.paths, words, device_plan ? 1 : 0, device_base, total);
    k_pool_scan<<<n_items, kScanThreads, 0, st>>>(items, s.paths, s.counts, s.backdrops, s.ranges, s.cursors, words);
}

void launch_path_totals(const SceneView& s, uint32_t* bumps, bool device_plan, const uint32_t* total,
                        cudaStream_t st) {
    if (s.path_count == 0) return;
    k_path_totals<<<(s.path_count + 255) / 256, 256, 0, st>>>(s.paths, s.path_count, s.ranges, s.pool_len, bumps,
                                                             device_plan ? 1 : 0, total);
}

void launch_scan_count_paths(const SceneView& s, const uint32_t* list, uint32_t n, cudaStream_t st) {
    if (n == 0) return;
    k_scan_count_paths<<<n, 256, 0, st>>>(s.lines, s.paths, s.path_count, list, s.backdrops, s.counts);
}

void launch_scan_emit_paths(const SceneView& s, const uint32_t* list, uint32_t n, cudaStream_t st) {
    if (n == 0) return;
    cudaMemsetAsync(s.emit_ticket, 0, sizeof(uint32_t), st);
    k_scan_emit<<<grid_for(uint64_t(n) * 32, kEmitThreads, 148 * 8), kEmitThreads, 0, st>>>(s.lines, s.paths, n, s.cursors, s.segments,
                                                                        s.segment_capacity, s.error, s.seg_line, list,
                                                                        s.emit_ticket);
}

void launch_check_path_totals(const SceneView& s, const uint32_t* bumps, const uint32_t* list, uint32_t n,
                              uint32_t* changed, cudaStream_t st) {
    cudaMemsetAsync(changed, 0, sizeof(uint32_t), st);
    if (n) k_check_path_totals<<<(n + 255) / 256, 256, 0, st>>>(s.paths, bumps, list, n, changed);
}

void launch_scan_emit(const SceneView& s, cudaStream_t st) {
    if (s.path_count == 0) return;
    uint64_t threads = uint64_t(s.path_count) * 32;
    cudaMemsetAsync(s.emit_ticket, 0, sizeof(uint32_t), st);
    k_scan_emit<<<grid_for(threads, kEmitThreads, 148 * 8), kEmitThreads, 0, st>>>(s.lines, s.paths, s.path_count, s.cursors,
                                                                s.segments, s.segment_capacity, s.error, s.seg_line,
                                                                s.emit_order, s.emit_ticket);
}

}  // namespace tk
