// Scratch for the allocation-free pool scan: one file-scope device array per
// device holding the per-item sums and prefixes, the work items, a copy of the path
// records and the counter words, plus the kernel that builds the work items
// from the path records on the device.
#include <cuda_runtime.h>

#include <mutex>

#include "kernels.h"

namespace tk {
namespace {

constexpr size_t align256(size_t n) { return (n + 255u) & ~size_t(255u); }

constexpr size_t kDescOff = 0;
constexpr size_t kItemsOff = kDescOff + align256(sizeof(unsigned long long) * TK_NOALLOC_MAX_SCAN_ITEMS);
constexpr size_t kPathsOff = kItemsOff + align256(sizeof(ScanItem) * TK_NOALLOC_MAX_SCAN_ITEMS);
constexpr size_t kWordsOff = kPathsOff + align256(sizeof(tk_path_record) * TK_NOALLOC_MAX_PATHS);
constexpr size_t kScratchBytes = kWordsOff + 256u;
static_assert(kScratchBytes == TK_NOALLOC_SCRATCH_BYTES, "header states the scratch size");

// Zero at module load; every call re-zeroes what it needs (see the launcher).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_base[kMaxDevices] = {};

constexpr unsigned kBuildThreads = 1024;

// Work items in the order the host builds them: path-major, rows ascending,
// whole rows of at most kScanItemElems elements per item.
__global__ void __launch_bounds__(kBuildThreads)
    k_build_scan_items(const tk_path_record* __restrict__ paths, uint32_t path_count, ScanItem* items) {
    __shared__ uint32_t s_warp[kBuildThreads / 32];
    __shared__ uint32_t s_base;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    if (tid == 0) s_base = 0u;
    __syncthreads();
    for (uint32_t c0 = 0; c0 < path_count; c0 += kBuildThreads) {
        const uint32_t p = c0 + tid;
        uint32_t n = 0u, height = 0u, rows_per = 1u;
        if (p < path_count) {
            const tk_path_record r = paths[p];
            const uint32_t stride = r.tile_x1 > r.tile_x0 ? r.tile_x1 - r.tile_x0 : 0u;
            height = r.tile_y1 > r.tile_y0 ? r.tile_y1 - r.tile_y0 : 0u;
            if (r.data_len && stride) {
                rows_per = kScanItemElems / stride;
                if (rows_per == 0u) rows_per = 1u;
                n = (height + rows_per - 1u) / rows_per;
            }
        }
        uint32_t incl = n;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= uint32_t(d)) incl += v;
        }
        if (lane == 31u) s_warp[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = s_warp[lane];
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                uint32_t v = __shfl_up_sync(0xffffffffu, w, d);
                if (lane >= uint32_t(d)) w += v;
            }
            s_warp[lane] = w;  // inclusive over warps
        }
        __syncthreads();
        const uint32_t base = s_base + (warp ? s_warp[warp - 1] : 0u) + incl - n;
        for (uint32_t j = 0; j < n; ++j) {
            const uint32_t row = j * rows_per;
            const uint32_t rows = height - row < rows_per ? height - row : rows_per;
            items[base + j] = ScanItem{p, row, rows, row == 0u ? 1u : 0u};
        }
        __syncthreads();
        if (tid == 0) s_base += s_warp[kBuildThreads / 32 - 1];
        __syncthreads();
    }
}

}  // namespace

cudaError_t noalloc_scratch(int device, NoAllocScratch* out) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_base[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_base[device] = static_cast<unsigned char*>(p);
    }
    unsigned char* b = g_base[device];
    out->desc = reinterpret_cast<unsigned long long*>(b + kDescOff);
    out->items = reinterpret_cast<ScanItem*>(b + kItemsOff);
    out->paths = reinterpret_cast<tk_path_record*>(b + kPathsOff);
    out->words = reinterpret_cast<uint32_t*>(b + kWordsOff);
    return cudaSuccess;
}

void launch_build_scan_items(const tk_path_record* paths, uint32_t path_count, ScanItem* items, cudaStream_t st) {
    if (path_count == 0) return;
    k_build_scan_items<<<1, kBuildThreads, 0, st>>>(paths, path_count, items);
}

}  // namespace tk
