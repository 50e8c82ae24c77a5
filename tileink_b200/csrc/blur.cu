// Separable Gaussian blur and surface composite.
//
// Shared route (radius <= 16, filter/blur_shared.hlsl:15-74): a CTA stages a
// 32x8 pixel tile plus the +-radius halo along the blurred axis in shared
// memory; every pixel accumulates its taps in the reference's order with
// fused multiply-adds. The Gaussian weight recurrence
// (w_{d+1} = w_d * ratio, ratio *= decay) and the normalising sum are the
// same for every pixel, so the host evaluates them once in f32 with the
// reference's operation order and passes them in.
// Global route (radius > 16, filter/blur.hlsli:40-94): one thread per pixel
// with the paired bilinear taps of filter/sample.hlsli:4-17.
#include <cmath>
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.h"

namespace tk {
namespace {

using namespace tkd;

constexpr int kBX = 32, kBY = 8;
constexpr int kMaxR = int(TK_SHARED_BLUR_MAX_RADIUS);

struct Weights {
    float w[kMaxR + 1];
    float inv_sum;
    int r;
    float weight0, decay;
};

__device__ __forceinline__ bool inside_b(int x, int y, const int4 b) { return x >= b.x && y >= b.y && x < b.z && y < b.w; }
__device__ __forceinline__ void acc_tap(float4& acc, uint32_t p, float w) {
    acc.x = mad(float(p & 255u), w, acc.x);
    acc.y = mad(float((p >> 8) & 255u), w, acc.y);
    acc.z = mad(float((p >> 16) & 255u), w, acc.z);
    acc.w = mad(float(p >> 24), w, acc.w);
}
__device__ __forceinline__ uint32_t pack_average(float4 acc, float inv) {
    return pack4(f2u(clampf(acc.x * inv + 0.5f, 0.0f, 255.0f)), f2u(clampf(acc.y * inv + 0.5f, 0.0f, 255.0f)),
                 f2u(clampf(acc.z * inv + 0.5f, 0.0f, 255.0f)), f2u(clampf(acc.w * inv + 0.5f, 0.0f, 255.0f)));
}

template <int AXIS>
__global__ void __launch_bounds__(kBX * kBY)
    k_blur_shared(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint32_t width, uint32_t height,
                  uint4 region, int4 bounds, Weights wt) {
    __shared__ uint32_t s[(kBY + 2 * kMaxR) * (kBX + 2 * kMaxR)];
    const int r = wt.r;
    const int ox = int(region.x) + int(blockIdx.x) * kBX, oy = int(region.y) + int(blockIdx.y) * kBY;
    const int sw = AXIS == 0 ? kBX + 2 * r : kBX;
    const int sh = AXIS == 0 ? kBY : kBY + 2 * r;
    const int hx = AXIS == 0 ? r : 0, hy = AXIS == 0 ? 0 : r;
    for (int i = threadIdx.x; i < sw * sh; i += kBX * kBY) {
        int x = ox - hx + i % sw, y = oy - hy + i / sw;
        uint32_t v = 0u;
        if (inside_b(x, y, bounds) && x >= 0 && y >= 0 && x < int(width) && y < int(height))
            v = src[uint64_t(y) * width + x];
        s[i] = v;
    }
    __syncthreads();
    const int lx = threadIdx.x % kBX, ly = threadIdx.x / kBX;
    const int x = ox + lx, y = oy + ly;
    if (x >= int(region.x + region.z) || y >= int(region.y + region.w) || x >= int(width) || y >= int(height)) return;
    const int c = (ly + hy) * sw + lx + hx;
    const int step = AXIS == 0 ? 1 : sw;
    uint32_t cp = s[c];
    float4 acc = make_float4(float(cp & 255u), float((cp >> 8) & 255u), float((cp >> 16) & 255u), float(cp >> 24));
    for (int d = 1; d <= r; ++d) {
        float w = wt.w[d];
        acc_tap(acc, s[c + d * step], w);
        acc_tap(acc, s[c - d * step], w);
    }
    dst[uint64_t(y) * width + x] = pack_average(acc, wt.inv_sum);
}

// filter/sample.hlsli:4-17 on an RGBA8 source (texel loads are k/255).
__device__ float4 sample_premul(const uint32_t* src, uint32_t w, uint32_t h, float px, float py) {
    int lastx = int(w) - 1, lasty = int(h) - 1;
    px = clampf(px, 0.0f, float(lastx));
    py = clampf(py, 0.0f, float(lasty));
    int fx = f2i(floorf(px)), fy = f2i(floorf(py));
    int nx = min(fx + 1, lastx), ny = min(fy + 1, lasty);
    float phx = px - float(fx), phy = py - float(fy);
    float4 a = texel_load(src[uint64_t(fy) * w + fx]), b = texel_load(src[uint64_t(fy) * w + nx]);
    float4 c = texel_load(src[uint64_t(ny) * w + fx]), d = texel_load(src[uint64_t(ny) * w + nx]);
    float4 top = make_float4(mad(b.x - a.x, phx, a.x), mad(b.y - a.y, phx, a.y), mad(b.z - a.z, phx, a.z),
                             mad(b.w - a.w, phx, a.w));
    float4 bot = make_float4(mad(d.x - c.x, phx, c.x), mad(d.y - c.y, phx, c.y), mad(d.z - c.z, phx, c.z),
                             mad(d.w - c.w, phx, c.w));
    return make_float4(mad(bot.x - top.x, phy, top.x), mad(bot.y - top.y, phy, top.y), mad(bot.z - top.z, phy, top.z),
                       mad(bot.w - top.w, phy, top.w));
}

__global__ void k_blur_global(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint32_t width,
                              uint32_t height, uint4 region, int4 bounds, uint32_t axis, int hw, float weight0,
                              float decay) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= region.z * region.w) return;
    int x = int(region.x + i % region.z), y = int(region.y + i / region.z);
    if (x >= int(width) || y >= int(height)) return;
    int ax = axis == 0u ? 1 : 0, ay = axis == 0u ? 0 : 1;
    bool interior = inside_b(x - ax * hw, y - ay * hw, bounds) && inside_b(x + ax * hw, y + ay * hw, bounds);
    float sum = 1.0f;
    uint32_t center = inside_b(x, y, bounds) ? src[uint64_t(y) * width + x] : 0u;
    float4 acc = make_float4(float(center & 255u), float((center >> 8) & 255u), float((center >> 16) & 255u),
                             float(center >> 24));
    float weight = weight0, ratio = weight0 * decay;
    auto tap = [&](int px, int py, float w) {
        if (interior || inside_b(px, py, bounds)) acc_tap(acc, src[uint64_t(py) * width + px], w);
    };
    auto pair_inside = [&](float off) {
        float fx = float(x) + float(ax) * off, fy = float(y) + float(ay) * off;
        float nx = fx + float(ax), ny = fy + float(ay);
        return fx >= float(bounds.x) && fy >= float(bounds.y) && nx < float(bounds.z) && ny < float(bounds.w);
    };
    auto pair = [&](float off, float w) {
        float4 sp = sample_premul(src, width, height, float(x) + float(ax) * off, float(y) + float(ay) * off);
        acc.x = mad(sp.x * 255.0f, w, acc.x);
        acc.y = mad(sp.y * 255.0f, w, acc.y);
        acc.z = mad(sp.z * 255.0f, w, acc.z);
        acc.w = mad(sp.w * 255.0f, w, acc.w);
    };
    for (int d = 1; d <= hw; d += 2) {
        int nd = d + 1;
        bool has_pair = nd <= hw;
        float next_weight = weight * ratio;
        float pw = weight + (has_pair ? next_weight : 0.0f);
        sum += 2.0f * pw;
        if (has_pair && (interior || pair_inside(float(d)))) {
            pair(float(d) + next_weight / pw, pw);
        } else {
            tap(x + ax * d, y + ay * d, weight);
            if (has_pair) tap(x + ax * nd, y + ay * nd, next_weight);
        }
        if (has_pair && (interior || pair_inside(-float(nd)))) {
            pair(-(float(d) + next_weight / pw), pw);
        } else {
            tap(x - ax * d, y - ay * d, weight);
            if (has_pair) tap(x - ax * nd, y - ay * nd, next_weight);
        }
        float next_ratio = ratio * decay;
        weight = next_weight * next_ratio;
        ratio = next_ratio * decay;
    }
    dst[uint64_t(y) * width + x] = sum <= 0.0f ? 0u : pack_average(acc, 1.0f / sum);
}

__global__ void k_copy_region(const uint32_t* src, uint32_t* dst, uint32_t width, uint4 region) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= region.z * region.w) return;
    uint64_t o = uint64_t(region.y + i / region.z) * width + region.x + i % region.z;
    dst[o] = src[o];
}

__global__ void k_fill(uint32_t* image, uint64_t n, uint32_t value) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        image[i] = value;
}

// filter_composite_surface_stack_region with an empty clip stack
// (filter/stack.hlsl:38-46, shared/composite_stack.hlsli:11-28).
__global__ void k_composite(uint32_t* dst, const uint32_t* src, uint32_t width, int4 b) {
    uint32_t w = uint32_t(b.z - b.x);
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * uint32_t(b.w - b.y)) return;
    uint64_t o = uint64_t(b.y + int(i / w)) * width + uint32_t(b.x) + i % w;
    dst[o] = src_over_premul_u8(dst[o], scale_premul_u8(src[o], 255u));
}

// One block row per scene of a batched pass: its image region to its clear colour.
// One CTA per listed tile, one thread per pixel.
__global__ void k_fill_tiles(uint32_t* image, uint32_t width, uint32_t height, uint32_t tw,
                             const uint32_t* __restrict__ tiles, uint32_t value) {
    const uint32_t t = tiles[blockIdx.x];
    const uint32_t x = (t % tw) * TK_TILE_SIZE + (threadIdx.x & 15u), y = (t / tw) * TK_TILE_SIZE + (threadIdx.x >> 4);
    if (x < width && y < height) image[uint64_t(y) * width + x] = value;
}

__global__ void k_fill_scenes(uint32_t* image, const BatchScene* __restrict__ scenes) {
    const BatchScene sc = scenes[blockIdx.y];
    const uint64_t n = uint64_t(sc.width) * sc.height;
    uint32_t* dst = image + sc.image_offset;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        dst[i] = sc.clear;
}

// Adds each batch scene's path base to the path ids of its lines; scene k owns
// lines [line_base[k], line_base[k + 1]).
__global__ void k_rebase_lines(tk_line* lines, uint64_t n, const uint64_t* __restrict__ line_base,
                               const uint32_t* __restrict__ path_base, uint32_t scenes) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        uint32_t lo = 0, hi = scenes;  // last scene with line_base <= i
        while (hi - lo > 1u) {
            const uint32_t mid = (lo + hi) >> 1;
            if (line_base[mid] <= i) lo = mid;
            else hi = mid;
        }
        lines[i].path_id += path_base[lo];
    }
}

}  // namespace

void launch_rebase_lines(tk_line* lines, uint64_t n, const uint64_t* line_base, const uint32_t* path_base,
                         uint32_t scenes, cudaStream_t st) {
    if (n == 0 || scenes == 0) return;
    k_rebase_lines<<<148 * 8, 256, 0, st>>>(lines, n, line_base, path_base, scenes);
}

void launch_fill(uint32_t* image, uint64_t n, uint32_t value, cudaStream_t st) {
    if (n == 0) return;
    uint64_t g = (n + 255) / 256;
    k_fill<<<unsigned(g > 148 * 16 ? 148 * 16 : g), 256, 0, st>>>(image, n, value);
}

void launch_fill_tiles(uint32_t* image, uint32_t width, uint32_t height, uint32_t tw, const uint32_t* tiles,
                       uint32_t n, uint32_t value, cudaStream_t st) {
    if (n) k_fill_tiles<<<n, TK_TILE_PIXELS, 0, st>>>(image, width, height, tw, tiles, value);
}

void launch_fill_scenes(uint32_t* image, const BatchScene* scenes, uint32_t scene_count, cudaStream_t st) {
    if (scene_count == 0) return;
    k_fill_scenes<<<dim3(8, scene_count), 256, 0, st>>>(image, scenes);
}

void launch_blur(const uint32_t* src, uint32_t* dst, const BlurParams& b, cudaStream_t st) {
    uint32_t rw = b.region[2], rh = b.region[3];
    if (rw == 0 || rh == 0) return;
    uint4 region = make_uint4(b.region[0], b.region[1], rw, rh);
    int4 bounds = make_int4(b.bounds[0], b.bounds[1], b.bounds[2], b.bounds[3]);
    float sd = std::fmax(b.sigma, 0.0f);
    if (sd <= 0.0f) {
        k_copy_region<<<(rw * rh + 255) / 256, 256, 0, st>>>(src, dst, b.width, region);
        return;
    }
    // filter/blur.hlsli:20 and the recurrence of filter/blur_shared.hlsl:62-72,
    // evaluated in f32 with the shader's operation order.
    int hw = int(std::fmax(std::ceil(sd * 3.0f), 1.0f));
    float sigma = std::fmax(sd, 0.0001f);
    float two = 2.0f * sigma * sigma;
    float weight0 = std::exp(-1.0f / two), decay = std::exp(-2.0f / two);
    if (hw > kMaxR) {
        k_blur_global<<<(rw * rh + 255) / 256, 256, 0, st>>>(src, dst, b.width, b.height, region, bounds, b.axis, hw,
                                                            weight0, decay);
        return;
    }
    Weights wt{};
    wt.r = hw;
    float sum = 1.0f, weight = weight0, ratio = weight0 * decay;
    for (int d = 1; d <= hw; ++d) {
        sum += 2.0f * weight;
        wt.w[d] = weight;
        weight = weight * ratio;
        ratio = ratio * decay;
    }
    wt.inv_sum = 1.0f / sum;
    dim3 grid((rw + kBX - 1) / kBX, (rh + kBY - 1) / kBY);
    if (b.axis == 0)
        k_blur_shared<0><<<grid, kBX * kBY, 0, st>>>(src, dst, b.width, b.height, region, bounds, wt);
    else
        k_blur_shared<1><<<grid, kBX * kBY, 0, st>>>(src, dst, b.width, b.height, region, bounds, wt);
}

namespace {

using namespace tkd;

// filter_downsample_pixel (filter/resample.hlsli): low-resolution texel (lx, ly)
// of the rect `rect` (x0, y0, x1, y1) reduced by `factor`: the centre source
// texel of its cell (filter 0, nearest) or the cell's byte average rounded
// half up (filter 1, box), transparent for a cell outside the rect.
__global__ void k_blur_downsample(const uint32_t* __restrict__ src, uint32_t* __restrict__ low, uint32_t width,
                                  int4 rect, int4 low_rect, uint32_t factor, uint32_t filter) {
    const uint32_t lx = uint32_t(low_rect.x) + blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t ly = uint32_t(low_rect.y) + blockIdx.y;
    if (lx >= uint32_t(low_rect.z) || ly >= uint32_t(low_rect.w)) return;
    const uint32_t x0 = uint32_t(rect.x), y0 = uint32_t(rect.y), x1 = uint32_t(rect.z), y1 = uint32_t(rect.w);
    const uint32_t bx = max(lx * factor, x0), by = max(ly * factor, y0);
    const uint32_t ex = min((lx + 1u) * factor, x1), ey = min((ly + 1u) * factor, y1);
    uint32_t out = 0u;
    if (bx < ex && by < ey) {
        if (filter == 0u) {
            const uint32_t px = min(max((bx + ex - 1u) / 2u, x0), x1 - 1u);
            const uint32_t py = min(max((by + ey - 1u) / 2u, y0), y1 - 1u);
            out = src[uint64_t(py) * width + px];
        } else {
            float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
            for (uint32_t sy = by; sy < ey; ++sy)
                for (uint32_t sx = bx; sx < ex; ++sx) {
                    const uint32_t p = src[uint64_t(sy) * width + sx];
                    sum.x += float(p & 255u);
                    sum.y += float((p >> 8) & 255u);
                    sum.z += float((p >> 16) & 255u);
                    sum.w += float(p >> 24);
                }
            const float inv = 1.0f / float((ex - bx) * (ey - by));
            out = pack4(f2u(clampf(mad(sum.x, inv, 0.5f), 0.0f, 255.0f)), f2u(clampf(mad(sum.y, inv, 0.5f), 0.0f, 255.0f)),
                        f2u(clampf(mad(sum.z, inv, 0.5f), 0.0f, 255.0f)), f2u(clampf(mad(sum.w, inv, 0.5f), 0.0f, 255.0f)));
        }
    }
    low[uint64_t(ly) * width + lx] = out;
}

// filter_upsample_pixel (filter/resample.hlsli): texel (x, y) of `rect` from the
// low-resolution rect: the nearest low texel (filter 0) or the bilinear sample
// of filter/sample.hlsli (filter 1) stored by pack_premul_rgba8.
__global__ void k_blur_upsample(const uint32_t* __restrict__ low, uint32_t* __restrict__ dst, uint32_t width,
                                uint32_t height, int4 rect, int4 low_rect, uint32_t factor, uint32_t filter) {
    const uint32_t x = uint32_t(rect.x) + blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = uint32_t(rect.y) + blockIdx.y;
    if (x >= uint32_t(rect.z) || y >= uint32_t(rect.w)) return;
    const float f = float(max(factor, 1u));
    const float px = clampf((float(x) + 0.5f) / f - 0.5f, float(low_rect.x), float(uint32_t(low_rect.z) - 1u));
    const float py = clampf((float(y) + 0.5f) / f - 0.5f, float(low_rect.y), float(uint32_t(low_rect.w) - 1u));
    uint32_t out;
    if (filter == 0u) {
        out = low[uint64_t(f2i(rintf(py))) * width + uint32_t(f2i(rintf(px)))];
    } else {
        const float4 p = sample_premul(low, width, height, px, py);
        out = pack4(f2u(clampf(p.x, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(p.y, 0.0f, 1.0f) * 255.0f + 0.5f),
                    f2u(clampf(p.z, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(p.w, 0.0f, 1.0f) * 255.0f + 0.5f));
    }
    dst[uint64_t(y) * width + x] = out;
}

}  // namespace

int32_t launch_blur_downsampled(uint32_t* surface, uint32_t* low, uint32_t* temp, uint32_t width, uint32_t height,
                                const int32_t rect[4], float sigma, uint32_t sampling, cudaStream_t st) {
    const uint32_t factor = sampling & 255u, down = (sampling >> 8) & 255u, up = (sampling >> 16) & 255u;
    // downsampled_bounds (render/filter_program/mod.rs:93-102): floor and ceil division
    auto fdiv = [](int32_t v, int32_t d) { return v >= 0 ? v / d : -((-v + d - 1) / d); };
    auto cdiv = [&](int32_t v, int32_t d) { return -fdiv(-v, d); };
    const int32_t f = int32_t(factor);
    const int4 r = make_int4(rect[0], rect[1], rect[2], rect[3]);
    const int4 lr = make_int4(fdiv(r.x, f), fdiv(r.y, f), cdiv(r.z, f), cdiv(r.w, f));
    if (r.z <= r.x || r.w <= r.y || lr.z <= lr.x || lr.w <= lr.y) return 0;
    const uint32_t lw = uint32_t(lr.z - lr.x), lh = uint32_t(lr.w - lr.y);
    k_blur_downsample<<<dim3((lw + 127) / 128, lh), 128, 0, st>>>(surface, low, width, r, lr, factor, down);
    // the Gaussian at low resolution: sigma / factor, horizontal then vertical
    // over the low rect (render/filter_program/blur.rs:31-62)
    BlurParams b{};
    b.width = width;
    b.height = height;
    b.region[0] = uint32_t(lr.x);
    b.region[1] = uint32_t(lr.y);
    b.region[2] = lw;
    b.region[3] = lh;
    b.bounds[0] = lr.x;
    b.bounds[1] = lr.y;
    b.bounds[2] = lr.z;
    b.bounds[3] = lr.w;
    b.sigma = sigma / float(factor);
    b.axis = 0;
    launch_blur(low, temp, b, st);
    b.axis = 1;
    launch_blur(temp, low, b, st);
    const uint32_t w = uint32_t(r.z - r.x), h = uint32_t(r.w - r.y);
    k_blur_upsample<<<dim3((w + 127) / 128, h), 128, 0, st>>>(low, surface, width, height, r, lr, factor, up);
    return 1;
}

void launch_composite(uint32_t* dst, const uint32_t* src, uint32_t width, const int32_t bounds[4], cudaStream_t st) {
    int w = bounds[2] - bounds[0], h = bounds[3] - bounds[1];
    if (w <= 0 || h <= 0) return;
    k_composite<<<(uint32_t(w) * uint32_t(h) + 255) / 256, 256, 0, st>>>(
        dst, src, width, make_int4(bounds[0], bounds[1], bounds[2], bounds[3]));
}

}  // namespace tk
