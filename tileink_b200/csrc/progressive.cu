// Progressive blur (Filter::ProgressiveBlur): a spatially varying Gaussian
// through a calibrated scale pyramid (native/runtime/program/filter/
// progressive/{mod,pyramid}.rs, filter/progressive.hlsl).
//
// The host plans the pyramid: level 0 is a copy of the blurred region, each
// further level is the previous one convolved with a paired Gaussian kernel
// along x then y and decimated by its step (1 or 2); levels carry their
// cumulative variance. The resolve pass then evaluates, per pixel, the
// standard deviation the gradient asks for and interpolates between the two
// levels that bracket its variance (or applies a 7-tap kernel directly for
// sigma <= 1). Levels and the reduction scratch are RGBA8 surfaces, as the
// reference's pooled textures are. The reference samples levels through the
// hardware bilinear filter inside them and through an explicit lerp at their
// edges; here both use the explicit lerp, `lerp(a, b, t)` as a + t (b - a),
// which the hardware filter approximates with 8-bit fractional weights.
#include <cmath>
#include <cuda_runtime.h>
#include <vector>

#include "device.cuh"
#include "kernels.h"
#include "sdf.cuh"

namespace tk {
namespace {

using namespace tkd;

constexpr uint32_t kMaxPairs = 48;

struct Taps {
    float offset[kMaxPairs], weight[kMaxPairs];
    uint32_t n;
};

struct Levels {
    uint32_t n;
    uint32_t w[kProgressiveMaxLevels], h[kProgressiveMaxLevels];
    uint64_t off[kProgressiveMaxLevels];
    float scale[kProgressiveMaxLevels], variance[kProgressiveMaxLevels];
};

__device__ __forceinline__ float4 fetch(const uint32_t* img, uint32_t w, uint32_t h, int32_t x, int32_t y) {
    if (x < 0 || y < 0 || x >= int32_t(w) || y >= int32_t(h)) return make_float4(0.f, 0.f, 0.f, 0.f);
    return texel_load(img[uint64_t(y) * w + uint32_t(x)]);
}
__device__ __forceinline__ float4 lerp4(float4 a, float4 b, float t) {
    return make_float4(a.x + t * (b.x - a.x), a.y + t * (b.y - a.y), a.z + t * (b.z - a.z), a.w + t * (b.w - a.w));
}
// sample_source / sample_level's bilinear read at texel position (px, py)
// with transparent texels outside the image.
__device__ __forceinline__ float4 bilinear(const uint32_t* img, uint32_t w, uint32_t h, float px, float py) {
    const float bx = floorf(px), by = floorf(py);
    const int32_t ix = f2i(bx), iy = f2i(by);
    const float fx = px - bx, fy = py - by;  // frac
    return lerp4(lerp4(fetch(img, w, h, ix, iy), fetch(img, w, h, ix + 1, iy), fx),
                 lerp4(fetch(img, w, h, ix, iy + 1), fetch(img, w, h, ix + 1, iy + 1), fx), fy);
}

// Level 0: the blurred region copied out of the surface.
__global__ void k_prog_copy(const uint32_t* __restrict__ surface, uint32_t width, int4 rect, uint32_t* level0) {
    const uint32_t w = uint32_t(rect.z - rect.x);
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w) return;
    level0[uint64_t(y) * w + x] = surface[uint64_t(uint32_t(rect.y) + y) * width + uint32_t(rect.x) + x];
}

// progressive_blur_reduce (filter/progressive.hlsl:38-51): output texel id
// sums the level's taps along `axis` around id (scaled by the step on that
// axis).
__global__ void k_prog_reduce(const uint32_t* __restrict__ src, uint32_t sw, uint32_t sh, uint32_t* dst, uint32_t dw,
                              uint32_t dh, uint32_t step, uint32_t axis, Taps taps) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= dw || y >= dh) return;
    float cx = float(x), cy = float(y);
    if (axis == 0u) cx *= float(step);
    else cy *= float(step);
    float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint32_t i = 0; i < taps.n; ++i) {
        float px = cx, py = cy;
        if (axis == 0u) px += taps.offset[i];
        else py += taps.offset[i];
        const float4 s = bilinear(src, sw, sh, px, py);
        const float wt = taps.weight[i];
        c = make_float4(c.x + wt * s.x, c.y + wt * s.y, c.z + wt * s.z, c.w + wt * s.w);
    }
    dst[uint64_t(y) * dw + x] = texel_store(c);
}

__device__ __forceinline__ float4 sample_level(const uint32_t* levels, const Levels& L, uint32_t i, float px, float py) {
    return bilinear(levels + L.off[i], L.w[i], L.h[i], px / L.scale[i] - 0.5f, py / L.scale[i] - 0.5f);
}

// progressive_blur_resolve (filter/progressive.hlsl:97-122) with
// shallow_blur (68-95) for sigma <= 1.
__global__ void k_prog_resolve(uint32_t* target, uint32_t width, int4 rect, const uint32_t* __restrict__ levels,
                               const Levels L, float4 gradient, float max_std_dev) {
    const uint32_t x = uint32_t(rect.x) + blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t y = uint32_t(rect.y) + blockIdx.y;
    if (x >= uint32_t(rect.z) || y >= uint32_t(rect.w)) return;
    float t = 1.0f;
    if (!(gradient.z == 0.0f && gradient.w == 0.0f))
        t = clampf(((float(x) + 0.5f) - gradient.x) * gradient.z + ((float(y) + 0.5f) - gradient.y) * gradient.w, 0.0f,
                   1.0f);
    const float sigma = max_std_dev * t * t * (3.0f - 2.0f * t);
    if (sigma < 0.125f) return;  // the pixel stays as it is
    const float px = float(x - uint32_t(rect.x)) + 0.5f, py = float(y - uint32_t(rect.y)) + 0.5f;
    float4 out;
    if (sigma <= 1.0f) {
        float wts[7], total = 0.0f;
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            const float d = float(k - 3);
            wts[k] = sdf_exp_nonpos(-0.5f * d * d / (sigma * sigma));
            total += wts[k];
        }
        float off[4], comb[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int first = 2 * k;
            const float second = first + 1 < 7 ? wts[first + 1] : 0.0f;
            comb[k] = wts[first] + second;
            off[k] = float(first - 3) + (comb[k] > 0.0f ? second / comb[k] : 0.0f);
        }
        float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int j = 0; j < 4; ++j)
            for (int k = 0; k < 4; ++k) {
                const float wt = comb[k] * comb[j];
                const float4 s = sample_level(levels, L, 0u, px + off[k], py + off[j]);
                c = make_float4(c.x + wt * s.x, c.y + wt * s.y, c.z + wt * s.z, c.w + wt * s.w);
            }
        const float tt = total * total;
        out = make_float4(c.x / tt, c.y / tt, c.z / tt, c.w / tt);
    } else {
        const float variance = sigma * sigma;
        uint32_t upper = 1u;
        while (upper + 1u < L.n && L.variance[upper] < variance) ++upper;
        const float lo = L.variance[upper - 1u], hi = L.variance[upper];
        const float weight = clampf((variance - lo) / (hi - lo), 0.0f, 1.0f);
        out = lerp4(sample_level(levels, L, upper - 1u, px, py), sample_level(levels, L, upper, px, py), weight);
    }
    target[uint64_t(y) * width + x] = texel_store(out);
}

cudaError_t grow(uint32_t*& ptr, uint64_t& cap, uint64_t need) {
    if (need <= cap) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&ptr, need * sizeof(uint32_t));
    if (e == cudaSuccess) cap = need;
    return e;
}

}  // namespace

// levels() and gaussian_kernel() (progressive/pyramid.rs:17-90), in f32 with
// the reference's operation order and the host's expf / powf / sqrtf.
std::vector<ProgressiveLevel> progressive_levels(uint32_t w, uint32_t h, float sigma, uint32_t quality) {
    const float octave_steps = quality == TK_PROGRESSIVE_HIGH ? 3.0f : 2.0f;
    const float min_sigma = quality == TK_PROGRESSIVE_HIGH ? 2.0f : 1.5f;
    const float support = quality == TK_PROGRESSIVE_HIGH ? 4.0f : 3.0f;
    std::vector<ProgressiveLevel> levels(1);
    levels[0].w = w;
    levels[0].h = h;
    levels[0].scale = 1.0f;
    levels[0].variance = 0.0f;
    levels[0].step = 1u;
    if (sigma <= 1.0f) return levels;
    float raw_variance = 0.0f, target_sigma = 1.0f;
    const float growth = std::pow(2.0f, 1.0f / octave_steps);
    while (levels.back().variance < sigma * sigma && levels.size() <= kProgressiveMaxLevels) {
        const ProgressiveLevel prev = levels.back();
        const uint32_t step = target_sigma >= min_sigma * prev.scale * 2.0f ? 2u : 1u;
        const float scale = prev.scale * float(step);
        const float reconstruction = scale == 1.0f ? 0.0f : (2.0f * scale * scale + 1.0f) / 12.0f;
        const float incremental =
            std::sqrt((target_sigma * target_sigma - reconstruction - raw_variance) / (prev.scale * prev.scale));
        // gaussian_kernel(incremental, step, support)
        const int32_t radius = int32_t(std::ceil(incremental * support));
        const float center = float(step - 1u) * 0.5f;
        std::vector<float> tx, tw;
        for (int32_t x = -radius; x < radius + int32_t(step); ++x) {
            const float d = (float(x) - center) / incremental;
            tx.push_back(float(x));
            tw.push_back(std::exp(-0.5f * (d * d)));
        }
        float total = 0.0f;
        for (float v : tw) total += v;
        float variance = 0.0f;
        for (size_t k = 0; k < tw.size(); ++k) {
            tw[k] /= total;
            const float d = tx[k] - center;
            variance += tw[k] * (d * d);
        }
        ProgressiveLevel L;
        for (size_t k = 0; k < tw.size(); k += 2) {  // adjacent taps paired, as a bilinear fetch combines them
            float weight = tw[k], moment = tx[k] * tw[k];
            if (k + 1 < tw.size()) {
                weight += tw[k + 1];
                moment += tx[k + 1] * tw[k + 1];
            }
            L.kernel.push_back({moment / weight, weight});
        }
        raw_variance += variance * prev.scale * prev.scale;
        L.w = (prev.w + step - 1u) / step;
        L.h = (prev.h + step - 1u) / step;
        L.scale = scale;
        L.variance = raw_variance + reconstruction;
        L.step = step;
        levels.push_back(std::move(L));
        target_sigma *= growth;
    }
    return levels;
}

int32_t launch_progressive_blur(uint32_t* surface, uint32_t width, uint32_t height, const int32_t rect[4],
                                const tk_progressive_blur& blur, ProgressiveScratch& s, cudaStream_t st) {
    const int32_t x0 = std::max(rect[0], 0), y0 = std::max(rect[1], 0);
    const int32_t x1 = std::min(rect[2], int32_t(width)), y1 = std::min(rect[3], int32_t(height));
    if (x1 <= x0 || y1 <= y0 || !(blur.max_std_dev > 0.0f)) return 0;
    const uint32_t w = uint32_t(x1 - x0), h = uint32_t(y1 - y0);
    const std::vector<ProgressiveLevel> plan = progressive_levels(w, h, blur.max_std_dev, blur.quality);
    if (plan.size() > kProgressiveMaxLevels) return -1;  // the reference's level-table overflow
    Levels L{};
    L.n = uint32_t(plan.size());
    uint64_t total = 0;
    for (uint32_t i = 0; i < L.n; ++i) {
        L.w[i] = plan[i].w;
        L.h[i] = plan[i].h;
        L.off[i] = total;
        L.scale[i] = plan[i].scale;
        L.variance[i] = plan[i].variance;
        total += uint64_t(plan[i].w) * plan[i].h;
        if (plan[i].kernel.size() > kMaxPairs) return -1;
    }
    if (grow(s.levels, s.levels_cap, total) != cudaSuccess) return -2;
    if (L.n > 1u && grow(s.scratch, s.scratch_cap, uint64_t(w) * h) != cudaSuccess) return -2;
    const int4 r = make_int4(x0, y0, x1, y1);
    k_prog_copy<<<dim3((w + 127) / 128, h), 128, 0, st>>>(surface, width, r, s.levels);
    for (uint32_t i = 1; i < L.n; ++i) {
        const ProgressiveLevel& lv = plan[i];
        Taps t{};
        t.n = uint32_t(lv.kernel.size());
        for (uint32_t k = 0; k < t.n; ++k) {
            t.offset[k] = lv.kernel[k].first;
            t.weight[k] = lv.kernel[k].second;
        }
        // horizontal into the scratch (level width x previous height), then vertical
        const uint32_t iw = lv.w, ih = L.h[i - 1];
        k_prog_reduce<<<dim3((iw + 127) / 128, ih), 128, 0, st>>>(s.levels + L.off[i - 1], L.w[i - 1], L.h[i - 1],
                                                                  s.scratch, iw, ih, lv.step, 0u, t);
        k_prog_reduce<<<dim3((lv.w + 127) / 128, lv.h), 128, 0, st>>>(s.scratch, iw, ih, s.levels + L.off[i], lv.w,
                                                                      lv.h, lv.step, 1u, t);
    }
    const float4 g = make_float4(blur.start_x, blur.start_y, blur.dir_x, blur.dir_y);
    k_prog_resolve<<<dim3((w + 127) / 128, h), 128, 0, st>>>(surface, width, r, s.levels, L, g, blur.max_std_dev);
    return 1;
}

void release_progressive(ProgressiveScratch& s) {
    if (s.levels) cudaFree(s.levels);
    if (s.scratch) cudaFree(s.scratch);
    s = ProgressiveScratch{};
}

}  // namespace tk
