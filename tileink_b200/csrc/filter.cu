// Filter layers (Canvas::push_filter_layer with Filter::Chain): the group's
// RGBA8 surface filtered in place, one chain filter after another, over the
// layer's processing bounds (render/filter_program/effects.rs:3-268).
//
// * Colour filters, the colour matrix and component transfers: one thread
//   per pixel applying a run of up to eight consecutive ones in order (one
//   read and one write per pixel for the run), each the
//   reference's filter_color_pixel / filter_color_matrix_pixel
//   (filter/color.hlsli:8-76) on the stored RGBA8 word. `mad` is an explicit
//   fused multiply-add; every other product and sum is rounded on its own.
//   Hue rotation takes cos / sin from the exactly rounded evaluation shared
//   with the SDF kinds (sdf.cuh), which the oracle restates.
// * Offset: out(x, y) = in(x - dx, y - dy) inside the bounds, transparent
//   where the source falls outside them (filter_offset_region,
//   filter/basic.hlsl:49-56), into the scratch surface and copied back.
// * Erode / dilate: per axis, the componentwise min / max of the
//   unpremultiplied texels within the radius along the surface line
//   (filter_morphology_pixel, filter/morphology.hlsli:8-27), x into the
//   scratch surface, then y back; an erosion clears texels within the radius
//   of the line's ends, and one whose doubled radius reaches the surface
//   size clears the bounds (render/filter_program/effects.rs:169-221).
// * Component transfer: each channel's table at its straight byte
//   (filter_transfer_pixel, filter/transfer.hlsli:5-19).
// * Convolution (filter_convolve_pixel, filter/convolve.hlsli:34-98): the
//   flipped kernel over the bounds with their edge mode, premultiplied taps
//   (straight with preserve_alpha), alpha in byte units, the divisor's
//   subnormal and huge ranges rescaled by 2^24, bias on the unbounded alpha.
// * Blur: the blur groups' Gaussian over the bounds, with its own deviation
//   along x and y (render/filter_program/blur.rs:194-244).
// * Flood: the bounds filled with the solid colour (filter_flood_region,
//   filter/brush.hlsl:19-26).
// * Drop shadow (render/filter_program/shadow.rs:3-52): the source alpha
//   copied to all four channels of a cleared scratch surface at the offset
//   position (filter_drop_shadow_mask_region, filter/basic.hlsl:58-66), the
//   Gaussian blur of the blur groups over the bounds (x, then y), then the
//   colour scaled by the shadow's alpha under the source
//   (filter_composite_drop_shadow_region, filter/brush.hlsl:27-36).
// The per-pixel kernels are HBM-bound: 8 bytes per pixel (read and write the
// word); a morphology pass reads 2r + 1 texels per pixel, mostly from L1.
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.h"
#include "sdf.cuh"

namespace tk {
namespace {

using namespace tkd;

struct FilterArgs {
    uint32_t kind;
    float amount;
    float m[20];
    const uint32_t* table;  // COMPONENT_TRANSFER: its table
};

// filter_transfer_pixel (filter/transfer.hlsli:5-19): the straight channel
// byte (rounded) indexes each channel's table, alpha its own.
__device__ __forceinline__ uint32_t straight_index(uint32_t premul, uint32_t alpha) {
    return alpha == 0u ? 0u : min((premul * 255u + alpha / 2u) / alpha, 255u);
}
__device__ uint32_t transfer_pixel(const uint32_t* __restrict__ t, uint32_t pixel) {
    const uint32_t alpha = pixel >> 24;
    const float r = float(__ldg(t + straight_index(pixel & 255u, alpha))) * CHANNEL_SCALE;
    const float g = float(__ldg(t + 256u + straight_index((pixel >> 8) & 255u, alpha))) * CHANNEL_SCALE;
    const float b = float(__ldg(t + 512u + straight_index((pixel >> 16) & 255u, alpha))) * CHANNEL_SCALE;
    const float a = float(__ldg(t + 768u + alpha)) * CHANNEL_SCALE;
    return pack4(f2u(clampf(r * a, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(g * a, 0.0f, 1.0f) * 255.0f + 0.5f),
                 f2u(clampf(b * a, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(a, 0.0f, 1.0f) * 255.0f + 0.5f));
}

// svg_luminance (filter/color.hlsli:7)
__device__ __forceinline__ float svg_luminance(float r, float g, float b) {
    return (0.2126f * r + 0.7152f * g) + 0.0722f * b;
}

// filter_color_pixel (filter/color.hlsli:9-45)
__device__ uint32_t color_filter_pixel(uint32_t pixel, uint32_t kind, float amount) {
    if ((kind == TK_FILTER_INVERT || kind == TK_FILTER_SEPIA) && (pixel >> 24) != 0u) {
        // byte channels, no normalize / unpremultiply round trip
        const float cr = float(pixel & 255u), cg = float((pixel >> 8) & 255u), cb = float((pixel >> 16) & 255u);
        const float alpha = float(pixel >> 24);
        float mr = alpha - cr, mg = alpha - cg, mb = alpha - cb;
        if (kind == TK_FILTER_SEPIA) {
            mr = mad(0.393f, cr, mad(0.769f, cg, 0.189f * cb));
            mg = mad(0.349f, cr, mad(0.686f, cg, 0.168f * cb));
            mb = mad(0.272f, cr, mad(0.534f, cg, 0.131f * cb));
        }
        const float t = clampf(amount, 0.0f, 1.0f);
        const uint32_t r = f2u(clampf(mad(mr - cr, t, cr), 0.0f, alpha) + 0.5f);
        const uint32_t g = f2u(clampf(mad(mg - cg, t, cg), 0.0f, alpha) + 0.5f);
        const uint32_t b = f2u(clampf(mad(mb - cb, t, cb), 0.0f, alpha) + 0.5f);
        return pack4(r, g, b, pixel >> 24);
    }
    float4 c = rgba8_to_unorm(pixel);
    if (kind == TK_FILTER_OPACITY) {
        const float a = clampf(amount, 0.0f, 1.0f);
        c = make_float4(c.x * a, c.y * a, c.z * a, c.w * a);
    } else if (c.w > 0.0f) {
        float r = c.x / c.w, g = c.y / c.w, b = c.z / c.w;
        if (kind == TK_FILTER_BRIGHTNESS) {
            r = r * amount;
            g = g * amount;
            b = b * amount;
        } else if (kind == TK_FILTER_CONTRAST) {
            r = (r - 0.5f) * amount + 0.5f;
            g = (g - 0.5f) * amount + 0.5f;
            b = (b - 0.5f) * amount + 0.5f;
        } else if (kind == TK_FILTER_GRAYSCALE) {
            // filter_lerp(straight, luminance, t) = mad(b - a, t, a)
            const float l = svg_luminance(r, g, b), t = clampf(amount, 0.0f, 1.0f);
            r = mad(l - r, t, r);
            g = mad(l - g, t, g);
            b = mad(l - b, t, b);
        } else if (kind == TK_FILTER_HUE_ROTATE) {
            const float angle = amount * 0.017453292f;
            float si, co;
            sdf_sincos(angle, si, co);
            const float nr = ((0.213f + co * 0.787f) - si * 0.213f) * r + ((0.715f - co * 0.715f) - si * 0.715f) * g +
                             ((0.072f - co * 0.072f) + si * 0.928f) * b;
            const float ng = ((0.213f - co * 0.213f) + si * 0.143f) * r + ((0.715f + co * 0.285f) + si * 0.140f) * g +
                             ((0.072f - co * 0.072f) - si * 0.283f) * b;
            const float nb = ((0.213f - co * 0.213f) - si * 0.787f) * r + ((0.715f - co * 0.715f) + si * 0.715f) * g +
                             ((0.072f + co * 0.928f) + si * 0.072f) * b;
            r = nr;
            g = ng;
            b = nb;
        } else if (kind == TK_FILTER_SATURATE) {
            const float l = svg_luminance(r, g, b);
            r = l + (r - l) * amount;
            g = l + (g - l) * amount;
            b = l + (b - l) * amount;
        }
        c = make_float4(clampf(r, 0.0f, 1.0f) * c.w, clampf(g, 0.0f, 1.0f) * c.w, clampf(b, 0.0f, 1.0f) * c.w, c.w);
    }
    // pack_premul_rgba8 (shared/pixel.hlsli:51-54)
    return pack4(f2u(clampf(c.x, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(c.y, 0.0f, 1.0f) * 255.0f + 0.5f),
                 f2u(clampf(c.z, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(c.w, 0.0f, 1.0f) * 255.0f + 0.5f));
}

// filter_dot4 (filter/color.hlsli:47)
__device__ __forceinline__ float dot4(const float* a, float x, float y, float z, float w) {
    return mad(a[0], x, mad(a[1], y, mad(a[2], z, a[3] * w)));
}

// filter_color_matrix_pixel (filter/color.hlsli:49-76); m is the 4 x 5
// row-major matrix (rows r g b a, columns r g b a bias).
__device__ uint32_t color_matrix_pixel(const float* m, uint32_t pixel) {
    const float alpha = float(pixel >> 24);
    const float cr = float(pixel & 255u), cg = float((pixel >> 8) & 255u), cb = float((pixel >> 16) & 255u);
    float sr = 0.0f, sg = 0.0f, sb = 0.0f;
    if ((pixel >> 24) == 255u) {
        sr = cr;
        sg = cg;
        sb = cb;
    } else if (alpha > 0.0f) {
        const float k = 255.0f / alpha;
        sr = cr * k;
        sg = cg * k;
        sb = cb * k;
    }
    const float out_a = floorf(clampf(dot4(m + 15, sr, sg, sb, alpha) + m[19] * 255.0f, 0.0f, 255.0f) + 0.5f);
    float rr, rg, rb;
    if (alpha > 0.0f) {
        const float sw = alpha * alpha * CHANNEL_SCALE;
        const float mr = mad(m[4], alpha, dot4(m + 0, cr, cg, cb, sw));
        const float mg = mad(m[9], alpha, dot4(m + 5, cr, cg, cb, sw));
        const float mb = mad(m[14], alpha, dot4(m + 10, cr, cg, cb, sw));
        const float scale = out_a == alpha ? 1.0f : out_a / alpha;
        rr = mr >= alpha ? out_a : clampf(mr, 0.0f, alpha) * scale;
        rg = mg >= alpha ? out_a : clampf(mg, 0.0f, alpha) * scale;
        rb = mb >= alpha ? out_a : clampf(mb, 0.0f, alpha) * scale;
    } else {
        rr = clampf(m[4], 0.0f, 1.0f) * out_a;
        rg = clampf(m[9], 0.0f, 1.0f) * out_a;
        rb = clampf(m[14], 0.0f, 1.0f) * out_a;
    }
    return pack4(f2u(clampf(rr, 0.0f, 255.0f) + 0.5f), f2u(clampf(rg, 0.0f, 255.0f) + 0.5f),
                 f2u(clampf(rb, 0.0f, 255.0f) + 0.5f), f2u(clampf(out_a, 0.0f, 255.0f) + 0.5f));
}

// A run of consecutive per-pixel filters of a chain, applied in order to each
// pixel in one pass (one read and one write per pixel for the whole run).
constexpr uint32_t kFilterRun = 8;
struct FilterRun {
    uint32_t n;
    FilterArgs f[kFilterRun];
};

__global__ void k_filter_color(uint32_t* surface, uint32_t width, int4 b, FilterRun run) {
    const uint32_t w = uint32_t(b.z - b.x);
    const uint64_t n = uint64_t(w) * uint32_t(b.w - b.y);
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t o = uint64_t(b.y + uint32_t(i / w)) * width + uint32_t(b.x) + uint32_t(i % w);
        uint32_t p = surface[o];
        for (uint32_t k = 0; k < run.n; ++k) {
            const FilterArgs& f = run.f[k];
            p = f.kind == TK_FILTER_COLOR_MATRIX         ? color_matrix_pixel(f.m, p)
                : f.kind == TK_FILTER_COMPONENT_TRANSFER ? transfer_pixel(f.table, p)
                                                         : color_filter_pixel(p, f.kind, f.amount);
        }
        surface[o] = p;
    }
}

__global__ void k_filter_offset(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint32_t width, int4 b,
                                int32_t dx, int32_t dy) {
    const uint32_t w = uint32_t(b.z - b.x);
    const uint64_t n = uint64_t(w) * uint32_t(b.w - b.y);
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const int64_t x = b.x + int64_t(i % w), y = b.y + int64_t(i / w);
        const int64_t sx = x - dx, sy = y - dy;
        uint32_t p = 0u;
        if (sx >= b.x && sy >= b.y && sx < b.z && sy < b.w) p = src[uint64_t(sy) * width + uint64_t(sx)];
        dst[uint64_t(y) * width + uint64_t(x)] = p;
    }
}

__global__ void k_filter_copy(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint32_t width, int4 b) {
    const uint32_t w = uint32_t(b.z - b.x);
    const uint64_t n = uint64_t(w) * uint32_t(b.w - b.y);
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t o = uint64_t(b.y + uint32_t(i / w)) * width + uint32_t(b.x) + uint32_t(i % w);
        dst[o] = src[o];
    }
}

// One morphology pass along x (horizontal) or y over bounds b, whose lines
// are the surface's (the bounds are the whole surface here).
__global__ void k_filter_morphology(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint32_t width,
                                    int4 b, uint32_t radius, bool dilate, bool horizontal) {
    const uint32_t w = uint32_t(b.z - b.x), h = uint32_t(b.w - b.y);
    const uint64_t n = uint64_t(w) * h;
    const uint32_t len = horizontal ? w : h;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t lx = uint32_t(i % w), ly = uint32_t(i / w);
        const uint64_t o = uint64_t(uint32_t(b.y) + ly) * width + uint32_t(b.x) + lx;
        const uint32_t pos = horizontal ? lx : ly;
        if (!dilate && (pos < radius || pos + radius >= len)) {
            dst[o] = 0u;
            continue;
        }
        float r = dilate ? 0.0f : 1.0f, g = r, bl = r, a = r;
        const uint32_t start = pos > radius ? pos - radius : 0u, end = min(len - 1u, pos + radius);
        for (uint32_t sp = start; sp <= end; ++sp) {
            const uint64_t so = horizontal ? uint64_t(uint32_t(b.y) + ly) * width + uint32_t(b.x) + sp
                                           : uint64_t(uint32_t(b.y) + sp) * width + uint32_t(b.x) + lx;
            const uint32_t p = __ldg(src + so), al = p >> 24;
            // straight_channel (shared/pixel.hlsli:24) and alpha / 255
            const float vr = al == 0u ? 0.0f : float(p & 255u) / float(al);
            const float vg = al == 0u ? 0.0f : float((p >> 8) & 255u) / float(al);
            const float vb = al == 0u ? 0.0f : float((p >> 16) & 255u) / float(al);
            const float va = float(al) / 255.0f;
            if (dilate) {
                r = fmaxf(r, vr);
                g = fmaxf(g, vg);
                bl = fmaxf(bl, vb);
                a = fmaxf(a, va);
            } else {
                r = fminf(r, vr);
                g = fminf(g, vg);
                bl = fminf(bl, vb);
                a = fminf(a, va);
            }
        }
        dst[o] = pack4(f2u(clampf(r * a, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(g * a, 0.0f, 1.0f) * 255.0f + 0.5f),
                       f2u(clampf(bl * a, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(a, 0.0f, 1.0f) * 255.0f + 0.5f));
    }
}

__global__ void k_filter_clear(uint32_t* dst, uint32_t width, int4 b) {
    const uint32_t w = uint32_t(b.z - b.x);
    const uint64_t n = uint64_t(w) * uint32_t(b.w - b.y);
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        dst[uint64_t(b.y + uint32_t(i / w)) * width + uint32_t(b.x) + uint32_t(i % w)] = 0u;
}

__global__ void k_filter_fill(uint32_t* dst, uint32_t width, int4 b, uint32_t color) {
    const uint32_t w = uint32_t(b.z - b.x);
    const uint64_t n = uint64_t(w) * uint32_t(b.w - b.y);
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        dst[uint64_t(b.y + uint32_t(i / w)) * width + uint32_t(b.x) + uint32_t(i % w)] = color;
}

// The source alpha in all four channels at the offset position, inside the
// bounds (the destination cleared beforehand).
__global__ void k_shadow_mask(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint32_t width, int4 b,
                              int32_t dx, int32_t dy) {
    const uint32_t w = uint32_t(b.z - b.x);
    const uint64_t n = uint64_t(w) * uint32_t(b.w - b.y);
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const int64_t x = b.x + int64_t(i % w), y = b.y + int64_t(i / w);
        const uint32_t a = src[uint64_t(y) * width + uint64_t(x)] >> 24;
        if (a == 0u) continue;
        const int64_t tx = x + dx, ty = y + dy;
        if (tx >= b.x && ty >= b.y && tx < b.z && ty < b.w) dst[uint64_t(ty) * width + uint64_t(tx)] = a * 0x01010101u;
    }
}

__global__ void k_shadow_composite(uint32_t* surface, const uint32_t* __restrict__ shadow, uint32_t width, int4 b,
                                   uint32_t color) {
    const uint32_t w = uint32_t(b.z - b.x);
    const uint64_t n = uint64_t(w) * uint32_t(b.w - b.y);
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t o = uint64_t(b.y + uint32_t(i / w)) * width + uint32_t(b.x) + uint32_t(i % w);
        surface[o] = src_over_premul_u8(scale_premul_u8(color, shadow[o] >> 24), surface[o]);
    }
}

// --- filter/convolve.hlsli:9-98 ----------------------------------------------
__device__ __forceinline__ int32_t conv_wrap(int32_t c, int32_t origin, int32_t len) {
    const int32_t r = (c - origin) % len;
    return origin + (r < 0 ? r + len : r);
}
// value x 2^24 through the exponent bits (subnormals scaled exactly)
__device__ __forceinline__ float conv_scale_24(float v) {
    const uint32_t bits = __float_as_uint(v), mag = bits & 0x7fffffffu, e = mag >> 23;
    if (e == 0u) {
        const float s = float(mag) * __uint_as_float(0x01000000u);
        return (bits & 0x80000000u) ? -s : s;
    }
    if (e >= 231u) return __uint_as_float((bits & 0x80000000u) | 0x7f800000u);
    return __uint_as_float(bits + (24u << 23));
}
__device__ __forceinline__ float conv_unscale_24(float v) {
    const uint32_t bits = __float_as_uint(v), e = (bits & 0x7fffffffu) >> 23;
    if (e <= 24u) return 0.0f;
    return __uint_as_float(bits - (24u << 23));
}

struct ConvArgs {
    const float* kernel;
    uint32_t columns, rows, target_x, target_y, edge_mode, preserve_alpha;
    float divisor, bias;
};

__global__ void k_filter_convolve(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint32_t width, int4 b,
                                  ConvArgs k) {
    const uint32_t w = uint32_t(b.z - b.x);
    const uint64_t n = uint64_t(w) * uint32_t(b.w - b.y);
    const uint32_t dmag = __float_as_uint(k.divisor) & 0x7fffffffu;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const int32_t x = b.x + int32_t(i % w), y = b.y + int32_t(i / w);
        const uint64_t o = uint64_t(y) * width + uint64_t(x);
        const uint32_t center = src[o];
        if (k.columns == 0u || k.rows == 0u || dmag == 0u) {
            dst[o] = center;
            continue;
        }
        float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f, s3 = 0.0f;
        for (uint32_t ky = 0; ky < k.rows; ++ky)
            for (uint32_t kx = 0; kx < k.columns; ++kx) {
                const float wt = __ldg(k.kernel + (k.rows - 1u - ky) * k.columns + (k.columns - 1u - kx));
                int32_t px = x + int32_t(kx) - int32_t(k.target_x), py = y + int32_t(ky) - int32_t(k.target_y);
                uint32_t p = 0u;
                if (k.edge_mode == TK_CONVOLVE_EDGE_DUPLICATE) {
                    px = min(max(px, b.x), b.z - 1);
                    py = min(max(py, b.y), b.w - 1);
                    p = src[uint64_t(py) * width + uint64_t(px)];
                } else if (k.edge_mode == TK_CONVOLVE_EDGE_WRAP) {
                    px = conv_wrap(px, b.x, b.z - b.x);
                    py = conv_wrap(py, b.y, b.w - b.y);
                    p = src[uint64_t(py) * width + uint64_t(px)];
                } else if (px >= b.x && py >= b.y && px < b.z && py < b.w) {
                    p = src[uint64_t(py) * width + uint64_t(px)];
                }
                const uint32_t al = p >> 24;
                float4 v = rgba8_to_unorm(p);
                if (k.preserve_alpha) {
                    v.x = al == 0u ? 0.0f : v.x / v.w;
                    v.y = al == 0u ? 0.0f : v.y / v.w;
                    v.z = al == 0u ? 0.0f : v.z / v.w;
                }
                v.w = float(al);
                s0 = mad(v.x, wt, s0);
                s1 = mad(v.y, wt, s1);
                s2 = mad(v.z, wt, s2);
                s3 = mad(v.w, wt, s3);
            }
        float q0, q1, q2, qa;
        if (dmag < 0x00800000u) {  // subnormal divisor: both sides scaled by 2^24
            float sd = float(dmag) * __uint_as_float(0x01000000u);
            if (__float_as_uint(k.divisor) & 0x80000000u) sd = -sd;
            q0 = conv_scale_24(s0) / sd;
            q1 = conv_scale_24(s1) / sd;
            q2 = conv_scale_24(s2) / sd;
            qa = conv_scale_24(s3) / (sd * 255.0f);
        } else if (dmag > 0x7e800000u) {  // huge divisor: both sides reduced by 2^24
            const float inv = 1.0f / conv_unscale_24(k.divisor);
            q0 = conv_unscale_24(s0) * inv;
            q1 = conv_unscale_24(s1) * inv;
            q2 = conv_unscale_24(s2) * inv;
            qa = conv_unscale_24(s3) * inv * CHANNEL_SCALE;
        } else {
            const float rc = 1.0f / k.divisor;
            q0 = s0 * rc;
            q1 = s1 * rc;
            q2 = s2 * rc;
            qa = (s3 * rc) * CHANNEL_SCALE;
        }
        const float ua = k.preserve_alpha ? float(center >> 24) * CHANNEL_SCALE : qa + k.bias;
        const float a = clampf(ua, 0.0f, 1.0f);
        const float bb = k.bias * ua;
        float c0 = q0 + bb, c1 = q1 + bb, c2 = q2 + bb;
        if (k.preserve_alpha) {
            c0 = clampf(c0, 0.0f, 1.0f) * a;
            c1 = clampf(c1, 0.0f, 1.0f) * a;
            c2 = clampf(c2, 0.0f, 1.0f) * a;
        } else {
            c0 = clampf(c0, 0.0f, a);
            c1 = clampf(c1, 0.0f, a);
            c2 = clampf(c2, 0.0f, a);
        }
        dst[o] = pack4(f2u(clampf(c0, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(c1, 0.0f, 1.0f) * 255.0f + 0.5f),
                       f2u(clampf(c2, 0.0f, 1.0f) * 255.0f + 0.5f), f2u(clampf(a, 0.0f, 1.0f) * 255.0f + 0.5f));
    }
}

unsigned filter_grid(uint64_t n) {
    const uint64_t g = (n + 255) / 256;
    return unsigned(g < 148ull * 32 ? (g ? g : 1) : 148ull * 32);
}

}  // namespace

void launch_filter_chain(uint32_t* surface, uint32_t* temp, uint32_t* temp2, const uint32_t* tables, uint32_t width,
                         uint32_t height, const int32_t bounds[4], const tk_filter* chain, uint32_t count,
                         cudaStream_t st) {
    const int4 b = make_int4(bounds[0], bounds[1], bounds[2], bounds[3]);
    if (b.z <= b.x || b.w <= b.y) return;
    const uint64_t n = uint64_t(b.z - b.x) * uint64_t(b.w - b.y);
    for (uint32_t k = 0; k < count; ++k) {
        const tk_filter& f = chain[k];
        if (f.kind == TK_FILTER_OFFSET) {
            if (f.dx == 0 && f.dy == 0) continue;
            k_filter_offset<<<filter_grid(n), 256, 0, st>>>(surface, temp, width, b, f.dx, f.dy);
            k_filter_copy<<<filter_grid(n), 256, 0, st>>>(temp, surface, width, b);
        } else if (f.kind == TK_FILTER_BLUR) {
            // apply_blur at full resolution (blur.rs:194-244): x into the
            // scratch surface, then y back, or the one axis and a copy back
            const float sx = fmaxf(f.std_dev, 0.0f), sy = fmaxf(f.amount, 0.0f);
            if (sx <= 0.0f && sy <= 0.0f) continue;
            BlurParams bp{};
            bp.width = width;
            bp.height = height;
            bp.region[0] = uint32_t(b.x);
            bp.region[1] = uint32_t(b.y);
            bp.region[2] = uint32_t(b.z - b.x);
            bp.region[3] = uint32_t(b.w - b.y);
            bp.bounds[0] = b.x;
            bp.bounds[1] = b.y;
            bp.bounds[2] = b.z;
            bp.bounds[3] = b.w;
            bp.sigma = sx > 0.0f ? sx : sy;
            bp.axis = sx > 0.0f ? 0 : 1;
            launch_blur(surface, temp, bp, st);
            if (sx > 0.0f && sy > 0.0f) {
                bp.sigma = sy;
                bp.axis = 1;
                launch_blur(temp, surface, bp, st);
            } else {
                k_filter_copy<<<filter_grid(n), 256, 0, st>>>(temp, surface, width, b);
            }
        } else if (f.kind == TK_FILTER_CONVOLVE) {
            // ConvolveMatrixToTarget into the scratch surface, copied back (effects.rs:115-133)
            const ConvArgs a{reinterpret_cast<const float*>(tables + f.color), f.columns, f.rows, f.target_x,
                             f.target_y, f.edge_mode, f.preserve_alpha, f.divisor, f.bias};
            k_filter_convolve<<<filter_grid(n), 256, 0, st>>>(surface, temp, width, b, a);
            k_filter_copy<<<filter_grid(n), 256, 0, st>>>(temp, surface, width, b);
        } else if (f.kind == TK_FILTER_FLOOD) {
            k_filter_fill<<<filter_grid(n), 256, 0, st>>>(surface, width, b, f.color);
        } else if (f.kind == TK_FILTER_DROP_SHADOW) {
            k_filter_fill<<<filter_grid(n), 256, 0, st>>>(temp, width, b, 0u);
            k_shadow_mask<<<filter_grid(n), 256, 0, st>>>(surface, temp, width, b, f.dx, f.dy);
            if (f.std_dev > 0.0f && temp2) {
                BlurParams bp{};
                bp.width = width;
                bp.height = height;
                bp.region[0] = uint32_t(b.x);
                bp.region[1] = uint32_t(b.y);
                bp.region[2] = uint32_t(b.z - b.x);
                bp.region[3] = uint32_t(b.w - b.y);
                bp.bounds[0] = b.x;
                bp.bounds[1] = b.y;
                bp.bounds[2] = b.z;
                bp.bounds[3] = b.w;
                bp.sigma = f.std_dev;
                bp.axis = 0;
                launch_blur(temp, temp2, bp, st);
                bp.axis = 1;
                launch_blur(temp2, temp, bp, st);
            }
            k_shadow_composite<<<filter_grid(n), 256, 0, st>>>(surface, temp, width, b, f.color);
        } else if (f.kind == TK_FILTER_ERODE || f.kind == TK_FILTER_DILATE) {
            if (f.dx == 0 && f.dy == 0) continue;
            const uint32_t sw = uint32_t(b.z - b.x), sh = uint32_t(b.w - b.y);
            const uint32_t rx = uint32_t(f.dx), ry = uint32_t(f.dy);
            const bool dilate = f.kind == TK_FILTER_DILATE;
            if (!dilate && (uint64_t(rx) * 2 >= sw || uint64_t(ry) * 2 >= sh)) {
                k_filter_clear<<<filter_grid(n), 256, 0, st>>>(surface, width, b);
                continue;
            }
            k_filter_morphology<<<filter_grid(n), 256, 0, st>>>(surface, temp, width, b, min(rx, sw - 1u), dilate,
                                                                 true);
            k_filter_morphology<<<filter_grid(n), 256, 0, st>>>(temp, surface, width, b, min(ry, sh - 1u), dilate,
                                                                 false);
        } else {
            // this filter and the per-pixel filters right after it, fused
            FilterRun run{};
            for (; k < count && run.n < kFilterRun; ++k) {
                const tk_filter& g = chain[k];
                if (g.kind < TK_FILTER_BRIGHTNESS || (g.kind > TK_FILTER_COLOR_MATRIX &&
                                                      g.kind != TK_FILTER_COMPONENT_TRANSFER))
                    break;
                FilterArgs& a = run.f[run.n++];
                a.kind = g.kind;
                a.amount = g.amount;
                for (int m = 0; m < 20; ++m) a.m[m] = g.matrix[m];
                a.table = g.kind == TK_FILTER_COMPONENT_TRANSFER ? tables + g.color : nullptr;
            }
            --k;  // the loop's increment moves past the run's last filter
            k_filter_color<<<filter_grid(n), 256, 0, st>>>(surface, width, b, run);
        }
    }
}

}  // namespace tk
