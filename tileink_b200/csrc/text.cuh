// Text compositing of glyph outline fills (PTCL_PATH_GLYPH): the coverage
// correction and source-over of fine/text/{gamma,auto,basic}.hlsli.
//
// The shaders' pow is evaluated here by text_pow, in double with exactly
// rounded operations only, so that this file and the oracle's restatement
// give the same bits; the shaders' other steps keep their f32 operation order
// (`lerp(a, b, t)` as a + t (b - a) and `dot` as (x x' + y y') + z z', each
// operation rounded, which is how the shader compiler lowers both).
#pragma once

#include <cstdint>

#include "device.cuh"

namespace tkd {

// x^y for finite x > 0 as exp(y ln x):
//   ln x = e ln 2 + ln m, x = m 2^e with m in [sqrt(1/2), sqrt(2)), and
//   ln m = 2 atanh(s), s = (m - 1) / (m + 1) (|s| <= 0.1716), by the odd
//   series of atanh to s^21;
//   exp t = 2^k exp(r), k = round(t / ln 2), r = t - k ln 2 (Cody-Waite
//   reduction with fdlibm's two-part ln 2, |r| <= 0.347), by the Taylor
//   polynomial of exp to degree 16.
__device__ __forceinline__ float text_pow(float x, float y) {
    int e = 0;
    double m = frexp(double(x), &e);  // m in [0.5, 1)
    if (m < 0.70710678118654752440) {
        m *= 2.0;
        --e;
    }
    const double s = (m - 1.0) / (m + 1.0), s2 = s * s;
    double p = 1.0 / 21.0;
    p = p * s2 + 1.0 / 19.0;
    p = p * s2 + 1.0 / 17.0;
    p = p * s2 + 1.0 / 15.0;
    p = p * s2 + 1.0 / 13.0;
    p = p * s2 + 1.0 / 11.0;
    p = p * s2 + 1.0 / 9.0;
    p = p * s2 + 1.0 / 7.0;
    p = p * s2 + 1.0 / 5.0;
    p = p * s2 + 1.0 / 3.0;
    p = p * s2 + 1.0;
    const double ln2_hi = 6.93147180369123816490e-01, ln2_lo = 1.90821492927058770002e-10;
    const double lnx = (double(e) * ln2_hi + 2.0 * s * p) + double(e) * ln2_lo;
    const double t = double(y) * lnx;
    const double k = rint(t * 1.44269504088896338700);
    const double r = (t - k * ln2_hi) - k * ln2_lo;
    double q = 1.0 / 20922789888000.0;  // 1/16!
    q = q * r + 1.0 / 1307674368000.0;
    q = q * r + 1.0 / 87178291200.0;
    q = q * r + 1.0 / 6227020800.0;
    q = q * r + 1.0 / 479001600.0;
    q = q * r + 1.0 / 39916800.0;
    q = q * r + 1.0 / 3628800.0;
    q = q * r + 1.0 / 362880.0;
    q = q * r + 1.0 / 40320.0;
    q = q * r + 1.0 / 5040.0;
    q = q * r + 1.0 / 720.0;
    q = q * r + 1.0 / 120.0;
    q = q * r + 1.0 / 24.0;
    q = q * r + 1.0 / 6.0;
    q = q * r + 0.5;
    q = q * r + 1.0;
    q = q * r + 1.0;
    return float(ldexp(q, int(k)));
}

// fine/text/gamma.hlsli:5-23
__device__ __forceinline__ float srgb_to_linear(float value) {
    const float v = clampf(value, 0.0f, 1.0f);
    float result = v / 12.92f;
    if (v > 0.04045f) result = text_pow((v + 0.055f) / 1.055f, 2.4f);
    return result;
}
__device__ __forceinline__ float linear_to_srgb(float value) {
    const float v = clampf(value, 0.0f, 1.0f);
    float result = v * 12.92f;
    if (v > 0.0031308f) result = 1.055f * text_pow(v, 1.0f / 2.4f) - 0.055f;
    return result;
}

// text_foreground (fine/text/auto.hlsli:6-9) reduced by the luminance
// weights, as src_over_mask_linear_auto_u8 uses it.
__device__ __forceinline__ float text_foreground_luma(uint32_t source) {
    const float alpha = float(source >> 24);
    if (!(alpha > 0.0f)) return 0.0f;
    const float r = clampf(float(source & 255u) / alpha, 0.0f, 1.0f);
    const float g = clampf(float((source >> 8) & 255u) / alpha, 0.0f, 1.0f);
    const float b = clampf(float((source >> 16) & 255u) / alpha, 0.0f, 1.0f);
    return (r * 0.2126f + g * 0.7152f) + b * 0.0722f;
}

// text_correcting_coverage (fine/text/auto.hlsli:15-26)
__device__ __forceinline__ float text_correcting_coverage(uint32_t coverage, float foreground) {
    if (coverage == 0u || coverage == 255u) return float(coverage) * (1.0f / 255.0f);
    const float raw = float(coverage) * (1.0f / 255.0f);
    const float background = 1.0f - foreground;
    const float bg_linear = srgb_to_linear(background);
    const float enhanced = raw + raw * (1.0f - raw) * bg_linear;
    const float difference = foreground - background;
    if (fabsf(difference) < (1.0f / 256.0f)) return enhanced;
    const float fg_linear = srgb_to_linear(foreground);
    const float output = linear_to_srgb(bg_linear + enhanced * (fg_linear - bg_linear));
    return clampf((output - background) / difference, 0.0f, 1.0f);
}

// src_over_subpixel_mask_f32 (fine/text/basic.hlsli:95-109) with the same
// coverage in all three channels.
__device__ __forceinline__ uint32_t src_over_gray_mask_f32(uint32_t destination, uint32_t source, float coverage) {
    if ((source >> 24) == 0u || coverage == 0.0f) return destination;
    float c = coverage;
    if ((destination >> 24) != 255u) c = (c + c + c) / 3.0f;  // the channel mean
    const float alpha = float(source >> 24) * (1.0f / 255.0f);
    const float amount = alpha * c;
    const float keep = 1.0f - amount;
    const float r = float(source & 255u) * c + float(destination & 255u) * keep;
    const float g = float((source >> 8) & 255u) * c + float((destination >> 8) & 255u) * keep;
    const float b = float((source >> 16) & 255u) * c + float((destination >> 16) & 255u) * keep;
    const float a = amount * 255.0f + float(destination >> 24) * keep;
    return pack4(f2u(r + 0.5f), f2u(g + 0.5f), f2u(b + 0.5f), f2u(a + 0.5f));
}

// src_over_mask_linear_auto_u8 (fine/text/auto.hlsli:28-33)
__device__ __forceinline__ uint32_t src_over_mask_linear_auto_u8(uint32_t destination, uint32_t source,
                                                                  uint32_t coverage) {
    if ((source >> 24) == 0u || coverage == 0u) return destination;
    const float corrected = text_correcting_coverage(coverage, text_foreground_luma(source));
    return src_over_gray_mask_f32(destination, source, corrected);
}

// text_foreground (fine/text/auto.hlsli:6-9)
__device__ __forceinline__ float3 text_foreground(uint32_t source) {
    const float alpha = float(source >> 24);
    if (!(alpha > 0.0f)) return make_float3(0.0f, 0.0f, 0.0f);
    return make_float3(clampf(float(source & 255u) / alpha, 0.0f, 1.0f),
                       clampf(float((source >> 8) & 255u) / alpha, 0.0f, 1.0f),
                       clampf(float((source >> 16) & 255u) / alpha, 0.0f, 1.0f));
}

// src_over_subpixel_mask_f32 (fine/text/basic.hlsli:95-109), one coverage
// per channel.
__device__ __forceinline__ uint32_t src_over_subpixel_mask_f32(uint32_t destination, uint32_t source, float3 cov) {
    if ((source >> 24) == 0u || (cov.x == 0.0f && cov.y == 0.0f && cov.z == 0.0f)) return destination;
    if ((destination >> 24) != 255u) {
        const float gray = (cov.x + cov.y + cov.z) / 3.0f;
        cov = make_float3(gray, gray, gray);
    }
    const float alpha = float(source >> 24) * (1.0f / 255.0f);
    const float ar = alpha * cov.x, ag = alpha * cov.y, ab = alpha * cov.z;
    const float r = float(source & 255u) * cov.x + float(destination & 255u) * (1.0f - ar);
    const float g = float((source >> 8) & 255u) * cov.y + float((destination >> 8) & 255u) * (1.0f - ag);
    const float b = float((source >> 16) & 255u) * cov.z + float((destination >> 16) & 255u) * (1.0f - ab);
    const float maximum = fmaxf(fmaxf(ar, ag), ab);
    const float a = maximum * 255.0f + float(destination >> 24) * (1.0f - maximum);
    return pack4(f2u(r + 0.5f), f2u(g + 0.5f), f2u(b + 0.5f), f2u(a + 0.5f));
}

// src_over_subpixel_mask_u8 with text_subpixel_coverage
// (fine/text/basic.hlsli:9-43): integer subpixel compositing.
__device__ __forceinline__ uint32_t src_over_subpixel_mask_u8(uint32_t dst, uint32_t src, uint32_t mask, uint32_t clip) {
    const uint32_t sa = src >> 24;
    if (sa == 0u || clip == 0u) return dst;
    uint32_t mr = mul_div255(mask & 255u, clip), mg = mul_div255((mask >> 8) & 255u, clip),
             mb = mul_div255((mask >> 16) & 255u, clip);
    if ((dst >> 24) != 255u) mr = mg = mb = (mr + mg + mb + 1u) / 3u;
    if (mr == 0u && mg == 0u && mb == 0u) return dst;
    const uint32_t cr = mul_div255(sa, mr), cg = mul_div255(sa, mg), cb = mul_div255(sa, mb);
    const uint32_t ca = max(max(cr, cg), cb);
    const uint32_t r = mul_div255(src & 255u, mr) + mul_div255(dst & 255u, 255u - cr);
    const uint32_t g = mul_div255((src >> 8) & 255u, mg) + mul_div255((dst >> 8) & 255u, 255u - cg);
    const uint32_t b = mul_div255((src >> 16) & 255u, mb) + mul_div255((dst >> 16) & 255u, 255u - cb);
    const uint32_t a = ca + mul_div255((dst >> 24) & 255u, 255u - ca);
    return pack4(r, g, b, a);
}

// A glyph image's texel, 0 outside it (fine/glyph.hlsli:17-21).
__device__ __forceinline__ uint32_t glyph_texel(const uint32_t* __restrict__ texels, const tk_glyph_image& im,
                                                int32_t x, int32_t y) {
    if (x < 0 || y < 0 || x >= int32_t(im.width) || y >= int32_t(im.height)) return 0u;
    return __ldg(texels + im.data_offset + uint32_t(y) * im.width + uint32_t(x));
}

// sample_glyph (fine/glyph.hlsli:22-30): bilinear in unorm, `lerp(a, b, t)`
// as a + t (b - a).
__device__ __forceinline__ float4 lerp4(float4 a, float4 b, float t) {
    return make_float4(a.x + t * (b.x - a.x), a.y + t * (b.y - a.y), a.z + t * (b.z - a.z), a.w + t * (b.w - a.w));
}
__device__ __forceinline__ uint32_t sample_glyph(const uint32_t* __restrict__ texels, const tk_glyph_image& im, float px,
                                                 float py) {
    const int32_t bx = f2i(floorf(px)), by = f2i(floorf(py));
    const float fx = px - float(bx), fy = py - float(by);
    const uint32_t a = glyph_texel(texels, im, bx, by);
    if (fx == 0.0f && fy == 0.0f) return a;
    const float4 top = lerp4(rgba8_to_unorm(a), rgba8_to_unorm(glyph_texel(texels, im, bx + 1, by)), fx);
    const float4 bottom = lerp4(rgba8_to_unorm(glyph_texel(texels, im, bx, by + 1)),
                                rgba8_to_unorm(glyph_texel(texels, im, bx + 1, by + 1)), fx);
    return unorm_to_rgba8(lerp4(top, bottom, fy));
}

// corrected_glyph_texel and sample_corrected_glyph (fine/glyph.hlsli:32-53)
__device__ __forceinline__ float3 corrected_glyph_texel(uint32_t data, float3 fg, bool lcd) {
    if (!lcd) {
        const float alpha = text_correcting_coverage(data & 255u, (fg.x * 0.2126f + fg.y * 0.7152f) + fg.z * 0.0722f);
        return make_float3(alpha, alpha, alpha);
    }
    return make_float3(text_correcting_coverage(data & 255u, fg.x), text_correcting_coverage((data >> 8) & 255u, fg.y),
                       text_correcting_coverage((data >> 16) & 255u, fg.z));
}
__device__ __forceinline__ float3 lerp3(float3 a, float3 b, float t) {
    return make_float3(a.x + t * (b.x - a.x), a.y + t * (b.y - a.y), a.z + t * (b.z - a.z));
}
__device__ __forceinline__ float3 sample_corrected_glyph(const uint32_t* __restrict__ texels, const tk_glyph_image& im,
                                                         float px, float py, float3 fg, bool lcd) {
    const int32_t bx = f2i(floorf(px)), by = f2i(floorf(py));
    const float fx = px - float(bx), fy = py - float(by);
    const float3 a = corrected_glyph_texel(glyph_texel(texels, im, bx, by), fg, lcd);
    if (fx == 0.0f && fy == 0.0f) return a;
    const float3 top = lerp3(a, corrected_glyph_texel(glyph_texel(texels, im, bx + 1, by), fg, lcd), fx);
    const float3 bottom = lerp3(corrected_glyph_texel(glyph_texel(texels, im, bx, by + 1), fg, lcd),
                                corrected_glyph_texel(glyph_texel(texels, im, bx + 1, by + 1), fg, lcd), fx);
    return lerp3(top, bottom, fy);
}

}  // namespace tkd
