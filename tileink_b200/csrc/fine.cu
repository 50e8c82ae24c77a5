// Fine stage: one CTA of 256 threads per 16x16 tile, one thread per pixel
// (fine/main.hlsl:23-40, fine/interpreter.hlsli:21-219,
// fine/specialized.hlsli:19-45).
//
// The tile's merged PTCL stream is processed in chunks of up to 64 records
// whose fills together reference at most 128 tile segments. Per chunk the CTA
// stages into shared memory, with coalesced loads and no dependent global
// round trips per record:
//   - the records and each fill's paint, one load of the draw's PaintInfo
//     (decoded once per upload by k_paint_table);
//   - the chunk's segments and, per tile row, the compacted list of segments
//     that cross the row (dy != 0) with their terms of segment_row_parts
//     (shared/coverage.hlsli:7-24). A segment crosses 4-5 of the 16 rows on
//     average; in the other rows it adds nothing to `running` or `partial`.
//   - for every crossing (row, segment) the partial-area products
//     segment_area_at(x) * dy of the pixels x in its partial range;
//   - per (record, row) the `base` sum: backdrop plus the row edges in segment
//     order. It is the same f32 sequence for every pixel of a row, and edges
//     of segments that do not touch the tile's left edge are +-0, which leave
//     the sum unchanged.
// Every pixel then accumulates `running` and `partial` in segment order over
// its row's crossing segments exactly as fill_alpha_at
// (shared/coverage.hlsli:34-51) does, so the f32 sums are the reference's.
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.h"
#include "sdf.cuh"
#include "text.cuh"

namespace tk {
namespace {

using namespace tkd;

constexpr int kFineThreads = 256;
constexpr uint32_t kRecChunk = 64;
constexpr uint32_t kSegBudget = 128;
constexpr uint32_t kProdCap = 2560;
static_assert(kRecChunk <= 64u && kSegBudget <= 256u, "offsets are scanned by one warp, two records a lane");
constexpr uint32_t kClipSpill = 28;
constexpr uint32_t kGroupDepth = 6;
constexpr uint32_t kGroupLocal = 2;  // FINE_LOCAL_GROUP_DEPTH (fine/constants.hlsli:11)
constexpr uint32_t kGradient = 0xFFFFFFFFu;
constexpr uint32_t kGradParams = 24;
constexpr uint32_t kGradConst = 0, kGradLinear = 1, kGradRadial = 2, kGradPattern = 3;  // decoded kinds
constexpr uint32_t kGradBilinear = 1u << 16;  // pattern: bilinear sampling
constexpr uint32_t kGradDenOk = 1u << 16;    // linear: den > GRADIENT_FLOAT_EPSILON
constexpr uint32_t kGradASmall = 1u << 16;   // radial: |a| <= RADIAL_QUADRATIC_EPSILON

// Record classes driving the per-pixel dispatch.
constexpr uint32_t kClsOther = 0, kClsFill = 1, kClsUniform = 2, kClsBatch = 3, kClsEnd = 4;

struct Group {
    uint32_t kind;
    float4 parent;
    uint32_t parent_clip, layer_alpha, payload;
};

// Crossing entry word: plo | phi << 5 | kEntSlow | (prod offset, or with
// kEntSlow the staged segment index) << 16, where [plo, phi) is the partial
// pixel range [clamp(floor(xmin)), clamp(ceil(xmax))) within [0, 16].
constexpr uint32_t kEntSlow = 1u << 10;  // products did not fit: evaluate per pixel

struct FineSmem {
    float2 ent[TK_TILE_SIZE][kSegBudget];        // crossing (row, segment) entries: dy, entry word
    uint16_t pos[TK_TILE_SIZE][kSegBudget + 1];  // crossing entries before staged segment j
    float prod[kProdCap];                        // segment_area_at(x) * dy per partial pixel
    float4 sgp[kSegBudget];                      // staged segments: p0x, p0y, p1x, p1y
    float2 sgx[kSegBudget];                      // y_edge, slope = (p1x - p0x) / (p1y - p0y)
    uint16_t rmask[kSegBudget];                  // rows the staged segment crosses (dy != 0)
    uint16_t rpre[kSegBudget + 1];               // crossings of staged segments before j
    float2 rb[kRecChunk][TK_TILE_SIZE];          // per (fill, row): base, k0 | k1 << 16
    float4 pfull[kRecChunk];                     // rgba8_to_unorm(paint) / uniform source
    float4 pcf[kRecChunk];                       // paint channels as floats
    uint4 rec_a[kRecChunk];                      // tag, backdrop, fill_rule, segment_start
    uint2 rec_b[kRecChunk];                      // segment_end, color
    uint32_t cls[kRecChunk];
    uint32_t ualpha[kRecChunk];
    uint32_t umode[kRecChunk];                   // uniform fills: 1 replace, 2 src-over, 3 no-op;
                                                 // SDF records: first word of the shape
    uint32_t paint[kRecChunk];                   // solid premul color, or kGradient
    alignas(16) float gp[kRecChunk][kGradParams];  // gradient terms of the chunk's fills (PaintInfo::g)
    uint4 gk[kRecChunk];                         // kind | flags, ramp word (or color), ramp length, extend
    uint32_t nseg[kRecChunk];
    uint32_t off[kRecChunk + 1];
    float unorm[256];                            // k / 255 for RGBA8 texel reloads
    uint32_t n, nprod;
};

__device__ __forceinline__ bool is_fill_like(uint32_t tag) {
    return tag == TK_PTCL_FILL || tag == TK_PTCL_BEGIN_CLIP || tag == TK_PTCL_BEGIN_OPACITY ||
           tag == TK_PTCL_BEGIN_BLEND || tag == TK_PTCL_PATH_GLYPH;
}

__device__ __forceinline__ float4 texel_load_lut(const FineSmem& S, uint32_t p) {
    return make_float4(S.unorm[p & 255u], S.unorm[(p >> 8) & 255u], S.unorm[(p >> 16) & 255u], S.unorm[p >> 24]);
}

// Decodes the gradient brush at word `db` of a fill whose draw has the inverse
// transform `m` into g[0..23] and gk: the transforms, and the terms of
// sample_gradient (fine/paint.hlsli:40-96) that depend on the brush alone,
// computed with the same f32 operations so that the per-pixel evaluation in
// gradient_at gives the same bits.
//   linear: gp[12..16] = sx, sy, dx = ex - sx, dy = ey - sy, den = dx*dx + dy*dy
//   radial: gp[12..22] = sx, sy, dcx, dcy, sr*dr, -sr*sr, a, -4*a, 2*a, dr, sr
//           with a = mad(dcx, dcx, mad(dcy, dcy, -dr*dr))
__device__ void decode_gradient(float* g, uint4& gk, const Paint& P, uint32_t db, const float* __restrict__ m,
                                const uint4* __restrict__ images, uint32_t image_count) {
#pragma unroll
    for (int k = 0; k < 6; ++k) g[k] = __ldg(m + k);
    const uint32_t kind = P.word(db), extend = P.word(db + 1u);
    const uint32_t payload = db + P.word(db + 2u);
    uint32_t len = P.word(db + 3u);
    const uint32_t base = db + TK_BRUSH_HEADER_WORDS;
    uint32_t code = kGradConst, flags = 0u, word = 0u;
    if (kind == TK_BRUSH_LINEAR) {
        code = kGradLinear;
        for (uint32_t k = 0; k < 6u; ++k) g[6 + k] = P.param(base, 4u + k);
        const float sx = P.param(base, 0), sy = P.param(base, 1), ex = P.param(base, 2), ey = P.param(base, 3);
        const float dx = ex - sx, dy = ey - sy;
        const float den = dx * dx + dy * dy;
        g[12] = sx;
        g[13] = sy;
        g[14] = dx;
        g[15] = dy;
        g[16] = den;
        if (den > GRADIENT_FLOAT_EPSILON) flags = kGradDenOk;
        word = payload;
    } else if (kind == TK_BRUSH_RADIAL) {
        code = kGradRadial;
        for (uint32_t k = 0; k < 6u; ++k) g[6 + k] = P.param(base, 6u + k);
        const float sx = P.param(base, 0), sy = P.param(base, 1), ex = P.param(base, 2), ey = P.param(base, 3);
        const float sr = P.param(base, 4), er = P.param(base, 5);
        const float dcx = ex - sx, dcy = ey - sy, dr = er - sr;
        const float a = mad(dcx, dcx, mad(dcy, dcy, -dr * dr));
        g[12] = sx;
        g[13] = sy;
        g[14] = dcx;
        g[15] = dcy;
        g[16] = sr * dr;
        g[17] = -sr * sr;
        g[18] = a;
        g[19] = -4.0f * a;
        g[20] = 2.0f * a;
        g[21] = dr;
        g[22] = sr;
        if (fabsf(a) <= RADIAL_QUADRATIC_EPSILON) flags = kGradASmall;
        word = payload;
    } else if (kind == TK_BRUSH_PATTERN_RESOURCE) {
        // sample_brush's texture-table branch (shared/brush/sample.hlsli:32-41):
        //   gp[6..11] the pattern transform, gp[12..13] the size as floats,
        //   gp[14..15] the size as integers; gk = kind, first texel, opacity, extend
        const uint32_t placement = P.word(db + 4u), w = P.word(db + 5u), h = P.word(db + 6u);
        const uint32_t ix = placement & ~TK_BRUSH_TEXTURE_PLACEMENT_BIT;
        if (w != 0u && h != 0u && (placement & TK_BRUSH_TEXTURE_PLACEMENT_BIT) && ix < image_count) {
            code = kGradPattern;
            for (uint32_t k = 0; k < 6u; ++k) g[6 + k] = P.param(base, k);
            g[12] = float(w);
            g[13] = float(h);
            g[14] = __uint_as_float(w);
            g[15] = __uint_as_float(h);
            if (P.word(db + 8u) == TK_PATTERN_BILINEAR) flags = kGradBilinear;
            word = images[ix].x;
            len = P.word(db + TK_BRUSH_IMAGE_ALPHA_WORD);
        }
    } else {
        word = kind == 6u ? 0u : P.word(db + TK_BRUSH_COLOR_WORD);  // BRUSH_PATTERN samples as 0
    }
    gk = make_uint4(code | flags, word, len, extend);
}

// One thread per draw: the draw's PaintInfo (solid colour, or the decoded
// gradient of its brush under its inverse transform).
__global__ void k_paint_table(const tk_draw_record* __restrict__ draws, uint32_t n, const uint32_t* __restrict__ brush,
                              uint64_t brush_words, uint32_t sdf_shadow_base, const uint4* __restrict__ images,
                              uint32_t image_count, PaintInfo* out) {
    const uint32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    const Paint P{brush, brush_words};
    const uint32_t bo = draws[d].brush_offset;
    PaintInfo info{};
    // sdf_coverage_from_draw (fine/draw.hlsli:21-26): the SDF record, else the shadow record
    const uint32_t so = draws[d].sdf_offset, ho = draws[d].sdf_shadow_offset;
    info.sdf = so != TK_INVALID_INDEX ? so : (ho != TK_INVALID_INDEX ? sdf_shadow_base + ho : TK_INVALID_INDEX);
    if (P.word(bo) == TK_BRUSH_SOLID) {
        info.paint = P.word(bo + TK_BRUSH_COLOR_WORD);
    } else {
        info.paint = kGradient;
        decode_gradient(info.g, info.gk, P, bo, &draws[d].inverse_transform.a, images, image_count);
    }
    out[d] = info;
}

// extend_coord_i32 (shared/brush/pattern.hlsli:9-17) with
// euclidean_remainder_i32 (shared/integer.hlsli:5-9).
__device__ __forceinline__ uint32_t extend_coord(int32_t v, uint32_t size, uint32_t extend) {
    if (size <= 1u) return 0u;
    if (extend == TK_EXTEND_REPEAT || extend == TK_EXTEND_REFLECT) {
        const uint32_t period = size * (extend == TK_EXTEND_REFLECT ? 2u : 1u);
        const uint32_t mag = v < 0 ? 0u - uint32_t(v) : uint32_t(v), rem = mag % period;
        const uint32_t coord = v < 0 && rem != 0u ? period - rem : rem;
        return coord < size ? coord : period - coord - 1u;
    }
    return uint32_t(min(max(v, 0), int32_t(size) - 1));
}

// lerp_premul_u8 (shared/pixel.hlsli:55-62): one fused interpolation per channel.
__device__ __forceinline__ uint32_t lerp_premul_u8(uint32_t a, uint32_t b, float t) {
    uint32_t out = 0u;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float l = float((a >> (8 * c)) & 255u), r = float((b >> (8 * c)) & 255u);
        out |= f2u(clampf(mad(r - l, t, l) + 0.5f, 0.0f, 255.0f)) << (8 * c);
    }
    return out;
}

// The image pattern decoded in g / k at brush-space point (x, y):
// pattern_transform_component (shared/pattern_transform.hlsli:7-11) and
// sample_resource_pattern_texture (shared/brush/texture.hlsli:11-31). Float to
// integer conversions saturate and take NaN to 0. The bilinear, pad-extended
// form is the texture unit's filter in the reference (SampleLevel with
// clamp-to-edge addressing); here it is that filter computed exactly: texel
// centres at half-integers, f32 weights, one rounding to 8 bits.
__device__ __noinline__ uint32_t pattern_at(const Paint& P, const float* g, uint4 k, float x, float y) {
    const float bx = g[8] * y, by = g[9] * y;
    const float tx = ((mad(g[6], x, bx) + mad(g[8], y, -bx)) + g[10]) * g[12];
    const float ty = ((mad(g[7], x, by) + mad(g[9], y, -by)) + g[11]) * g[13];
    const uint32_t w = __float_as_uint(g[14]), h = __float_as_uint(g[15]), extend = k.w;
    const uint32_t* __restrict__ tex = P.texels + k.y;
    uint32_t color;
    if ((k.x & kGradBilinear) && extend == TK_EXTEND_PAD) {
        const float sx = clampf(tx, 0.0f, g[12]) - 0.5f, sy = clampf(ty, 0.0f, g[13]) - 0.5f;
        const float fx0 = floorf(sx), fy0 = floorf(sy), fx = sx - fx0, fy = sy - fy0;
        const int32_t ix = __float2int_rz(fx0), iy = __float2int_rz(fy0);
        const uint32_t x0 = uint32_t(min(max(ix, 0), int32_t(w) - 1)), x1 = uint32_t(min(max(ix + 1, 0), int32_t(w) - 1));
        const uint32_t y0 = uint32_t(min(max(iy, 0), int32_t(h) - 1)), y1 = uint32_t(min(max(iy + 1, 0), int32_t(h) - 1));
        const float4 tl = rgba8_to_unorm(__ldg(tex + uint64_t(y0) * w + x0)), tr = rgba8_to_unorm(__ldg(tex + uint64_t(y0) * w + x1));
        const float4 bl = rgba8_to_unorm(__ldg(tex + uint64_t(y1) * w + x0)), br = rgba8_to_unorm(__ldg(tex + uint64_t(y1) * w + x1));
        const float4 top = make_float4(mad(tr.x - tl.x, fx, tl.x), mad(tr.y - tl.y, fx, tl.y), mad(tr.z - tl.z, fx, tl.z),
                                       mad(tr.w - tl.w, fx, tl.w));
        const float4 bot = make_float4(mad(br.x - bl.x, fx, bl.x), mad(br.y - bl.y, fx, bl.y), mad(br.z - bl.z, fx, bl.z),
                                       mad(br.w - bl.w, fx, bl.w));
        color = unorm_to_rgba8(make_float4(mad(bot.x - top.x, fy, top.x), mad(bot.y - top.y, fy, top.y),
                                           mad(bot.z - top.z, fy, top.z), mad(bot.w - top.w, fy, top.w)));
    } else if (k.x & kGradBilinear) {
        const float sx = tx - 0.5f, sy = ty - 0.5f;
        const float fx0 = floorf(sx), fy0 = floorf(sy), fx = sx - fx0, fy = sy - fy0;
        const int32_t ix = __float2int_rz(fx0), iy = __float2int_rz(fy0);
        const int32_t jx = int32_t(uint32_t(ix) + 1u), jy = int32_t(uint32_t(iy) + 1u);
        const uint64_t r0 = uint64_t(extend_coord(iy, h, extend)) * w, r1 = uint64_t(extend_coord(jy, h, extend)) * w;
        const uint32_t c0 = extend_coord(ix, w, extend), c1 = extend_coord(jx, w, extend);
        const uint32_t top = lerp_premul_u8(__ldg(tex + r0 + c0), __ldg(tex + r0 + c1), fx);
        const uint32_t bot = lerp_premul_u8(__ldg(tex + r1 + c0), __ldg(tex + r1 + c1), fx);
        color = lerp_premul_u8(top, bot, fy);
    } else {
        const uint32_t c = extend_coord(__float2int_rz(floorf(tx)), w, extend);
        const uint32_t r = extend_coord(__float2int_rz(floorf(ty)), h, extend);
        color = __ldg(tex + uint64_t(r) * w + c);
    }
    return scale_premul_u8(color, k.z);
}

// sample_gradient at pixel centre (px, py) for the gradient decoded in slot i.
// IMG: whether image patterns can occur (only SDF draws carry them).
template <bool IMG>
__device__ __forceinline__ uint32_t gradient_at(const FineSmem& S, const Paint& P, uint32_t i, float px, float py) {
    const float* g = S.gp[i];
    const uint4 k = S.gk[i];
    const uint32_t code = k.x & 255u, extend = k.w;
    if (code == kGradConst) return k.y;
    const float x = mad(g[0], px, mad(g[2], py, g[4]));
    const float y = mad(g[1], px, mad(g[3], py, g[5]));
    if (IMG && code == kGradPattern) return pattern_at(P, g, k, x, y);
    const float tx = mad(g[6], x, mad(g[8], y, g[10]));
    const float ty = mad(g[7], x, mad(g[9], y, g[11]));
    float t = 0.0f;
    if (code == kGradLinear) {
        if (k.x & kGradDenOk) t = mad(tx - g[12], g[14], (ty - g[13]) * g[15]) / g[16];
    } else {
        const float qx = tx - g[12], qy = ty - g[13];
        const float b = -2.0f * mad(qx, g[14], mad(qy, g[15], g[16]));
        const float c = mad(qx, qx, mad(qy, qy, g[17]));
        const float dr = g[21], sr = g[22];
        bool has_t = false;
        if (k.x & kGradASmall) {
            if (fabsf(b) > RADIAL_QUADRATIC_EPSILON) {
                const float cand = -c / b;
                if (mad(cand, dr, sr) >= 0.0f) {
                    has_t = true;
                    t = cand;
                }
            }
        } else {
            const float disc = mad(b, b, g[19] * c);
            if (disc >= 0.0f) {
                const float root = sqrtf(disc);
                const float t0 = (-b - root) / g[20], t1 = (-b + root) / g[20];
                const bool v0 = mad(t0, dr, sr) >= 0.0f, v1 = mad(t1, dr, sr) >= 0.0f;
                if (v0) {
                    has_t = true;
                    t = v1 ? fmaxf(t0, t1) : t0;
                } else if (v1) {
                    has_t = true;
                    t = t1;
                }
            }
        }
        if (!has_t) return 0u;
    }
    return sample_ramp(P, k.y, k.z, t, extend);
}

// segment_row_parts (shared/coverage.hlsli:7-24) of staged segment j for
// tile row `row`, with the slope division done once per segment at staging.
__device__ __forceinline__ RowParts staged_row_parts(const FineSmem& S, uint32_t j, uint32_t row) {
    const float4 g = S.sgp[j];
    const float row_y = float(row), local_y = g.y - row_y, far_y = g.w - row_y;
    const float y0 = clampf(local_y, 0.0f, 1.0f), y1 = clampf(far_y, 0.0f, 1.0f);
    const float dy = y0 - y1;
    if (dy == 0.0f) return {0.0f, dy, 0.0f, 0.0f};
    const float slope = S.sgx[j].y;
    const bool nearer_p0 = fabsf(local_y - 0.5f) <= fabsf(far_y - 0.5f);
    const float anchor_x = nearer_p0 ? g.x : g.z;
    const float anchor_y = nearer_p0 ? local_y : far_y;
    const float sx0 = mad(y0 - anchor_y, slope, anchor_x);
    const float sx1 = mad(y1 - anchor_y, slope, anchor_x);
    return {0.0f, dy, fminf(sx0, sx1), fmaxf(sx0, sx1)};
}

// The rows a segment crosses, i.e. where segment_row_parts gives dy != 0:
// with lo < hi the segment's y extent, clamp(y - row, 0, 1) differs between
// its ends exactly for rows floor(lo) .. ceil(hi) - 1 (y - row is exact for y
// in [row, row + 1], and rounds to the same side of that interval otherwise).
__device__ __forceinline__ uint32_t crossed_rows(float p0y, float p1y) {
    const float lo = fminf(p0y, p1y), hi = fmaxf(p0y, p1y);
    if (!(lo < hi)) return 0u;
    const int32_t r0 = max(f2i(floorf(lo)), 0), r1 = min(f2i(ceilf(hi)) - 1, int32_t(TK_TILE_SIZE) - 1);
    if (r1 < r0) return 0u;
    return ((2u << r1) - 1u) & ~((1u << r0) - 1u);
}

// Crossing lists and partial products for staged segments [0, total) of the
// chunk's first n records, and the per (fill, row) base sums.
// Positions: warp w ranks rows 2w and 2w + 1, lanes walk the segments in
// order and rank the crossing ones by ballot (warp 0 also prefixes the
// segments' crossing counts). Entries: the (segment, row) crossings are spread
// evenly over the CTA, and only they evaluate segment_row_parts and their
// partial-area products.
__device__ void stage_rows(FineSmem& S, uint32_t total, uint32_t n) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    for (uint32_t rr = 0; rr < 2u; ++rr) {
        const uint32_t row = warp * 2u + rr;
        uint32_t count = 0;
        for (uint32_t j0 = 0; j0 < total; j0 += 32u) {
            const uint32_t j = j0 + lane;
            const bool crossing = j < total && ((S.rmask[j] >> row) & 1u);
            const uint32_t ballot = __ballot_sync(0xffffffffu, crossing);
            if (j < total) S.pos[row][j] = uint16_t(count + __popc(ballot & lt));
            count += __popc(ballot);
        }
        if (lane == 0) S.pos[row][total] = uint16_t(count);
    }
    if (warp == 0) {
        uint32_t run = 0;
        for (uint32_t j0 = 0; j0 < total; j0 += 32u) {
            const uint32_t j = j0 + lane;
            const uint32_t c = j < total ? __popc(S.rmask[j]) : 0u;
            uint32_t incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= uint32_t(d)) incl += v;
            }
            if (j < total) S.rpre[j] = uint16_t(run + incl - c);
            run += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) S.rpre[total] = uint16_t(run);
    }
    __syncthreads();
    // per (fill, row): the base sum and the row's entry range (needs the
    // positions only, so it shares this phase with the entries below)
    for (uint32_t k = threadIdx.x; k < n * TK_TILE_SIZE; k += kFineThreads) {
        const uint32_t ri = k >> 4, row = k & 15u;
        const uint32_t j0 = S.off[ri], ns = S.nseg[ri];
        if (ns == 0u) continue;
        float bsum = float(int32_t(S.rec_a[ri].y));
        for (uint32_t j = j0; j < j0 + ns; ++j) {
            const float ye = S.sgx[j].x;
            if (ye < 1000000000.0f) {  // y_edge set: the segment touches the tile's left edge
                const float4 g = S.sgp[j];
                bsum += signum_f32(g.z - g.x) * clampf(float(row) - ye + 1.0f, 0.0f, 1.0f);
            }
        }
        const uint32_t k0 = S.pos[row][j0], k1 = S.pos[row][j0 + ns];
        S.rb[ri][row] = make_float2(bsum, __uint_as_float(k0 | (k1 << 16)));
    }
    const uint32_t items = S.rpre[total];
    for (uint32_t it = threadIdx.x; it < items; it += kFineThreads) {
        uint32_t lo = 0, hi = total;  // staged segment j with rpre[j] <= it < rpre[j + 1]
        while (hi - lo > 1u) {
            const uint32_t mid = (lo + hi) >> 1;
            if (S.rpre[mid] <= it) lo = mid;
            else hi = mid;
        }
        const uint32_t j = lo;
        uint32_t m = S.rmask[j];  // the row of this crossing: its (it - rpre[j])-th set bit
        for (uint32_t k = it - S.rpre[j]; k; --k) m &= m - 1u;
        const uint32_t row = uint32_t(__ffs(m) - 1);
        const RowParts rp = staged_row_parts(S, j, row);
        const uint32_t plo = uint32_t(min(max(f2i(floorf(rp.xmin)), 0), int32_t(TK_TILE_SIZE)));
        const uint32_t phi = uint32_t(min(max(f2i(ceilf(rp.xmax)), 0), int32_t(TK_TILE_SIZE)));
        const uint32_t span = phi > plo ? phi - plo : 0u;
        uint32_t word = plo | (phi << 5);
        const uint32_t o = span ? atomicAdd(&S.nprod, span) : 0u;
        if (o + span <= kProdCap) {
            for (uint32_t x = 0; x < span; ++x) S.prod[o + x] = segment_area_at(rp.xmin, rp.xmax, plo + x) * rp.dy;
            word |= o << 16;
        } else {
            word |= kEntSlow | (j << 16);
        }
        S.ent[row][S.pos[row][j]] = make_float2(rp.dy, __uint_as_float(word));
    }
}

// fill_alpha_at's coverage sum (shared/coverage.hlsli:34-51) of staged fill
// i at pixel (lx, ly): base + running + partial over the row's crossing
// entries in segment order.
__device__ __forceinline__ float staged_coverage(const FineSmem& S, uint32_t i, uint32_t lx, uint32_t ly) {
    float running = 0.0f, partial = 0.0f;
    const float2* row = S.ent[ly];
    const float2 rb = S.rb[i][ly];
    const uint32_t kk = __float_as_uint(rb.y);
    for (uint32_t k = kk & 0xFFFFu, k1 = kk >> 16; k < k1; ++k) {
        const float2 e = row[k];
        const uint32_t pk = __float_as_uint(e.y);
        const uint32_t plo = pk & 31u, phi = (pk >> 5) & 31u;
        if (lx >= phi) running += e.x;
        if (lx >= plo && lx < phi) {
            if (!(pk & kEntSlow)) {
                partial += S.prod[(pk >> 16) + lx - plo];
            } else {
                const RowParts q = staged_row_parts(S, pk >> 16, ly);
                partial += segment_area_at(q.xmin, q.xmax, lx) * q.dy;
            }
        }
    }
    return rb.x + running + partial;
}

// Analytic coverage of the SDF record `w` at the centre of pixel (gx, gy)
// mapped to draw space by the draw's inverse transform (affine_record_point,
// shared/affine.hlsli:14-18). Inlined: an out-of-line call costs the record
// loop more (register saves around the call) than the shape switch does.
template <bool EXT>
static __device__ __forceinline__ float sdf_coverage_at(const uint32_t* w, const tk_affine* t, uint32_t gx, uint32_t gy) {
    const tk_affine inv{__ldg(&t->a), __ldg(&t->b), __ldg(&t->c), __ldg(&t->d), __ldg(&t->e), __ldg(&t->f)};
    const float sx = float(gx) + 0.5f, sy = float(gy) + 0.5f;
    const float ux = __fmaf_rn(inv.a, sx, __fmaf_rn(inv.c, sy, inv.e));
    const float uy = __fmaf_rn(inv.b, sx, __fmaf_rn(inv.d, sy, inv.f));
    return sdf_coverage<EXT>(w, ux, uy, inv);
}

// Paints a fill's masked coverage over px (the brush branch of
// fine/interpreter.hlsli's fill handling, fine/draw.hlsli:16-21).
template <bool IMG>
__device__ __forceinline__ void paint_fill(const FineSmem& S, const Paint& P, uint32_t i, uint32_t masked,
                                           uint32_t gx, uint32_t gy, float4& px) {
    const uint32_t paint = S.paint[i];
    if (paint != kGradient) {
        if (masked == 255u && premul_u8_is_opaque(paint)) {
            px = S.pfull[i];
        } else {
            // scale_premul_u8_to_unorm with the channels staged as floats
            const float sc = float(masked) * (1.0f / 65025.0f);
            const float4 c = S.pcf[i];
            if (c.w != 0.0f) px = src_over_premul_unorm(px, make_float4(c.x * sc, c.y * sc, c.z * sc, c.w * sc));
        }
    } else {
        const uint32_t g = gradient_at<IMG>(S, P, i, float(gx) + 0.5f, float(gy) + 0.5f);
        if (masked == 255u && premul_u8_is_opaque(g)) px = rgba8_to_unorm(g);
        else px = src_over_premul_unorm(px, scale_premul_u8_to_unorm(g, masked));
    }
}

// Paints a glyph outline fill's masked coverage over px: the brush colour
// composited by src_over_mask_linear_auto_u8 on the stored RGBA8 value
// (fine/interpreter.hlsli:205-206).
// Out of line: glyph fills are rare outside text, and the double-precision
// pow would otherwise weigh on the record loop's registers.
template <bool IMG>
__device__ __noinline__ float4 paint_glyph_fill(const FineSmem& S, const Paint P, uint32_t i, uint32_t masked,
                                                uint32_t gx, uint32_t gy, float4 px) {
    const uint32_t paint = S.paint[i];
    const uint32_t color =
        paint != kGradient ? paint : gradient_at<IMG>(S, P, i, float(gx) + 0.5f, float(gy) + 0.5f);
    return rgba8_to_unorm(src_over_mask_linear_auto_u8(unorm_to_rgba8(px), color, masked));
}

// The text blob as fine raster reads it: the pass's glyph lists, the glyph
// records, the glyph images and their texels.
struct GlyphView {
    const uint32_t* list;
    const tk_glyph* glyphs;
    const tk_glyph_image* images;
    const uint32_t* texels;
};

// composite_glyphs_at (fine/glyph.hlsli:55-111): the glyphs list[g0, g1) of
// a glyph run draw over px at pixel (gx, gy), each by its image's content.
// Out of line like the glyph outline paint.
template <bool IMG>
__device__ __noinline__ float4 composite_glyphs(const FineSmem& S, const Paint P, uint32_t i, const GlyphView G,
                                                const tk_draw_record* dr, uint32_t g0, uint32_t g1, uint32_t gx,
                                                uint32_t gy, uint32_t clip, float4 px) {
    const tk_affine& t = dr->inverse_transform;
    const float a = __ldg(&t.a), b = __ldg(&t.b), c = __ldg(&t.c), d = __ldg(&t.d), e = __ldg(&t.e), f = __ldg(&t.f);
    const float sx = float(gx) + 0.5f, sy = float(gy) + 0.5f;
    const float lx = __fmaf_rn(a, sx, __fmaf_rn(c, sy, e)) - 0.5f;
    const float ly = __fmaf_rn(b, sx, __fmaf_rn(d, sy, f)) - 0.5f;
    for (uint32_t g = g0; g < g1; ++g) {
        const tk_glyph glyph = G.glyphs[__ldg(G.list + g)];
        if (glyph.image == TK_INVALID_INDEX) continue;
        const tk_glyph_image im = G.images[glyph.image];
        const int32_t x0 = int32_t(uint32_t(glyph.x) + uint32_t(im.left));
        const int32_t y0 = int32_t(uint32_t(glyph.y) - uint32_t(im.top));
        const float ux = lx - float(x0), uy = ly - float(y0);
        if (!(ux > -1.0f && uy > -1.0f && ux < float(int32_t(im.width)) && uy < float(int32_t(im.height)))) continue;
        const uint32_t content = im.content;
        auto brush = [&]() {
            const uint32_t paint = S.paint[i];
            return paint != kGradient ? paint : gradient_at<IMG>(S, P, i, sx, sy);
        };
        if (content == TK_GLYPH_LINEAR_MASK || content == TK_GLYPH_LINEAR_SUBPIXEL_MASK) {
            const uint32_t color = brush();
            float3 cov = sample_corrected_glyph(G.texels, im, ux, uy, text_foreground(color),
                                                content == TK_GLYPH_LINEAR_SUBPIXEL_MASK);
            const float k = float(clip) * (1.0f / 255.0f);
            cov = make_float3(cov.x * k, cov.y * k, cov.z * k);
            px = rgba8_to_unorm(src_over_subpixel_mask_f32(unorm_to_rgba8(px), color, cov));
        } else {
            const uint32_t data = sample_glyph(G.texels, im, ux, uy);
            if (content == TK_GLYPH_MASK) {
                const uint32_t alpha = combine_alpha(data, clip);
                if (alpha != 0u) px = src_over_premul_unorm(px, scale_premul_u8_to_unorm(brush(), alpha));
            } else if (content == TK_GLYPH_COLOR) {
                px = src_over_premul_unorm(px, scale_premul_u8_to_unorm(data, clip));
            } else if (content == TK_GLYPH_LINEAR_COLOR) {
                px = rgba8_to_unorm(src_over_mask_linear_auto_u8(unorm_to_rgba8(px), data, clip));
            } else if (content == TK_GLYPH_SUBPIXEL_MASK) {
                px = rgba8_to_unorm(src_over_subpixel_mask_u8(unorm_to_rgba8(px), brush(), data, clip));
            }
        }
    }
    return px;
}

// SDF: 0 for scenes without SDF records, 1 with SDF records of the base
// kinds, 2 with the extended kinds (candlestick, dash line, triangle,
// checkerboard). Path-only scenes run the instance without the PTCL_SDF
// branch, which costs the record loop about 3% even when never taken; the
// extended kinds' code costs the base kinds more, so it has its own instance,
// with the registers of 3 CTAs per SM.
// TEXT: the scene has glyph outline fills or glyph runs; their compositing
// runs out of line, and only this instance holds the calls, so that scenes
// without text keep the record loop's registers.
template <uint32_t SDF, bool TEXT>
__global__ void __launch_bounds__(kFineThreads, SDF == 2u ? 3 : 4)
    k_fine(const tk_tile_record* __restrict__ tiles, const tk_ptcl_record* __restrict__ ptcl,
           const SegmentRec* __restrict__ segments, const PaintInfo* __restrict__ paints,
           const uint32_t* __restrict__ brush, uint64_t brush_words, const uint32_t* __restrict__ texels,
           const tk_draw_record* __restrict__ draws, const uint32_t* __restrict__ sdf, uint64_t seg_capacity, uint32_t* target,
           uint32_t width, uint32_t height, uint32_t tw, uint32_t* error, const BatchScene* __restrict__ scenes,
           const uint32_t* __restrict__ tile_scene, const uint32_t* __restrict__ tile_list, const GlyphView glyphs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FineSmem& S = *reinterpret_cast<FineSmem*>(smem_raw);
    const uint32_t tile = tile_list ? tile_list[blockIdx.x] : blockIdx.x;
    const tk_tile_record rec = tiles[tile];
    if (rec.ptcl_start >= rec.ptcl_end) return;
    uint32_t ltile = tile;
    if (scenes) {  // batched pass: this tile's canvas and image
        const BatchScene& sc = scenes[tile_scene[tile]];
        ltile = tile - sc.tile_base;
        tw = sc.tw;
        width = sc.width;
        height = sc.height;
        target += sc.image_offset;
    }
    const uint32_t tid = threadIdx.x;
    const uint32_t lx = tid & 15u, ly = tid >> 4;
    const uint32_t gx = (ltile % tw) * TK_TILE_SIZE + lx, gy = (ltile / tw) * TK_TILE_SIZE + ly;
    const bool inside = gx < width && gy < height;
    const uint64_t pix = uint64_t(gy) * width + gx;
    const Paint P{brush, brush_words, texels};
    S.unorm[tid] = float(tid) / 255.0f;
    __syncthreads();
    float4 px = inside ? texel_load_lut(S, target[pix]) : make_float4(0.f, 0.f, 0.f, 0.f);

    uint32_t clip = 255u, cdepth = 0u, cregs = 0u;
    uint32_t cspill[kClipSpill];
    Group groups[kGroupDepth];
    uint32_t gdepth = 0u;
    uint32_t mode = TK_TILE_KIND_INTERPRETER;

    uint64_t r = rec.ptcl_start;
    const uint64_t end = rec.ptcl_end;
    bool done = false;
    while (r < end && !done) {
        // ---- stage a chunk of records ----------------------------------------
        __syncthreads();
        const uint32_t avail = uint32_t(min(uint64_t(kRecChunk), end - r));
        if (tid < avail) {
            const uint2* w = reinterpret_cast<const uint2*>(ptcl + r + tid);
            const uint2 a = __ldg(w), b = __ldg(w + 1), c = __ldg(w + 2);
            S.rec_a[tid] = make_uint4(a.x, a.y, b.x, b.y);
            S.rec_b[tid] = c;
            uint32_t n = 0, cls = kClsOther;
            if (a.x == TK_PTCL_END) cls = kClsEnd;
            else if (a.x == TK_PTCL_BATCH_BEGIN) cls = kClsBatch;
            if (is_fill_like(a.x)) {
                uint32_t s0 = b.y, s1 = c.x;
                if (s1 > seg_capacity || s0 > s1) {  // inconsistent scan inputs
                    atomicOr(error, ERR_SEGMENT_OVERFLOW);
                    s1 = s0 > seg_capacity ? s0 : uint32_t(seg_capacity);
                    if (s0 > s1) s1 = s0;
                    S.rec_b[tid].x = s1;
                }
                n = s1 - s0;
                if (n == 0u) S.ualpha[tid] = coverage_to_alpha(float(int32_t(a.y)), b.x);
                if (a.x == TK_PTCL_FILL && n != 0u) cls = kClsFill;  // row sums staged below
            }
            S.nseg[tid] = n;
            if (SDF != 0u && a.x == TK_PTCL_BEGIN_SDF_CLIP) S.umode[tid] = __ldg(&paints[c.y].sdf);
            if (a.x == TK_PTCL_FILL || a.x == TK_PTCL_PATH_GLYPH || (TEXT && a.x == TK_PTCL_GLYPH) ||
                (SDF != 0u && (a.x == TK_PTCL_SDF || a.x == TK_PTCL_IMAGE))) {
                const PaintInfo* pi = paints + c.y;
                if (SDF != 0u && a.x == TK_PTCL_SDF) S.umode[tid] = __ldg(&pi->sdf);  // SDF records: the shape's first word
                const uint32_t paint = __ldg(&pi->paint);
                if (paint != kGradient) {
                    S.paint[tid] = paint;
                    S.pcf[tid] = make_float4(float(paint & 255u), float((paint >> 8) & 255u),
                                             float((paint >> 16) & 255u), float(paint >> 24));
                    S.pfull[tid] = rgba8_to_unorm(paint);
                    if (n == 0u && a.x == TK_PTCL_FILL) {
                        // segment-free solid fill: with clip == 255 the source is uniform
                        const uint32_t masked = S.ualpha[tid];
                        cls = kClsUniform;
                        if (masked == 0u) {
                            S.umode[tid] = 3u;
                        } else if (masked == 255u && premul_u8_is_opaque(paint)) {
                            S.umode[tid] = 1u;
                        } else {
                            S.umode[tid] = 2u;
                            S.pfull[tid] = scale_premul_u8_to_unorm(paint, masked);
                        }
                    }
                } else {
                    S.paint[tid] = kGradient;
                    S.gk[tid] = __ldg(&pi->gk);
                    const float4* g = reinterpret_cast<const float4*>(pi->g);
                    float4* dst = reinterpret_cast<float4*>(S.gp[tid]);
#pragma unroll
                    for (int k = 0; k < kGradParams / 4; ++k) dst[k] = __ldg(g + k);
                }
            }
            S.cls[tid] = cls;
        }
        if (tid == 0) S.nprod = 0u;
        __syncthreads();
        if (tid < 32) {  // segment offsets and chunk length (warp 0)
            const uint32_t a0 = tid * 2u < avail ? S.nseg[tid * 2u] : 0u;
            const uint32_t a1 = tid * 2u + 1u < avail ? S.nseg[tid * 2u + 1u] : 0u;
            const uint32_t v = a0 + a1;
            uint32_t incl = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t q = __shfl_up_sync(0xffffffffu, incl, o);
                if (tid >= uint32_t(o)) incl += q;
            }
            const uint32_t excl = incl - v;
            if (tid * 2u <= kRecChunk) S.off[tid * 2u] = excl;
            if (tid * 2u + 1u <= kRecChunk) S.off[tid * 2u + 1u] = excl + a0;
            if (tid == 31 && kRecChunk == 64u) S.off[kRecChunk] = incl;
            const bool fit0 = tid * 2u < avail && excl + a0 <= kSegBudget;
            const bool fit1 = tid * 2u + 1u < avail && excl + a0 + a1 <= kSegBudget;
            const uint32_t nfit = __popc(__ballot_sync(0xffffffffu, fit0)) + __popc(__ballot_sync(0xffffffffu, fit1));
            if (tid == 0) S.n = nfit == 0u ? 1u : nfit;
        }
        __syncthreads();
        const uint32_t n = S.n;
        const bool big = S.off[n] > kSegBudget;  // one record with more than kSegBudget segments
        if (!big) {
            const uint32_t total = S.off[n];
            for (uint32_t sg = tid; sg < total; sg += kFineThreads) {
                uint32_t lo = 0, hi = n;  // record owning staged segment sg
                while (hi - lo > 1u) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (S.off[mid] <= sg) lo = mid;
                    else hi = mid;
                }
                const float4* g = reinterpret_cast<const float4*>(segments + S.rec_a[lo].w + (sg - S.off[lo]));
                const float4 q = __ldg(g);
                const float4 e = __ldg(g + 1);  // y_edge, slope
                S.sgp[sg] = q;
                S.sgx[sg] = make_float2(e.x, e.y);
                S.rmask[sg] = uint16_t(crossed_rows(q.y, q.w));
            }
            __syncthreads();
            stage_rows(S, total, n);
            __syncthreads();
        }
        // ---- interpret the chunk -------------------------------------------------
        uint32_t i = 0;
        while (i < n) {
            const uint32_t cls = S.cls[i];
            if (cls == kClsEnd) {
                done = true;
                break;
            }
            if (cls == kClsFill && mode != TK_TILE_KIND_COLOR && !big) {
                // the common record: a path fill with segments in the tile
                const uint32_t alpha = coverage_to_alpha(staged_coverage(S, i, lx, ly), S.rec_a[i].z);
                const uint32_t masked = clip == 255u ? alpha : combine_alpha(alpha, clip);
                if (masked != 0u) paint_fill<SDF != 0u>(S, P, i, masked, gx, gy, px);
                ++i;
                continue;
            }
            const uint2 qb = S.rec_b[i];
            if (cls == kClsBatch) {
                // A new reference batch dispatch: store / reload the target
                // texel and start from the interpreter's initial state.
                px = texel_load_lut(S, texel_store(px));
                clip = 255u;
                cdepth = 0u;
                cregs = 0u;
                gdepth = 0u;
                mode = qb.y & TK_TILE_KIND_MASK;
                i += 1u + (qb.y >> TK_TILE_PREFIX_SHIFT);
                continue;
            }
            if (mode == TK_TILE_KIND_COLOR) {  // color_only_no_stack_tile_pixel
                if (premul_u8_is_opaque(qb.y)) px = rgba8_to_unorm(qb.y);
                else px = src_over_premul_unorm(px, rgba8_to_unorm(qb.y));
                ++i;
                continue;
            }
            if (cls == kClsUniform && clip == 255u) {
                const uint32_t um = S.umode[i];
                if (um == 1u) px = S.pfull[i];
                else if (um == 2u) px = src_over_premul_unorm(px, S.pfull[i]);
                ++i;
                continue;
            }
            const uint4 qa = S.rec_a[i];
            const uint32_t tag = qa.x;
            if (tag == TK_PTCL_COLOR) {
                if (clip != 0u) {
                    if (clip == 255u && premul_u8_is_opaque(qb.y)) px = rgba8_to_unorm(qb.y);
                    else px = src_over_premul_unorm(px, scale_premul_u8_to_unorm(qb.y, clip));
                }
            } else if (tag == TK_PTCL_END_CLIP) {
                if (cdepth > 0u) {
                    --cdepth;
                    if (cdepth < 4u) clip = (cregs >> (8u * cdepth)) & 255u;
                    else clip = cspill[cdepth - 4u];
                } else {
                    clip = 255u;
                }
            } else if (tag == TK_PTCL_END_OPACITY || tag == TK_PTCL_END_BLEND) {
                if (gdepth > 0u) {
                    --gdepth;
                    const Group v = groups[gdepth];
                    if (v.kind == TK_PTCL_BEGIN_OPACITY) {
                        uint32_t a = combine_alpha(combine_alpha(v.layer_alpha, v.parent_clip), v.payload);
                        px = src_over_premul_unorm(v.parent, scale_premul_u8_to_unorm(unorm_to_rgba8(px), a));
                    }
                }
            } else if (SDF != 0u && (tag == TK_PTCL_SDF || tag == TK_PTCL_BEGIN_SDF_CLIP || tag == TK_PTCL_IMAGE)) {
                // PTCL_SDF (fine/interpreter.hlsli:70-84) and BEGIN_SDF_CLIP (131-150):
                // the shape's quantized coverage, one evaluation for both;
                // PTCL_IMAGE (65-69): the brush over the whole tile
                uint32_t alpha = 0u;
                if (clip != 0u)
                    alpha = tag == TK_PTCL_IMAGE ? 255u
                                                 : coverage_to_u8(sdf_coverage_at<SDF == 2u>(
                                                       sdf + S.umode[i], &draws[qb.y].inverse_transform, gx, gy));
                if (tag == TK_PTCL_BEGIN_SDF_CLIP) {  // push the mask, then narrow it
                    if (cdepth < 4u) {
                        cregs = (cregs & ~(255u << (8u * cdepth))) | (clip << (8u * cdepth));
                        ++cdepth;
                    } else if (cdepth - 4u < kClipSpill) {
                        cspill[cdepth - 4u] = clip;
                        ++cdepth;
                    } else {
                        atomicOr(error, ERR_STACK_DEPTH);
                    }
                    clip = combine_alpha(clip, alpha);
                } else if (tag == TK_PTCL_IMAGE && (mode == TK_TILE_KIND_SDF || mode == TK_TILE_KIND_MIXED)) {
                    // analytic tiles (fine/specialized.hlsli:84-90): the sample over the pixel, unscaled
                    const uint32_t g = gradient_at<true>(S, P, i, float(gx) + 0.5f, float(gy) + 0.5f);
                    px = premul_u8_is_opaque(g) ? rgba8_to_unorm(g) : src_over_premul_unorm(px, rgba8_to_unorm(g));
                } else {
                    const uint32_t masked = combine_alpha(alpha, clip);
                    if (masked != 0u) paint_fill<SDF != 0u>(S, P, i, masked, gx, gy, px);
                }
            } else if (TEXT && tag == TK_PTCL_GLYPH) {
                // fine/interpreter.hlsli:93-106: the run's glyphs inside the
                // draw's exact pixel bounds
                const tk_draw_record* dr = draws + qb.y;
                const int32_t x = int32_t(gx), y = int32_t(gy);
                if (clip != 0u && x >= __ldg(&dr->pixel_bounds.x0) && y >= __ldg(&dr->pixel_bounds.y0) &&
                    x < __ldg(&dr->pixel_bounds.x1) && y < __ldg(&dr->pixel_bounds.y1))
                    px = composite_glyphs<SDF != 0u>(S, P, i, glyphs, dr, qa.w, qb.x, gx, gy, clip, px);
            } else if (is_fill_like(tag)) {
                uint32_t alpha;
                if (S.nseg[i] == 0u) {
                    alpha = S.ualpha[i];
                } else if (!big) {
                    alpha = coverage_to_alpha(staged_coverage(S, i, lx, ly), qa.z);
                } else {
                    // more segments than one chunk holds: per-pixel evaluation
                    // of fill_alpha_at over 128-segment slices
                    float base = float(int32_t(qa.y)), running = 0.0f, partial = 0.0f;
                    for (uint32_t c0 = qa.w; c0 < qb.x; c0 += kSegBudget) {
                        const uint32_t m = min(kSegBudget, qb.x - c0);
                        __syncthreads();
                        for (uint32_t j = tid; j < m; j += kFineThreads) {
                            S.sgp[j] = __ldg(reinterpret_cast<const float4*>(segments + c0 + j));
                            S.sgx[j] = make_float2(__ldg(&segments[c0 + j].y_edge), 0.0f);
                        }
                        __syncthreads();
                        for (uint32_t j = 0; j < m; ++j) {
                            const float4 g = S.sgp[j];
                            const RowParts q = segment_row_parts(g.x, g.y, g.z, g.w, S.sgx[j].x, ly);
                            base += q.edge;
                            if (q.dy != 0.0f) {
                                const int32_t hi = min(max(f2i(ceilf(q.xmax)), 0), int32_t(TK_TILE_SIZE));
                                if (hi < int32_t(TK_TILE_SIZE) && int32_t(lx) >= hi) running += q.dy;
                                const int32_t lo = min(max(f2i(floorf(q.xmin)), 0), int32_t(TK_TILE_SIZE));
                                if (int32_t(lx) >= lo && int32_t(lx) < hi)
                                    partial += segment_area_at(q.xmin, q.xmax, lx) * q.dy;
                            }
                        }
                    }
                    alpha = coverage_to_alpha(base + running + partial, qa.z);
                }
                if (tag == TK_PTCL_BEGIN_CLIP) {
                    if (cdepth < 4u) {
                        cregs = (cregs & ~(255u << (8u * cdepth))) | (clip << (8u * cdepth));
                        ++cdepth;
                    } else if (cdepth - 4u < kClipSpill) {
                        cspill[cdepth - 4u] = clip;
                        ++cdepth;
                    } else {
                        atomicOr(error, ERR_STACK_DEPTH);
                    }
                    clip = combine_alpha(clip, alpha);
                } else if (tag == TK_PTCL_BEGIN_OPACITY || tag == TK_PTCL_BEGIN_BLEND) {
                    if (gdepth < kGroupDepth) {
                        // Parents beyond the local slots are kept as RGBA8
                        // (fine/group.hlsli:21-36).
                        const float4 parent = gdepth < kGroupLocal ? px : rgba8_to_unorm(unorm_to_rgba8(px));
                        groups[gdepth] = Group{tag, parent, clip, alpha, qb.y};
                        ++gdepth;
                        px = make_float4(0.f, 0.f, 0.f, 0.f);
                    } else {
                        atomicOr(error, ERR_STACK_DEPTH);
                    }
                } else {
                    const uint32_t masked = clip == 255u ? alpha : combine_alpha(alpha, clip);
                    if (masked != 0u) {
                        if (TEXT && tag == TK_PTCL_PATH_GLYPH) {
                            px = paint_glyph_fill<SDF != 0u>(S, P, i, masked, gx, gy, px);
                        } else {
                            // text instances take every glyph outline fill
                            if (!TEXT && tag == TK_PTCL_PATH_GLYPH) atomicOr(error, ERR_UNSUPPORTED);
                            paint_fill<SDF != 0u>(S, P, i, masked, gx, gy, px);
                        }
                    }
                }
            }
            ++i;
        }
        r += i;
    }
    if (inside) target[pix] = texel_store(px);
}

// g_star_dir: the star vertex directions, by the same sdf_sincos the pixels
// would call.
__global__ void k_star_table() {
    if (threadIdx.x < 10u) {
        float s, c;
        sdf_sincos(float(threadIdx.x) * 0.62831855f, s, c);
        g_star_dir[threadIdx.x] = make_float2(c, s);
    }
}

}  // namespace

void launch_paint_table(const tk_draw_record* draws, uint32_t draw_count, const uint32_t* brush,
                        uint64_t brush_words, uint32_t sdf_shadow_base, const uint4* images, uint32_t image_count,
                        PaintInfo* out, cudaStream_t st) {
    if (draw_count)
        k_paint_table<<<(draw_count + 255) / 256, 256, 0, st>>>(draws, draw_count, brush, brush_words,
                                                                sdf_shadow_base, images, image_count, out);
}

void launch_fine(const SceneView& s, const PassView& p, uint32_t* target, cudaStream_t st) {
    const uint32_t T = p.tile_list ? p.tile_list_n : (p.scenes ? p.total_tiles : s.tw * s.th);
    if (T == 0) return;
    static bool configured = false;
    if (!configured) {
        for (auto k : {k_fine<0u, false>, k_fine<1u, false>, k_fine<2u, false>, k_fine<0u, true>, k_fine<1u, true>,
                       k_fine<2u, true>})
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(FineSmem)));
        configured = true;
    }
    if (s.sdf_ext) k_star_table<<<1, 32, 0, st>>>();
    auto kernel = s.text ? (!s.sdf_words ? k_fine<0u, true> : (s.sdf_ext ? k_fine<2u, true> : k_fine<1u, true>))
                         : (!s.sdf_words ? k_fine<0u, false> : (s.sdf_ext ? k_fine<2u, false> : k_fine<1u, false>));
    const GlyphView glyphs{p.glyph_list, s.glyphs, s.glyph_images, s.glyph_texels};
    kernel<<<T, kFineThreads, sizeof(FineSmem), st>>>(p.tiles, p.ptcl, s.segments, s.paints, s.brush, s.brush_words,
                                                      s.texels, s.draws, s.sdf, s.segment_capacity, target, s.width, s.height,
                                                      s.tw, s.error, p.scenes, p.tile_scene, p.tile_list, glyphs);
}

}  // namespace tk
