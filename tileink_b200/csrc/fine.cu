// Fine stage: one CTA of 256 threads per 16x16 tile, one thread per pixel
// (fine/main.hlsl:23-40, fine/interpreter.hlsli:21-219,
// fine/specialized.hlsli:19-45).
//
// The tile's merged PTCL stream is processed in chunks of up to 64 records
// whose fills together reference at most 128 tile segments. Per chunk the CTA
// stages into shared memory, with coalesced loads and no dependent global
// round trips per record:
//   - the records and each fill's paint, resolved from draw -> brush once per
//     record;
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

namespace tk {
namespace {

using namespace tkd;

constexpr int kFineThreads = 256;
constexpr uint32_t kRecChunk = 64;
constexpr uint32_t kSegBudget = 128;
constexpr uint32_t kProdCap = 4096;
constexpr uint32_t kNoProd = 0xFFFFu;
constexpr uint32_t kClipSpill = 28;
constexpr uint32_t kGroupDepth = 6;
constexpr uint32_t kGroupLocal = 2;  // FINE_LOCAL_GROUP_DEPTH (fine/constants.hlsli:11)
constexpr uint32_t kGradient = 0xFFFFFFFFu;

// Record classes driving the per-pixel dispatch.
constexpr uint32_t kClsOther = 0, kClsFill = 1, kClsUniform = 2, kClsBatch = 3, kClsEnd = 4;

struct Group {
    uint32_t kind;
    float4 parent;
    uint32_t parent_clip, layer_alpha, payload;
};

struct FineSmem {
    // crossing (row, segment) entries: dy, xmin, xmax, and
    // plo | phi << 8 | prod offset << 16 (plo/phi: the partial pixel range
    // [clamp(floor(xmin)), clamp(ceil(xmax))) within [0, 16])
    float4 ent[TK_TILE_SIZE][kSegBudget];
    uint16_t pos[TK_TILE_SIZE][kSegBudget + 1];  // crossing entries before staged segment j
    float prod[kProdCap];                        // segment_area_at(x) * dy per partial pixel
    float seg[kSegBudget * 5];
    float base[kRecChunk][TK_TILE_SIZE];
    float4 pfull[kRecChunk];                     // rgba8_to_unorm(paint) / uniform source
    float4 pcf[kRecChunk];                       // paint channels as floats
    uint4 rec_a[kRecChunk];                      // tag, backdrop, fill_rule, segment_start
    uint2 rec_b[kRecChunk];                      // segment_end, color
    uint32_t cls[kRecChunk];
    uint32_t ualpha[kRecChunk];
    uint32_t umode[kRecChunk];                   // uniform fills: 1 replace, 2 src-over, 3 no-op
    uint32_t paint[kRecChunk];                   // solid premul color, or kGradient
    uint32_t brush_off[kRecChunk];
    float inv[kRecChunk][6];
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

// Crossing lists and partial products for staged segments [0, total): warp w
// builds rows 2w and 2w + 1, lanes walk the segments in order.
__device__ void stage_rows(FineSmem& S, uint32_t total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    for (uint32_t rr = 0; rr < 2u; ++rr) {
        const uint32_t row = warp * 2u + rr;
        uint32_t count = 0;
        for (uint32_t j0 = 0; j0 < total; j0 += 32u) {
            const uint32_t j = j0 + lane;
            RowParts rp{0.f, 0.f, 0.f, 0.f};
            if (j < total) {
                const float* g = S.seg + j * 5u;
                rp = segment_row_parts(g[0], g[1], g[2], g[3], g[4], row);
            }
            const bool crossing = j < total && rp.dy != 0.0f;
            const uint32_t ballot = __ballot_sync(0xffffffffu, crossing);
            const uint32_t k = count + __popc(ballot & lt);
            if (j < total) S.pos[row][j] = uint16_t(k);
            if (crossing) {
                const int32_t plo = min(max(f2i(floorf(rp.xmin)), 0), int32_t(TK_TILE_SIZE));
                const int32_t phi = min(max(f2i(ceilf(rp.xmax)), 0), int32_t(TK_TILE_SIZE));
                const uint32_t span = phi > plo ? uint32_t(phi - plo) : 0u;
                uint32_t o = atomicAdd(&S.nprod, span);
                if (o + span <= kProdCap) {
                    for (uint32_t x = 0; x < span; ++x)
                        S.prod[o + x] = segment_area_at(rp.xmin, rp.xmax, uint32_t(plo) + x) * rp.dy;
                } else {
                    o = kNoProd;
                }
                S.ent[row][k] = make_float4(rp.dy, rp.xmin, rp.xmax,
                                            __uint_as_float(uint32_t(plo) | (uint32_t(phi) << 8) | (o << 16)));
            }
            count += __popc(ballot);
        }
        if (lane == 0) S.pos[row][total] = uint16_t(count);
    }
}

__global__ void __launch_bounds__(kFineThreads, 3)
    k_fine(const tk_tile_record* __restrict__ tiles, const tk_ptcl_record* __restrict__ ptcl,
           const tk_line_segment* __restrict__ segments, const tk_draw_record* __restrict__ draws,
           const uint32_t* __restrict__ brush, uint64_t brush_words, uint64_t seg_capacity, uint32_t* target,
           uint32_t width, uint32_t height, uint32_t tw, uint32_t* error) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FineSmem& S = *reinterpret_cast<FineSmem*>(smem_raw);
    const uint32_t tile = blockIdx.x;
    const tk_tile_record rec = tiles[tile];
    if (rec.ptcl_start >= rec.ptcl_end) return;
    const uint32_t tid = threadIdx.x;
    const uint32_t lx = tid & 15u, ly = tid >> 4;
    const uint32_t gx = (tile % tw) * TK_TILE_SIZE + lx, gy = (tile / tw) * TK_TILE_SIZE + ly;
    const bool inside = gx < width && gy < height;
    const uint64_t pix = uint64_t(gy) * width + gx;
    const Paint P{brush, brush_words};
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
                if (a.x == TK_PTCL_FILL) cls = kClsFill;
            }
            S.nseg[tid] = n;
            if (a.x == TK_PTCL_FILL || a.x == TK_PTCL_PATH_GLYPH) {
                const tk_draw_record& d = draws[c.y];
                const uint32_t bo = __ldg(&d.brush_offset);
                S.brush_off[tid] = bo;
                if (P.word(bo) == TK_BRUSH_SOLID) {
                    const uint32_t paint = P.word(bo + TK_BRUSH_COLOR_WORD);
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
                    const float* m = &d.inverse_transform.a;
#pragma unroll
                    for (int k = 0; k < 6; ++k) S.inv[tid][k] = __ldg(m + k);
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
            S.off[tid * 2u] = excl;
            S.off[tid * 2u + 1u] = excl + a0;
            if (tid == 31) S.off[kRecChunk] = incl;
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
            for (uint32_t j = tid; j < total * 5u; j += kFineThreads) {
                const uint32_t sg = j / 5u, comp = j - sg * 5u;
                uint32_t lo = 0, hi = n;  // record owning staged segment sg
                while (hi - lo > 1u) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (S.off[mid] <= sg) lo = mid;
                    else hi = mid;
                }
                const uint32_t g = S.rec_a[lo].w + (sg - S.off[lo]);
                S.seg[j] = __ldg(reinterpret_cast<const float*>(segments + g) + comp);
            }
            __syncthreads();
            stage_rows(S, total);
            for (uint32_t k = tid; k < n * TK_TILE_SIZE; k += kFineThreads) {
                const uint32_t ri = k >> 4, row = k & 15u;
                if (S.nseg[ri] == 0u) continue;
                float bsum = float(int32_t(S.rec_a[ri].y));
                for (uint32_t j = S.off[ri], e = S.off[ri] + S.nseg[ri]; j < e; ++j) {
                    const float* g = S.seg + j * 5u;
                    if (g[4] < 1000000000.0f)  // y_edge set: the segment touches the tile's left edge
                        bsum += signum_f32(g[2] - g[0]) * clampf(float(row) - g[4] + 1.0f, 0.0f, 1.0f);
                }
                S.base[ri][row] = bsum;
            }
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
            } else if (is_fill_like(tag)) {
                uint32_t alpha;
                if (S.nseg[i] == 0u) {
                    alpha = S.ualpha[i];
                } else if (!big) {
                    float running = 0.0f, partial = 0.0f;
                    const float4* row = S.ent[ly];
                    const uint32_t k0 = S.pos[ly][S.off[i]], k1 = S.pos[ly][S.off[i] + S.nseg[i]];
                    for (uint32_t k = k0; k < k1; ++k) {
                        const float4 e = row[k];
                        const uint32_t pk = __float_as_uint(e.w);
                        const uint32_t plo = pk & 0xFFu, phi = (pk >> 8) & 0xFFu;
                        if (lx >= phi) running += e.x;
                        if (lx >= plo && lx < phi) {
                            const uint32_t o = pk >> 16;
                            partial += o != kNoProd ? S.prod[o + lx - plo] : segment_area_at(e.y, e.z, lx) * e.x;
                        }
                    }
                    alpha = coverage_to_alpha(S.base[i][ly] + running + partial, qa.z);
                } else {
                    // more segments than one chunk holds: per-pixel evaluation
                    // of fill_alpha_at over 128-segment slices
                    float base = float(int32_t(qa.y)), running = 0.0f, partial = 0.0f;
                    for (uint32_t c0 = qa.w; c0 < qb.x; c0 += kSegBudget) {
                        const uint32_t m = min(kSegBudget, qb.x - c0);
                        __syncthreads();
                        for (uint32_t j = tid; j < m * 5u; j += kFineThreads)
                            S.seg[j] = __ldg(reinterpret_cast<const float*>(segments + c0) + j);
                        __syncthreads();
                        for (uint32_t j = 0; j < m; ++j) {
                            const float* g = S.seg + j * 5u;
                            const RowParts q = segment_row_parts(g[0], g[1], g[2], g[3], g[4], ly);
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
                        if (tag == TK_PTCL_PATH_GLYPH) atomicOr(error, ERR_UNSUPPORTED);
                        const uint32_t paint = S.paint[i];
                        if (paint != kGradient) {
                            if (masked == 255u && premul_u8_is_opaque(paint)) {
                                px = S.pfull[i];
                            } else {
                                // scale_premul_u8_to_unorm with the channels staged as floats
                                const float sc = float(masked) * (1.0f / 65025.0f);
                                const float4 c = S.pcf[i];
                                if (c.w != 0.0f)
                                    px = src_over_premul_unorm(px, make_float4(c.x * sc, c.y * sc, c.z * sc, c.w * sc));
                            }
                        } else {
                            const float sx = float(gx) + 0.5f, sy = float(gy) + 0.5f;
                            const float* m = S.inv[i];
                            const float lxf = mad(m[0], sx, mad(m[2], sy, m[4]));
                            const float lyf = mad(m[1], sx, mad(m[3], sy, m[5]));
                            const uint32_t g = sample_gradient(P, S.brush_off[i], lxf, lyf);
                            if (masked == 255u && premul_u8_is_opaque(g)) px = rgba8_to_unorm(g);
                            else px = src_over_premul_unorm(px, scale_premul_u8_to_unorm(g, masked));
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

}  // namespace

void launch_fine(const SceneView& s, const PassView& p, uint32_t* target, cudaStream_t st) {
    const uint32_t T = s.tw * s.th;
    if (T == 0) return;
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(k_fine, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(FineSmem)));
        configured = true;
    }
    k_fine<<<T, kFineThreads, sizeof(FineSmem), st>>>(p.tiles, p.ptcl, s.segments, s.draws, s.brush, s.brush_words,
                                                      s.segment_capacity, target, s.width, s.height, s.tw, s.error);
}

}  // namespace tk
