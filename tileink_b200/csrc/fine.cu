// Fine stage: one CTA of 256 threads per 16x16 tile, one thread per pixel
// (fine/main.hlsl:23-40, fine/interpreter.hlsli:21-219,
// fine/specialized.hlsli:19-45).
//
// The tile's merged PTCL stream is walked uniformly by the whole CTA. For a
// fill record its tile-local segments are staged in shared memory and the
// per-row terms of shared/coverage.hlsli:7-24 (segment_row_parts) are computed
// once per (row, segment) instead of once per pixel; every pixel then
// accumulates base / running / partial in segment order exactly as
// fill_alpha_at (shared/coverage.hlsli:34-51) does, so the sums are the same
// f32 sequence.
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.h"

namespace tk {
namespace {

using namespace tkd;

constexpr int kFineThreads = 256;
constexpr uint32_t kSegChunk = 128;
constexpr uint32_t kClipSpill = 28;
constexpr uint32_t kGroupDepth = 6;
constexpr uint32_t kGroupLocal = 2;  // FINE_LOCAL_GROUP_DEPTH (fine/constants.hlsli:11)

struct Group {
    uint32_t kind;
    float4 parent;
    uint32_t parent_clip, layer_alpha, payload;
};

__device__ __forceinline__ tk_ptcl_record load_ptcl(const tk_ptcl_record* p, uint64_t i) {
    const uint2* w = reinterpret_cast<const uint2*>(p + i);
    uint2 a = __ldg(w), b = __ldg(w + 1), c = __ldg(w + 2);
    tk_ptcl_record r;
    r.tag = a.x;
    r.backdrop = int32_t(a.y);
    r.fill_rule = b.x;
    r.segment_start = b.y;
    r.segment_end = c.x;
    r.color = c.y;
    return r;
}

__global__ void __launch_bounds__(kFineThreads)
    k_fine(const tk_tile_record* __restrict__ tiles, const tk_ptcl_record* __restrict__ ptcl,
           const tk_line_segment* __restrict__ segments, const tk_draw_record* __restrict__ draws,
           const uint32_t* __restrict__ brush, uint64_t brush_words, uint64_t seg_capacity, uint32_t* target,
           uint32_t width, uint32_t height, uint32_t tw, uint32_t* error) {
    __shared__ float s_seg[kSegChunk * 5];
    __shared__ float4 s_parts[TK_TILE_SIZE * kSegChunk];
    const uint32_t tile = blockIdx.x;
    const tk_tile_record rec = tiles[tile];
    if (rec.ptcl_start >= rec.ptcl_end) return;
    const uint32_t tid = threadIdx.x;
    const uint32_t lx = tid & 15u, ly = tid >> 4;
    const uint32_t gx = (tile % tw) * TK_TILE_SIZE + lx, gy = (tile / tw) * TK_TILE_SIZE + ly;
    const bool inside = gx < width && gy < height;
    const uint64_t pix = uint64_t(gy) * width + gx;
    const Paint P{brush, brush_words};
    float4 px = inside ? texel_load(target[pix]) : make_float4(0.f, 0.f, 0.f, 0.f);

    uint32_t clip = 255u, cdepth = 0u, cregs = 0u;
    uint32_t cspill[kClipSpill];
    Group groups[kGroupDepth];
    uint32_t gdepth = 0u;
    uint32_t mode = TK_TILE_KIND_INTERPRETER;

    uint64_t r = rec.ptcl_start;
    const uint64_t end = rec.ptcl_end;
    while (r < end) {
        const tk_ptcl_record q = load_ptcl(ptcl, r);
        const uint32_t tag = q.tag;
        if (tag == TK_PTCL_END) break;
        if (tag == TK_PTCL_BATCH_BEGIN) {
            // A new reference batch dispatch: store/reload the target texel
            // and start from the fine interpreter's initial state.
            px = texel_load(texel_store(px));
            clip = 255u;
            cdepth = 0u;
            cregs = 0u;
            gdepth = 0u;
            mode = q.color & TK_TILE_KIND_MASK;
            r += 1u + (q.color >> TK_TILE_PREFIX_SHIFT);
            continue;
        }
        ++r;
        if (mode == TK_TILE_KIND_COLOR) {  // color_only_no_stack_tile_pixel
            if (premul_u8_is_opaque(q.color)) px = rgba8_to_unorm(q.color);
            else px = src_over_premul_unorm(px, rgba8_to_unorm(q.color));
            continue;
        }
        if (tag == TK_PTCL_COLOR) {
            if (clip != 0u) {
                if (clip == 255u && premul_u8_is_opaque(q.color)) px = rgba8_to_unorm(q.color);
                else px = src_over_premul_unorm(px, scale_premul_u8_to_unorm(q.color, clip));
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
                Group v = groups[gdepth];
                if (v.kind == TK_PTCL_BEGIN_OPACITY) {
                    uint32_t a = combine_alpha(combine_alpha(v.layer_alpha, v.parent_clip), v.payload);
                    px = src_over_premul_unorm(v.parent, scale_premul_u8_to_unorm(unorm_to_rgba8(px), a));
                }
            }
        } else if (tag == TK_PTCL_FILL || tag == TK_PTCL_BEGIN_CLIP || tag == TK_PTCL_BEGIN_OPACITY ||
                   tag == TK_PTCL_BEGIN_BLEND || tag == TK_PTCL_PATH_GLYPH) {
            float base = float(q.backdrop), running = 0.0f, partial = 0.0f;
            uint32_t seg_end = q.segment_end;
            if (seg_end > seg_capacity || q.segment_start > seg_end) {  // inconsistent scan inputs
                if (tid == 0) atomicOr(error, ERR_SEGMENT_OVERFLOW);
                seg_end = q.segment_start > seg_capacity ? q.segment_start : uint32_t(seg_capacity);
                if (q.segment_start > seg_end) seg_end = q.segment_start;
            }
            for (uint32_t c0 = q.segment_start; c0 < seg_end; c0 += kSegChunk) {
                const uint32_t m = min(kSegChunk, seg_end - c0);
                __syncthreads();
                for (uint32_t i = tid; i < m * 5u; i += kFineThreads)
                    s_seg[i] = __ldg(reinterpret_cast<const float*>(segments + c0) + i);
                __syncthreads();
                for (uint32_t i = tid; i < m * TK_TILE_SIZE; i += kFineThreads) {
                    uint32_t row = i & 15u, j = i >> 4;
                    const float* g = s_seg + j * 5u;
                    RowParts rp = segment_row_parts(g[0], g[1], g[2], g[3], g[4], row);
                    s_parts[row * kSegChunk + j] = make_float4(rp.edge, rp.dy, rp.xmin, rp.xmax);
                }
                __syncthreads();
                const float4* rowp = s_parts + ly * kSegChunk;
                for (uint32_t j = 0; j < m; ++j) {
                    float4 p4 = rowp[j];
                    base += p4.x;
                    if (p4.y != 0.0f) {
                        int32_t hi = min(max(f2i(ceilf(p4.w)), 0), int32_t(TK_TILE_SIZE));
                        if (hi < int32_t(TK_TILE_SIZE) && int32_t(lx) >= hi) running += p4.y;
                        int32_t lo = min(max(f2i(floorf(p4.z)), 0), int32_t(TK_TILE_SIZE));
                        if (int32_t(lx) >= lo && int32_t(lx) < hi) partial += segment_area_at(p4.z, p4.w, lx) * p4.y;
                    }
                }
            }
            const uint32_t alpha = coverage_to_alpha(base + running + partial, q.fill_rule);
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
                    float4 parent = gdepth < kGroupLocal ? px : rgba8_to_unorm(unorm_to_rgba8(px));
                    groups[gdepth] = Group{tag, parent, clip, alpha, q.color};
                    ++gdepth;
                    px = make_float4(0.f, 0.f, 0.f, 0.f);
                } else {
                    atomicOr(error, ERR_STACK_DEPTH);
                }
            } else {
                const uint32_t masked = combine_alpha(alpha, clip);
                if (masked != 0u) {
                    if (tag == TK_PTCL_PATH_GLYPH) atomicOr(error, ERR_UNSUPPORTED);
                    const tk_draw_record& d = draws[q.color];
                    const uint32_t bo = d.brush_offset;
                    uint32_t color;
                    if (P.word(bo) == TK_BRUSH_SOLID) {
                        color = P.word(bo + TK_BRUSH_COLOR_WORD);
                    } else {
                        const tk_affine m = d.inverse_transform;
                        float sx = float(gx) + 0.5f, sy = float(gy) + 0.5f;
                        float lxf = mad(m.a, sx, mad(m.c, sy, m.e));
                        float lyf = mad(m.b, sx, mad(m.d, sy, m.f));
                        color = sample_gradient(P, bo, lxf, lyf);
                    }
                    if (masked == 255u && premul_u8_is_opaque(color)) px = rgba8_to_unorm(color);
                    else px = src_over_premul_unorm(px, scale_premul_u8_to_unorm(color, masked));
                }
            }
        }
    }
    if (inside) target[pix] = texel_store(px);
}

}  // namespace

void launch_fine(const SceneView& s, const PassView& p, uint32_t* target, cudaStream_t st) {
    uint32_t T = s.tw * s.th;
    if (T == 0) return;
    k_fine<<<T, kFineThreads, 0, st>>>(p.tiles, p.ptcl, s.segments, s.draws, s.brush, s.brush_words,
                                       s.segment_capacity, target, s.width, s.height, s.tw, s.error);
}

}  // namespace tk
