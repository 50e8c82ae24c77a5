// Coarse stage: tile binning, per-tile PTCL counting, tile prefix, emission.
//
// Binning replaces the reference's CPU TileDrawBins
// (src/shared/gpu_plan/tile_bins/build.rs:4-83): one CTA per 16x16-tile bin
// scans the pass's draws in painter order and compacts those whose tile bbox
// meets the bin, preserving order.
//
// Counting and emission follow coarse_count_bins / coarse_emit_bins
// (coarse/count.hlsl:48-73, coarse/emit.hlsl:82-142): one thread per tile
// walks the bin's candidates in painter order. All draw batches of a target
// pass are emitted into one merged stream per tile: each batch with particles
// in the tile contributes TK_PTCL_BATCH_BEGIN{segment_start = batch id,
// segment_end = record count, color = kind | skip << 3} followed by the
// reference batch stream without its END; one END closes the tile.
#include <cuda_runtime.h>

#include "device.cuh"
#include "kernels.h"
#include "sdf.cuh"

namespace tk {
namespace {

using namespace tkd;

constexpr int kBinSide = 16;
// Coarse runs one CTA per 8x8-tile quadrant of a bin (four per bin), so that a
// 4096^2 canvas gives 1024 CTAs instead of 256; each quadrant walks its bin's
// candidate list.
constexpr int kQuadSide = 8;
constexpr int kQuads = (kBinSide / kQuadSide) * (kBinSide / kQuadSide);
constexpr int kCoarseThreads = kQuadSide * kQuadSide;
constexpr uint32_t kChunkClassColor = 1u, kChunkClassSdf = 2u, kChunkClassOther = 4u, kChunkClassOccluder = 8u;
// DrawInfo::meta bits (the draw's batch ordinal above them, from bit kMetaBatchShift)
constexpr uint32_t kMetaPath = 16u, kMetaSolid = 32u, kMetaSdf = 64u, kMetaSdfSolidClass = 128u, kMetaGlyph = 256u;
constexpr uint32_t kMetaBatchShift = 9u;
// DrawInfo::py bits of an SDF draw (px holds its first SDF word)
constexpr uint32_t kSdfPlain = 256u, kSdfIdentity = 512u, kSdfImage = 1024u;
// Candidates whose tile loads are in flight together, per pass (emission
// keeps more state live and holds fewer).
constexpr uint32_t kPrefetchCount = 8, kPrefetchEmit = 4;

__device__ __forceinline__ uint32_t tile_min_(int32_t px, uint32_t lim) {
    return px > 0 ? min(uint32_t(px) / TK_TILE_SIZE, lim) : 0u;
}
__device__ __forceinline__ uint32_t tile_max_(int32_t px, uint32_t lim) {
    return px > 0 ? min((uint32_t(px) + TK_TILE_SIZE - 1u) / TK_TILE_SIZE, lim) : 0u;
}

// ---------------------------------------------------------------------------
// Binning.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    k_bins(const tk_draw_record* __restrict__ draws, const uint32_t* __restrict__ order, uint32_t order0,
           uint32_t draw_n, uint32_t tw, uint32_t th, uint32_t nbx, uint32_t* bin_lists, uint32_t* bin_counts,
           const BatchScene* __restrict__ scenes, const uint32_t* __restrict__ bin_scene) {
    __shared__ uint32_t s_warp[8];
    __shared__ uint32_t s_base;
    const uint32_t bin = blockIdx.x;
    uint32_t lbin = bin;
    uint64_t list = uint64_t(bin) * draw_n;
    if (scenes) {  // batched pass: this bin's canvas
        const BatchScene& sc = scenes[bin_scene[bin]];
        lbin = bin - sc.bin_base;
        tw = sc.tw;
        th = sc.th;
        nbx = sc.nbx;
        order0 = sc.order0;
        draw_n = sc.draw_n;
        list = sc.list_base + uint64_t(lbin) * sc.draw_n;
    }
    const uint32_t bx0 = (lbin % nbx) * kBinSide, by0 = (lbin / nbx) * kBinSide;
    const uint32_t bx1 = min(bx0 + kBinSide, tw), by1 = min(by0 + kBinSide, th);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_base = 0u;
    __syncthreads();
    uint32_t* out = bin_lists + list;
    for (uint32_t c = 0; c < draw_n; c += 256u) {
        uint32_t j = c + threadIdx.x;
        bool hit = false;
        uint32_t d = 0;
        if (j < draw_n) {
            d = __ldg(order + order0 + j);
            const tk_pixel_bounds pb = draws[d].pixel_bounds;
            uint32_t x0 = tile_min_(pb.x0, tw), y0 = tile_min_(pb.y0, th);
            uint32_t x1 = tile_max_(pb.x1, tw), y1 = tile_max_(pb.y1, th);
            hit = x0 < x1 && y0 < y1 && x0 < bx1 && x1 > bx0 && y0 < by1 && y1 > by0;
        }
        uint32_t ballot = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) s_warp[warp] = __popc(ballot);
        __syncthreads();
        uint32_t before = s_base;
        for (int w = 0; w < warp; ++w) before += s_warp[w];
        if (hit) out[before + __popc(ballot & ((1u << lane) - 1u))] = d;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = 0;
            for (int w = 0; w < 8; ++w) t += s_warp[w];
            s_base += t;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) bin_counts[bin] = s_base;
}

// ---------------------------------------------------------------------------
// Coarse count / emit.
// ---------------------------------------------------------------------------
struct DrawInfo {
    uint32_t draw;
    uint32_t tx, ty;         // draw tile bbox: x0 | x1 << 16, y0 | y1 << 16
    uint32_t px, py;         // path tile bbox packed the same way; SDF draws: first SDF word, kind | flags
    uint32_t data_offset;
    uint32_t meta;           // tag | fill << 3 | kMeta* bits | batch << kMetaBatchShift
    uint32_t color;
};

struct Ctx {
    const tk_draw_record* draws;
    const tk_path_record* paths;
    uint32_t path_count;
    const tk_layer_record* layers;
    const uint32_t* brush;
    uint64_t brush_words;
    const uint32_t* sdf;
    uint64_t sdf_shadow_base;
    const int32_t* backdrops;
    const tk_segment_range* ranges;
    uint32_t tw, th;
    // the text blob (glyph_runs null: no text)
    const tk_glyph_run* glyph_runs;
    const tk_glyph* glyphs;
    const tk_glyph_image* glyph_images;
    uint32_t glyph_run_count;
};

// count_draw_glyphs / store_draw_glyphs (coarse/text.hlsli:8-35): the glyphs
// [first, first + count) of a run whose image, widened by a pixel each way
// (bilinear reach), meets tile (tx, ty) under the draw transform
// (transformed_rect_hits_tile, shared/draw.hlsli:52-61); with `out`, their
// indices are stored from `at` on. Out of line: only text draws reach it.
static __device__ __noinline__ uint32_t draw_glyphs(const Ctx& c, uint32_t di, uint32_t first, uint32_t count,
                                                   uint32_t tx, uint32_t ty, uint32_t* out, uint64_t at,
                                                   uint64_t cap, uint32_t* error) {
    const tk_affine t = c.draws[di].transform;
    const float tlx = float(tx * TK_TILE_SIZE), tly = float(ty * TK_TILE_SIZE);
    uint32_t n = 0;
    for (uint32_t k = first; k < first + count; ++k) {
        const tk_glyph g = c.glyphs[k];
        if (g.image == TK_INVALID_INDEX) continue;
        const tk_glyph_image im = c.glyph_images[g.image];
        if (im.width == 0u || im.height == 0u) continue;
        // int2(x + left, y - top) - 1 and + size + 1, in wrapping 32-bit arithmetic
        const uint32_t lx = uint32_t(g.x) + uint32_t(im.left), ly = uint32_t(g.y) - uint32_t(im.top);
        const float x0 = float(int32_t(lx - 1u)), y0 = float(int32_t(ly - 1u));
        const float x1 = float(int32_t(lx + im.width + 1u)), y1 = float(int32_t(ly + im.height + 1u));
        // draw_point of the four corners: (a x + c y) + e, (b x + d y) + f
        const float p0x = t.a * x0 + t.c * y0 + t.e, p0y = t.b * x0 + t.d * y0 + t.f;
        const float p1x = t.a * x1 + t.c * y0 + t.e, p1y = t.b * x1 + t.d * y0 + t.f;
        const float p2x = t.a * x0 + t.c * y1 + t.e, p2y = t.b * x0 + t.d * y1 + t.f;
        const float p3x = t.a * x1 + t.c * y1 + t.e, p3y = t.b * x1 + t.d * y1 + t.f;
        const float lox = fminf(fminf(p0x, p1x), fminf(p2x, p3x)), loy = fminf(fminf(p0y, p1y), fminf(p2y, p3y));
        const float hix = fmaxf(fmaxf(p0x, p1x), fmaxf(p2x, p3x)), hiy = fmaxf(fmaxf(p0y, p1y), fmaxf(p2y, p3y));
        if (!(lox < tlx + float(TK_TILE_SIZE) && loy < tly + float(TK_TILE_SIZE) && hix > tlx && hiy > tly)) continue;
        if (out) {
            if (at + n < cap) out[at + n] = k;
            else atomicOr(error, ERR_PTCL_OVERFLOW);
        }
        ++n;
    }
    return n;
}

__device__ __forceinline__ uint32_t brush_word(const Ctx& c, uint32_t i) {
    return i < c.brush_words ? __ldg(c.brush + i) : 0u;
}

// draw_backdrop (shared/draw.hlsli:40-47) reading records from global memory.
__device__ uint32_t draw_backdrop_g(const Ctx& c, uint32_t di, uint32_t tx, uint32_t ty) {
    const tk_draw_record& d = c.draws[di];
    if (d.path_id == TK_INVALID_INDEX || d.tag > TK_DRAW_PATH_GLYPH || d.path_id >= c.path_count) return TK_INVALID_INDEX;
    uint32_t lx = tile_min_(d.pixel_bounds.x0, c.tw), ly = tile_min_(d.pixel_bounds.y0, c.th);
    uint32_t ux = tile_max_(d.pixel_bounds.x1, c.tw), uy = tile_max_(d.pixel_bounds.y1, c.th);
    if (!(tx >= lx && ty >= ly && tx < ux && ty < uy)) return TK_INVALID_INDEX;
    const tk_path_record& p = c.paths[d.path_id];
    if (p.tile_x1 <= p.tile_x0 || tx < p.tile_x0 || ty < p.tile_y0 || tx >= p.tile_x1 || ty >= p.tile_y1)
        return TK_INVALID_INDEX;
    return p.data_offset + (ty - p.tile_y0) * (p.tile_x1 - p.tile_x0) + tx - p.tile_x0;
}

// An SDF clip layer's draw (coarse/sdf_clip.hlsli:35-40): a rect with an
// identity linear part that covers the whole tile clips nothing there.
__device__ __forceinline__ bool sdf_clip_draw(const Ctx& c, uint32_t di, uint32_t tx, uint32_t ty, bool& covers,
                                              bool& hits) {
    const tk_draw_record& d = c.draws[di];
    if (d.sdf_offset == TK_INVALID_INDEX && d.sdf_shadow_offset == TK_INVALID_INDEX) return false;
    covers = false;
    if (d.sdf_offset != TK_INVALID_INDEX && d.sdf_shadow_offset == TK_INVALID_INDEX && d.sdf_len >= 9u &&
        __ldg(c.sdf + d.sdf_offset) == TK_SDF_RECT && d.transform.a == 1.0f && d.transform.b == 0.0f &&
        d.transform.c == 0.0f && d.transform.d == 1.0f)
        covers = sdf_rect_covers(c.sdf + d.sdf_offset, d.transform.e, d.transform.f, tx, ty);
    // draw_hits_tile (shared/draw.hlsli:36-40)
    hits = tx >= tile_min_(d.pixel_bounds.x0, c.tw) && ty >= tile_min_(d.pixel_bounds.y0, c.th) &&
           tx < tile_max_(d.pixel_bounds.x1, c.tw) && ty < tile_max_(d.pixel_bounds.y1, c.th);
    return true;
}

// stack_wrapper_count (coarse/classify.hlsli:11-33).
template <bool SDF>
__device__ uint32_t stack_wrappers(const Ctx& c, const PassBatch& b, uint32_t tx, uint32_t ty) {
    uint32_t count = 0;
    for (uint32_t i = b.layer_start; i < b.layer_end; ++i) {
        tk_layer_record L = c.layers[i];
        bool covers, hits;
        if (SDF && sdf_clip_draw(c, L.draw, tx, ty, covers, hits)) {
            if (covers) continue;
            if (!hits) return TK_INVALID_INDEX;
            ++count;
            continue;
        }
        uint32_t bd = draw_backdrop_g(c, L.draw, tx, ty);
        if (bd == TK_INVALID_INDEX) return TK_INVALID_INDEX;
        tk_segment_range r = c.ranges[bd];
        int32_t w = c.backdrops[bd];
        uint32_t rule = c.draws[L.draw].fill_rule;
        bool full = rule == TK_FILL_EVEN_ODD ? (uint32_t(w) & 1u) != 0u : w != 0;
        if (L.tag == TK_LAYER_CLIP && r.start == r.end && full) continue;
        if (r.start == r.end && w == 0) return TK_INVALID_INDEX;
        ++count;
    }
    return count;
}

__device__ __forceinline__ void store_ptcl(tk_ptcl_record* ptcl, uint64_t cap, uint64_t at, uint32_t tag,
                                           uint32_t winding, uint32_t rule, uint32_t s0, uint32_t s1, uint32_t color,
                                           uint32_t* error) {
    if (at >= cap) {
        atomicOr(error, ERR_PTCL_OVERFLOW);
        return;
    }
    uint2* w = reinterpret_cast<uint2*>(ptcl + at);
    w[0] = make_uint2(tag, winding);
    w[1] = make_uint2(rule, s0);
    w[2] = make_uint2(s1, color);
}

// emit_stack_begins / emit_stack_ends (coarse/emit_stack.hlsli:9-44); SDF
// clips open with BEGIN_SDF_CLIP naming their draw.
template <bool SDF>
__device__ uint64_t emit_stack(const Ctx& c, const PassBatch& b, uint32_t tx, uint32_t ty, bool begin,
                               tk_ptcl_record* ptcl, uint64_t cap, uint64_t at, uint32_t* error) {
    uint32_t n = b.layer_end - b.layer_start;
    for (uint32_t k = 0; k < n; ++k) {
        uint32_t i = begin ? b.layer_start + k : b.layer_end - 1u - k;
        tk_layer_record L = c.layers[i];
        bool covers, hits;
        if (SDF && sdf_clip_draw(c, L.draw, tx, ty, covers, hits)) {
            if (covers) continue;  // noop_stack_clip
            if (begin) store_ptcl(ptcl, cap, at++, TK_PTCL_BEGIN_SDF_CLIP, 0u, 0u, 0u, 0u, L.draw, error);
            else store_ptcl(ptcl, cap, at++, TK_PTCL_END_CLIP, 0u, 0u, 0u, 0u, 0u, error);
            continue;
        }
        uint32_t bd = draw_backdrop_g(c, L.draw, tx, ty);
        tk_segment_range r = c.ranges[bd];
        uint32_t w = uint32_t(c.backdrops[bd]);
        uint32_t rule = c.draws[L.draw].fill_rule;
        bool noop = L.tag == TK_LAYER_CLIP && r.start == r.end &&
                    (rule == TK_FILL_EVEN_ODD ? (w & 1u) != 0u : w != 0u);
        if (noop) continue;
        if (begin) {
            uint32_t tag = L.tag == TK_LAYER_OPACITY ? TK_PTCL_BEGIN_OPACITY
                           : (L.tag == TK_LAYER_BLEND ? TK_PTCL_BEGIN_BLEND : TK_PTCL_BEGIN_CLIP);
            store_ptcl(ptcl, cap, at++, tag, w, rule, r.start, r.end, L.payload, error);
        } else {
            uint32_t tag = L.tag == TK_LAYER_OPACITY ? TK_PTCL_END_OPACITY
                           : (L.tag == TK_LAYER_BLEND ? TK_PTCL_END_BLEND : TK_PTCL_END_CLIP);
            store_ptcl(ptcl, cap, at++, tag, 0u, 0u, 0u, 0u, 0u, error);
        }
    }
    return at;
}

// occluded_particle_prefix (coarse/occlusion.hlsli:12-34) over records
// [start, end) of one batch stream whose END is implied at `end`.
__device__ uint32_t occluded_prefix_g(const tk_ptcl_record* ptcl, uint64_t start, uint64_t end) {
    if (end - start + 1u <= 2u) return 0u;  // stream length incl. END
    uint32_t depth = 0;
    for (uint64_t cur = end; cur > start;) {
        --cur;
        uint32_t tag = ptcl[cur].tag;
        if (tag == TK_PTCL_END_CLIP || tag == TK_PTCL_END_OPACITY || tag == TK_PTCL_END_BLEND) ++depth;
        else if (tag == TK_PTCL_BEGIN_CLIP || tag == TK_PTCL_BEGIN_SDF_CLIP || tag == TK_PTCL_BEGIN_OPACITY ||
                 tag == TK_PTCL_BEGIN_BLEND) {
            if (depth == 0u) return 0u;
            --depth;
        } else if (tag == TK_PTCL_COLOR && depth == 0u && (ptcl[cur].color >> 24) == 255u) {
            return uint32_t(cur - start);
        }
    }
    return 0u;
}

// draw_particle for an SDF draw in tile (tx, ty) (coarse/emit_draw.hlsli:22-30):
// 0 inside a rect stroke's hole (sdf_stroke_empty), TK_PTCL_COLOR for a solid
// rect that covers the tile (full_tile_solid), else TK_PTCL_SDF. Out of line
// so that the walk over path candidates keeps its registers.
static __device__ __noinline__ uint32_t sdf_particle(const tk_draw_record* draws, const uint32_t* sdf, uint32_t draw,
                                                     uint32_t word, uint32_t bits, uint32_t meta, uint32_t tx,
                                                     uint32_t ty) {
    const uint32_t kind = bits & 255u;
    const bool proof = (bits & kSdfPlain) && (bits & kSdfIdentity) &&
                       (kind == TK_SDF_RECT_STROKE ||
                        (kind == TK_SDF_RECT && ((meta & kMetaSolid) || (bits & kSdfImage))));
    if (!proof) return TK_PTCL_SDF;
    const float ex = draws[draw].transform.e, ey = draws[draw].transform.f;
    if (kind == TK_SDF_RECT_STROKE) return sdf_stroke_empty(sdf + word, ex, ey, tx, ty) ? 0u : TK_PTCL_SDF;
    // full_tile_solid, then full_tile_image (coarse/paint.hlsli:27-34)
    if (!sdf_rect_covers(sdf + word, ex, ey, tx, ty)) return TK_PTCL_SDF;
    return (meta & kMetaSolid) ? TK_PTCL_COLOR : TK_PTCL_IMAGE;
}

// SDF: whether the scene has SDF records; path-only scenes run the instance
// without the SDF candidate handling. TEXT: whether it has glyph runs; the
// glyph particle handling (and its calls) lives only in those instances.
template <bool EMIT, bool SDF, bool TEXT>
__global__ void __launch_bounds__(kCoarseThreads)
    k_coarse(Ctx c, const uint32_t* __restrict__ bin_lists, const uint32_t* __restrict__ bin_counts, uint32_t draw_n,
             uint32_t nbx, const uint32_t* __restrict__ batch_ids, const PassBatch* __restrict__ batches,
             uint32_t batch0, tk_tile_record* tiles, tk_ptcl_record* ptcl, uint64_t cap,
             unsigned long long* stats, uint32_t* error, const BatchScene* __restrict__ scenes,
             const uint32_t* __restrict__ bin_scene, const uint8_t* __restrict__ tile_active, uint32_t* glyph_list,
             uint64_t glyph_cap) {
    __shared__ DrawInfo s_d[kCoarseThreads];
    const uint32_t bin = blockIdx.x / kQuads, quad = blockIdx.x % kQuads;
    uint32_t lbin = bin, tile_base = 0u;
    uint64_t list_at = uint64_t(bin) * draw_n;
    if (scenes) {  // batched pass: this bin's canvas
        const BatchScene& sc = scenes[bin_scene[bin]];
        lbin = bin - sc.bin_base;
        c.tw = sc.tw;
        c.th = sc.th;
        nbx = sc.nbx;
        draw_n = sc.draw_n;
        tile_base = sc.tile_base;
        list_at = sc.list_base + uint64_t(lbin) * sc.draw_n;
    }
    const uint32_t qx = quad % (kBinSide / kQuadSide), qy = quad / (kBinSide / kQuadSide);
    const uint32_t tx = (lbin % nbx) * kBinSide + qx * kQuadSide + (threadIdx.x % kQuadSide);
    const uint32_t ty = (lbin / nbx) * kBinSide + qy * kQuadSide + (threadIdx.x / kQuadSide);
    const bool in_canvas = tx < c.tw && ty < c.th;
    const uint32_t tile = tile_base + ty * c.tw + tx;
    // incremental render: tiles that are not redrawn get no particles
    const bool live = in_canvas && (!tile_active || tile_active[tile]);
    if (!__syncthreads_or(live)) {
        if (!EMIT && in_canvas) {
            tiles[tile].ptcl_count = 0u;
            tiles[tile].glyph_count = 0u;
        }
        return;
    }
    const uint32_t* list = bin_lists + list_at;
    const uint32_t n = bin_counts[bin];

    uint64_t at = 0, gat = 0;
    if (EMIT && live) {
        at = tiles[tile].ptcl_start;
        if (TEXT) gat = tiles[tile].glyph_start;
    }
    uint32_t total = 0, glyph_total = 0;
    uint32_t cur = 0xFFFFFFFFu, wrappers = 0, nb = 0, flags = 0;
    bool rejected = false;
    uint64_t section = 0;
    unsigned long long fills = 0, visits = 0;

    auto close = [&]() {
        if (cur == 0xFFFFFFFFu || rejected || nb == 0u) return;
        total += nb + 2u * wrappers + 1u;
        if (EMIT) {
            const PassBatch& b = batches[cur];
            uint64_t end = emit_stack<SDF>(c, b, tx, ty, false, ptcl, cap, at, error);
            uint32_t skip = 0;
            if (flags & kChunkClassOccluder) skip = wrappers ? 0u : occluded_prefix_g(ptcl, section + 1u, end);
            // classify_tile_flags (coarse/tile_classification.hlsli:6-10)
            uint32_t kind = TK_TILE_KIND_EMPTY;
            if (flags & kChunkClassOther) kind = TK_TILE_KIND_INTERPRETER;
            else if (flags & kChunkClassSdf) kind = (flags & kChunkClassColor) ? TK_TILE_KIND_MIXED : TK_TILE_KIND_SDF;
            else if (flags & kChunkClassColor) kind = TK_TILE_KIND_COLOR;
            store_ptcl(ptcl, cap, section, TK_PTCL_BATCH_BEGIN, 0u, 0u, b.batch_id, nb + 2u * wrappers,
                       kind | (skip << TK_TILE_PREFIX_SHIFT), error);
            at = end;
        }
    };

    for (uint32_t c0 = 0; c0 < n; c0 += kCoarseThreads) {
        __syncthreads();
        uint32_t j = c0 + threadIdx.x;
        if (j < n) {
            uint32_t di = list[j];
            const tk_draw_record& d = c.draws[di];
            DrawInfo info;
            info.draw = di;
            info.tx = tile_min_(d.pixel_bounds.x0, c.tw) | (tile_max_(d.pixel_bounds.x1, c.tw) << 16);
            info.ty = tile_min_(d.pixel_bounds.y0, c.th) | (tile_max_(d.pixel_bounds.y1, c.th) << 16);
            bool valid_path = d.path_id != TK_INVALID_INDEX && d.tag <= TK_DRAW_PATH_GLYPH && d.path_id < c.path_count;
            info.px = 0; info.py = 0; info.data_offset = 0;
            if (valid_path) {
                const tk_path_record& p = c.paths[d.path_id];
                info.px = p.tile_x0 | (p.tile_x1 << 16);
                info.py = p.tile_y0 | (p.tile_y1 << 16);
                info.data_offset = p.data_offset;
            }
            bool color_candidate = false;
            info.color = di;
            // nontransparent_solid (coarse/paint.hlsli:13-17), read only for the
            // draws that can use it
            auto solid_paint = [&]() {
                return d.brush_offset != TK_INVALID_INDEX && brush_word(c, d.brush_offset) == TK_BRUSH_SOLID &&
                       brush_word(c, d.brush_offset + TK_BRUSH_COLOR_WORD) != 0u;
            };
            // a glyph run draw gives a PTCL_GLYPH particle or none
            // (coarse/emit_draw.hlsli:15-22)
            const bool glyph = TEXT && c.glyph_runs && d.glyph_run_id != TK_INVALID_INDEX;
            const bool has_sdf = !glyph && SDF &&
                                 (d.sdf_offset != TK_INVALID_INDEX || d.sdf_shadow_offset != TK_INVALID_INDEX);
            uint32_t sdf_bits = 0u;
            if (glyph) {
                valid_path = false;
                if (d.tag == TK_DRAW_BRUSH && d.glyph_run_id < c.glyph_run_count) {
                    const tk_glyph_run run = c.glyph_runs[d.glyph_run_id];
                    info.px = run.first;
                    info.py = run.count;
                    sdf_bits |= kMetaGlyph;
                }
            } else if (has_sdf) {
                // draw_has_sdf (shared/draw.hlsli:31): only brush draws give a particle
                valid_path = false;
                const bool plain = d.sdf_offset != TK_INVALID_INDEX;
                info.px = plain ? d.sdf_offset : uint32_t(c.sdf_shadow_base) + d.sdf_shadow_offset;
                const uint32_t kind = __ldg(c.sdf + info.px);
                const bool ident = d.transform.a == 1.0f && d.transform.b == 0.0f && d.transform.c == 0.0f &&
                                   d.transform.d == 1.0f;
                // full_tile_image's brush test: an image pattern at full opacity
                const bool image = d.brush_offset != TK_INVALID_INDEX &&
                                   brush_word(c, d.brush_offset) == TK_BRUSH_PATTERN_RESOURCE &&
                                   brush_word(c, d.brush_offset + TK_BRUSH_IMAGE_ALPHA_WORD) == 255u;
                info.py = (kind & 255u) | (plain ? kSdfPlain : 0u) | (ident ? kSdfIdentity : 0u) |
                          (image ? kSdfImage : 0u);
                if (d.tag == TK_DRAW_BRUSH) sdf_bits |= kMetaSdf;
                const bool solid = solid_paint();
                if (solid) {
                    color_candidate = true;
                    info.color = brush_word(c, d.brush_offset + TK_BRUSH_COLOR_WORD);
                }
                // solid_supported_sdf (coarse/paint.hlsli:21-25)
                if (solid && plain && (kind == TK_SDF_RECT || kind == TK_SDF_CANDLESTICK || kind == TK_SDF_CHECKERBOARD))
                    sdf_bits |= kMetaSdfSolidClass;
            } else if (d.tag == TK_DRAW_BRUSH && d.solid_rect != 0u && d.transform.b == 0.0f &&
                       d.transform.c == 0.0f && solid_paint()) {
                color_candidate = true;
                info.color = brush_word(c, d.brush_offset + TK_BRUSH_COLOR_WORD);
            }
            if (d.tag == TK_DRAW_CLIP) info.color = 0u;
            uint32_t batch = batch_ids[di] - batch0;
            const uint32_t rule = has_sdf ? 0u : (d.fill_rule & 1u);  // SDF particles carry rule 0
            info.meta = (d.tag & 7u) | (rule << 3) | (valid_path ? kMetaPath : 0u) |
                        (color_candidate ? kMetaSolid : 0u) | sdf_bits | (batch << kMetaBatchShift);
            s_d[threadIdx.x] = info;
        }
        __syncthreads();
        if (!live) continue;
        uint32_t m = min(uint32_t(kCoarseThreads), n - c0);
        // Candidates in groups of kPrefetch: the tile tests and the range /
        // backdrop loads of a whole group are issued first, so that their
        // latencies overlap; the group is then walked in painter order.
        constexpr uint32_t kPrefetch = EMIT ? kPrefetchEmit : kPrefetchCount;
        for (uint32_t k0 = 0; k0 < m; k0 += kPrefetch) {
            tk_segment_range rr[kPrefetch];
            uint32_t ww[kPrefetch];
            uint32_t hit = 0u, sdf_hit = 0u, glyph_hit = 0u;
#pragma unroll
            for (uint32_t q = 0; q < kPrefetch; ++q) {
                rr[q] = tk_segment_range{0u, 0u};
                ww[q] = 0u;
                const uint32_t k = k0 + q;
                if (k >= m) continue;
                const DrawInfo& d = s_d[k];
                if (!(tx >= (d.tx & 0xFFFFu) && tx < (d.tx >> 16) && ty >= (d.ty & 0xFFFFu) && ty < (d.ty >> 16))) continue;
                const uint32_t meta = d.meta;
                if (SDF && (meta & kMetaSdf)) {
                    sdf_hit |= 1u << q;
                    continue;
                }
                if (TEXT && (meta & kMetaGlyph)) {
                    glyph_hit |= 1u << q;
                    continue;
                }
                if (!(meta & kMetaPath)) continue;
                const uint32_t px0 = d.px & 0xFFFFu, px1 = d.px >> 16, py0 = d.py & 0xFFFFu, py1 = d.py >> 16;
                if (px1 <= px0 || tx < px0 || ty < py0 || tx >= px1 || ty >= py1) continue;
                const uint32_t tag = meta & 7u;
                if (tag != TK_DRAW_BRUSH && tag != TK_DRAW_PATH_GLYPH && tag != TK_DRAW_CLIP) continue;
                const uint32_t bd = d.data_offset + (ty - py0) * (px1 - px0) + tx - px0;
                rr[q] = c.ranges[bd];
                ww[q] = uint32_t(c.backdrops[bd]);
                hit |= 1u << q;
            }
#pragma unroll
            for (uint32_t q = 0; q < kPrefetch; ++q) {
                if (!((hit | sdf_hit | glyph_hit) & (1u << q))) continue;
                const DrawInfo& d = s_d[k0 + q];
                const uint32_t meta = d.meta, tag = meta & 7u;
                tk_segment_range r = rr[q];
                const uint32_t w = ww[q];  // 0 for SDF and glyph draws
                uint32_t ptag = TK_PTCL_FILL;
                uint32_t glyphs_here = 0u;
                if (TEXT && (glyph_hit & (1u << q))) {
                    glyphs_here = draw_glyphs(c, d.draw, d.px, d.py, tx, ty, nullptr, 0u, 0u, error);
                    if (glyphs_here == 0u) continue;
                    ptag = TK_PTCL_GLYPH;
                } else if (SDF && (sdf_hit & (1u << q))) {
                    ptag = sdf_particle(c.draws, c.sdf, d.draw, d.px, d.py, meta, tx, ty);
                    if (ptag == 0u) continue;
                    // an SDF particle names its draw in segment_start (coarse/emit_draw.hlsli:28)
                    r = ptag == TK_PTCL_SDF ? tk_segment_range{d.draw, 0u} : tk_segment_range{0u, 0u};
                } else {
                    if (r.start == r.end && w == 0u) continue;
                    if (tag == TK_DRAW_CLIP) ptag = TK_PTCL_BEGIN_CLIP;
                    else if (tag == TK_DRAW_PATH_GLYPH) ptag = TK_PTCL_PATH_GLYPH;
                    else if ((meta & kMetaSolid) && r.start == r.end) ptag = TK_PTCL_COLOR;
                }
                uint32_t batch = meta >> kMetaBatchShift;
                if (batch != cur) {
                    close();
                    cur = batch;
                    nb = 0;
                    wrappers = stack_wrappers<SDF>(c, batches[batch], tx, ty);
                    rejected = wrappers == TK_INVALID_INDEX;
                    flags = (!rejected && wrappers) ? kChunkClassOther : 0u;
                    if (EMIT && !rejected) {
                        section = at;
                        at = emit_stack<SDF>(c, batches[batch], tx, ty, true, ptcl, cap, at + 1u, error);
                    }
                }
                if (rejected) continue;
                if (EMIT) {
                    // particle_class_flags (coarse/paint.hlsli:35-40)
                    uint32_t cls = kChunkClassOther;
                    if (ptag == TK_PTCL_COLOR) cls = kChunkClassColor;
                    else if (ptag == TK_PTCL_IMAGE || (ptag == TK_PTCL_SDF && (meta & kMetaSdfSolidClass)))
                        cls = kChunkClassSdf;
                    flags |= cls;
                    uint32_t color = ptag == TK_PTCL_COLOR ? d.color : (tag == TK_DRAW_CLIP ? 0u : d.draw);
                    if (wrappers == 0u && ptag == TK_PTCL_COLOR && (color >> 24) == 255u && nb > 0u) flags |= kChunkClassOccluder;
                    if (TEXT && ptag == TK_PTCL_GLYPH) {
                        // the tile's glyph list continues at gat (coarse/emit.hlsl:54-58)
                        draw_glyphs(c, d.draw, d.px, d.py, tx, ty, glyph_list, gat, glyph_cap, error);
                        store_ptcl(ptcl, cap, at++, ptag, 0u, 0u, uint32_t(gat), uint32_t(gat + glyphs_here), color,
                                   error);
                        gat += glyphs_here;
                    } else {
                        store_ptcl(ptcl, cap, at++, ptag, w, (meta >> 3) & 1u, r.start, r.end, color, error);
                    }
                    if (ptag != TK_PTCL_COLOR && ptag != TK_PTCL_SDF && ptag != TK_PTCL_GLYPH) {
                        fills += 1;
                        visits += r.end - r.start;
                    }
                } else {
                    glyph_total += glyphs_here;
                }
                ++nb;
            }
        }
    }
    if (!live) {
        if (!EMIT && in_canvas) {
            tiles[tile].ptcl_count = 0u;
            tiles[tile].glyph_count = 0u;
        }
        return;
    }
    close();
    if (total) total += 1u;
    if (EMIT) {
        if (total) store_ptcl(ptcl, cap, at, TK_PTCL_END, 0u, 0u, 0u, 0u, 0u, error);
        if (fills) {
            atomicAdd(stats + 0, fills);
            atomicAdd(stats + 1, visits);
        }
    } else {
        tiles[tile].ptcl_count = total;
        tiles[tile].glyph_count = glyph_total;
    }
}

// Exclusive scan of tile counts into ptcl_start / ptcl_end (coarse/prefix.hlsl:11-63),
// single pass with decoupled look-back over 4096-tile blocks. Blocks take
// their position from a ticket, so every predecessor a block waits for is
// already running; each wait still gives up after `poll_limit` polls, sets
// ERR_LOOKBACK_TIMEOUT and carries on, so the kernel always ends.
constexpr int kTileScanThreads = 256, kTilePer = 16, kTileBlock = kTileScanThreads * kTilePer;
constexpr unsigned long long kAgg = 1ull << 62, kIncl = 2ull << 62;

// GLYPH: the same scan of glyph_count into glyph_start / glyph_end (the
// second component of coarse/prefix.hlsl's uint2 scan), for text scenes.
template <bool GLYPH>
__global__ void __launch_bounds__(kTileScanThreads)
    k_tile_prefix(tk_tile_record* tiles, uint32_t T, unsigned long long* desc, uint32_t* ticket, uint32_t* total,
                  uint32_t* error, uint32_t poll_limit) {
    __shared__ uint32_t s_warp[8];
    __shared__ uint32_t s_blk, s_prefix;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_blk = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t blk = s_blk;
    const uint32_t base = blk * kTileBlock;
    uint32_t v[kTilePer];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kTilePer; ++k) {
        uint32_t t = base + tid * kTilePer + k;
        v[k] = t < T ? (GLYPH ? tiles[t].glyph_count : tiles[t].ptcl_count) : 0u;
        sum += v[k];
    }
    uint32_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t p = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += p;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint32_t wpre = 0, agg = 0;
    for (int w = 0; w < 8; ++w) {
        if (w < warp) wpre += s_warp[w];
        agg += s_warp[w];
    }
    if (tid == 0) {
        uint32_t prefix = 0;
        if (blk == 0) {
            atomicExch(desc, kIncl | (unsigned long long)agg);
        } else {
            atomicExch(desc + blk, kAgg | (unsigned long long)agg);
            uint32_t j = blk - 1, spins = 0;
            for (;;) {
                unsigned long long d = *((volatile unsigned long long*)(desc + j));
                unsigned long long st = d & (3ull << 62);
                if (st == 0ull) {
                    if (++spins > poll_limit) { atomicOr(error, ERR_LOOKBACK_TIMEOUT); break; }
                    __nanosleep(64);
                    continue;
                }
                prefix += uint32_t(d);
                if (st == kIncl) break;
                --j;
            }
            __threadfence();
            atomicExch(desc + blk, kIncl | (unsigned long long)(prefix + agg));
        }
        if ((blk + 1u) * kTileBlock >= T) *total = prefix + agg;
        s_prefix = prefix;
    }
    __syncthreads();
    uint32_t run = s_prefix + wpre + incl - sum;
#pragma unroll
    for (int k = 0; k < kTilePer; ++k) {
        uint32_t t = base + tid * kTilePer + k;
        if (t < T) {
            if (GLYPH) {
                tiles[t].glyph_start = run;
                tiles[t].glyph_end = run + v[k];
            } else {
                tiles[t].ptcl_start = run;
                tiles[t].ptcl_end = run + v[k];
                tiles[t].glyph_start = 0u;
                tiles[t].glyph_end = 0u;
            }
        }
        run += v[k];
    }
}

}  // namespace

void launch_bins(const SceneView& s, const PassView& p, cudaStream_t st) {
    const uint32_t nbins = p.scenes ? p.total_bins : p.nbx * p.nby;
    if (nbins == 0) return;
    if (!p.scenes && p.draw_n == 0) {
        cudaMemsetAsync(p.bin_counts, 0, sizeof(uint32_t) * nbins, st);
        return;
    }
    k_bins<<<nbins, 256, 0, st>>>(s.draws, s.order, p.order0, p.draw_n, s.tw, s.th, p.nbx, p.bin_lists, p.bin_counts,
                                  p.scenes, p.bin_scene);
}

void launch_coarse(const SceneView& s, const PassView& p, bool emit, cudaStream_t st) {
    Ctx c{s.draws, s.paths, s.path_count, s.layers, s.brush, s.brush_words, s.sdf, s.sdf_shadow_base, s.backdrops,
          s.ranges, s.tw, s.th, s.glyph_runs, s.glyphs, s.glyph_images, s.glyph_run_count};
    const uint32_t nbins = p.scenes ? p.total_bins : p.nbx * p.nby;
    if (nbins == 0) return;
    const bool sdf = s.sdf_words != 0, text = s.glyph_runs != nullptr;
    using Kernel = decltype(&k_coarse<true, true, true>);
    const Kernel table[2][2][2] = {
        {{k_coarse<false, false, false>, k_coarse<false, false, true>},
         {k_coarse<false, true, false>, k_coarse<false, true, true>}},
        {{k_coarse<true, false, false>, k_coarse<true, false, true>},
         {k_coarse<true, true, false>, k_coarse<true, true, true>}}};
    const Kernel kernel = table[emit][sdf][text];
    kernel<<<nbins * kQuads, kCoarseThreads, 0, st>>>(c, p.bin_lists, p.bin_counts, p.draw_n, p.nbx, s.batch_ids,
                                                      p.batches, p.batch0, p.tiles, p.ptcl, p.ptcl_capacity, p.stats,
                                                      s.error, p.scenes, p.bin_scene, p.tile_active, p.glyph_list,
                                                      p.glyph_capacity);
}

void launch_tile_prefix(const SceneView& s, const PassView& p, cudaStream_t st) {
    uint32_t T = p.scenes ? p.total_tiles : s.tw * s.th;
    launch_tile_prefix_on(p.tiles, T, p.tile_desc, p.ticket, p.ptcl_total, s.error, kTilePrefixPollLimit, 0u, st);
    if (s.glyph_runs) {  // text scenes: the glyph lists' prefix too
        const uint32_t blocks = tile_prefix_blocks(T);
        cudaMemsetAsync(p.tile_desc, 0, sizeof(unsigned long long) * blocks, st);
        cudaMemsetAsync(p.ticket, 0, sizeof(uint32_t), st);
        if (blocks)
            k_tile_prefix<true><<<blocks, kTileScanThreads, 0, st>>>(p.tiles, T, p.tile_desc, p.ticket, p.glyph_total,
                                                                     s.error, kTilePrefixPollLimit);
    }
}

uint32_t tile_prefix_blocks(uint32_t T) { return (T + kTileBlock - 1) / kTileBlock; }

void launch_tile_prefix_on(tk_tile_record* tiles, uint32_t T, unsigned long long* desc, uint32_t* ticket,
                           uint32_t* total, uint32_t* error, uint32_t poll_limit, uint32_t first_ticket,
                           cudaStream_t st) {
    const uint32_t blocks = tile_prefix_blocks(T);
    cudaMemsetAsync(desc, 0, sizeof(unsigned long long) * (blocks + first_ticket), st);
    cudaMemsetAsync(ticket, 0, sizeof(uint32_t), st);
    if (first_ticket) cudaMemcpyAsync(ticket, &first_ticket, sizeof(uint32_t), cudaMemcpyHostToDevice, st);
    if (blocks)
        k_tile_prefix<false><<<blocks, kTileScanThreads, 0, st>>>(tiles, T, desc, ticket, total, error, poll_limit);
}

}  // namespace tk
