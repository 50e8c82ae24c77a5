// Host-side launchers of the device pipeline (implemented in *.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>
#include <vector>

#include "../../include/tileink.h"

namespace tkf {
struct Pt;
}

namespace tk {

// Error bits raised by kernels into a device word.
constexpr uint32_t ERR_LOOKBACK_TIMEOUT = 1u << 0;
constexpr uint32_t ERR_LINE_PATH_MISMATCH = 1u << 1;
constexpr uint32_t ERR_SEGMENT_OVERFLOW = 1u << 2;
constexpr uint32_t ERR_PTCL_OVERFLOW = 1u << 3;
constexpr uint32_t ERR_STACK_DEPTH = 1u << 4;
constexpr uint32_t ERR_UNSUPPORTED = 1u << 5;

// One work item of the pool scan: whole rows [row0, row0 + rows) of `path`,
// at most kScanItemElems elements.
struct ScanItem {
    uint32_t path, row0, rows, first;  // first: 1 when row0 == 0
};
constexpr uint32_t kScanItemElems = 4096;

// Per draw-batch data of one target pass.
struct PassBatch {
    uint32_t batch_id, layer_start, layer_end, pad;
};

// A tile segment as the device stores it: the LineSegment fields
// (src/shared/line_seg.rs:1-9) padded to one 32-byte sector, so that every
// segment write covers whole sectors (20-byte records left partly written
// sectors at the edges of short tile ranges, which HBM had to read back), plus
// the slope (p1x - p0x) / (p1y - p0y) (0 when p1y == p0y) that fine raster
// needs per segment. Debug readback strips it to the 20-byte record.
struct alignas(32) SegmentRec {
    float p0x, p0y, p1x, p1y, y_edge, slope;
    uint32_t pad[2];
};
static_assert(sizeof(SegmentRec) == 32, "one sector per segment");

// A draw's paint as fine raster needs it, decoded once per upload from the
// draw record and its brush (fine.cu): the solid premultiplied colour, or
// kGradient with the gradient's brush-only terms, and the first word of the
// draw's SDF record in the device SDF buffer (TK_INVALID_INDEX for none).
struct alignas(16) PaintInfo {
    uint32_t paint;      // premultiplied RGBA8, or 0xFFFFFFFF for a gradient
    uint32_t sdf;
    uint32_t pad[2];
    uint4 gk;            // kind | flags, ramp word (or colour), ramp length, extend
    float g[24];         // transforms and brush terms (fine.cu stage_gradient)
};
static_assert(sizeof(PaintInfo) == 128, "two 64-byte halves");

struct SceneView {
    const tk_line* lines;
    uint64_t line_count;
    tk_path_record* paths;
    uint32_t path_count;
    const tk_draw_record* draws;
    uint32_t draw_count;
    const uint32_t* brush;
    uint64_t brush_words;
    // SDF records: the scene's sdf_blob followed by its sdf_shadow_blob
    const uint32_t* sdf;
    uint64_t sdf_words;
    uint64_t sdf_shadow_base;
    bool sdf_ext;  // some record is of an extended kind (fine's k_fine<2>)
    bool text;     // glyph outline fills or glyph runs (fine's text instances)
    const uint32_t* texels;  // the scene's images, concatenated (premultiplied RGBA8)
    // the text blob (null without glyph runs)
    const tk_glyph_run* glyph_runs;
    const tk_glyph* glyphs;
    const tk_glyph_image* glyph_images;
    const uint32_t* glyph_texels;
    uint32_t glyph_run_count;
    const tk_layer_record* layers;
    const uint32_t* batch_ids;
    const uint32_t* order;
    uint32_t width, height, tw, th;
    // pool
    int32_t* backdrops;
    uint32_t* counts;
    tk_segment_range* ranges;
    uint32_t* cursors;
    uint64_t pool_len;
    SegmentRec* segments;
    uint64_t segment_capacity;
    uint32_t* error;
    uint32_t* seg_line;  // optional: line index of every emitted segment
    const PaintInfo* paints;     // per draw (launch_paint_table)
    const uint32_t* emit_order;  // paths by decreasing line count (optional)
    uint32_t* emit_ticket;       // path queue of scan_emit
};

void launch_scan_count(const SceneView& s, cudaStream_t st);
// Row-blocked pool scan: segment ranges + cursors (per-path prefix from
// segment_start, or one chain over all paths when device_plan), and the
// row-wise backdrop cumsum, in three passes (item sums, item prefixes, apply).
// item_scratch holds 8 bytes per item; `total` receives the last inclusive
// value.
void launch_pool_scan(const SceneView& s, const ScanItem* items, uint32_t n_items, unsigned long long* item_scratch,
                      bool device_plan, uint32_t device_base, uint32_t* total, cudaStream_t st);
void launch_path_totals(const SceneView& s, uint32_t* bumps, bool device_plan, const uint32_t* total,
                        cudaStream_t st);
void launch_scan_emit(const SceneView& s, cudaStream_t st);
// The scan of the listed paths only (n entries of `list`, device memory):
// clear their backdrop and count slices and count their lines; emit their
// segments. Their pool scan runs through launch_pool_scan with their items.
void launch_scan_count_paths(const SceneView& s, const uint32_t* list, uint32_t n, cudaStream_t st);
void launch_scan_emit_paths(const SceneView& s, const uint32_t* list, uint32_t n, cudaStream_t st);
// *changed = 1 when a listed path's segment total (bumps, from
// launch_path_totals) differs from its planned segment_capacity.
void launch_check_path_totals(const SceneView& s, const uint32_t* bumps, const uint32_t* list, uint32_t n,
                              uint32_t* changed, cudaStream_t st);

// Fixed scratch of the allocation-free pool scan (one array per device).
struct NoAllocScratch {
    unsigned long long* desc;  // TK_NOALLOC_MAX_SCAN_ITEMS item sum / prefix pairs
    ScanItem* items;           // TK_NOALLOC_MAX_SCAN_ITEMS work items
    tk_path_record* paths;     // TK_NOALLOC_MAX_PATHS path records
    uint32_t* words;           // [0] error [1] unused [2] total
};
// Resolves the scratch address of `device` (which must be current) once and
// caches it.
cudaError_t noalloc_scratch(int device, NoAllocScratch* out);
void launch_build_scan_items(const tk_path_record* paths, uint32_t path_count, ScanItem* items, cudaStream_t st);

// One canvas of a batched pass: several independent scenes go through each
// stage in one launch; their tiles, bins and images are concatenated.
struct BatchScene {
    uint32_t tile_base, bin_base;  // first global tile / bin of the scene
    uint64_t list_base;            // first word of the scene's bin lists
    uint32_t tw, th, nbx;          // tile grid and bins per row
    uint32_t order0, draw_n;       // draw_order[order0 .. order0 + draw_n)
    uint32_t width, height;
    uint32_t clear;                // premultiplied RGBA8 clear colour
    uint64_t image_offset;         // first pixel of the scene's image
};

// Target pass: binning, coarse count, tile prefix, coarse emit, fine.
struct PassView {
    uint32_t order0, draw_n;          // draw_order[order0 .. order0 + draw_n)
    const PassBatch* batches;         // indexed by batch ordinal within the pass
    uint32_t batch0;                  // first batch_id of the pass
    uint32_t batch_n;
    uint32_t nbx, nby;                // 16x16-tile bins
    uint32_t* bin_lists;              // nbins * draw_n
    uint32_t* bin_counts;             // nbins
    tk_tile_record* tiles;            // T
    tk_ptcl_record* ptcl;
    uint64_t ptcl_capacity;
    unsigned long long* tile_desc;    // lookback descriptors for the tile scan
    uint32_t* ticket;
    uint32_t* ptcl_total;
    // glyph lists: the glyph indices PTCL_GLYPH records name (text scenes)
    uint32_t* glyph_list;
    uint64_t glyph_capacity;
    uint32_t* glyph_total;
    unsigned long long* stats;        // [0] fill records, [1] segment visits
    // batched pass (null for one canvas): per-scene geometry and the scene
    // of every global bin and tile
    const BatchScene* scenes;
    const uint32_t* bin_scene;
    const uint32_t* tile_scene;
    uint32_t total_bins, total_tiles, scene_count;
    // incremental render (null: every tile): per tile 1 when it is redrawn,
    // and the list of those tiles
    const uint8_t* tile_active;
    const uint32_t* tile_list;
    uint32_t tile_list_n;
};
void launch_bins(const SceneView& s, const PassView& p, cudaStream_t st);
void launch_coarse(const SceneView& s, const PassView& p, bool emit, cudaStream_t st);
void launch_tile_prefix(const SceneView& s, const PassView& p, cudaStream_t st);
// The tile prefix on explicit buffers: `desc` holds tile_prefix_blocks(T) +
// first_ticket words. The block ticket starts at `first_ticket` (1 leaves
// block 0's descriptor unpublished: the bounded-wait test); each look-back
// wait gives up after `poll_limit` polls.
constexpr uint32_t kTilePrefixPollLimit = 1u << 22;
uint32_t tile_prefix_blocks(uint32_t T);
void launch_tile_prefix_on(tk_tile_record* tiles, uint32_t T, unsigned long long* desc, uint32_t* ticket,
                           uint32_t* total, uint32_t* error, uint32_t poll_limit, uint32_t first_ticket,
                           cudaStream_t st);
void launch_fine(const SceneView& s, const PassView& p, uint32_t* target, cudaStream_t st);
// The per-draw PaintInfo table of the uploaded draws and brush blob; shadow
// records start at word sdf_shadow_base of the device SDF buffer.
// images: per image of the texture table its first texel, width and height.
void launch_paint_table(const tk_draw_record* draws, uint32_t draw_count, const uint32_t* brush,
                        uint64_t brush_words, uint32_t sdf_shadow_base, const uint4* images, uint32_t image_count,
                        PaintInfo* out, cudaStream_t st);

// Images.
void launch_fill(uint32_t* image, uint64_t n, uint32_t value, cudaStream_t st);
// Batch upload: lines of scene k occupy [line_base[k], line_base[k + 1]) and
// get path_base[k] added to their path ids.
void launch_rebase_lines(tk_line* lines, uint64_t n, const uint64_t* line_base, const uint32_t* path_base,
                         uint32_t scenes, cudaStream_t st);
// Sets the pixels of the listed 16x16 tiles of a width x height image to value.
void launch_fill_tiles(uint32_t* image, uint32_t width, uint32_t height, uint32_t tw, const uint32_t* tiles,
                       uint32_t n, uint32_t value, cudaStream_t st);
// Clears every scene's image region of a batched pass to its clear colour.
void launch_fill_scenes(uint32_t* image, const BatchScene* scenes, uint32_t scene_count, cudaStream_t st);
struct BlurParams {
    uint32_t width, height;
    uint32_t region[4];   // x0, y0, width, height
    int32_t bounds[4];    // sample bounds x0, y0, x1, y1
    float sigma;
    uint32_t axis;
};
void launch_blur(const uint32_t* src, uint32_t* dst, const BlurParams& b, cudaStream_t st);
void launch_composite(uint32_t* dst, const uint32_t* src, uint32_t width, const int32_t bounds[4], cudaStream_t st);
// A filter layer's chain applied in place to `surface` over `bounds`
// (filter.cu); `temp` is a scratch surface of the same size, `temp2` a second
// one that drop shadows need (null for chains without one), `tables` the
// scene's component transfer tables on the device.
void launch_filter_chain(uint32_t* surface, uint32_t* temp, uint32_t* temp2, const uint32_t* tables, uint32_t width,
                         uint32_t height, const int32_t bounds[4], const tk_filter* chain, uint32_t count,
                         cudaStream_t st);

// Progressive blur (progressive.cu). A pyramid level: its size, scale and
// cumulative variance, its decimation step and its paired kernel (offset,
// weight); level 0 is the blurred region itself.
constexpr uint32_t kProgressiveMaxLevels = 64;  // the reference's level table
struct ProgressiveLevel {
    uint32_t w = 0, h = 0;
    float scale = 1.0f, variance = 0.0f;
    uint32_t step = 1;
    std::vector<std::pair<float, float>> kernel;
};
std::vector<ProgressiveLevel> progressive_levels(uint32_t w, uint32_t h, float sigma, uint32_t quality);
// Device memory the context keeps for it (levels concatenated, one scratch).
struct ProgressiveScratch {
    uint32_t* levels = nullptr;
    uint64_t levels_cap = 0;
    uint32_t* scratch = nullptr;
    uint64_t scratch_cap = 0;
};
// The progressive blur of `surface` inside `rect` (clipped to the surface):
// 1 when it ran, 0 for an empty rect or no blur, -1 for a pyramid beyond
// kProgressiveMaxLevels or too many taps, -2 when memory ran out.
int32_t launch_progressive_blur(uint32_t* surface, uint32_t width, uint32_t height, const int32_t rect[4],
                                const tk_progressive_blur& blur, ProgressiveScratch& s, cudaStream_t st);
void release_progressive(ProgressiveScratch& s);
// The blur of `surface` inside `rect` (x0, y0, x1, y1) through a reduced copy
// (BlurSampling with factor > 1, filter/resample.hlsli): downsample into
// `low`, blur there at sigma / factor (`temp` holds the horizontal pass),
// upsample back into `surface` over `rect`. `sampling` = factor | downsample
// filter << 8 | upsample filter << 16 (TK_BLUR_SAMPLING_*). All three buffers
// are width x height. Returns 0 when the rect is empty.
int32_t launch_blur_downsampled(uint32_t* surface, uint32_t* low, uint32_t* temp, uint32_t width, uint32_t height,
                                const int32_t rect[4], float sigma, uint32_t sampling, cudaStream_t st);


// Device flattening (flatten.cu): per-element line counts, exclusive offsets
// in `counts` and the total; then path line ranges and the lines themselves.
void launch_flatten_count(const tk_flatten_el* els, uint64_t n, uint32_t* counts, uint32_t* block_sums,
                          uint32_t* total, uint32_t* error, cudaStream_t st);
void launch_flatten_emit(const tk_flatten_el* els, uint64_t n, const uint32_t* offsets, const uint32_t* total,
                         tk_path_record* paths, uint32_t path_count, const uint32_t* path_els, tk_line* lines,
                         uint64_t line_base, uint64_t line_end, uint32_t* error, cudaStream_t st);
size_t flatten_block_sums(uint64_t n);
// Exclusive scan of n u32 values in place (1024 per block; block totals in
// block_sums, flatten_block_sums(n) words); `total` receives the sum.
void launch_exclusive_scan(uint32_t* v, uint64_t n, uint32_t* block_sums, uint32_t* total, cudaStream_t st);

// Device stroking (stroke.cu). launch_stroke_count: raw centerline points per
// stroke element, scanned into exclusive offsets (u32 total, plus the exact
// u64 sum to catch wrap-around). launch_stroke_outline_count: writes the
// points, cleans each polyline and counts its outline lines into line_off,
// scanned into exclusive offsets. launch_stroke_emit: writes the lines and
// the stroked paths' line ranges.
struct StrokeView {
    const tk_flatten_el* els;
    uint64_t n_els;
    const uint32_t* offsets;   // per element: first raw point
    const uint32_t* pt_total;  // raw points
    tkf::Pt* pts;
    uint64_t pt_cap;
    const tk_stroke_polyline* polys;
    uint32_t npl;
    const tk_stroke_desc* strokes;
    uint32_t n_strokes;
    uint32_t* poly_n;    // per polyline: points kept
    uint32_t* line_off;  // per polyline: lines, then their exclusive offsets
    uint32_t* error;
    uint32_t* unit_lines;  // per outline unit: its lines (2 slots per raw point)
};
void launch_stroke_count(const tk_flatten_el* els, uint64_t n, uint32_t* counts, uint32_t* block_sums,
                         uint32_t* total, unsigned long long* total64, uint32_t* error, cudaStream_t st);
void launch_stroke_outline_count(const StrokeView& v, uint32_t* block_sums, uint32_t* line_total,
                                 unsigned long long* line_total64, cudaStream_t st);
void launch_stroke_emit(const StrokeView& v, const uint32_t* line_total, tk_path_record* paths, tk_line* lines,
                        uint64_t line_base, uint64_t line_end, cudaStream_t st);

// Differentiable rendering (diff.cu): float forward and adjoint.
void launch_diff_fine_fwd(const SceneView& s, const PassView& p, const float4* colp, float4* layer, cudaStream_t st);
void launch_diff_blur(const float4* in, float4* out, const float* w, int32_t r, uint32_t width, uint32_t height,
                      int32_t axis, cudaStream_t st);
void launch_diff_composite(const float4* B, const float4* target, float4 bg, uint64_t n, uint64_t lo, uint64_t hi,
                           float4* image, float4* gI, double* loss, cudaStream_t st);
void launch_diff_blur_bwd(const float4* dout_src, const float4* fwd_in, float4* din, const float* w, const float* wd,
                          int32_t r, uint32_t width, uint32_t height, int32_t axis, bool from_gI, float4 bg,
                          double* sig, cudaStream_t st);
void launch_diff_composite_bwd(const float4* gI, float4 bg, uint64_t n, float4* dL, cudaStream_t st);
void launch_diff_fine_bwd(const SceneView& s, const PassView& p, const uint32_t* seg_line, const float4* colp,
                          const float4* dlayer, float2* scratch, float2* line_acc, float* color_acc, cudaStream_t st);
void launch_diff_lines_to_points(const tk_line* lines, const float2* line_acc, const uint32_t* ep_base,
                                 const float* ep_w, uint64_t n, float* dpoints, cudaStream_t st);

}  // namespace tk
