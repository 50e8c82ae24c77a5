/*
 * Oracle: CPU restatement of the reference's tile rasterization path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load it. The product (tileink_b200) never links or calls it.
 *
 * It restates, sequentially (or on host threads where the reference runs
 * independent GPU threads), the HLSL kernels and CPU planners of
 * Jianqoq/tileink:
 *   scan    src/shaders/hlsl/scan/{geometry.hlsli,count.hlsl,clip.hlsli,
 *           emit.hlsl,prefix_chunks.hlsl,chunk_offsets.hlsl,
 *           apply_chunk_offsets.hlsl}, cumsum.hlsl
 *   planner src/shared/scan_line.rs, src/shared/gpu_plan/tile_bins/build.rs
 *   coarse  src/shaders/hlsl/coarse/{count.hlsl,emit.hlsl,classify.hlsli,
 *           emit_draw.hlsli,emit_stack.hlsli,occlusion.hlsli,prefix.hlsl,
 *           tile_classification.hlsli}, shared/draw.hlsli
 *   fine    src/shaders/hlsl/fine/{main.hlsl,interpreter.hlsli,
 *           specialized.hlsli,clip.hlsli,group.hlsli}, shared/{coverage,
 *           pixel,affine}.hlsli, shared/brush/{sample,linear,radial,ramp,
 *           extend}.hlsli
 *   blur    src/shaders/hlsl/filter/{blur.hlsli,blur_shared.hlsl,blur.hlsl,
 *           sample.hlsli}, shared/composite_stack.hlsli
 *
 * Arithmetic contract: IEEE f32 with no contraction (built with
 * -ffp-contract=off); HLSL `mad` is a fused multiply-add (std::fma); HLSL
 * `round` rounds half to even; float->int conversions saturate; RGBA8 target
 * loads are k/255 and stores round to nearest even. The only freedom the
 * reference leaves open, the order of atomic increments, is fixed to the
 * sequential order: a path's lines in order, each line's tile steps in order
 * (emit_path in oracle.cpp).
 */
#ifndef TILEINK_ORACLE_H
#define TILEINK_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/tileink.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_scene or_scene;

/* Run the full reference frame (scan, cumsum, bins, per-batch coarse+fine,
 * blur layers) on `threads` host threads. tile_y0/tile_y1 restrict coarse
 * and fine to tile rows [tile_y0, tile_y1) (tile_y1 == 0: all rows); the
 * scan always covers every line. */
int32_t or_run(const tk_scene_desc* scene, int32_t threads, uint32_t tile_y0,
               uint32_t tile_y1, or_scene** out);
void or_free(or_scene* s);
const char* or_error(void);
/* The same frame in two steps: or_prepare runs the scan (count, prefix +
 * cumsum, emit) over every line and bins every draw; or_raster then runs
 * coarse and fine of every pass, and the blur layers, over the tile rows
 * ty (tile_y0 <= ty < tile_y1, tile_y1 == 0: to the last row) with
 * (ty - tile_y0) % row_step == 0, replacing the previous raster's passes and
 * image. A scan serves any number of rasters (row bands of one frame). */
int32_t or_prepare(const tk_scene_desc* scene, int32_t threads, or_scene** out);
int32_t or_raster(or_scene* s, int32_t threads, uint32_t tile_y0, uint32_t tile_y1, uint32_t row_step);

/* Output access. Returns bytes needed; copies min(bytes, needed) into dst
 * when dst != NULL. */
#define OR_COUNTS 0u       /* u32[B] */
#define OR_BACKDROPS 1u    /* i32[B] after cumsum */
#define OR_RANGES 2u       /* tk_segment_range[B] */
#define OR_SEGMENTS 3u     /* tk_line_segment[segment capacity], canonical order */
#define OR_BATCH_PTCL 4u   /* reference layout PTCL of draw batch `index` */
#define OR_BATCH_TILES 5u  /* tk_tile_record[T] of draw batch `index` */
#define OR_BATCH_KINDS 6u  /* u32[T] of draw batch `index` */
#define OR_IMAGE 7u        /* u32[W*H] final image */
#define OR_PASS_PTCL 8u    /* merged PTCL of target pass `index` */
#define OR_PASS_TILES 9u   /* tk_tile_record[T] of target pass `index` */
#define OR_PASS_KINDS 10u  /* u32[T] of target pass `index` */
#define OR_PATHS 11u       /* tk_path_record[P] as used */
#define OR_BUMPS 12u       /* u32[P] per-path segment totals */
#define OR_PASS_GLYPHS 13u /* u32[] glyph list of target pass `index` */
size_t or_get(const or_scene* s, uint32_t what, uint32_t index, void* dst, size_t bytes);
/* Elements [first, first + count) of OR_COUNTS, OR_BACKDROPS, OR_RANGES,
 * OR_SEGMENTS, OR_IMAGE or OR_BUMPS (count clipped); returns the array's
 * element count. */
uint64_t or_get_range(const or_scene* s, uint32_t what, uint64_t first, uint64_t count, void* dst);
/* Number of draw batches / target passes in the run. */
uint32_t or_batch_count(const or_scene* s);
uint32_t or_pass_count(const or_scene* s);
/* Stage wall times in seconds: [scan_count, prefix+cumsum, emit, bins,
 * coarse, fine, blur+composite]. */
void or_stage_times(const or_scene* s, double out[7]);

/* --- Kernel-level restatements used by the golden tests --------------- */

/* CPU planner: tiles visited by one line inside a tile bbox
 * (src/shared/scan_line.rs:17-31). */
uint32_t or_line_scanned_tile_count(const tk_line* line, uint32_t x0, uint32_t y0,
                                    uint32_t x1, uint32_t y1);

/* scan_count for the given lines into backdrops/counts (accumulating). */
void or_scan_count(const tk_line* lines, uint64_t line_count, const tk_path_record* paths,
                   uint32_t path_count, int32_t* backdrops, uint32_t* counts);

/* Per-path prefix (scan_prefix_chunks + chunk_offsets + apply). */
void or_scan_prefix(const uint32_t* counts, const tk_path_record* paths, uint32_t path_count,
                    tk_segment_range* ranges, uint32_t* cursors, uint32_t* bumps);

/* One blur pass (filter_blur_shared_region with its global fallback). */
void or_blur_pass(const uint32_t* src, uint32_t* dst, uint32_t width, uint32_t height,
                  const uint32_t region[4], const uint32_t source[4], float sigma,
                  uint32_t axis);

/* Analytic coverage of one pixel by a PTCL fill over the given tile-local
 * segments, returned before u8 quantization (shared/coverage.hlsli:34-51). */
float or_fill_value(const tk_line_segment* segments, uint32_t count, int32_t backdrop,
                    uint32_t x, uint32_t y);

/* Coverage of one SDF record (TK_SDF_RECORD_WORDS words) at local point
 * (x, y) under the draw inverse transform `inv` (sdf_coverage_from_blob,
 * shared/sdf/coverage.hlsli:13-236), and the library's exp(x) for x <= 0
 * used by shadow falloffs. */
float or_sdf_coverage(const uint32_t* record, float x, float y, const tk_affine* inv);
float or_exp_nonpos(float x);
/* The library's sin / cos and atan2 for the arc and star kinds. */
void or_sincos(float x, float* s, float* c);
float or_atan2(float y, float x);
/* The library's pow for the text gamma (x > 0), and the glyph outline
 * composite src_over_mask_linear_auto_u8 (fine/text/auto.hlsli:28-33). */
float or_text_pow(float x, float y);
/* The filter layer chain (filter/color.hlsli, filter/basic.hlsl) applied in
 * place over rect = {x0, y0, x1, y1} of a width-wide RGBA8 surface;
 * `tables` holds the filter words (transfer tables, kernels) it indexes. */
void or_filter_chain(uint32_t* surface, uint32_t width, const int32_t rect[4], const tk_filter* chain, uint32_t count,
                     const uint32_t* tables);
/* The progressive blur of `surface` (width x height, RGBA8) inside `rect`,
 * and its pyramid plan: per level w, h, scale, variance, step, kernel weight
 * sum and kernel radius (max ceil(|offset - centre|) + 1), 7 floats each;
 * returns the level count. */
int32_t or_progressive_blur(uint32_t* surface, uint32_t width, uint32_t height, const int32_t rect[4],
                            const tk_progressive_blur* blur);
uint32_t or_progressive_levels(uint32_t w, uint32_t h, float sigma, uint32_t quality, float* out, uint32_t cap);
uint32_t or_glyph_over(uint32_t destination, uint32_t source, uint32_t coverage);
/* Fine-only image of a scene of SDF draws: every draw interpreted in every
 * tile as a PTCL_SDF particle, from the clear colour (no coarse stage). */
int32_t or_interpret_sdf_draws(const tk_scene_desc* scene, uint32_t* image);
/* Fine-only image of a scene of path (and SDF) draws in clip and opacity
 * layers: after the scan, every batch's whole layer stack and every draw of
 * the batch are interpreted in every tile with the tile's segment range and
 * backdrop (empty outside a path's bbox), batch after batch, with no tile
 * bins, coarse elision, colour promotion or occlusion skip. No blur layers. */
int32_t or_interpret_path_draws(const tk_scene_desc* scene, int32_t threads, uint32_t* image);
/* The same with the given particle stream in every tile. */
int32_t or_interpret_particles(const tk_scene_desc* scene, const tk_ptcl_record* particles, uint32_t count,
                               uint32_t* image);

/* FP64 loss of the differentiable model (include/tileink_diff.h) for the
 * flattening `lines` / endpoint weights of a forward and the parameters
 * `points` ([point][x, y]), `colors` ([path][rgba] straight), `sigma` with the
 * blur radius held at `radius` (0: no blur). `target` is [H][W][4]; `image`
 * (optional) receives the rendered image. diff_oracle.cpp. */
double or_diff_loss(uint32_t width, uint32_t height, uint32_t path_count, uint64_t line_count,
                    const tk_line* lines, const uint32_t* endpoint_point, const float* endpoint_weights,
                    const double* points, const double* colors, double sigma, int32_t radius,
                    const double* background, const float* target, double* image, int32_t threads);

#ifdef __cplusplus
}
#endif

#endif /* TILEINK_ORACLE_H */
