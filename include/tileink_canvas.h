/*
 * tileink_b200 — host-side scene recording (the reference's `Canvas`).
 *
 * Mirrors the recording API of the reference's Canvas for the vector path:
 *   push_path            src/canvas/primitives/paths.rs:50-60 -> canvas/paths.rs:42-156
 *   push_stroke          src/canvas/primitives/paths.rs:24-48
 *   push_rect / push_circle / push_line and their strokes and shadows
 *                        src/canvas/primitives/{rectangles,shapes,shadows}.rs
 *   push_clip_layer      src/canvas/layers.rs:7-28
 *   push_blur_group      src/canvas/layers.rs:205-212
 *   pop_layer            src/canvas/layers.rs
 * and its compilation into draw batches (src/canvas/compile.rs:39-331,
 * src/shared/execution/batches.rs). `tk_canvas_scene` exposes the recorded
 * records as a tk_scene_desc for tk_scene_upload / tk_render_to_image.
 *
 * Flattening uses the project's own flattener (quadratic flattening by the
 * parabola-integral method, cubics first approximated by quadratics); the
 * reference delegates this to the kurbo crate (0.13.1).
 */
#ifndef TILEINK_B200_CANVAS_H
#define TILEINK_B200_CANVAS_H

#include "tileink.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tk_canvas tk_canvas;
typedef struct tk_path tk_path;

/* Path builder (kurbo::BezPath, f64 coordinates). */
tk_path* tk_path_new(void);
void tk_path_free(tk_path* p);
void tk_path_move_to(tk_path* p, double x, double y);
void tk_path_line_to(tk_path* p, double x, double y);
void tk_path_quad_to(tk_path* p, double x1, double y1, double x2, double y2);
void tk_path_cubic_to(tk_path* p, double x1, double y1, double x2, double y2, double x3, double y3);
void tk_path_close(tk_path* p);

/* Flatten a path into lines (PathFlatten::flatten, src/shared/path_flatten.rs:20-82).
 * Returns the number of lines; writes at most `cap` into `out`. */
uint64_t tk_path_flatten(const tk_path* p, float tolerance, uint32_t path_id, tk_line* out, uint64_t cap);

/* Brushes. Colors are straight (unpremultiplied) sRGB RGBA in [0,1]. */
#define TK_BRUSH_KIND_SOLID 0u
#define TK_BRUSH_KIND_LINEAR 1u
#define TK_BRUSH_KIND_RADIAL 2u
typedef struct tk_gradient_stop {
    float offset;
    float rgba[4];
} tk_gradient_stop;
typedef struct tk_brush_desc {
    uint32_t kind;
    uint32_t extend;        /* TK_EXTEND_* */
    float rgba[4];          /* SOLID */
    float p0[2], p1[2];     /* LINEAR start/end; RADIAL start/end centers */
    float r0, r1;           /* RADIAL radii */
    uint32_t stop_count;
    const tk_gradient_stop* stops;
} tk_brush_desc;

/* Canvas with logical size and scale factor (Canvas::new, canvas/surface.rs:16-21). */
tk_canvas* tk_canvas_new(uint32_t logical_width, uint32_t logical_height, float scale);
void tk_canvas_free(tk_canvas* c);
/* When set (default), segment capacities are planned on the host with the
 * scan-line planner at record time (canvas/storage.rs:131-142); otherwise the
 * scene asks the device to plan them (TK_SCENE_SEGMENTS_FROM_DEVICE). */
void tk_canvas_set_host_segment_plan(tk_canvas* c, int32_t enabled);
/* Fill paths and stroke centerlines recorded after this keep their Bezier
 * elements for tk_scene_upload_flatten, which flattens and strokes them on the
 * device, instead of being flattened on the host. Turns host segment planning
 * off. */
void tk_canvas_set_device_flatten(tk_canvas* c, int32_t enabled);
/* The recorded elements and per-path element ranges (valid until the canvas
 * changes). */
int32_t tk_canvas_flatten_desc(const tk_canvas* c, tk_flatten_desc* out);
void tk_canvas_set_clear_color(tk_canvas* c, uint32_t premul_rgba8);

/* transform: 6 coefficients [a b c d e f] or NULL for identity. Returns the
 * draw index, or -1 on error. */
int64_t tk_canvas_push_path(tk_canvas* c, const tk_path* path, const tk_brush_desc* brush,
                            const double* transform, uint32_t fill_rule, double tolerance);
int64_t tk_canvas_push_stroke(tk_canvas* c, const tk_path* path, const tk_brush_desc* brush,
                              double width, const double* transform, double tolerance);
/* A rasterized glyph image (a glyph cache entry of the caller's text stack)
 * for glyph runs: placement (the image covers x + left .. + width,
 * y - top .. + height for a glyph at pen position (x, y)), size, content
 * (TK_GLYPH_*) and width * height texels. The same texels with the same
 * placement register once. Returns the image index, or -1. */
int32_t tk_canvas_add_glyph_image(tk_canvas* c, int32_t left, int32_t top, uint32_t width, uint32_t height,
                                  uint32_t content, const uint32_t* texels);
/* Canvas::push_text_layout / push_text_layout_clipped
 * (src/canvas/primitives/text.rs:11-100) after layout: `count` glyphs at pen
 * positions in device pixels, drawn with `brush` as one glyph run. Its pixel
 * bounds are the union of its glyph images, intersected with `clip` (x0, y0,
 * x1, y1 in device pixels, or NULL); glyph runs take no transform. Returns
 * the draw index, or -1 (no glyphs, an unknown image, or empty bounds). */
int64_t tk_canvas_push_glyph_run(tk_canvas* c, const tk_glyph* glyphs, uint32_t count, const tk_brush_desc* brush,
                                 const int32_t* clip);
/* Canvas::push_text_layout_as_path (src/canvas/primitives/text.rs:107-147)
 * after shaping: `path` holds the glyph outlines of a laid-out text run (the
 * caller's shaping and outline extraction), filled nonzero with `brush` as a
 * DrawTag::PathGlyph draw, which fine raster composites with the text
 * coverage correction (src_over_mask_linear_auto_u8,
 * fine/text/auto.hlsli:28-33) instead of plain source-over. Returns the draw
 * index, or -1 on error. */
int64_t tk_canvas_push_glyph_outlines(tk_canvas* c, const tk_path* path, const tk_brush_desc* brush,
                                      const double* transform, double tolerance);
/* Analytic SDF shapes (Canvas::push_rect, push_rect_stroke(_widths),
 * push_circle, push_circle_stroke, push_line and push_{rect,circle,line}_shadow,
 * src/canvas/primitives/{rectangles,shapes,shadows}.rs:5-110), in logical
 * coordinates. kind selects the fields used:
 *   TK_SDF_RECT           p0, p1 corners; radii
 *   TK_SDF_RECT_STROKE    p0, p1; radii; widths (full side widths)
 *   TK_SDF_CIRCLE         p0 centre; radius
 *   TK_SDF_CIRCLE_STROKE  p0; radius; width (full stroke width)
 *   TK_SDF_LINE           p0, p1 ends; width; cap
 *   TK_SDF_DASH_LINE      p0, p1; width; cap; dash (dash and gap lengths, offset)
 *   TK_SDF_TRIANGLE       p0, p1, p2 vertices; radius (corner radius)
 *   TK_SDF_CHECKERBOARD   p0, p1 corners; radius (cell size): the even cells
 *                         only (Canvas::push_checkerboard adds the base rect)
 *   TK_SDF_CANDLESTICK    p0 = (centre x, high y), p1 = (body top y, body
 *                         bottom y), p2 = (low y, unused), widths[0] body and
 *                         widths[1] wick width (whole pixels, > 0)
 *   TK_SDF_ARC            p0 centre; radius; width; cap; angle = start,
 *                         sweep (radians)
 *   TK_SDF_STAR(_STROKE)  p0 centre; radius (outer radius); widths[0] inner
 *                         and widths[1] corner radius; angle[0] rotation;
 *                         strokes: width (full stroke width)
 *   TK_SDF_CALLOUT(_STROKE)  p0, p1 body corners; radius (body corner
 *                         radius); cap = tail side (0 top, 1 right, 2 bottom,
 *                         3 left); widths = tail offset, width, length and
 *                         corner radius; flags bit 0 hides the tail; strokes:
 *                         width (full stroke width)
 *   TK_SDF_*_SHADOW       the shape's fields plus shadow
 * The draw is recorded as one SDF record (identity draw transform) whose
 * pixel bounds follow the reference's Sdf::bounds / SdfShadow::bounds. */
typedef struct tk_sdf_shape {
    uint32_t kind;       /* TK_SDF_* */
    uint32_t cap;        /* lines: TK_SDF_CAP_* */
    double p0[2], p1[2], p2[2];
    double radius;       /* circles; triangle corner radius; checkerboard cell size */
    double width;        /* circle strokes and lines */
    float radii[4];      /* corner radii: top-left, top-right, bottom-left, bottom-right */
    float widths[4];     /* rect stroke side widths: top, right, bottom, left */
    float shadow[4];     /* offset x, offset y, expand (falloff length), intensity */
    float dash[3];       /* dash lines: dash length, gap length, dash offset */
    uint32_t flags;      /* callouts: TK_SDF_CALLOUT_TAIL_HIDDEN */
    float angle[2];      /* arcs: start and sweep; stars: rotation */
} tk_sdf_shape;
#define TK_SDF_CALLOUT_TAIL_HIDDEN 1u
/* Returns the draw index, -2 when the shape draws nothing (a non-positive
 * stroke width, an empty line, a shadow of zero intensity: the reference's
 * None), or -1 on error. */
int64_t tk_canvas_push_sdf(tk_canvas* c, const tk_sdf_shape* shape, const tk_brush_desc* brush);
/* Clip layer of an SDF shape (Canvas::push_clip_sdf_layer and its rect,
 * circle, arc and line forms, canvas/layers.rs:34-78): later draws until the
 * matching pop are masked by the shape's coverage. Shadows are not clips;
 * a shape that draws nothing is rejected (-1). */
int32_t tk_canvas_push_clip_sdf_layer(tk_canvas* c, const tk_sdf_shape* shape);
/* Registers an image with the canvas (Canvas::register_scene_image,
 * canvas/primitives/images.rs:42-52): the texels (premultiplied RGBA8, red in
 * the low byte, width * height words, row-major) are copied. Returns the
 * image's index, or -1 for an empty image or one wider or taller than
 * TK_MAX_IMAGE_DIMENSION. */
int32_t tk_canvas_add_image(tk_canvas* c, const uint32_t* premul_rgba8, uint32_t width, uint32_t height);
/* Canvas::push_image (canvas/primitives/images.rs:9-26): a rect from
 * (x0, y0) to (x1, y1), in logical coordinates, filled with registered image
 * `image` scaled into it (Brush::for_rect_resource, shared/brush.rs:557-580),
 * with extend TK_EXTEND_*, sampling TK_PATTERN_* and opacity 0..255 (the
 * reference's push_image uses 255). Returns the draw index, or -1 for an
 * empty or non-finite rect or an unknown image. */
int64_t tk_canvas_push_image(tk_canvas* c, const double rect[4], uint32_t image, uint32_t extend,
                             uint32_t sampling, uint32_t opacity);
int32_t tk_canvas_push_clip_layer(tk_canvas* c, const tk_path* path, const double* transform,
                                  uint32_t fill_rule, double tolerance);
int32_t tk_canvas_push_blur_group(tk_canvas* c, float sigma);
/* The same group blurred with a BlurSampling (TK_BLUR_SAMPLING(factor,
 * downsample filter, upsample filter); factor <= TK_BLUR_MAX_FACTOR): the
 * reference's Filter::Blur { std_dev, std_dev, sampling }
 * (src/shared/layer/filter.rs:53-60) over the group's output bounds.
 * Returns -1 for a bad sigma or sampling word. */
int32_t tk_canvas_push_blur_group_sampled(tk_canvas* c, float sigma, uint32_t sampling);
/* A group blurred by Filter::ProgressiveBlur (src/shared/layer/filter/
 * progressive.rs:14-103): unchanged before `start`, max_std_dev after `end`,
 * smoothstep between along the start-end direction (start == end: a uniform
 * blur of max_std_dev), in logical coordinates; quality TK_PROGRESSIVE_*.
 * Returns -1 for a non-finite or out-of-range parameter. */
int32_t tk_canvas_push_progressive_blur_group(tk_canvas* c, double start_x, double start_y, double end_x,
                                              double end_y, float max_std_dev, uint32_t quality);
/* One filter of a filter layer's chain, in logical units: a colour filter
 * (TK_FILTER_BRIGHTNESS .. TK_FILTER_SEPIA with its amount; hue rotation in
 * degrees), TK_FILTER_COLOR_MATRIX (matrix: 4 rows of r g b a bias),
 * TK_FILTER_OFFSET (dx, dy), TK_FILTER_ERODE / TK_FILTER_DILATE (dx, dy:
 * the radii along x and y), TK_FILTER_FLOOD (rgba: a straight colour) or
 * TK_FILTER_DROP_SHADOW (dx, dy: the offset, std_dev, rgba) or
 * TK_FILTER_COMPONENT_TRANSFER (table: TK_TRANSFER_TABLE_WORDS words, each
 * 0..255, copied by the call) or TK_FILTER_CONVOLVE (kernel: columns x rows
 * floats, copied; target, divisor, bias, edge_mode, preserve_alpha) or
 * TK_FILTER_BLUR (dx, dy: the standard deviations along x and y). */
typedef struct tk_canvas_filter {
    uint32_t kind;
    float amount;
    float dx, dy;
    float rgba[4];
    float std_dev;
    float matrix[20];
    const uint32_t* table;
    const float* kernel;
    uint32_t columns, rows, target_x, target_y, edge_mode, preserve_alpha;
    float divisor, bias;
} tk_canvas_filter;
/* Canvas::push_filter_layer with Filter::Chain { filters, fixed_region } and
 * a Region::Rect sample region without corner radii (src/canvas/layers.rs:
 * 222-233; physical_filter / physical_region, canvas/surface.rs:197-326):
 * the children until the matching pop are rendered into a surface, filtered
 * in place by the chain and composited over the output bounds (the region's
 * pixel bounds grown by the chain's reach unless fixed_region, clipped to
 * the canvas; shared/layer/filter.rs:510-597). `rect` = {x0, y0, x1, y1}.
 * Returns -1 for an unknown kind or a non-finite value. */
int32_t tk_canvas_push_filter_layer(tk_canvas* c, const tk_canvas_filter* filters, uint32_t count, const double rect[4],
                                    int32_t fixed_region);
/* The same with a Region::Path sample region: the region's bounds are the
 * tight box of `path` under `transform` (may be null) and the canvas scale.
 * Corner radii of a rect region do not change its bounds, so a rounded rect
 * region is its rect. */
int32_t tk_canvas_push_filter_layer_path(tk_canvas* c, const tk_canvas_filter* filters, uint32_t count,
                                         const tk_path* path, const double* transform, int32_t fixed_region);
/* Canvas::push_opacity_layer (src/canvas/layers.rs:122-140): the children
 * until the matching pop are composited at `opacity` (clamped to [0, 1],
 * stored as opacity_f32_to_u8) through the nonzero coverage of `path`. The
 * layer is fused into each batch's layer stack (a BEGIN_OPACITY / END_OPACITY
 * pair per tile), which is how the reference compiles it when the subtree
 * draws in one stack (src/canvas/compile.rs:342-353). A subtree that does not
 * (a blur group below it, or draws both beside and inside a nested layer)
 * needs the reference's offscreen group: tk_canvas_scene then fails and
 * tk_canvas_last_error says why. Returns -1 for a null path, a tolerance
 * <= 0 or a non-finite opacity. */
int32_t tk_canvas_push_opacity_layer(tk_canvas* c, const tk_path* path, const double* transform,
                                     double tolerance, float opacity);
int32_t tk_canvas_pop_layer(tk_canvas* c);
/* Why the last tk_canvas_scene failed ("" when it did not). */
const char* tk_canvas_last_error(const tk_canvas* c);

/* Compile (if needed) and describe the recorded scene. Pointers stay valid
 * until the canvas is modified or freed. */
int32_t tk_canvas_scene(tk_canvas* c, tk_scene_desc* out);

/* Command log: when set, the canvas also keeps every later push / pop call
 * with its original geometry, brush and transform, so that it can be replayed
 * into another canvas (and become a retained scene node). */
void tk_canvas_set_keep_commands(tk_canvas* c, int32_t enabled);
/* Replays `src`'s logged calls into `dst`, each call's transform preceded by
 * `transform` (NULL: as recorded). `src` must keep commands and have every
 * layer it opened closed. */
int32_t tk_canvas_replay(tk_canvas* dst, const tk_canvas* src, const double* transform);

/* ------------------------------------------------------------------------ */
/* Retained scene (RetainedScene, src/retained_scene/scene.rs:14-140 and     */
/* transaction.rs:74-255): nodes in painter order, each a copy of a          */
/* command-keeping canvas's calls under a node transform. Every mutation     */
/* bumps the version. tk_retained_materialize records the nodes into one     */
/* canvas and reports the damage since the previous materialization: the     */
/* pixel bounds, before and after, of every node inserted, replaced,         */
/* transformed, moved or removed, plus invalidated rectangles; everything    */
/* on the first call, after invalidate_all or a clear colour change, and     */
/* when a changed node has clip or blur layers (which can regroup the draw   */
/* batches of other nodes). That damage drives tk_render_incremental.        */
/* ------------------------------------------------------------------------ */
typedef struct tk_retained tk_retained;
tk_retained* tk_retained_new(uint32_t logical_width, uint32_t logical_height, float scale);
void tk_retained_free(tk_retained* rs);
void tk_retained_set_clear_color(tk_retained* rs, uint32_t premul_rgba8);
/* Materialized canvases record fills and stroke centerlines as elements for
 * device flattening (the lines are the same either way). */
void tk_retained_set_device_flatten(tk_retained* rs, int32_t enabled);
uint64_t tk_retained_version(const tk_retained* rs);
/* id != 0 and unused; before = 0 appends, else the node goes in front of
 * node `before`. transform NULL = identity. Returns 0, or -1 on error. */
int32_t tk_retained_insert(tk_retained* rs, uint64_t id, const tk_canvas* content, const double* transform,
                           uint64_t before);
int32_t tk_retained_replace(tk_retained* rs, uint64_t id, const tk_canvas* content);
int32_t tk_retained_set_transform(tk_retained* rs, uint64_t id, const double* transform);
/* sibling = 0 moves the node to the end (painted last). */
int32_t tk_retained_move_before(tk_retained* rs, uint64_t id, uint64_t sibling);
int32_t tk_retained_remove(tk_retained* rs, uint64_t id);
/* rect: {x0, y0, x1, y1} in physical pixels, half-open. */
int32_t tk_retained_invalidate_rect(tk_retained* rs, const int32_t rect[4]);
int32_t tk_retained_invalidate_all(tk_retained* rs);
/* The scene as one canvas (owned by `rs`, valid until the next call or
 * tk_retained_free) and, in `damage` (may be NULL), what changed since the
 * previous call; damage->rects points into `rs` with the same lifetime. */
tk_canvas* tk_retained_materialize(tk_retained* rs, tk_damage* damage);

/* Seeded synthetic workloads. `config`: 1 = 640x360 240 cubic fills;
 * 2 = 4096x4096 50k mixed fills/strokes/gradients/clips; 3 = 1920x1080 20k
 * quadratic glyphs; 4 = one scene of the uneven batch (index = `variant`);
 * 5 = 1024x1024 256 cubic paths inside a sigma-4 blur group. Zero fields in
 * `overrides` keep the workload's defaults. */
typedef struct tk_gen_params {
    uint32_t width, height;   /* canvas size */
    uint32_t paths;           /* path / glyph count */
    uint32_t variant;         /* config 4: scene index */
    float sigma;              /* config 5: blur sigma */
    float jitter;             /* config 5: control point jitter (px) */
    uint32_t flags;           /* 1: host segment planning off; 2: device flattening of fills */
    uint32_t reserved;
} tk_gen_params;
tk_canvas* tk_generate(uint32_t config, uint64_t seed, const tk_gen_params* overrides);

/* Differentiable parameters of configs 1 and 5 (fills of cubic paths with
 * solid colors): control points per path element and straight RGBA colors.
 * Returns the number of floats of each array when the pointer is NULL. */
uint64_t tk_canvas_param_points(const tk_canvas* c, double* out);  /* all path points, x,y */
uint64_t tk_canvas_param_colors(const tk_canvas* c, float* out);   /* per draw straight RGBA */

#ifdef __cplusplus
}
#endif

#endif /* TILEINK_B200_CANVAS_H */
