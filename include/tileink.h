/*
 * tileink_b200 — C ABI of the B200-native tile rasterization path.
 *
 * This header is the drop-in boundary. It replaces, for the vector
 * rasterization path, the reference's internal compute boundary:
 *   - `ComputeBatch` + `Adapter::submit_compute` + `Receipt::readback`
 *     (src/native/runtime/compute.rs:68-120,195,307; adapter.rs:159;
 *      submission.rs:120), and
 *   - the public wrapper `NativeRenderer::render_to_image`
 *     (src/native/renderer.rs:177-190).
 * A thin Rust FFI crate binds these symbols with `#[repr(C)]` mirrors of the
 * records below; the records are byte-identical to the reference's Pod types,
 * so a `Canvas` can hand its vectors over unchanged.
 *
 * Conventions (all entry points):
 *   - every call returns an int32 status: 0 = ok, negative = error
 *     (TK_E_*); `tk_last_error(ctx)` returns the message of the last failure;
 *   - no C++ exception crosses this ABI;
 *   - a context is used by one host thread at a time (the reference's
 *     `Rc<RefCell<..>>` runtime is `!Send` for the same reason);
 *   - host pointers passed in are borrowed for the duration of the call only;
 *     outputs go to caller-allocated buffers.
 */
#ifndef TILEINK_B200_H
#define TILEINK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Algorithm constants (src/shaders/hlsl/constants.hlsli:7-19).              */
/* ------------------------------------------------------------------------ */
#define TK_TILE_SIZE 16u
#define TK_TILE_PIXELS (TK_TILE_SIZE * TK_TILE_SIZE)
#define TK_INVALID_INDEX 0xFFFFFFFFu
#define TK_SHARED_BLUR_MAX_RADIUS 16u

/* Draw tags (src/shared/draw_record.rs:7-17, shaders/hlsl/shared/draw_tags.hlsli) */
#define TK_DRAW_BRUSH 0u
#define TK_DRAW_CLIP 1u
#define TK_DRAW_OPACITY 2u
#define TK_DRAW_BLEND 3u
#define TK_DRAW_ISOLATE 4u
#define TK_DRAW_PATH_GLYPH 5u

/* Layer stack tags (shaders/hlsl/shared/draw_tags.hlsli:7-9) */
#define TK_LAYER_CLIP 0u
#define TK_LAYER_OPACITY 1u
#define TK_LAYER_BLEND 2u

/* Fill rules (src/shared/fill.rs:1-6) */
#define TK_FILL_NONZERO 0u
#define TK_FILL_EVEN_ODD 1u

/* PTCL tags (shaders/hlsl/shared/particle_tags.hlsli:3-16). */
#define TK_PTCL_END 0u
#define TK_PTCL_FILL 1u
#define TK_PTCL_COLOR 2u
#define TK_PTCL_BEGIN_CLIP 3u
#define TK_PTCL_END_CLIP 4u
#define TK_PTCL_BEGIN_OPACITY 5u
#define TK_PTCL_END_OPACITY 6u
#define TK_PTCL_BEGIN_BLEND 7u
#define TK_PTCL_END_BLEND 8u
#define TK_PTCL_SDF 9u
#define TK_PTCL_GLYPH 10u
#define TK_PTCL_PATH_GLYPH 11u
#define TK_PTCL_BEGIN_SDF_CLIP 12u
#define TK_PTCL_IMAGE 13u
/* Merged-stream extension (no reference counterpart). All draw batches of a
 * target pass share one PTCL stream per tile; each batch with particles in
 * the tile opens its section with BATCH_BEGIN {segment_start = batch id,
 * segment_end = record count of the section, color = tile kind | skip << 3
 * of that batch}, followed by the reference's batch stream without its END;
 * one END closes the tile. Fine stores the pixel to RGBA8 and reloads it at
 * each BATCH_BEGIN (the reference's per-batch target store/load) and resets
 * the clip/group state. */
#define TK_PTCL_BATCH_BEGIN 14u

/* Tile kinds (shaders/hlsl/shared/tile_kinds.hlsli:3-11) */
#define TK_TILE_KIND_INTERPRETER 0u
#define TK_TILE_KIND_EMPTY 1u
#define TK_TILE_KIND_COLOR 2u
#define TK_TILE_KIND_SDF 3u
#define TK_TILE_KIND_MIXED 4u
#define TK_TILE_KIND_MASK 7u
#define TK_TILE_PREFIX_SHIFT 3u

/* SDF records (src/shared/gpu_sdf.rs:27-46, shaders/hlsl/shared/sdf/
 * constants.hlsli:3-21): TK_SDF_RECORD_WORDS words per shape, word 0 the kind,
 * then four coordinate, four radius, four stroke and four shadow words as
 * floats (coverage.hlsli:13-30). A draw's sdf_offset indexes the scene's
 * sdf_blob, its sdf_shadow_offset the sdf_shadow_blob. The kinds below are
 * the ones this library renders; other kinds are rejected at upload. */
#define TK_SDF_RECORD_WORDS 17u
#define TK_SDF_RECT 1u
#define TK_SDF_CIRCLE 2u
#define TK_SDF_RECT_STROKE 3u
#define TK_SDF_CIRCLE_STROKE 4u
#define TK_SDF_CANDLESTICK 5u
#define TK_SDF_LINE 6u
#define TK_SDF_RECT_SHADOW 7u
#define TK_SDF_ARC 8u
#define TK_SDF_ARC_SHADOW 9u
#define TK_SDF_CIRCLE_SHADOW 10u
#define TK_SDF_LINE_SHADOW 11u
#define TK_SDF_DASH_LINE 12u
#define TK_SDF_TRIANGLE 13u
#define TK_SDF_CHECKERBOARD 14u
#define TK_SDF_STAR 15u
#define TK_SDF_STAR_STROKE 16u
#define TK_SDF_CALLOUT 17u
#define TK_SDF_CALLOUT_STROKE 18u
#define TK_SDF_CALLOUT_SHADOW 19u
#define TK_SDF_CAP_BUTT 0u
#define TK_SDF_CAP_SQUARE 1u
#define TK_SDF_CAP_ROUND 2u

/* Brush blob layout (shaders/hlsl/shared/brush/constants.hlsli:3-22,
 * src/shared/brush.rs:249-340). A brush record is a 9-word header followed by
 * 12 parameter words and an optional payload (gradient ramp). */
#define TK_BRUSH_HEADER_WORDS 9u
#define TK_BRUSH_PARAM_WORDS 12u
#define TK_BRUSH_SOLID 1u
#define TK_BRUSH_LINEAR 2u
#define TK_BRUSH_RADIAL 3u
#define TK_BRUSH_COLOR_WORD 4u
/* Image pattern brush (BRUSH_PATTERN_RESOURCE, shared/brush/constants.hlsli:9-21,
 * src/shared/brush.rs:325-339): header word 1 extend, 4 placement
 * (TK_BRUSH_TEXTURE_PLACEMENT_BIT | index into tk_scene_desc.images), 5 and 6
 * the image's width and height, 7 opacity (0..255), 8 sampling; parameter
 * words 0..5 the f32 transform [a b c d e f] from pixel space to the unit
 * square of the image. */
#define TK_BRUSH_PATTERN_RESOURCE 7u
#define TK_BRUSH_IMAGE_ALPHA_WORD 7u
#define TK_BRUSH_TEXTURE_PLACEMENT_BIT 0x80000000u
#define TK_PATTERN_NEAREST 0u
#define TK_PATTERN_BILINEAR 1u
#define TK_EXTEND_PAD 0u
#define TK_EXTEND_REPEAT 1u
#define TK_EXTEND_REFLECT 2u

/* One image of a scene's texture table: premultiplied RGBA8 texels (red in
 * the low byte), row-major and tightly packed, width * height words. Width
 * and height are at most TK_MAX_IMAGE_DIMENSION: the reference rejects a
 * texture larger than the device's 2D image limit
 * (src/native/runtime/vulkan/limits.rs:111-121), 16384 on its DX12 and
 * Vulkan targets, and the pattern sampler's reflect period (twice the size)
 * must stay inside 32-bit arithmetic. */
#define TK_MAX_IMAGE_DIMENSION 16384u
typedef struct tk_image_desc {
    const uint32_t* premul_rgba8;
    uint32_t width;
    uint32_t height;
} tk_image_desc;

/* Glyph runs drawn from rasterized glyph images (Canvas::push_text_layout,
 * src/canvas/primitives/text.rs:11-100; the text blob records of
 * draw_records.hlsli:19-21). A draw whose glyph_run_id is a run index
 * composites that run's glyphs (coarse/text.hlsli, fine/glyph.hlsli). */
typedef struct tk_glyph_run {  /* TextRun, 8 bytes */
    uint32_t first;            /* first glyph */
    uint32_t count;
} tk_glyph_run;
typedef struct tk_glyph {      /* a positioned glyph, 12 bytes */
    uint32_t image;            /* glyph image, TK_INVALID_INDEX for none */
    int32_t x, y;              /* pen position in device pixels */
} tk_glyph;
typedef struct tk_glyph_image {  /* 24 bytes */
    int32_t left, top;           /* image placement: x + left, y - top */
    uint32_t width, height;
    uint32_t content;            /* TK_GLYPH_* */
    uint32_t data_offset;        /* first texel in the glyph texels, rows of `width` */
} tk_glyph_image;
/* Glyph image contents (fine/constants.hlsli:4-9). Texels are 32-bit words:
 * masks keep the coverage in the low byte, subpixel masks one coverage per
 * byte (red in the low byte), colour glyphs premultiplied RGBA8. */
#define TK_GLYPH_MASK 0u
#define TK_GLYPH_COLOR 1u
#define TK_GLYPH_SUBPIXEL_MASK 2u
#define TK_GLYPH_LINEAR_MASK 3u
#define TK_GLYPH_LINEAR_COLOR 4u
#define TK_GLYPH_LINEAR_SUBPIXEL_MASK 5u

/* ------------------------------------------------------------------------ */
/* Records. Layouts equal the reference's #[repr(C)] Pod types.              */
/* ------------------------------------------------------------------------ */

/* GpuAffine (src/shared/affine.rs:5-18): (x,y) -> (a x + c y + e, b x + d y + f) */
typedef struct tk_affine {
    float a, b, c, d, e, f;
} tk_affine; /* 24 B */

/* Line (src/shared/line.rs:1-9) */
typedef struct tk_line {
    uint32_t path_id;
    float pad;
    float p0[2];
    float p1[2];
} tk_line; /* 24 B */

/* PathRecord (src/shared/path.rs:4-23; offsets scene_records.hlsli:5-19) */
typedef struct tk_path_record {
    uint32_t path_id;
    uint32_t line_count;
    uint32_t line_start;
    uint32_t flags;
    uint32_t data_offset;  /* first word of the path's backdrop slice */
    uint32_t data_len;     /* bbox tile count */
    uint32_t tile_x0, tile_y0, tile_x1, tile_y1;
    uint32_t segment_start;
    uint32_t segment_capacity;
    uint32_t segment_count;
    tk_affine transform;
} tk_path_record; /* 76 B */

/* PixelBounds (src/shared/bounds.rs:76-83) */
typedef struct tk_pixel_bounds {
    int32_t x0, y0, x1, y1;
} tk_pixel_bounds;

/* DrawRecord (src/shared/draw_record.rs:51-81; offsets draw_records.hlsli:5-17) */
typedef struct tk_draw_record {
    uint32_t path_id;
    uint32_t glyph_run_id;
    uint32_t sdf_offset;
    uint32_t sdf_len;
    uint32_t sdf_shadow_offset;
    uint32_t sdf_shadow_len;
    uint32_t brush_offset;
    uint32_t brush_len;
    uint32_t tag;
    uint32_t fill_rule;
    tk_pixel_bounds pixel_bounds;
    tk_pixel_bounds local_pixel_bounds;
    uint32_t solid_rect;
    tk_affine transform;
    tk_affine inverse_transform;
} tk_draw_record; /* 124 B */

/* LayerStackRecord (src/shared/gpu_coarse.rs:47-53) */
typedef struct tk_layer_record {
    uint32_t tag;
    uint32_t draw;
    uint32_t payload;
} tk_layer_record; /* 12 B */

/* PtclRecord (src/shared/gpu_coarse.rs:55-65) */
typedef struct tk_ptcl_record {
    uint32_t tag;
    int32_t backdrop;
    uint32_t fill_rule;
    uint32_t segment_start;
    uint32_t segment_end;
    uint32_t color;
} tk_ptcl_record; /* 24 B */

/* LineSegment (src/shared/line_seg.rs:1-9): tile-local clipped segment */
typedef struct tk_line_segment {
    float p0x, p0y, p1x, p1y, y_edge;
} tk_line_segment; /* 20 B */

/* TileSegmentRange (src/shared/tile_seg_range.rs:1-6) */
typedef struct tk_segment_range {
    uint32_t start, end;
} tk_segment_range; /* 8 B */

/* TileCoarseRecord (src/shared/gpu_coarse.rs:1-10) */
typedef struct tk_tile_record {
    uint32_t ptcl_count, ptcl_start, ptcl_end;
    uint32_t glyph_count, glyph_start, glyph_end;
} tk_tile_record; /* 24 B */

/* Linearised execution plan (the reference's ExecPlan ops,
 * src/shared/execution.rs:98-124). DRAW_BATCH renders one batch into the
 * current target; BLUR_BEGIN opens a transparent offscreen surface for the
 * ops that follow (OffscreenLayer::Filter{Blur}); BLUR_END blurs it
 * horizontally then vertically inside `bounds` and composites it src-over
 * onto the enclosing target (render/filter_program/blur.rs:194-245,
 * shared/composite_stack.hlsli:11-28). */
#define TK_OP_DRAW_BATCH 0u
#define TK_OP_BLUR_BEGIN 1u
#define TK_OP_BLUR_END 2u
/* A progressive blur group: the group's surface blurred with a spatially
 * varying standard deviation (Filter::ProgressiveBlur), closed by
 * TK_OP_BLUR_END. batch_id indexes the scene's progressive blurs. */
#define TK_OP_PROGRESSIVE_BEGIN 3u
/* BLUR_BEGIN's batch_id word is the blur's sampling (Filter::Blur's
 * BlurSampling, src/shared/layer/filter.rs:183-227): factor | downsample
 * filter << 8 | upsample filter << 16. Factor 0 or 1 blurs at full
 * resolution; a factor f > 1 reduces the output bounds by f (nearest or box
 * filter), blurs there at sigma / f and restores them (nearest or bilinear),
 * render/filter_program/blur.rs:24-73, filter/resample.hlsli. */
#define TK_BLUR_SAMPLING(factor, down, up) ((uint32_t)(factor) | ((uint32_t)(down) << 8) | ((uint32_t)(up) << 16))
#define TK_BLUR_DOWNSAMPLE_NEAREST 0u
#define TK_BLUR_DOWNSAMPLE_BOX 1u
#define TK_BLUR_UPSAMPLE_NEAREST 0u
#define TK_BLUR_UPSAMPLE_BILINEAR 1u
#define TK_BLUR_MAX_FACTOR 64u
typedef struct tk_op {
    uint32_t kind;
    uint32_t batch_id;     /* DRAW_BATCH: draw_batch_ids value of its draws;
                              BLUR_BEGIN: TK_BLUR_SAMPLING word (0: full resolution);
                              PROGRESSIVE_BEGIN: index of its tk_progressive_blur */
    uint32_t layer_start;  /* DRAW_BATCH: fused layer stack range */
    uint32_t layer_end;
    float sigma;           /* BLUR_BEGIN: physical standard deviation */
    int32_t bounds[4];     /* BLUR_BEGIN: output bounds x0,y0,x1,y1 (children's
                              paint bounds outset by ceil(3 sigma));
                              PROGRESSIVE_BEGIN: outset by ceil(20 max_std_dev + 8) */
} tk_op; /* 36 B */

/* Filter::ProgressiveBlur (src/shared/layer/filter/progressive.rs:14-103) in
 * device pixels: the blur's projection (projection(): the start point and
 * (end - start) / |end - start|^2, zero for a uniform blur), its maximum
 * standard deviation (0..65536) and its quality. */
typedef struct tk_progressive_blur {
    float start_x, start_y;
    float dir_x, dir_y;
    float max_std_dev;
    uint32_t quality;  /* TK_PROGRESSIVE_BALANCED or TK_PROGRESSIVE_HIGH */
} tk_progressive_blur;
#define TK_PROGRESSIVE_BALANCED 0u
#define TK_PROGRESSIVE_HIGH 1u

/* A filter layer (Canvas::push_filter_layer with Filter::Chain,
 * src/canvas/layers.rs:222-233, src/shared/layer/filter.rs:28-95): the
 * group's surface filtered in place by a chain of filters, each over the
 * layer's processing bounds, then composited src-over onto the enclosing
 * target (render/filters.rs:71-243, render/filter_program/effects.rs:3-268).
 * TK_OP_FILTER_BEGIN opens it (batch_id indexes the scene's filter layers;
 * the output bounds are the layer's surface bounds clipped to the canvas,
 * derived by the library, and the op's own bounds are not read);
 * TK_OP_BLUR_END closes it. */
#define TK_OP_FILTER_BEGIN 4u
/* Filter kinds: the colour filters of filter/constants.hlsli, then the
 * colour matrix and the offset. */
#define TK_FILTER_BRIGHTNESS 1u
#define TK_FILTER_CONTRAST 2u
#define TK_FILTER_GRAYSCALE 3u
#define TK_FILTER_HUE_ROTATE 4u
#define TK_FILTER_INVERT 5u
#define TK_FILTER_OPACITY 6u
#define TK_FILTER_SATURATE 7u
#define TK_FILTER_SEPIA 8u
#define TK_FILTER_COLOR_MATRIX 9u /* Filter::ColorMatrix: 4 rows of 5 (r g b a bias), filter/color.hlsli:47-76 */
#define TK_FILTER_OFFSET 10u      /* Filter::Offset: dx, dy already whole pixels (ceil(d - 0.5)) */
/* Filter::Morphology (filter/morphology.hlsli): dx, dy are the whole-pixel
 * radii ceil(max(radius, 0)) along x and y */
#define TK_FILTER_ERODE 11u
#define TK_FILTER_DILATE 12u
/* Filter::Flood and Filter::DropShadow with a solid brush (filter/brush.hlsl,
 * render/filter_program/shadow.rs): color is the premultiplied RGBA8 colour;
 * a drop shadow's dx, dy are its offset rounded to whole pixels and std_dev
 * its Gaussian standard deviation. */
#define TK_FILTER_FLOOD 13u
#define TK_FILTER_DROP_SHADOW 14u
/* Filter::ComponentTransfer (filter/transfer.hlsli): color is the first word
 * of its table in the scene's filter_words, TK_TRANSFER_TABLE_WORDS words:
 * 256 entries (0..255) for red, green, blue and alpha in that order, indexed
 * by the straight (unpremultiplied) channel byte. */
#define TK_FILTER_COMPONENT_TRANSFER 15u
#define TK_TRANSFER_TABLE_WORDS 1024u
/* Filter::ConvolveMatrix (filter/convolve.hlsli): color is the first word of
 * its columns x rows kernel (f32 bits, row-major) in filter_words; target,
 * divisor, bias, edge mode and preserve_alpha as in the reference. */
#define TK_FILTER_CONVOLVE 16u
#define TK_CONVOLVE_EDGE_NONE 0u
#define TK_CONVOLVE_EDGE_DUPLICATE 1u
#define TK_CONVOLVE_EDGE_WRAP 2u
#define TK_CONVOLVE_MAX_TAPS 4096u
/* Filter::Blur at full resolution inside a chain (render/filter_program/
 * blur.rs:194-244): std_dev along x, amount along y, each through the blur
 * groups' Gaussian over the layer's bounds. */
#define TK_FILTER_BLUR 17u
typedef struct tk_filter {
    uint32_t kind;
    float amount;      /* the colour filters' argument (hue rotation in degrees) */
    int32_t dx, dy;    /* OFFSET, DROP_SHADOW: the offset; ERODE / DILATE: the radii */
    uint32_t color;    /* FLOOD, DROP_SHADOW: the colour; COMPONENT_TRANSFER, CONVOLVE: first filter word */
    float std_dev;     /* DROP_SHADOW */
    float matrix[20];  /* TK_FILTER_COLOR_MATRIX, row-major */
    /* TK_FILTER_CONVOLVE */
    uint32_t columns, rows, target_x, target_y, edge_mode, preserve_alpha;
    float divisor, bias;
} tk_filter; /* 136 B */
/* One filter layer: its chain filters[first, first + count), and the surface
 * bounds the chain reads (the sample region's pixel bounds grown by the
 * chain's reach, filter.rs:510-575; may extend past the canvas). */
typedef struct tk_filter_layer {
    uint32_t first, count;
    int32_t surface[4];  /* x0, y0, x1, y1 */
} tk_filter_layer; /* 24 B */

/* Scene flags */
#define TK_SCENE_SEGMENTS_FROM_DEVICE 1u /* recompute segment_start on device */

typedef struct tk_scene_desc {
    uint32_t width, height;   /* physical canvas size in pixels */
    uint32_t clear_color;     /* premultiplied RGBA8 (set_clear_color) */
    uint32_t flags;
    const tk_line* lines;
    uint64_t line_count;
    const tk_path_record* paths;
    uint32_t path_count;
    uint32_t draw_count;
    const tk_draw_record* draws;
    const uint32_t* brush_blob;
    uint64_t brush_word_count;
    const tk_layer_record* layers;
    uint32_t layer_count;
    uint32_t draw_order_count;
    const uint32_t* draw_order;      /* painter order of drawn draws */
    const uint32_t* draw_batch_ids;  /* per draw; TK_INVALID_INDEX = hidden */
    const tk_op* ops;
    uint32_t op_count;
    uint32_t reserved;
    /* Canvas::sdf_blob / sdf_shadow_blob (src/canvas.rs:92-93) */
    const uint32_t* sdf_blob;
    uint64_t sdf_word_count;
    const uint32_t* sdf_shadow_blob;
    uint64_t sdf_shadow_word_count;
    /* The texture table that image pattern brushes index (the scene's
     * registered images, canvas/primitives/images.rs:42-52). */
    const tk_image_desc* images;
    uint32_t image_count;
    uint32_t image_reserved;
    /* The text blob: glyph runs, their glyphs, the glyph images and their
     * texels (all may be empty). */
    const tk_glyph_run* glyph_runs;
    const tk_glyph* glyphs;
    const tk_glyph_image* glyph_images;
    const uint32_t* glyph_texels;
    uint32_t glyph_run_count;
    uint32_t glyph_count;
    uint32_t glyph_image_count;
    uint32_t glyph_reserved;
    uint64_t glyph_texel_count;
    /* the progressive blurs PROGRESSIVE_BEGIN ops index */
    const tk_progressive_blur* progressive_blurs;
    uint32_t progressive_count;
    uint32_t progressive_reserved;
    /* the filter layers FILTER_BEGIN ops index, and their chains' filters */
    const tk_filter_layer* filter_layers;
    const tk_filter* filters;
    uint32_t filter_layer_count;
    uint32_t filter_count;
    /* words the filters index: component transfer tables, convolution kernels */
    const uint32_t* filter_words;
    uint32_t filter_word_count;
    uint32_t filter_reserved;
} tk_scene_desc;

/* Per-scene counts measured by the device pipeline. */
typedef struct tk_stats {
    uint64_t lines;          /* L */
    uint64_t backdrop_len;   /* B: sum of path bbox tiles */
    uint64_t segments;       /* S: tile segments emitted */
    uint64_t ptcl_records;   /* K: PTCL records over all target passes */
    uint64_t tile_draw_refs; /* sum over draws of bbox tiles */
    uint64_t fill_particles; /* fill-like PTCL records */
    uint64_t segment_visits; /* sum over fill records of segment counts */
    uint32_t passes;         /* coarse+fine passes (target segments) */
    uint32_t tiles;          /* T */
} tk_stats;

/* Status codes */
#define TK_OK 0
#define TK_E_INVALID -1
#define TK_E_CAPACITY -2
#define TK_E_CUDA -3
#define TK_E_TIMEOUT -4
#define TK_E_STATE -5
#define TK_E_ALLOC -6

typedef struct tk_ctx tk_ctx;

/* Library version string. */
const char* tk_version(void);

/* Layout of every struct in tileink.h, tileink_canvas.h and tileink_diff.h as
 * the library was compiled: one entry per struct (field "" with its size)
 * followed by one per field (byte offset and size). A binding (the Rust
 * #[repr(C)] mirrors, ctypes) checks its own declarations against it, as the
 * reference checks its record layouts (src/shared/gpu_coarse.rs:210-286,
 * src/shared/draw_record.rs:165-175). Returns the entry count; the table is
 * static. Needs no device. */
typedef struct tk_abi_field {
    const char* type;
    const char* field;
    uint32_t offset;
    uint32_t size;
} tk_abi_field;
uint32_t tk_abi_layout(const tk_abi_field** table);

/* Context on CUDA device `device` with its own stream. */
int32_t tk_ctx_create(int32_t device, tk_ctx** out);
void tk_ctx_destroy(tk_ctx* ctx);
const char* tk_last_error(const tk_ctx* ctx);
/* The context's cudaStream_t (as void*), for callers that order their work. */
void* tk_ctx_stream(tk_ctx* ctx);
int32_t tk_synchronize(tk_ctx* ctx);

/* Copy a recorded scene to the device and validate it (replaces the
 * reference's per-frame record upload, native/runtime/renderer.rs:91-112).
 * Host records are copied; the caller may free them after the call. */
int32_t tk_scene_upload(tk_ctx* ctx, const tk_scene_desc* scene);

/* Upload a scene that replaces the context's current one path for path,
 * keeping the current scan for every path that did not change (the
 * reference's selective rescan of its scan history,
 * src/native/runtime/program/scene_scan.rs:116-192). `changed` lists the
 * paths whose lines differ from the last upload (the caller's journal; their
 * lines are uploaded, the others' stay on the device); the library adds
 * every path whose record changed. The next render rescans only those paths
 * (their slices cleared, counted, prefixed and emitted), which gives the
 * scan of the whole new scene. It applies when the current scene was
 * scanned, the new one has the same path and line counts, the same kind of
 * segment plan, and keeps the backdrop pool (and, with host plans, the
 * segment layout); otherwise the scene is uploaded whole and scanned in
 * full. With device segment plans (TK_SCENE_SEGMENTS_FROM_DEVICE) every path
 * keeps the segment slice the last scan planned; the next render counts the
 * replaced paths and, if any of their segment totals changed (which moves
 * every later slice), scans the whole scene instead. `*rescan_paths` (may be
 * null) receives the number of paths the next render scans (with device
 * plans: unless that check finds a changed total). */
int32_t tk_scene_upload_delta(tk_ctx* ctx, const tk_scene_desc* scene, const uint32_t* changed,
                              uint32_t changed_count, uint32_t* rescan_paths);

/* Enqueue the whole frame on the context stream: scan (count, prefix,
 * cumsum, emit), tile binning, and per target pass coarse + fine, with blur
 * layers (replaces frame::record, native/runtime/renderer/frame.rs:6-80). */
int32_t tk_render(tk_ctx* ctx);

/* Wait for the frame and copy the premultiplied RGBA8 image
 * (NativeImageSubmission::readback, src/native/submission.rs:120). */
int32_t tk_readback(tk_ctx* ctx, uint32_t* rgba8, size_t pixel_count);

/* upload + render + readback in one call
 * (NativeRenderer::render_to_image, src/native/renderer.rs:177-190). */
int32_t tk_render_to_image(tk_ctx* ctx, const tk_scene_desc* scene,
                           uint32_t* rgba8, size_t pixel_count);

int32_t tk_get_stats(tk_ctx* ctx, tk_stats* out);

/* Debug readback of an intermediate buffer for parity tests. `index`
 * selects the target pass for PTCL/TILES/KINDS. When `dst` is NULL only
 * `*needed` (bytes) is written. */
#define TK_STAGE_COUNTS 0u     /* u32[B] segment tile counts */
#define TK_STAGE_BACKDROPS 1u  /* i32[B] after row cumsum */
#define TK_STAGE_RANGES 2u     /* tk_segment_range[B] */
#define TK_STAGE_SEGMENTS 3u   /* tk_line_segment[segment total] */
#define TK_STAGE_PTCL 4u       /* tk_ptcl_record[] of pass `index` */
#define TK_STAGE_TILES 5u      /* tk_tile_record[T] of pass `index` */
#define TK_STAGE_KINDS 6u      /* u32[T] tile kind words of pass `index` */
#define TK_STAGE_IMAGE 7u      /* u32[W*H] current target image */
#define TK_STAGE_PATHS 8u      /* tk_path_record[P] (segment plan applied) */
#define TK_STAGE_LINES 9u      /* tk_line[L] (device-flattened lines included) */
#define TK_STAGE_GLYPHS 10u    /* u32[] glyph list of pass `index` (the glyph indices PTCL_GLYPH ranges name) */
int32_t tk_debug_readback(tk_ctx* ctx, uint32_t stage, uint32_t index,
                          void* dst, size_t bytes, size_t* needed);
/* Elements [first, first + count) of the same buffers (count clipped to the
 * buffer), for buffers larger than a host copy should hold at once (the
 * 4096^2 / 50,000-path frame has 335 M segments); *total receives the
 * buffer's element count. */
int32_t tk_debug_readback_range(tk_ctx* ctx, uint32_t stage, uint32_t index, uint64_t first,
                                uint64_t count, void* dst, uint64_t* total);

/* Band split (multi-GPU): one rank per GPU renders tile rows
 * [tile_y0, tile_y1) of the frame. The next tk_scene_upload (or
 * tk_scene_upload_flatten) clamps every path's tile bbox to those rows, so
 * the rank scans only the lines that reach its band (tile rows are
 * independent after the scan: a backdrop is the row-wise cumsum of its own
 * row's deltas), repacks the backdrop slices and plans segments on the
 * device; tk_render then runs coarse and fine on the band's tiles only.
 * Rows outside the band are left unwritten. tile_y0 == tile_y1 returns to
 * whole frames. Scenes with blur layers are rejected in band mode (a blur
 * reaches across bands). Band pixels equal the whole frame's. */
int32_t tk_set_band(tk_ctx* ctx, uint32_t tile_y0, uint32_t tile_y1);
/* The path records tk_set_band uploads for a band (host only, no device):
 * each tile bbox clamped to rows [tile_y0, tile_y1) (a path that misses the
 * band gets rows [tile_y0, tile_y0) and data_len 0), backdrop slices repacked
 * contiguously in path order, segment_start and segment_capacity 0 for the
 * device's segment plan (TK_SCENE_SEGMENTS_FROM_DEVICE). */
void tk_band_paths(const tk_path_record* paths, uint32_t path_count, uint32_t tile_y0, uint32_t tile_y1,
                   tk_path_record* out);
/* Pixel rows [row0, row1) of the current image into `rgba8` (host or device
 * memory: cudaMemcpyDefault), width * (row1 - row0) words. */
int32_t tk_readback_rows(tk_ctx* ctx, uint32_t row0, uint32_t row1, uint32_t* rgba8, size_t pixel_count);

/* Stage timing with CUDA events recorded on the context stream around each
 * stage of tk_render (no reference counterpart; measurement support).
 * Stages: 0 pool clear, 1 scan_count, 2 pool prefix + cumsum, 3 scan_emit,
 * 4 tile binning, 5 coarse count + tile prefix, 6 coarse emit, 7 fine,
 * 8 blur + composite. Times are summed over the passes of the last frame. */
#define TK_TIMED_STAGES 9u
int32_t tk_set_timing(tk_ctx* ctx, int32_t enabled);
int32_t tk_get_stage_times(tk_ctx* ctx, float* ms, uint32_t count);

/* ------------------------------------------------------------------------ */
/* Stage harnesses on host buffers (the reference's per-kernel GPU test      */
/* harnesses, src/native/runtime/tests/scan_cases.rs:8-213 and               */
/* tests/shared_blur_gpu.rs:9-155).                                          */
/* ------------------------------------------------------------------------ */

/* Per path p: ranges[t] over [data_offset, data_offset+data_len) is the
 * exclusive/inclusive prefix of counts starting at segment_start (wrapping
 * u32); cursors[t] = ranges[t].start; bumps[p] = path total. Elements outside
 * every path slice are left as given. (scan/prefix_chunks.hlsl:16-38,
 * scan/chunk_offsets.hlsl:14-26, scan/apply_chunk_offsets.hlsl:15-27) */
int32_t tk_stage_scan_prefix(tk_ctx* ctx, const uint32_t* counts, uint64_t pool_len,
                             const tk_path_record* paths, uint32_t path_count,
                             tk_segment_range* ranges, uint32_t* cursors,
                             uint32_t* bumps);

/* Tile prefix (coarse/prefix.hlsl:11-63) on host tile records: the exclusive
 * scan of tiles[i].ptcl_count into ptcl_start / ptcl_end (glyph_start /
 * glyph_end cleared, glyph_count kept: text scenes scan it after) and the
 * total record count. The scan's look-back wait gives up
 * after `poll_limit` polls (0: the renderer's limit, 2^22), and the call then
 * returns TK_E_TIMEOUT with the context still usable; this is the library's
 * bounded-wait failure path (the reference latches a failed submission on
 * its context instead, src/native/runtime/adapter.rs:8-15). withhold_first = 1
 * is the test of that path: the block tickets start at 1, so block 0's
 * descriptor is never published and every look-back reaches a predecessor
 * that never publishes. */
int32_t tk_stage_tile_prefix(tk_ctx* ctx, tk_tile_record* tiles, uint32_t tile_count,
                             uint32_t poll_limit, uint32_t withhold_first, uint32_t* total);

/* scan_count on the given lines/paths (scan/count.hlsl:13-40). `backdrops`
 * and `counts` are read, accumulated into and written back. */
int32_t tk_stage_scan_count(tk_ctx* ctx, const tk_line* lines, uint64_t line_count,
                            const tk_path_record* paths, uint32_t path_count,
                            int32_t* backdrops, uint32_t* counts, uint64_t pool_len);

/* One separable blur pass over an RGBA8 image (filter/blur_shared.hlsl:15-74,
 * filter/blur.hlsl:10-17). Pixels outside `region` keep `dst`'s contents;
 * samples outside `source` (x0,y0,x1,y1; empty = region) are transparent. */
int32_t tk_stage_blur(tk_ctx* ctx, const uint32_t* src, uint32_t* dst,
                      uint32_t width, uint32_t height, const uint32_t region[4],
                      const uint32_t source[4], float sigma, uint32_t axis);

/* ------------------------------------------------------------------------ */
/* Device flattening: fill paths arrive as Bezier elements and are flattened */
/* on the GPU at upload (the flattening step of Canvas::push_path,           */
/* src/shared/path_flatten.rs:20-82). The lines are bit-identical to the     */
/* host Canvas's: both run the same double-precision flattener.              */
/* ------------------------------------------------------------------------ */

#define TK_EL_LINE 1u
#define TK_EL_QUAD 2u
#define TK_EL_CUBIC 3u

/* One element of a fill path with its start point: p[0] = start, then the
 * end point (line), control + end point (quadratic) or two controls + end
 * point (cubic). move_to / close are already resolved into line elements. */
typedef struct tk_flatten_el {
    uint32_t verb;
    uint32_t path;        /* path index: the lines' path_id */
    double tolerance;     /* flattening tolerance in device pixels */
    double p[4][2];
} tk_flatten_el; /* 80 B */

/* Stroke centerlines (the stroking step of Canvas::push_stroke,
 * src/canvas/primitives/paths.rs:24-48, kurbo::stroke with round joins and
 * caps) are elements too, in the path's local units: each polyline is a
 * TK_EL_MOVE element (p[0] = its start) followed by line / quadratic / cubic
 * elements whose p[0] is the current point; `path` holds the polyline index and
 * `tolerance` the stroking tolerance. The device flattens, offsets, joins, caps
 * and transforms them into the stroke's outline lines. */
#define TK_EL_MOVE 4u

typedef struct tk_stroke_polyline {
    uint32_t stroke;        /* index into tk_flatten_desc.strokes */
    uint32_t element0;      /* its TK_EL_MOVE in stroke_elements */
    uint32_t element_count; /* >= 1, the move included */
    uint32_t closed;        /* 1 after a close */
} tk_stroke_polyline; /* 16 B */

typedef struct tk_stroke_desc {
    uint32_t path;           /* the outline's path: its lines' path_id */
    uint32_t polyline0;      /* first polyline */
    uint32_t polyline_count;
    uint32_t reserved;
    double half_width;       /* width / 2 in local units, (0, 1e6] */
    double tolerance;        /* arc tolerance in local units, >= 1e-3 */
    double transform[6];     /* local -> device pixels: x' = t0 x + t2 y + t4, y' = t1 x + t3 y + t5 */
} tk_stroke_desc; /* 80 B */

typedef struct tk_flatten_desc {
    const tk_flatten_el* elements;
    uint64_t element_count;
    const uint32_t* path_elements; /* [path_count][first, count]; count 0: the
                                      path's lines are in tk_scene_desc.lines
                                      or come from a stroke */
    const tk_flatten_el* stroke_elements;
    uint64_t stroke_element_count;
    const tk_stroke_polyline* polylines;
    uint32_t polyline_count;
    uint32_t stroke_count;
    const tk_stroke_desc* strokes;
} tk_flatten_desc;

/* tk_scene_upload for a scene whose paths with elements or strokes are
 * flattened on the device. tk_scene_desc.lines holds the other paths' lines;
 * the fills' device lines follow them, then the strokes' outline lines.
 * Requires TK_SCENE_SEGMENTS_FROM_DEVICE. */
int32_t tk_scene_upload_flatten(tk_ctx* ctx, const tk_scene_desc* scene, const tk_flatten_desc* flatten);

/* ------------------------------------------------------------------------ */
/* Incremental rendering: the damage-driven redraw of the retained path      */
/* (NativeRenderer::render_retained, src/native/renderer/retained.rs:17-218; */
/* damage planning, src/render/incremental.rs:1-297). The uploaded scene is  */
/* scanned in full, then coarse and fine run only on the tiles under the     */
/* damage; every other pixel keeps the context's previous frame. The result  */
/* equals a full tk_render of the scene whenever the damage covers every     */
/* pixel whose value changed since that frame (tk_retained_materialize       */
/* reports such damage).                                                     */
/* ------------------------------------------------------------------------ */

typedef struct tk_damage {
    uint32_t full;          /* 1: redraw everything */
    uint32_t rect_count;
    const int32_t* rects;   /* rect_count x {x0, y0, x1, y1}, physical pixels, half-open */
} tk_damage;

/* Why a frame was drawn in full (FullRedrawReason,
 * src/render/incremental/config.rs:52-63). */
#define TK_FULL_NONE 0u         /* incremental */
#define TK_FULL_REQUESTED 1u    /* damage.full (ExplicitInvalidation) */
#define TK_FULL_NO_HISTORY 2u   /* no previous frame of this size and clear colour in the context (FirstFrame) */
#define TK_FULL_THRESHOLD 3u    /* dirty tiles >= full_redraw_ratio of all (DirtyTileThreshold) */
#define TK_FULL_FILTERS 4u      /* the scene has blur layers, whose reach crosses tiles */

typedef struct tk_incremental_stats {
    uint32_t total_tiles;
    uint32_t dirty_tiles;   /* tiles redrawn */
    uint32_t full_redraw;   /* 1 when every tile was redrawn */
    uint32_t reason;        /* TK_FULL_* */
    uint32_t scan_reused;   /* 1 when the uploaded scene's last scan served the frame */
    uint32_t scanned_paths; /* paths scanned for the frame (all, those a delta upload replaced, or 0) */
} tk_incremental_stats;

/* Renders the uploaded scene, redrawing only the tiles that meet `damage`
 * unless a full redraw is needed (see TK_FULL_*; full_redraw_ratio in (0, 1],
 * the reference's default is 0.7). A partial redraw of a scene that has not
 * been re-uploaded since its last scan reuses that scan (counts, backdrops,
 * ranges, segments) and runs only coarse and fine of the damaged tiles.
 * `stats` may be null. */
int32_t tk_render_incremental(tk_ctx* ctx, const tk_damage* damage, float full_redraw_ratio,
                              tk_incremental_stats* stats);

/* ------------------------------------------------------------------------ */
/* Batched mode: many independent scenes of uneven size rendered together.   */
/* Every stage runs once for the whole batch (the scenes' paths, tiles, bins */
/* and images are concatenated) and the stage sequence is one CUDA graph,    */
/* instantiated on the first tk_batch_render and replayed after that.        */
/* Each scene's PTCL equals its serial tk_render PTCL with the offsets of    */
/* tk_batch_info added to segment, draw and batch indices.                   */
/* ------------------------------------------------------------------------ */

typedef struct tk_batch_info {
    uint32_t width, height;
    uint32_t tile_base, tile_count;   /* the scene's tile records in the batch pass */
    uint32_t path_base, draw_base, batch_base, line_base;
    uint32_t layer_base, reserved;
    uint64_t segment_base, pool_base; /* added to its segment / backdrop indices */
    uint64_t image_offset;            /* its first pixel in the batch image */
} tk_batch_info;

/* Scenes with one target pass (draw batches and clip layers; no blur
 * groups) and host segment planning. Replaces any uploaded scene. */
int32_t tk_batch_upload(tk_ctx* ctx, const tk_scene_desc* scenes, uint32_t scene_count);
/* Renders the whole batch on the context stream; asynchronous. */
int32_t tk_batch_render(tk_ctx* ctx);
int32_t tk_batch_info_get(tk_ctx* ctx, uint32_t scene, tk_batch_info* out);
/* All images, scene after scene (tk_batch_info.image_offset). */
int32_t tk_batch_readback(tk_ctx* ctx, uint32_t* rgba8, size_t pixel_count);

/* Autotuner: renders the uploaded scene or batch with each pool-scan work
 * item size (512, 1024, 2048, 4096 tiles; bbox rows are never split), keeps
 * the fastest for later renders and reports the timings. Tiles are 16x16. */
typedef struct tk_tune_result {
    uint32_t scan_item_elems;     /* chosen */
    uint32_t tile_width, tile_height;
    uint32_t candidates;
    uint32_t candidate_elems[8];
    float candidate_ms[8];        /* median frame time of each candidate */
} tk_tune_result;
int32_t tk_autotune(tk_ctx* ctx, uint32_t iterations, tk_tune_result* out);

/* ------------------------------------------------------------------------ */
/* Allocation-free pool scan. No reference counterpart: the reference's      */
/* scan runs on buffers its runtime allocated up front, and this entry point */
/* gives C callers the same property.                                        */
/* ------------------------------------------------------------------------ */

#define TK_NOALLOC_MAX_PATHS 16384u
#define TK_NOALLOC_MAX_SCAN_ITEMS 65536u   /* work items: whole bbox rows, <= 4096 tiles each */
#define TK_NOALLOC_SCRATCH_BYTES 2818304u  /* per device, inside the library's module */

/* The pool scan of tk_stage_scan_prefix (segment ranges, cursors, per-path
 * totals) plus the row-wise backdrop cumsum, on DEVICE buffers the caller
 * owns (`d_*`, pool_len elements each; d_bumps path_count elements) and
 * `paths` on the host. It makes no device allocation and frees nothing: its
 * per-item sums and prefixes, work items, copy of `paths` and counter words live
 * in one fixed array of TK_NOALLOC_SCRATCH_BYTES in device memory, one per
 * device. For callers that cannot allocate: an application whose own
 * allocator has reserved the device's memory, where cudaMalloc fails at an
 * arbitrary point, or one that must not stall other streams, which
 * cudaMalloc/cudaFree can do by synchronizing the whole device. The call
 * orders its work on tk_ctx_stream(ctx) and waits for that stream only.
 *
 * Limits: path_count <= TK_NOALLOC_MAX_PATHS and at most
 * TK_NOALLOC_MAX_SCAN_ITEMS work items; larger inputs return TK_E_CAPACITY
 * with a message and launch nothing.
 * State between calls: the per-item sums and prefixes, the work items and
 * the copy of `paths` are rewritten by every call before it reads them, so
 * nothing a previous call left there is used; the call clears its counter
 * words on the stream before it launches. d_backdrops holds the per-tile
 * backdrop deltas (0 where none) and is replaced by its row-wise inclusive
 * cumsum; d_counts is read only; d_ranges, d_cursors, d_bumps are written
 * (elements outside every path slice are left as they are).
 * First call per device: it looks up the scratch address
 * (cudaGetSymbolAddress with the context's device current), which may load
 * the library's module; make that first call before any stream capture.
 * Concurrency: the scratch is shared by every call on one device, so two
 * calls in flight at the same time on one device race; serialize them. */
int32_t tk_pool_scan_noalloc(tk_ctx* ctx, const tk_path_record* paths, uint32_t path_count,
                             const uint32_t* d_counts, int32_t* d_backdrops,
                             tk_segment_range* d_ranges, uint32_t* d_cursors,
                             uint64_t pool_len, uint32_t* d_bumps);

#ifdef __cplusplus
}
#endif

#endif /* TILEINK_B200_H */
