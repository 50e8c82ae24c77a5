"""ctypes binding of libtileink_b200.so (include/tileink.h, include/tileink_canvas.h).

The record types below are byte-identical to the reference's #[repr(C)] Pod
records (src/shared/{line,path,draw_record,gpu_coarse,line_seg,tile_seg_range}.rs)
and are exposed both as ctypes structures and as numpy structured dtypes.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libtileink_b200.so"

TILE_SIZE = 16
INVALID = 0xFFFFFFFF

# Status codes
TK_OK, TK_E_INVALID, TK_E_CAPACITY, TK_E_CUDA, TK_E_TIMEOUT, TK_E_STATE, TK_E_ALLOC = 0, -1, -2, -3, -4, -5, -6

# Debug stages
STAGE_COUNTS, STAGE_BACKDROPS, STAGE_RANGES, STAGE_SEGMENTS = 0, 1, 2, 3
STAGE_PTCL, STAGE_TILES, STAGE_KINDS, STAGE_IMAGE, STAGE_PATHS, STAGE_LINES = 4, 5, 6, 7, 8, 9

# PTCL tags (shaders/hlsl/shared/particle_tags.hlsli) + merged-stream marker
PTCL_END, PTCL_FILL, PTCL_COLOR, PTCL_BEGIN_CLIP, PTCL_END_CLIP = 0, 1, 2, 3, 4
PTCL_BEGIN_OPACITY, PTCL_END_OPACITY = 5, 6
PTCL_PATH_GLYPH = 11
# Draw tags (src/shared/draw_record.rs:7-13)
DRAW_BRUSH, DRAW_CLIP, DRAW_OPACITY, DRAW_PATH_GLYPH = 0, 1, 2, 5
FILL_NONZERO, FILL_EVEN_ODD = 0, 1
# Layer stack tags (shaders/hlsl/shared/draw_tags.hlsli:7-9)
LAYER_CLIP, LAYER_OPACITY, LAYER_BLEND = 0, 1, 2
PTCL_BATCH_BEGIN = 14
PTCL_SDF = 9
PTCL_IMAGE = 13
PATTERN_NEAREST, PATTERN_BILINEAR = 0, 1
MAX_IMAGE_DIMENSION = 16384  # TK_MAX_IMAGE_DIMENSION
BLUR_DOWNSAMPLE_NEAREST, BLUR_DOWNSAMPLE_BOX = 0, 1
BLUR_UPSAMPLE_NEAREST, BLUR_UPSAMPLE_BILINEAR = 0, 1


def blur_sampling(factor: int, down: int = BLUR_DOWNSAMPLE_BOX, up: int = BLUR_UPSAMPLE_BILINEAR) -> int:
    """TK_BLUR_SAMPLING(factor, downsample filter, upsample filter)."""
    return int(factor) | (int(down) << 8) | (int(up) << 16)
PTCL_BEGIN_SDF_CLIP = 12
TILE_KIND_INTERPRETER, TILE_KIND_EMPTY, TILE_KIND_COLOR, TILE_KIND_SDF, TILE_KIND_MIXED = 0, 1, 2, 3, 4
# SDF kinds (src/shared/gpu_types.rs) and line caps
SDF_RECT, SDF_CIRCLE, SDF_RECT_STROKE, SDF_CIRCLE_STROKE, SDF_LINE = 1, 2, 3, 4, 6
SDF_RECT_SHADOW, SDF_CIRCLE_SHADOW, SDF_LINE_SHADOW = 7, 10, 11
SDF_CANDLESTICK, SDF_DASH_LINE, SDF_TRIANGLE, SDF_CHECKERBOARD = 5, 12, 13, 14
SDF_CALLOUT, SDF_CALLOUT_STROKE, SDF_CALLOUT_SHADOW = 17, 18, 19
SDF_ARC, SDF_ARC_SHADOW, SDF_STAR, SDF_STAR_STROKE = 8, 9, 15, 16
SIDE_TOP, SIDE_RIGHT, SIDE_BOTTOM, SIDE_LEFT = 0, 1, 2, 3
SDF_RECORD_WORDS = 17
CAP_BUTT, CAP_SQUARE, CAP_ROUND = 0, 1, 2

OP_DRAW_BATCH, OP_BLUR_BEGIN, OP_BLUR_END = 0, 1, 2
SCENE_SEGMENTS_FROM_DEVICE = 1

LINE_DTYPE = np.dtype([("path_id", "<u4"), ("pad", "<f4"), ("p0", "<f4", 2), ("p1", "<f4", 2)])
AFFINE_DTYPE = np.dtype([(k, "<f4") for k in "abcdef"])
PATH_DTYPE = np.dtype(
    [(k, "<u4") for k in ("path_id", "line_count", "line_start", "flags", "data_offset", "data_len",
                          "tile_x0", "tile_y0", "tile_x1", "tile_y1", "segment_start",
                          "segment_capacity", "segment_count")]
    + [("transform", AFFINE_DTYPE)]
)
BOUNDS_DTYPE = np.dtype([(k, "<i4") for k in ("x0", "y0", "x1", "y1")])
DRAW_DTYPE = np.dtype(
    [(k, "<u4") for k in ("path_id", "glyph_run_id", "sdf_offset", "sdf_len", "sdf_shadow_offset",
                          "sdf_shadow_len", "brush_offset", "brush_len", "tag", "fill_rule")]
    + [("pixel_bounds", BOUNDS_DTYPE), ("local_pixel_bounds", BOUNDS_DTYPE), ("solid_rect", "<u4"),
       ("transform", AFFINE_DTYPE), ("inverse_transform", AFFINE_DTYPE)]
)
LAYER_DTYPE = np.dtype([("tag", "<u4"), ("draw", "<u4"), ("payload", "<u4")])
PTCL_DTYPE = np.dtype([("tag", "<u4"), ("backdrop", "<i4"), ("fill_rule", "<u4"), ("segment_start", "<u4"),
                       ("segment_end", "<u4"), ("color", "<u4")])
SEGMENT_DTYPE = np.dtype([(k, "<f4") for k in ("p0x", "p0y", "p1x", "p1y", "y_edge")])
RANGE_DTYPE = np.dtype([("start", "<u4"), ("end", "<u4")])
TILE_DTYPE = np.dtype([(k, "<u4") for k in ("ptcl_count", "ptcl_start", "ptcl_end", "glyph_count",
                                            "glyph_start", "glyph_end")])
OP_DTYPE = np.dtype([("kind", "<u4"), ("batch_id", "<u4"), ("layer_start", "<u4"), ("layer_end", "<u4"),
                     ("sigma", "<f4"), ("bounds", "<i4", 4)])
# the text blob (tk_glyph_run, tk_glyph, tk_glyph_image; draw_records.hlsli:19-21)
GLYPH_RUN_DTYPE = np.dtype([("first", "<u4"), ("count", "<u4")])
GLYPH_DTYPE = np.dtype([("image", "<u4"), ("x", "<i4"), ("y", "<i4")])
GLYPH_IMAGE_DTYPE = np.dtype([("left", "<i4"), ("top", "<i4"), ("width", "<u4"), ("height", "<u4"),
                              ("content", "<u4"), ("data_offset", "<u4")])
PROGRESSIVE_DTYPE = np.dtype([("start_x", "<f4"), ("start_y", "<f4"), ("dir_x", "<f4"), ("dir_y", "<f4"),
                              ("max_std_dev", "<f4"), ("quality", "<u4")])
PROGRESSIVE_BALANCED, PROGRESSIVE_HIGH = 0, 1
OP_PROGRESSIVE_BEGIN = 3
OP_FILTER_BEGIN = 4
FILTER_DTYPE = np.dtype([("kind", "<u4"), ("amount", "<f4"), ("dx", "<i4"), ("dy", "<i4"), ("color", "<u4"),
                         ("std_dev", "<f4"), ("matrix", "<f4", (20,)), ("columns", "<u4"), ("rows", "<u4"),
                         ("target_x", "<u4"), ("target_y", "<u4"), ("edge_mode", "<u4"), ("preserve_alpha", "<u4"),
                         ("divisor", "<f4"), ("bias", "<f4")])
CANVAS_FILTER_DTYPE = np.dtype([("kind", "<u4"), ("amount", "<f4"), ("dx", "<f4"), ("dy", "<f4"),
                                ("rgba", "<f4", (4,)), ("std_dev", "<f4"), ("matrix", "<f4", (20,)),
                                ("table", "<u8"), ("kernel", "<u8"), ("columns", "<u4"), ("rows", "<u4"),
                                ("target_x", "<u4"), ("target_y", "<u4"), ("edge_mode", "<u4"),
                                ("preserve_alpha", "<u4"), ("divisor", "<f4"), ("bias", "<f4")], align=True)
FILTER_LAYER_DTYPE = np.dtype([("first", "<u4"), ("count", "<u4"), ("surface", "<i4", (4,))])
(FILTER_BRIGHTNESS, FILTER_CONTRAST, FILTER_GRAYSCALE, FILTER_HUE_ROTATE, FILTER_INVERT, FILTER_OPACITY,
 FILTER_SATURATE, FILTER_SEPIA, FILTER_COLOR_MATRIX, FILTER_OFFSET, FILTER_ERODE, FILTER_DILATE, FILTER_FLOOD,
 FILTER_DROP_SHADOW, FILTER_COMPONENT_TRANSFER, FILTER_CONVOLVE, FILTER_BLUR) = range(1, 18)
CONVOLVE_EDGE_NONE, CONVOLVE_EDGE_DUPLICATE, CONVOLVE_EDGE_WRAP = 0, 1, 2
TRANSFER_TABLE_WORDS = 1024
GLYPH_MASK, GLYPH_COLOR, GLYPH_SUBPIXEL_MASK = 0, 1, 2
GLYPH_LINEAR_MASK, GLYPH_LINEAR_COLOR, GLYPH_LINEAR_SUBPIXEL_MASK = 3, 4, 5
PTCL_GLYPH = 10
STAGE_GLYPHS = 10
EL_LINE, EL_QUAD, EL_CUBIC, EL_MOVE = 1, 2, 3, 4
FLATTEN_EL_DTYPE = np.dtype([("verb", "<u4"), ("path", "<u4"), ("tolerance", "<f8"), ("p", "<f8", (4, 2))])
POLYLINE_DTYPE = np.dtype([("stroke", "<u4"), ("element0", "<u4"), ("element_count", "<u4"), ("closed", "<u4")])
STROKE_DTYPE = np.dtype([("path", "<u4"), ("polyline0", "<u4"), ("polyline_count", "<u4"), ("reserved", "<u4"),
                         ("half_width", "<f8"), ("tolerance", "<f8"), ("transform", "<f8", (6,))])
assert FLATTEN_EL_DTYPE.itemsize == 80 and POLYLINE_DTYPE.itemsize == 16 and STROKE_DTYPE.itemsize == 80
assert LINE_DTYPE.itemsize == 24 and PATH_DTYPE.itemsize == 76 and DRAW_DTYPE.itemsize == 124
assert LAYER_DTYPE.itemsize == 12 and PTCL_DTYPE.itemsize == 24 and SEGMENT_DTYPE.itemsize == 20
assert TILE_DTYPE.itemsize == 24 and OP_DTYPE.itemsize == 36
assert GLYPH_RUN_DTYPE.itemsize == 8 and GLYPH_DTYPE.itemsize == 12 and GLYPH_IMAGE_DTYPE.itemsize == 24


class SceneDesc(C.Structure):
    _fields_ = [
        ("width", C.c_uint32), ("height", C.c_uint32), ("clear_color", C.c_uint32), ("flags", C.c_uint32),
        ("lines", C.c_void_p), ("line_count", C.c_uint64),
        ("paths", C.c_void_p), ("path_count", C.c_uint32),
        ("draw_count", C.c_uint32), ("draws", C.c_void_p),
        ("brush_blob", C.c_void_p), ("brush_word_count", C.c_uint64),
        ("layers", C.c_void_p), ("layer_count", C.c_uint32),
        ("draw_order_count", C.c_uint32), ("draw_order", C.c_void_p),
        ("draw_batch_ids", C.c_void_p),
        ("ops", C.c_void_p), ("op_count", C.c_uint32), ("reserved", C.c_uint32),
        ("sdf_blob", C.c_void_p), ("sdf_word_count", C.c_uint64),
        ("sdf_shadow_blob", C.c_void_p), ("sdf_shadow_word_count", C.c_uint64),
        ("images", C.c_void_p), ("image_count", C.c_uint32), ("image_reserved", C.c_uint32),
        ("glyph_runs", C.c_void_p), ("glyphs", C.c_void_p), ("glyph_images", C.c_void_p),
        ("glyph_texels", C.c_void_p), ("glyph_run_count", C.c_uint32), ("glyph_count", C.c_uint32),
        ("glyph_image_count", C.c_uint32), ("glyph_reserved", C.c_uint32), ("glyph_texel_count", C.c_uint64),
        ("progressive_blurs", C.c_void_p), ("progressive_count", C.c_uint32), ("progressive_reserved", C.c_uint32),
        ("filter_layers", C.c_void_p), ("filters", C.c_void_p), ("filter_layer_count", C.c_uint32),
        ("filter_count", C.c_uint32), ("filter_words", C.c_void_p), ("filter_word_count", C.c_uint32),
        ("filter_reserved", C.c_uint32),
    ]


class ImageDesc(C.Structure):
    """tk_image_desc: premultiplied RGBA8 texels (red in the low byte), row-major."""
    _fields_ = [("premul_rgba8", C.c_void_p), ("width", C.c_uint32), ("height", C.c_uint32)]


class Stats(C.Structure):
    _fields_ = [("lines", C.c_uint64), ("backdrop_len", C.c_uint64), ("segments", C.c_uint64),
                ("ptcl_records", C.c_uint64), ("tile_draw_refs", C.c_uint64), ("fill_particles", C.c_uint64),
                ("segment_visits", C.c_uint64), ("passes", C.c_uint32), ("tiles", C.c_uint32)]


class GradientStop(C.Structure):
    _fields_ = [("offset", C.c_float), ("rgba", C.c_float * 4)]


class BrushDesc(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("extend", C.c_uint32), ("rgba", C.c_float * 4), ("p0", C.c_float * 2),
                ("p1", C.c_float * 2), ("r0", C.c_float), ("r1", C.c_float), ("stop_count", C.c_uint32),
                ("stops", C.POINTER(GradientStop))]


class SdfShape(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("cap", C.c_uint32), ("p0", C.c_double * 2), ("p1", C.c_double * 2),
                ("p2", C.c_double * 2), ("radius", C.c_double), ("width", C.c_double), ("radii", C.c_float * 4),
                ("widths", C.c_float * 4), ("shadow", C.c_float * 4), ("dash", C.c_float * 3),
                ("flags", C.c_uint32), ("angle", C.c_float * 2)]


class FlattenDesc(C.Structure):
    """tk_flatten_desc (include/tileink.h)."""
    _fields_ = [("elements", C.c_void_p), ("element_count", C.c_uint64), ("path_elements", C.c_void_p),
                ("stroke_elements", C.c_void_p), ("stroke_element_count", C.c_uint64), ("polylines", C.c_void_p),
                ("polyline_count", C.c_uint32), ("stroke_count", C.c_uint32), ("strokes", C.c_void_p)]


class DiffScene(C.Structure):
    """tk_diff_scene (include/tileink_diff.h)."""
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("path_count", C.c_uint32),
                ("cubics_per_path", C.c_uint32), ("points", C.c_void_p), ("colors", C.c_void_p),
                ("sigma", C.c_float), ("tolerance", C.c_float), ("background", C.c_float * 4),
                ("loss_row0", C.c_uint32), ("loss_row1", C.c_uint32)]


class BatchInfo(C.Structure):
    """tk_batch_info (include/tileink.h)."""
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("tile_base", C.c_uint32), ("tile_count", C.c_uint32),
                ("path_base", C.c_uint32), ("draw_base", C.c_uint32), ("batch_base", C.c_uint32),
                ("line_base", C.c_uint32), ("layer_base", C.c_uint32), ("reserved", C.c_uint32),
                ("segment_base", C.c_uint64), ("pool_base", C.c_uint64), ("image_offset", C.c_uint64)]


class TuneResult(C.Structure):
    """tk_tune_result (include/tileink.h)."""
    _fields_ = [("scan_item_elems", C.c_uint32), ("tile_width", C.c_uint32), ("tile_height", C.c_uint32),
                ("candidates", C.c_uint32), ("candidate_elems", C.c_uint32 * 8), ("candidate_ms", C.c_float * 8)]


class GenParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("paths", C.c_uint32), ("variant", C.c_uint32),
                ("sigma", C.c_float), ("jitter", C.c_float), ("flags", C.c_uint32), ("reserved", C.c_uint32)]


class Damage(C.Structure):
    """tk_damage (include/tileink.h)."""
    _fields_ = [("full", C.c_uint32), ("rect_count", C.c_uint32), ("rects", C.c_void_p)]


class IncrementalStats(C.Structure):
    """tk_incremental_stats (include/tileink.h)."""
    _fields_ = [("total_tiles", C.c_uint32), ("dirty_tiles", C.c_uint32), ("full_redraw", C.c_uint32),
                ("reason", C.c_uint32), ("scan_reused", C.c_uint32), ("scanned_paths", C.c_uint32)]


class AbiField(C.Structure):
    """tk_abi_field (include/tileink.h)."""
    _fields_ = [("type", C.c_char_p), ("field", C.c_char_p), ("offset", C.c_uint32), ("size", C.c_uint32)]


def abi_layout() -> dict:
    """{struct: {"": size, field: (offset, size), ...}} as the library was
    compiled (tk_abi_layout)."""
    t = C.POINTER(AbiField)()
    n = library().tk_abi_layout(C.byref(t))
    out: dict = {}
    for k in range(n):
        e = t[k]
        d = out.setdefault(e.type.decode(), {})
        if e.field:
            d[e.field.decode()] = (e.offset, e.size)
        else:
            d[""] = e.size
    return out


FULL_NONE, FULL_REQUESTED, FULL_NO_HISTORY, FULL_THRESHOLD, FULL_FILTERS = 0, 1, 2, 3, 4

_LIB = None


def library() -> C.CDLL:
    """Load the in-tree native library; raise if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m tileink_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(str(LIB_PATH))
    P, U32, U64, I32, I64, F32, F64 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_int64, C.c_float, C.c_double
    sig = {
        "tk_version": (C.c_char_p, []),
        "tk_abi_layout": (U32, [C.POINTER(C.POINTER(AbiField))]),
        "tk_ctx_create": (I32, [I32, C.POINTER(P)]),
        "tk_ctx_destroy": (None, [P]),
        "tk_last_error": (C.c_char_p, [P]),
        "tk_ctx_stream": (P, [P]),
        "tk_synchronize": (I32, [P]),
        "tk_scene_upload": (I32, [P, C.POINTER(SceneDesc)]),
        "tk_scene_upload_flatten": (I32, [P, C.POINTER(SceneDesc), C.POINTER(FlattenDesc)]),
        "tk_canvas_set_device_flatten": (None, [P, I32]),
        "tk_canvas_flatten_desc": (I32, [P, C.POINTER(FlattenDesc)]),
        "tk_render": (I32, [P]),
        "tk_render_incremental": (I32, [P, C.POINTER(Damage), F32, C.POINTER(IncrementalStats)]),
        "tk_readback": (I32, [P, P, C.c_size_t]),
        "tk_render_to_image": (I32, [P, C.POINTER(SceneDesc), P, C.c_size_t]),
        "tk_get_stats": (I32, [P, C.POINTER(Stats)]),
        "tk_debug_readback": (I32, [P, U32, U32, P, C.c_size_t, C.POINTER(C.c_size_t)]),
        "tk_stage_scan_prefix": (I32, [P, P, U64, P, U32, P, P, P]),
        "tk_stage_tile_prefix": (I32, [P, P, U32, U32, U32, C.POINTER(U32)]),
        "tk_debug_readback_range": (I32, [P, U32, U32, U64, U64, P, C.POINTER(U64)]),
        "tk_set_band": (I32, [P, U32, U32]),
        "tk_scene_upload_delta": (I32, [P, C.POINTER(SceneDesc), P, U32, C.POINTER(U32)]),
        "tk_band_paths": (None, [P, U32, U32, U32, P]),
        "tk_readback_rows": (I32, [P, U32, U32, P, C.c_size_t]),
        "tk_stage_scan_count": (I32, [P, P, U64, P, U32, P, P, U64]),
        "tk_stage_blur": (I32, [P, P, P, U32, U32, P, P, F32, U32]),
        "tk_pool_scan_noalloc": (I32, [P, P, U32, P, P, P, P, U64, P]),
        "tk_batch_upload": (I32, [P, P, U32]),
        "tk_batch_render": (I32, [P]),
        "tk_batch_info_get": (I32, [P, U32, C.POINTER(BatchInfo)]),
        "tk_batch_readback": (I32, [P, P, C.c_size_t]),
        "tk_autotune": (I32, [P, U32, C.POINTER(TuneResult)]),
        "tk_diff_forward": (I32, [P, C.POINTER(DiffScene), P, C.POINTER(C.c_double), P]),
        "tk_diff_backward": (I32, [P, P, P, P]),
        "tk_diff_flatten": (U64, [C.POINTER(DiffScene), P, P, P, U64]),
        "tk_set_timing": (I32, [P, I32]),
        "tk_get_stage_times": (I32, [P, P, U32]),
        "tk_path_new": (P, []),
        "tk_path_free": (None, [P]),
        "tk_path_move_to": (None, [P, F64, F64]),
        "tk_path_line_to": (None, [P, F64, F64]),
        "tk_path_quad_to": (None, [P, F64, F64, F64, F64]),
        "tk_path_cubic_to": (None, [P, F64, F64, F64, F64, F64, F64]),
        "tk_path_close": (None, [P]),
        "tk_path_flatten": (U64, [P, F32, U32, P, U64]),
        "tk_canvas_new": (P, [U32, U32, F32]),
        "tk_canvas_free": (None, [P]),
        "tk_canvas_set_host_segment_plan": (None, [P, I32]),
        "tk_canvas_set_clear_color": (None, [P, U32]),
        "tk_canvas_push_path": (I64, [P, P, C.POINTER(BrushDesc), P, U32, F64]),
        "tk_canvas_push_stroke": (I64, [P, P, C.POINTER(BrushDesc), F64, P, F64]),
        "tk_canvas_push_glyph_outlines": (I64, [P, P, C.POINTER(BrushDesc), P, F64]),
        "tk_canvas_push_progressive_blur_group": (I32, [P, F64, F64, F64, F64, C.c_float, U32]),
        "tk_canvas_push_filter_layer": (I32, [P, P, U32, P, C.c_int32]),
        "tk_canvas_push_filter_layer_path": (I32, [P, P, U32, P, P, C.c_int32]),
        "tk_canvas_push_sdf": (I64, [P, C.POINTER(SdfShape), C.POINTER(BrushDesc)]),
        "tk_canvas_push_clip_sdf_layer": (I32, [P, C.POINTER(SdfShape)]),
        "tk_canvas_add_image": (I32, [P, P, U32, U32]),
        "tk_canvas_add_glyph_image": (I32, [P, C.c_int32, C.c_int32, U32, U32, U32, P]),
        "tk_canvas_push_glyph_run": (I64, [P, P, U32, C.POINTER(BrushDesc), P]),
        "tk_canvas_push_image": (C.c_int64, [P, C.POINTER(C.c_double), U32, U32, U32, U32]),
        "tk_canvas_push_clip_layer": (I32, [P, P, P, U32, F64]),
        "tk_canvas_push_opacity_layer": (I32, [P, P, P, F64, F32]),
        "tk_canvas_push_blur_group_sampled": (I32, [P, F32, U32]),
        "tk_canvas_last_error": (C.c_char_p, [P]),
        "tk_canvas_push_blur_group": (I32, [P, F32]),
        "tk_canvas_pop_layer": (I32, [P]),
        "tk_canvas_scene": (I32, [P, C.POINTER(SceneDesc)]),
        "tk_canvas_set_keep_commands": (None, [P, I32]),
        "tk_canvas_replay": (I32, [P, P, P]),
        "tk_retained_new": (P, [U32, U32, F32]),
        "tk_retained_free": (None, [P]),
        "tk_retained_set_clear_color": (None, [P, U32]),
        "tk_retained_set_device_flatten": (None, [P, I32]),
        "tk_retained_version": (U64, [P]),
        "tk_retained_insert": (I32, [P, U64, P, P, U64]),
        "tk_retained_replace": (I32, [P, U64, P]),
        "tk_retained_set_transform": (I32, [P, U64, P]),
        "tk_retained_move_before": (I32, [P, U64, U64]),
        "tk_retained_remove": (I32, [P, U64]),
        "tk_retained_invalidate_rect": (I32, [P, P]),
        "tk_retained_invalidate_all": (I32, [P]),
        "tk_retained_materialize": (P, [P, C.POINTER(Damage)]),
        "tk_generate": (P, [U32, U64, C.POINTER(GenParams)]),
        "tk_canvas_param_points": (U64, [P, P]),
        "tk_canvas_param_colors": (U64, [P, P]),
        "tk_plan_line_tile_count": (U32, [P, U32, U32, U32, U32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def ptr(a: np.ndarray | None) -> int | None:
    return None if a is None or a.size == 0 else a.ctypes.data


def desc_to_arrays(d: SceneDesc) -> dict:
    """Copy a scene description into numpy arrays."""
    def arr(p, n, dt):
        if n == 0 or not p:
            return np.zeros(0, dtype=dt)
        buf = (C.c_uint8 * (n * np.dtype(dt).itemsize)).from_address(p)
        return np.frombuffer(buf, dtype=dt).copy()
    return {
        "width": d.width, "height": d.height, "clear_color": d.clear_color, "flags": d.flags,
        "lines": arr(d.lines, d.line_count, LINE_DTYPE),
        "paths": arr(d.paths, d.path_count, PATH_DTYPE),
        "draws": arr(d.draws, d.draw_count, DRAW_DTYPE),
        "brush": arr(d.brush_blob, d.brush_word_count, np.uint32),
        "layers": arr(d.layers, d.layer_count, LAYER_DTYPE),
        "draw_order": arr(d.draw_order, d.draw_order_count, np.uint32),
        "draw_batch_ids": arr(d.draw_batch_ids, d.draw_count, np.uint32),
        "ops": arr(d.ops, d.op_count, OP_DTYPE),
        "sdf": arr(d.sdf_blob, d.sdf_word_count, np.uint32),
        "sdf_shadow": arr(d.sdf_shadow_blob, d.sdf_shadow_word_count, np.uint32),
        "images": [arr(im.premul_rgba8, im.width * im.height, np.uint32).reshape(im.height, im.width)
                   for im in (C.cast(d.images, C.POINTER(ImageDesc))[k] for k in range(d.image_count))],
        "glyph_runs": arr(d.glyph_runs, d.glyph_run_count, GLYPH_RUN_DTYPE),
        "glyphs": arr(d.glyphs, d.glyph_count, GLYPH_DTYPE),
        "glyph_images": arr(d.glyph_images, d.glyph_image_count, GLYPH_IMAGE_DTYPE),
        "glyph_texels": arr(d.glyph_texels, d.glyph_texel_count, np.uint32),
        "progressive": arr(d.progressive_blurs, d.progressive_count, PROGRESSIVE_DTYPE),
        "filter_layers": arr(d.filter_layers, d.filter_layer_count, FILTER_LAYER_DTYPE),
        "filters": arr(d.filters, d.filter_count, FILTER_DTYPE),
        "filter_words": arr(d.filter_words, d.filter_word_count, np.uint32),
    }


class ArrayScene:
    """A scene held in numpy arrays with a SceneDesc pointing into them."""

    def __init__(self, arrays: dict):
        self.a = {k: (np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v) for k, v in arrays.items()}
        a = self.a
        d = SceneDesc()
        d.width, d.height, d.clear_color, d.flags = a["width"], a["height"], a["clear_color"], a.get("flags", 0)
        d.lines, d.line_count = ptr(a["lines"]), len(a["lines"])
        d.paths, d.path_count = ptr(a["paths"]), len(a["paths"])
        d.draws, d.draw_count = ptr(a["draws"]), len(a["draws"])
        d.brush_blob, d.brush_word_count = ptr(a["brush"]), len(a["brush"])
        d.layers, d.layer_count = ptr(a["layers"]), len(a["layers"])
        d.draw_order, d.draw_order_count = ptr(a["draw_order"]), len(a["draw_order"])
        d.draw_batch_ids = ptr(a["draw_batch_ids"])
        d.ops, d.op_count = ptr(a["ops"]), len(a["ops"])
        sdf, shadow = a.get("sdf"), a.get("sdf_shadow")
        if sdf is not None and len(sdf):
            d.sdf_blob, d.sdf_word_count = ptr(sdf), len(sdf)
        if shadow is not None and len(shadow):
            d.sdf_shadow_blob, d.sdf_shadow_word_count = ptr(shadow), len(shadow)
        for key, cnt in (("glyph_runs", "glyph_run_count"), ("glyphs", "glyph_count"),
                         ("glyph_images", "glyph_image_count"), ("glyph_texels", "glyph_texel_count"),
                         ("progressive", "progressive_count"), ("filter_layers", "filter_layer_count"),
                         ("filters", "filter_count")):
            v = a.get(key)
            if v is not None and len(v):
                setattr(d, "progressive_blurs" if key == "progressive" else key, ptr(v))
                setattr(d, cnt, len(v))
        words = a.get("filter_words")
        if words is not None and len(words):
            d.filter_words, d.filter_word_count = ptr(words), len(words)
        images = [np.ascontiguousarray(im, dtype=np.uint32) for im in a.get("images", [])]
        if images:
            self._images = images
            self._image_table = (ImageDesc * len(images))(*[ImageDesc(ptr(im), im.shape[1], im.shape[0])
                                                            for im in images])
            d.images, d.image_count = C.addressof(self._image_table), len(images)
        self.desc = d
        self.flatten = None
        els, strokes = a.get("elements"), a.get("strokes")
        if (els is not None and len(els)) or (strokes is not None and len(strokes)):
            f = FlattenDesc()
            f.elements, f.element_count, f.path_elements = ptr(els), len(els), ptr(a["path_elements"])
            if strokes is not None and len(strokes):
                f.stroke_elements, f.stroke_element_count = ptr(a["stroke_elements"]), len(a["stroke_elements"])
                f.polylines, f.polyline_count = ptr(a["polylines"]), len(a["polylines"])
                f.strokes, f.stroke_count = ptr(strokes), len(strokes)
            self.flatten = f
