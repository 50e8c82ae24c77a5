"""Scene recording: the reference's `Canvas` recording API for the vector path.

    Canvas.push_path        src/canvas/primitives/paths.rs:50-60
    Canvas.push_stroke      src/canvas/primitives/paths.rs:24-48
    Canvas.push_rect / push_rect_stroke / push_circle / push_circle_stroke /
    push_line / push_dash_line / push_triangle / push_checkerboard /
    push_candlestick and push_{rect,circle,line}_shadow
                            src/canvas/primitives/{rectangles,shapes,shadows}.rs
    Canvas.push_clip_layer  src/canvas/layers.rs:7-28
    Canvas.push_blur_group  src/canvas/layers.rs:205-212
    Canvas.pop_layer        src/canvas/layers.rs

Recording, flattening, stroking, brush encoding and batch compilation run in
the native library (tileink_b200/csrc/canvas.cpp).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import _native as N

FILL_NONZERO, FILL_EVEN_ODD = 0, 1
EXTEND_PAD, EXTEND_REPEAT, EXTEND_REFLECT = 0, 1, 2


class BezPath:
    """Path builder (kurbo::BezPath): f64 move/line/quad/cubic/close."""

    def __init__(self):
        self._lib = N.library()
        self._h = self._lib.tk_path_new()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.tk_path_free(h)
            self._h = None

    def move_to(self, x, y):
        self._lib.tk_path_move_to(self._h, float(x), float(y))
        return self

    def line_to(self, x, y):
        self._lib.tk_path_line_to(self._h, float(x), float(y))
        return self

    def quad_to(self, x1, y1, x2, y2):
        self._lib.tk_path_quad_to(self._h, float(x1), float(y1), float(x2), float(y2))
        return self

    def cubic_to(self, x1, y1, x2, y2, x3, y3):
        self._lib.tk_path_cubic_to(self._h, *(float(v) for v in (x1, y1, x2, y2, x3, y3)))
        return self

    def close(self):
        self._lib.tk_path_close(self._h)
        return self

    def flatten(self, tolerance: float, path_id: int = 0) -> np.ndarray:
        """PathFlatten::flatten (src/shared/path_flatten.rs:20-82) -> Line records."""
        n = self._lib.tk_path_flatten(self._h, float(tolerance), int(path_id), None, 0)
        out = np.zeros(n, dtype=N.LINE_DTYPE)
        self._lib.tk_path_flatten(self._h, float(tolerance), int(path_id), N.ptr(out), n)
        return out


@dataclass
class Brush:
    """Solid color or linear/radial gradient with straight RGBA colors in [0, 1]."""
    kind: int = 0
    rgba: Sequence[float] = (0.0, 0.0, 0.0, 1.0)
    p0: Sequence[float] = (0.0, 0.0)
    p1: Sequence[float] = (0.0, 0.0)
    r0: float = 0.0
    r1: float = 0.0
    stops: Sequence[tuple] = field(default_factory=list)  # (offset, (r, g, b, a))
    extend: int = EXTEND_PAD

    @staticmethod
    def solid(r, g, b, a=1.0) -> "Brush":
        return Brush(kind=0, rgba=(r, g, b, a))

    @staticmethod
    def linear(p0, p1, stops, extend=EXTEND_PAD) -> "Brush":
        return Brush(kind=1, p0=p0, p1=p1, stops=list(stops), extend=extend)

    @staticmethod
    def radial(c0, r0, c1, r1, stops, extend=EXTEND_PAD) -> "Brush":
        return Brush(kind=2, p0=c0, p1=c1, r0=r0, r1=r1, stops=list(stops), extend=extend)

    def _desc(self):
        d = N.BrushDesc()
        d.kind, d.extend = self.kind, self.extend
        d.rgba[:] = [float(v) for v in self.rgba]
        d.p0[:] = [float(v) for v in self.p0]
        d.p1[:] = [float(v) for v in self.p1]
        d.r0, d.r1 = float(self.r0), float(self.r1)
        stops = (N.GradientStop * max(1, len(self.stops)))()
        for i, (off, rgba) in enumerate(self.stops):
            stops[i].offset = float(off)
            stops[i].rgba[:] = [float(v) for v in rgba]
        d.stop_count = len(self.stops)
        d.stops = C.cast(stops, C.POINTER(N.GradientStop))
        return d, stops


def _four(v):
    """One value for all four corners / sides, or four values."""
    if np.ndim(v) == 0:
        return [float(v)] * 4
    v = [float(x) for x in v]
    if len(v) != 4:
        raise ValueError("expected one value or four")
    return v


def _affine(transform):
    if transform is None:
        return None, None
    arr = (C.c_double * 6)(*[float(v) for v in transform])
    return C.cast(arr, C.c_void_p), arr


class Canvas:
    """Immediate-mode recording canvas (src/canvas.rs:86-126)."""

    def __init__(self, width: int, height: int, scale: float = 1.0, *, _handle=None, _owner=None):
        self._lib = N.library()
        self._h = _handle if _handle is not None else self._lib.tk_canvas_new(int(width), int(height), float(scale))
        self._owner = _owner  # a canvas owned by another object (a retained scene's materialization)
        if not self._h:
            raise ValueError("invalid canvas surface")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and getattr(self, "_owner", None) is None:
            self._lib.tk_canvas_free(h)
        self._h = None

    def keep_commands(self, enabled: bool = True):
        """Keep every later push / pop call with its original geometry, so
        the canvas can be replayed or become a RetainedScene node."""
        self._lib.tk_canvas_set_keep_commands(self._h, 1 if enabled else 0)

    def replay(self, src: "Canvas", transform=None):
        """Replays `src`'s kept calls into this canvas under `transform`."""
        t, keep = _affine(transform)
        if self._lib.tk_canvas_replay(self._h, src._h, t) != 0:
            raise ValueError("replay needs a command-keeping source with its layers closed")

    def set_clear_color(self, premul_rgba8: int):
        self._lib.tk_canvas_set_clear_color(self._h, int(premul_rgba8) & 0xFFFFFFFF)

    def set_host_segment_plan(self, enabled: bool):
        self._lib.tk_canvas_set_host_segment_plan(self._h, 1 if enabled else 0)

    def set_device_flatten(self, enabled: bool):
        """Fills and strokes recorded from now on are flattened (and stroked)
        on the GPU at upload."""
        self._lib.tk_canvas_set_device_flatten(self._h, 1 if enabled else 0)

    def flatten_desc(self) -> N.FlattenDesc | None:
        """The elements and strokes to flatten on the device, or None when
        there are none."""
        f = N.FlattenDesc()
        self._lib.tk_canvas_flatten_desc(self._h, C.byref(f))
        return f if (f.element_count or f.stroke_count) else None

    def flatten_arrays(self) -> dict:
        """Copies of the device-flattening elements, per-path element ranges
        and strokes (empty when the canvas flattens on the host)."""
        f = self.flatten_desc()
        n_paths = self.scene_desc().path_count

        def arr(addr, n, dtype):
            if not n:
                return np.zeros(0, dtype)
            raw = np.ctypeslib.as_array((C.c_uint8 * (n * dtype.itemsize)).from_address(addr))
            return raw.view(dtype).copy()

        if f is None:
            f = N.FlattenDesc()
            n_paths = 0
        return {"elements": arr(f.elements, f.element_count, N.FLATTEN_EL_DTYPE),
                "path_elements": arr(f.path_elements, 2 * n_paths, np.dtype(np.uint32)),
                "stroke_elements": arr(f.stroke_elements, f.stroke_element_count, N.FLATTEN_EL_DTYPE),
                "polylines": arr(f.polylines, f.polyline_count, N.POLYLINE_DTYPE),
                "strokes": arr(f.strokes, f.stroke_count, N.STROKE_DTYPE)}

    def push_path(self, path: BezPath, brush: Brush, transform=None, fill_rule=FILL_NONZERO,
                  tolerance: float = 0.1) -> int:
        d, keep = brush._desc()
        t, tk = _affine(transform)
        r = self._lib.tk_canvas_push_path(self._h, path._h, C.byref(d), t, int(fill_rule), float(tolerance))
        if r < 0:
            raise ValueError("push_path rejected its arguments")
        return r

    def push_stroke(self, path: BezPath, brush: Brush, width: float, transform=None, tolerance: float = 0.1) -> int:
        d, keep = brush._desc()
        t, tk = _affine(transform)
        r = self._lib.tk_canvas_push_stroke(self._h, path._h, C.byref(d), float(width), t, float(tolerance))
        if r < 0:
            raise ValueError("push_stroke rejected its arguments")
        return r

    def push_glyph_outlines(self, path: BezPath, brush: Brush, transform=None, tolerance: float = 0.1) -> int:
        """Canvas::push_text_layout_as_path (src/canvas/primitives/text.rs:107-147)
        after shaping: the glyph outlines of a laid-out run as one nonzero
        DrawTag::PathGlyph fill, composited with the text coverage
        correction (fine/text/auto.hlsli)."""
        d, keep = brush._desc()
        t, tk = _affine(transform)
        r = self._lib.tk_canvas_push_glyph_outlines(self._h, path._h, C.byref(d), t, float(tolerance))
        if r < 0:
            raise ValueError("push_glyph_outlines rejected its arguments")
        return r

    # -- analytic SDF shapes (src/canvas/primitives/{rectangles,shapes,shadows}.rs) --
    @staticmethod
    def _shape(kind: int, p0=(0.0, 0.0), p1=(0.0, 0.0), radius=0.0, width=0.0, radii=0.0, widths=0.0, shadow=None,
               cap=N.CAP_BUTT, p2=(0.0, 0.0), dash=(0.0, 0.0, 0.0), flags=0, angle=(0.0, 0.0)) -> N.SdfShape:
        s = N.SdfShape()
        s.kind, s.cap = kind, int(cap)
        s.p0[:] = [float(v) for v in p0]
        s.p1[:] = [float(v) for v in p1]
        s.p2[:] = [float(v) for v in p2]
        s.dash[:] = [float(v) for v in dash]
        s.flags = int(flags)
        s.angle[:] = [float(v) for v in angle]
        s.radius, s.width = float(radius), float(width)
        s.radii[:] = _four(radii)
        s.widths[:] = _four(widths)
        if shadow is not None:
            s.shadow[:] = [float(v) for v in shadow]
        return s

    def _push_sdf(self, brush: Brush, kind: int, *args, **fields):
        s = self._shape(kind, *args, **fields)
        d, keep = brush._desc()
        r = self._lib.tk_canvas_push_sdf(self._h, C.byref(s), C.byref(d))
        if r == -2:
            return None  # the shape draws nothing
        if r < 0:
            raise ValueError("SDF shape rejected its arguments")
        return r

    def add_image(self, premul_rgba8) -> int:
        """Registers an image (H, W) uint32 array of premultiplied RGBA8
        texels, red in the low byte (Canvas::register_scene_image); returns
        its index for push_image."""
        im = np.ascontiguousarray(premul_rgba8, dtype=np.uint32)
        if im.ndim != 2:
            raise ValueError("image must be a (height, width) uint32 array")
        r = self._lib.tk_canvas_add_image(self._h, im.ctypes.data, im.shape[1], im.shape[0])
        if r < 0:
            raise ValueError(f"empty image, or a side above {N.MAX_IMAGE_DIMENSION} texels")
        return r

    def add_glyph_image(self, left: int, top: int, texels, content=N.GLYPH_MASK) -> int:
        """Registers a rasterized glyph image: (H, W) uint32 texels (masks:
        coverage in the low byte; subpixel masks: r, g, b coverages; colour
        glyphs: premultiplied RGBA8), placed at pen + (left, -top)."""
        im = np.ascontiguousarray(texels, dtype=np.uint32)
        if im.ndim != 2:
            raise ValueError("glyph texels must be a (height, width) uint32 array")
        r = self._lib.tk_canvas_add_glyph_image(self._h, int(left), int(top), im.shape[1], im.shape[0], int(content),
                                                im.ctypes.data)
        if r < 0:
            raise ValueError("bad glyph image")
        return r

    def push_glyph_run(self, glyphs, brush: Brush, clip=None) -> int:
        """Canvas::push_text_layout(_clipped) after layout: glyphs as (image,
        x, y) rows (pen positions in device pixels), one glyph run draw."""
        g = np.zeros(len(glyphs), dtype=N.GLYPH_DTYPE)
        for k, (image, x, y) in enumerate(glyphs):
            g[k] = (N.INVALID if image is None else int(image), int(x), int(y))
        d, keep = brush._desc()
        cl = None if clip is None else (C.c_int32 * 4)(*[int(v) for v in clip])
        r = self._lib.tk_canvas_push_glyph_run(self._h, g.ctypes.data, len(g), C.byref(d), cl)
        if r < 0:
            raise ValueError("push_glyph_run rejected the run")
        return r

    def push_image(self, x0, y0, x1, y1, image: int, extend=EXTEND_PAD, sampling=N.PATTERN_NEAREST, opacity=255):
        """Canvas::push_image: registered image `image` scaled into the rect
        (x0, y0)-(x1, y1) with extend EXTEND_* and sampling PATTERN_*."""
        rect = (C.c_double * 4)(x0, y0, x1, y1)
        r = self._lib.tk_canvas_push_image(self._h, rect, int(image), int(extend), int(sampling), int(opacity))
        if r == -2:
            return None  # the rect draws nothing
        if r < 0:
            raise ValueError("image rect or options rejected")
        return r

    def _push_clip_sdf(self, kind: int, **fields):
        if self._lib.tk_canvas_push_clip_sdf_layer(self._h, C.byref(self._shape(kind, **fields))) != 0:
            raise ValueError("SDF clip layer rejected its arguments")

    def push_clip_sdf_rect_layer(self, x0, y0, x1, y1, radius=0.0):
        """Canvas::push_clip_sdf_rect_layer: later draws until pop_layer are
        masked by the (rounded) rectangle's analytic coverage."""
        self._push_clip_sdf(N.SDF_RECT, p0=(x0, y0), p1=(x1, y1), radii=radius)

    def push_clip_sdf_circle_layer(self, cx, cy, r):
        self._push_clip_sdf(N.SDF_CIRCLE, p0=(cx, cy), radius=r)

    def push_clip_sdf_line_layer(self, x0, y0, x1, y1, width, cap=N.CAP_BUTT):
        self._push_clip_sdf(N.SDF_LINE, p0=(x0, y0), p1=(x1, y1), width=width, cap=cap)

    def push_clip_sdf_arc_layer(self, cx, cy, radius, start_angle, sweep_angle, width, cap=N.CAP_BUTT):
        self._push_clip_sdf(N.SDF_ARC, p0=(cx, cy), radius=radius, width=width, cap=cap,
                            angle=(start_angle, sweep_angle))

    def push_rect(self, x0, y0, x1, y1, brush: Brush, radius=0.0):
        """Canvas::push_rect: a filled rectangle, corner radii one value or
        (top-left, top-right, bottom-left, bottom-right)."""
        return self._push_sdf(brush, N.SDF_RECT, (x0, y0), (x1, y1), radii=radius)

    def push_rect_stroke(self, x0, y0, x1, y1, widths, brush: Brush, radius=0.0):
        """Canvas::push_rect_stroke(_widths): a centred stroke, full widths one
        value or (top, right, bottom, left). None when every width is <= 0."""
        return self._push_sdf(brush, N.SDF_RECT_STROKE, (x0, y0), (x1, y1), radii=radius, widths=widths)

    def push_circle(self, cx, cy, r, brush: Brush):
        return self._push_sdf(brush, N.SDF_CIRCLE, (cx, cy), radius=r)

    def push_circle_stroke(self, cx, cy, r, width, brush: Brush):
        """None when width <= 0."""
        return self._push_sdf(brush, N.SDF_CIRCLE_STROKE, (cx, cy), radius=r, width=width)

    def push_line(self, x0, y0, x1, y1, width, brush: Brush, cap=N.CAP_BUTT):
        """Canvas::push_line (SdfLine): None for an empty line (width <= 0, or a
        butt-capped point)."""
        return self._push_sdf(brush, N.SDF_LINE, (x0, y0), (x1, y1), width=width, cap=cap)

    def push_dash_line(self, x0, y0, x1, y1, width, dash_length, gap_length, brush: Brush, cap=N.CAP_BUTT,
                       dash_offset=0.0):
        """Canvas::push_dash_line (SdfDashLine::with_offset): None when no dash
        is visible."""
        return self._push_sdf(brush, N.SDF_DASH_LINE, (x0, y0), (x1, y1), width=width, cap=cap,
                              dash=(dash_length, gap_length, dash_offset))

    def push_triangle(self, a, b, c, brush: Brush, corner_radius=0.0):
        """Canvas::push_triangle: None for collinear or non-finite vertices."""
        return self._push_sdf(brush, N.SDF_TRIANGLE, a, b, p2=c, radius=corner_radius)

    def push_checkerboard(self, x0, y0, x1, y1, cell_size, first: Brush, second: Brush):
        """Canvas::push_checkerboard (src/canvas/primitives/rectangles.rs:9-26):
        the rectangle in `second`, then the even cells in `first`; returns the
        two draw ids, or None (and no draw) for an invalid rectangle or cell."""
        import math
        ok = all(math.isfinite(v) for v in (x0, y0, x1, y1)) and x1 - x0 > 0 and y1 - y0 > 0
        if not ok or not (math.isfinite(cell_size) and cell_size > 0):
            return None
        base = self.push_rect(x0, y0, x1, y1, second)
        return base, self._push_sdf(first, N.SDF_CHECKERBOARD, (x0, y0), (x1, y1), radius=cell_size)

    def push_candlestick(self, center_x, high_y, low_y, body_top_y, body_bottom_y, body_width: int,
                         wick_width: int, brush: Brush):
        """Canvas::push_candlestick (SdfCandleStick): a wick from high to low and
        a body between its top and bottom; widths whole pixels > 0."""
        return self._push_sdf(brush, N.SDF_CANDLESTICK, (center_x, high_y), (body_top_y, body_bottom_y),
                              p2=(low_y, 0.0), widths=(float(body_width), float(wick_width), 0.0, 0.0))

    def push_sdf_arc(self, cx, cy, radius, start_angle, sweep_angle, width, brush: Brush, cap=N.CAP_BUTT):
        """Canvas::push_sdf_arc (SdfArc): a circular stroke from start_angle
        over sweep_angle (radians); None when radius, width or sweep is 0."""
        return self._push_sdf(brush, N.SDF_ARC, (cx, cy), radius=radius, width=width, cap=cap,
                              angle=(start_angle, sweep_angle))

    def push_arc_shadow(self, cx, cy, radius, start_angle, sweep_angle, width, brush: Brush, offset=(0.0, 0.0),
                        expand=0.0, intensity=1.0, cap=N.CAP_BUTT):
        return self._push_sdf(brush, N.SDF_ARC_SHADOW, (cx, cy), radius=radius, width=width, cap=cap,
                              angle=(start_angle, sweep_angle), shadow=(offset[0], offset[1], expand, intensity))

    def push_star(self, cx, cy, outer_radius, inner_radius, brush: Brush, corner_radius=0.0, rotation=0.0):
        """Canvas::push_star (SdfStar): a five-point star; None for invalid radii."""
        return self._push_sdf(brush, N.SDF_STAR, (cx, cy), radius=outer_radius,
                              widths=(inner_radius, corner_radius, 0.0, 0.0), angle=(rotation, 0.0))

    def push_star_stroke(self, cx, cy, outer_radius, inner_radius, width, brush: Brush, corner_radius=0.0,
                         rotation=0.0):
        return self._push_sdf(brush, N.SDF_STAR_STROKE, (cx, cy), radius=outer_radius, width=width,
                              widths=(inner_radius, corner_radius, 0.0, 0.0), angle=(rotation, 0.0))

    def _callout(self, brush, kind, rect, body_radius, tail, width=0.0, shadow=None):
        if tail is None:  # CalloutTail::hidden()
            return self._push_sdf(brush, kind, rect[:2], rect[2:], radius=body_radius, width=width, shadow=shadow,
                                  cap=N.SIDE_BOTTOM, flags=1)
        side, offset, tail_width, length, radius = tail
        return self._push_sdf(brush, kind, rect[:2], rect[2:], radius=body_radius, width=width, shadow=shadow,
                              cap=side, widths=(offset, tail_width, length, radius))

    def push_callout(self, rect, body_radius, tail, brush: Brush):
        """Canvas::push_callout: a rounded body (x0, y0, x1, y1) and a tail
        (side, offset, width, length, corner radius), or tail None for none."""
        return self._callout(brush, N.SDF_CALLOUT, rect, body_radius, tail)

    def push_callout_stroke(self, rect, body_radius, tail, width, brush: Brush):
        return self._callout(brush, N.SDF_CALLOUT_STROKE, rect, body_radius, tail, width=width)

    def push_callout_shadow(self, rect, body_radius, tail, brush: Brush, offset=(0.0, 0.0), expand=0.0,
                            intensity=1.0):
        return self._callout(brush, N.SDF_CALLOUT_SHADOW, rect, body_radius, tail,
                             shadow=(offset[0], offset[1], expand, intensity))

    def push_rect_shadow(self, x0, y0, x1, y1, brush: Brush, offset=(0.0, 0.0), expand=0.0, intensity=1.0,
                         radius=0.0):
        """Canvas::push_rect_shadow: exponential falloff over `expand` pixels
        (a plain antialiased edge when 0). None when intensity <= 0."""
        return self._push_sdf(brush, N.SDF_RECT_SHADOW, (x0, y0), (x1, y1), radii=radius,
                              shadow=(offset[0], offset[1], expand, intensity))

    def push_circle_shadow(self, cx, cy, r, brush: Brush, offset=(0.0, 0.0), expand=0.0, intensity=1.0):
        return self._push_sdf(brush, N.SDF_CIRCLE_SHADOW, (cx, cy), radius=r,
                              shadow=(offset[0], offset[1], expand, intensity))

    def push_line_shadow(self, x0, y0, x1, y1, width, brush: Brush, offset=(0.0, 0.0), expand=0.0,
                         intensity=1.0, cap=N.CAP_BUTT):
        return self._push_sdf(brush, N.SDF_LINE_SHADOW, (x0, y0), (x1, y1), width=width, cap=cap,
                              shadow=(offset[0], offset[1], expand, intensity))

    def push_clip_layer(self, path: BezPath, transform=None, fill_rule=FILL_NONZERO, tolerance: float = 0.1):
        t, tk = _affine(transform)
        if self._lib.tk_canvas_push_clip_layer(self._h, path._h, t, int(fill_rule), float(tolerance)) != 0:
            raise ValueError("push_clip_layer rejected its arguments")

    def push_opacity_layer(self, path: BezPath, opacity: float, transform=None, tolerance: float = 0.1):
        """Canvas::push_opacity_layer: the children until pop_layer are
        composited at `opacity` through the nonzero coverage of `path`."""
        t, tk = _affine(transform)
        if self._lib.tk_canvas_push_opacity_layer(self._h, path._h, t, float(tolerance), float(opacity)) != 0:
            raise ValueError("push_opacity_layer rejected its arguments")

    def push_progressive_blur_group(self, start, end, max_std_dev: float, quality=N.PROGRESSIVE_BALANCED) -> None:
        """Children until pop_layer() are blurred by Filter::ProgressiveBlur
        (src/shared/layer/filter/progressive.rs:14-103): unchanged before
        `start`, max_std_dev after `end`, smoothstep between (start == end: a
        uniform blur)."""
        r = self._lib.tk_canvas_push_progressive_blur_group(self._h, float(start[0]), float(start[1]), float(end[0]),
                                                            float(end[1]), float(max_std_dev), int(quality))
        if r != 0:
            raise ValueError("bad progressive blur")

    def push_filter_layer(self, filters, rect, fixed_region: bool = False, transform=None) -> None:
        """Canvas::push_filter_layer with a chain of filters over a Region::Rect
        sample region (src/canvas/layers.rs:222-233): children until
        pop_layer() are rendered into a surface, filtered in place by each
        filter in turn and composited over the region's pixel bounds grown by
        the chain's reach. `filters`: (kind, value) pairs, kind one of
        N.FILTER_* — a colour filter's amount (hue rotation in degrees), a
        20-float matrix for FILTER_COLOR_MATRIX, (dx, dy) for FILTER_OFFSET,
        (radius_x, radius_y) for FILTER_ERODE / FILTER_DILATE, a straight
        (r, g, b, a) for FILTER_FLOOD, (dx, dy, std_dev, (r, g, b, a)) for
        FILTER_DROP_SHADOW, 1024 bytes (R, G, B, A tables of 256) for
        FILTER_COMPONENT_TRANSFER, {"kernel": rows x columns floats, "target",
        "divisor", "bias", "edge_mode", "preserve_alpha"} for FILTER_CONVOLVE
        (defaults: the centre, the kernel's sum or 1, 0, duplicate, False),
        (std_dev_x, std_dev_y) for FILTER_BLUR.
        `rect` = (x0, y0, x1, y1) in logical units, or a BezPath (a
        Region::Path, under the optional `transform`)."""
        chain = np.zeros(len(filters), dtype=N.CANVAS_FILTER_DTYPE)
        keep = []  # the transfer tables, alive for the call (the canvas copies them)
        for k, (kind, value) in enumerate(filters):
            chain[k]["kind"] = kind
            if kind == N.FILTER_COLOR_MATRIX:
                chain[k]["matrix"] = np.asarray(value, dtype=np.float32).reshape(20)
            elif kind in (N.FILTER_OFFSET, N.FILTER_ERODE, N.FILTER_DILATE, N.FILTER_BLUR):
                chain[k]["dx"], chain[k]["dy"] = value
            elif kind == N.FILTER_FLOOD:
                chain[k]["rgba"] = value
            elif kind == N.FILTER_DROP_SHADOW:
                dx, dy, std_dev, rgba = value
                chain[k]["dx"], chain[k]["dy"], chain[k]["std_dev"], chain[k]["rgba"] = dx, dy, std_dev, rgba
            elif kind == N.FILTER_COMPONENT_TRANSFER:
                table = np.ascontiguousarray(np.asarray(value, dtype=np.uint32).reshape(N.TRANSFER_TABLE_WORDS))
                keep.append(table)
                chain[k]["table"] = table.ctypes.data
            elif kind == N.FILTER_CONVOLVE:
                kern = np.ascontiguousarray(np.asarray(value["kernel"], dtype=np.float32))
                keep.append(kern)
                rows, cols = kern.shape
                chain[k]["kernel"] = kern.ctypes.data
                chain[k]["columns"], chain[k]["rows"] = cols, rows
                chain[k]["target_x"] = value.get("target", (cols // 2, rows // 2))[0]
                chain[k]["target_y"] = value.get("target", (cols // 2, rows // 2))[1]
                chain[k]["edge_mode"] = value.get("edge_mode", N.CONVOLVE_EDGE_DUPLICATE)
                chain[k]["preserve_alpha"] = 1 if value.get("preserve_alpha", False) else 0
                chain[k]["divisor"] = value.get("divisor", float(kern.sum()) or 1.0)
                chain[k]["bias"] = value.get("bias", 0.0)
            else:
                chain[k]["amount"] = value
        if isinstance(rect, BezPath):  # Region::Path (the path's bounds under `transform`)
            t = None if transform is None else np.asarray(transform, dtype=np.float64).reshape(6)
            rc = self._lib.tk_canvas_push_filter_layer_path(self._h, N.ptr(chain) if len(chain) else None, len(chain),
                                                            rect._h, None if t is None else N.ptr(t),
                                                            1 if fixed_region else 0)
        else:
            r = np.asarray(rect, dtype=np.float64).reshape(4)
            rc = self._lib.tk_canvas_push_filter_layer(self._h, N.ptr(chain) if len(chain) else None, len(chain),
                                                       N.ptr(r), 1 if fixed_region else 0)
        if rc != 0:
            raise ValueError("bad filter layer")

    def push_blur_group(self, sigma: float, factor: int = 1, downsample: int = N.BLUR_DOWNSAMPLE_BOX,
                        upsample: int = N.BLUR_UPSAMPLE_BILINEAR):
        """Canvas::push_blur_group; factor > 1 blurs through a copy reduced
        by `factor` (the BlurSampling of Filter::Blur)."""
        word = N.blur_sampling(factor, downsample, upsample) if factor > 1 else 0
        if self._lib.tk_canvas_push_blur_group_sampled(self._h, float(sigma), word) != 0:
            raise ValueError("blur sigma must be finite and nonnegative, and the sampling valid")

    def pop_layer(self):
        if self._lib.tk_canvas_pop_layer(self._h) != 0:
            raise ValueError("no layer to pop")

    def scene_desc(self) -> N.SceneDesc:
        d = N.SceneDesc()
        if self._lib.tk_canvas_scene(self._h, C.byref(d)) != 0:
            raise RuntimeError("canvas compile failed: " + (self._lib.tk_canvas_last_error(self._h) or b"").decode())
        return d

    def scene_arrays(self) -> dict:
        return N.desc_to_arrays(self.scene_desc())

    def param_points(self) -> np.ndarray:
        n = self._lib.tk_canvas_param_points(self._h, None)
        out = np.zeros(n, dtype=np.float64)
        self._lib.tk_canvas_param_points(self._h, N.ptr(out))
        return out.reshape(-1, 2)

    def param_colors(self) -> np.ndarray:
        n = self._lib.tk_canvas_param_colors(self._h, None)
        out = np.zeros(n, dtype=np.float32)
        self._lib.tk_canvas_param_colors(self._h, N.ptr(out))
        return out.reshape(-1, 4)


def generate(config: int, seed: int, *, width=0, height=0, paths=0, variant=0, sigma=0.0, jitter=0.0,
             device_segment_plan=False, device_flatten=False) -> Canvas:
    """Seeded synthetic workload (1: 640x360 cubic fills, 2: 4096^2 50k mixed,
    3: 1920x1080 glyphs, 4: one uneven batch scene, 5: 1024^2 blur group).
    device_flatten keeps the fills as Bezier elements for GPU flattening
    (and implies device segment planning)."""
    lib = N.library()
    flags = (1 if device_segment_plan else 0) | (2 if device_flatten else 0)
    p = N.GenParams(width, height, paths, variant, sigma, jitter, flags, 0)
    h = lib.tk_generate(int(config), int(seed), C.byref(p))
    if not h:
        raise ValueError(f"unknown workload {config}")
    return Canvas(0, 0, _handle=h)


def plan_line_tile_count(line: np.ndarray, bbox) -> int:
    """Host scan-line planner (src/shared/scan_line.rs:17-31)."""
    l = np.ascontiguousarray(np.asarray(line, dtype=N.LINE_DTYPE).reshape(1))
    return N.library().tk_plan_line_tile_count(N.ptr(l), *[int(v) for v in bbox])


class RetainedScene:
    """Retained scene (RetainedScene, src/retained_scene/scene.rs:14-140;
    transaction.rs:74-255): nodes in painter order, each a command-keeping
    Canvas under a node transform. `materialize()` gives the scene as one
    Canvas and the damage since the previous call, which
    NativeRenderer.render_incremental turns into a redraw of those tiles."""

    def __init__(self, width: int, height: int, scale: float = 1.0, device_flatten: bool = False):
        self._lib = N.library()
        self._h = self._lib.tk_retained_new(int(width), int(height), float(scale))
        if not self._h:
            raise ValueError("invalid retained scene surface")
        self._lib.tk_retained_set_device_flatten(self._h, 1 if device_flatten else 0)
        self._canvas = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._canvas = None
            self._lib.tk_retained_free(h)
            self._h = None

    def _check(self, rc: int, what: str):
        if rc != 0:
            raise ValueError(f"retained scene: {what} rejected its arguments")

    @property
    def version(self) -> int:
        return int(self._lib.tk_retained_version(self._h))

    def set_clear_color(self, premul_rgba8: int):
        self._lib.tk_retained_set_clear_color(self._h, int(premul_rgba8) & 0xFFFFFFFF)

    def insert(self, node_id: int, content: Canvas, transform=None, before: int = 0):
        t, keep = _affine(transform)
        self._check(self._lib.tk_retained_insert(self._h, int(node_id), content._h, t, int(before)), "insert")

    def replace(self, node_id: int, content: Canvas):
        self._check(self._lib.tk_retained_replace(self._h, int(node_id), content._h), "replace")

    def set_transform(self, node_id: int, transform=None):
        t, keep = _affine(transform)
        self._check(self._lib.tk_retained_set_transform(self._h, int(node_id), t), "set_transform")

    def move_before(self, node_id: int, sibling: int = 0):
        self._check(self._lib.tk_retained_move_before(self._h, int(node_id), int(sibling)), "move_before")

    def remove(self, node_id: int):
        self._check(self._lib.tk_retained_remove(self._h, int(node_id)), "remove")

    def invalidate_rect(self, x0: int, y0: int, x1: int, y1: int):
        r = (C.c_int32 * 4)(int(x0), int(y0), int(x1), int(y1))
        self._check(self._lib.tk_retained_invalidate_rect(self._h, r), "invalidate_rect")

    def invalidate_all(self):
        self._check(self._lib.tk_retained_invalidate_all(self._h), "invalidate_all")

    def materialize(self):
        """(Canvas, damage): the scene recorded as one canvas (valid until the
        next materialize) and a dict {full, rects (n x 4 int32 array)}."""
        d = N.Damage()
        h = self._lib.tk_retained_materialize(self._h, C.byref(d))
        if not h:
            raise ValueError("retained scene: materialization failed")
        if self._canvas is not None:
            self._canvas._h = None  # its native canvas was just replaced
        self._canvas = Canvas(0, 0, _handle=h, _owner=self)
        rects = np.zeros((0, 4), np.int32)
        if d.rect_count:
            rects = np.ctypeslib.as_array((C.c_int32 * (4 * d.rect_count)).from_address(d.rects)).reshape(-1, 4).copy()
        return self._canvas, {"full": bool(d.full), "rects": rects}
