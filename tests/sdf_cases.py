"""Scenes of the reference's coarse known-answer pixel tests for SDF rects
(src/native/runtime/tests/coarse_count/rect_pixels.rs:110-283 and
occlusion_pixels.rs:34-116), restated on this library's Canvas: the full
pipeline must give the pixels of the fine-only oracle, which interprets every
draw in every tile and so bypasses coarse's full-tile, hollow-stroke and
occlusion proofs."""
from __future__ import annotations

import math

import numpy as np

import tileink_b200 as tk
from tileink_b200 import _native as N

W, H = 129, 113
BLACK = 0xFF000000


def rgba8(r, g, b, a=255):
    """peniko Color::from_rgba8: straight sRGB bytes."""
    return tk.Brush.solid(r / 255.0, g / 255.0, b / 255.0, a / 255.0)


def inset(rect, v):
    """kurbo Rect::inset: a positive inset grows the rectangle."""
    x0, y0, x1, y1 = rect
    return (x0 - v, y0 - v, x1 + v, y1 + v)


def affine_arrays(t):
    """GpuAffine of a kurbo Affine [a b c d e f] and its inverse, in f32."""
    a, b, c, d, e, f = t
    det = a * d - b * c
    inv = (d / det, -b / det, -c / det, a / det, (c * f - d * e) / det, (b * e - a * f) / det)
    return np.float32(t), np.float32(inv)


def rect_mode_scene(mode: int) -> dict:
    """rect_pixels.rs:138-231: a translucent full-canvas rect under a rect
    stroke (modes 0-10) or rect (11, 12) of edge, huge and far-away geometry,
    modes >= 4 under a draw transform with pixel bounds the whole canvas."""
    c = tk.Canvas(W, H)
    c.set_clear_color(BLACK)
    c.push_rect(0, 0, 129, 113, rgba8(90, 140, 210, 177))
    rect = {11: (1e7, 0.25, 1e7 + 128.0, 112.75), 12: (1.70e38, 0.25, 1.705e38, 112.75),
            9: (65400.25, 0.25, 65528.0, 112.75), 10: (-65528.0, 0.25, -65400.25, 112.75),
            7: (1e7 - 1.0, 0.25, 1e7 + 129.0, 112.75), 8: (1.69e38, 0.25, 1.705e38, 112.75),
            3: (16.25, 16.25, 31.75, 31.75)}.get(mode, (0.25, 0.25, 128.75, 112.75))
    if mode in (7, 8, 11, 12):
        radius = 0.0
    elif mode == 1:
        radius = 39.5
    else:
        radius = (4.0, 16.0, 7.5, 26.0)  # top-left, top-right, bottom-left, bottom-right
    widths = {7: 2.0, 8: (0.0, 0.0, 0.0, 2e36), 2: 150.0}.get(mode, (1.0, 7.5, 4.0, 2.25))
    brush = rgba8(240, 70, 30, 193)
    if mode >= 11:
        draw = c.push_rect(*rect, brush, radius=radius)
    else:
        draw = c.push_rect_stroke(*rect, widths, brush, radius=radius)
    a = c.scene_arrays()
    if mode >= 4:
        t = {4: (1, 0, 0, 1, 0.375, -0.25), 5: (0.8, 0, 0, 0.9, 0, 0),
             6: (math.cos(0.15), math.sin(0.15), -math.sin(0.15), math.cos(0.15), 0, 0),
             7: (1, 0, 0, 1, -1e7, 0), 11: (1, 0, 0, 1, -1e7, 0), 9: (1, 0, 0, 1, -65408.0, 0),
             10: (1, 0, 0, 1, 65512.0, 0)}.get(mode, (1, 0, 0, 1, -1.702e38, 0))
        fwd, inv = affine_arrays(t)
        draws = a["draws"].copy()
        draws["transform"][draw] = tuple(fwd)
        draws["inverse_transform"][draw] = tuple(inv)
        draws["pixel_bounds"][draw] = (0, 0, 129, 113)
        a["draws"] = draws
    return a


def specialization_scene(count: int, alpha: int, mode: int) -> tk.Canvas:
    """rect_pixels.rs:244-283: `count` rects, full-canvas or rounded partial,
    switching among empty, colour, analytic, mixed and general streams (the
    reference's four-corner gradient mode 3 has no counterpart here)."""
    c = tk.Canvas(W, H)
    c.set_clear_color(BLACK)
    for i in range(count):
        partial = mode == 1 or (mode == 2 and i % 2 == 0)
        rect = (3.25, 7.75, 124.5, 107.25) if partial else (0.0, 0.0, 129.0, 113.0)
        a = 0 if mode == 4 else alpha
        c.push_rect(*rect, rgba8((i * 37) % 256, (i * 71) % 256, (i * 97) % 256, a),
                    radius=19.5 if partial else 0.0)
    return c


def occlusion_scene(alpha: int, radius: float, grow: float) -> tk.Canvas:
    """occlusion_pixels.rs:34-46, 85-116: 40 translucent full-canvas rects,
    then a cover of the given alpha that may hide them, then a translucent
    rect on top."""
    c = tk.Canvas(W, H)
    c.set_clear_color(BLACK)
    for i in range(40):
        c.push_rect(0, 0, 129, 113, rgba8((i * 37) % 256, (i * 71) % 256, (i * 97) % 256, 119), radius=float(i % 8))
    c.push_rect(*inset((16.0, 0.0, 129.0, 113.0), grow), rgba8(230, 70, 35, alpha), radius=radius)
    c.push_rect(0, 32.25, 90, 79.75, rgba8(20, 130, 240, 130), radius=3.0)
    return c


def all_cases():
    """(name, scene) pairs: Canvas objects or scene-array dicts."""
    cases = [(f"rect_mode_{m}", rect_mode_scene(m)) for m in range(13)]
    cases += [(f"spec_{n}_{a}_{m}", specialization_scene(n, a, m)) for n in (0, 1, 17, 257) for a in (0, 127, 255)
              for m in (2, 0, 1, 4)]
    cases += [(f"occlusion_{a}_{r}_{g}", occlusion_scene(a, r, g)) for a in (0, 254, 255) for r in (0.0, 19.0)
              for g in (0.0, 0.375)]
    return cases


def desc_of(scene):
    if isinstance(scene, dict):
        s = N.ArrayScene(scene)
        return s, s.desc
    return scene, scene.scene_desc()


def particles(records):
    """PTCL records (tag, color) for the fine-only oracle's tile stream."""
    out = np.zeros(len(records), N.PTCL_DTYPE)
    for k, (tag, color) in enumerate(records):
        out[k]["tag"], out[k]["color"] = tag, color
    return out


def partial_clip_cases():
    """occlusion_pixels.rs:48-83: an opaque background, then, inside a
    (rounded, grown) SDF rect clip, 128 translucent full-canvas rects and an
    opaque cover; the expected stream interprets every draw in every tile
    inside the clip. (name, canvas, particle stream) triples."""
    out = []
    for radius in (0.0, 41.0):
        for grow in (0.0, 4.375):
            c = tk.Canvas(W, H)
            c.set_clear_color(BLACK)
            c.push_rect(0, 0, 129, 113, rgba8(0, 0, 0, 255))
            c.push_clip_sdf_rect_layer(*inset((0.0, 0.0, 129.0, 113.0), grow), radius=radius)
            for i in range(128):
                c.push_rect(0, 0, 129, 113, rgba8((i * 17) % 256, (i * 29) % 256, (i * 3) % 256, 120))
            c.push_rect(0, 0, 129, 113, rgba8(23, 47, 93, 255))
            c.pop_layer()
            n = len(c.scene_arrays()["draws"])
            stream = [(N.PTCL_SDF, 0), (N.PTCL_BEGIN_SDF_CLIP, 1)] + [(N.PTCL_SDF, d) for d in range(2, n)] + \
                     [(N.PTCL_END_CLIP, 0)]
            out.append((f"partial_clip_{radius}_{grow}", c, particles(stream)))
    return out
