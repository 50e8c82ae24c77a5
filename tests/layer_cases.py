"""Scenes with clip, SDF-clip and opacity layers (the reference's fused
layer stacks, src/canvas/compile.rs:342-353 and src/shared/gpu_coarse.rs:
314-332), shared by the oracle and GPU tests."""
from __future__ import annotations

import numpy as np

import tileink_b200 as tk


def blob(rng, cx, cy, r, n=7):
    """A closed cubic blob around (cx, cy)."""
    a = np.sort(rng.uniform(0, 2 * np.pi, n))
    pts = [(cx + r * rng.uniform(0.5, 1.2) * np.cos(t), cy + r * rng.uniform(0.5, 1.2) * np.sin(t)) for t in a]
    p = tk.BezPath().move_to(*pts[0])
    for k in range(1, n + 1):
        q0, q1 = pts[(k - 1) % n], pts[k % n]
        p.cubic_to(q0[0] + (q1[0] - q0[0]) / 3 + rng.normal(0, r / 6), q0[1] + (q1[1] - q0[1]) / 3,
                   q0[0] + 2 * (q1[0] - q0[0]) / 3, q0[1] + 2 * (q1[1] - q0[1]) / 3 + rng.normal(0, r / 6),
                   q1[0], q1[1])
    return p.close()


def opacity_scene(seed, w=256, h=192):
    """Opacity layers (path-masked, opacities 0..1) nested with path clips and
    SDF clips, over fills with solid and gradient paint; layers open and close
    between draws so batches split and merge."""
    rng = np.random.default_rng(seed)
    c = tk.Canvas(w, h)
    c.set_clear_color(0xFFFFFFFF)

    def fill(k):
        x, y = rng.uniform(0, w), rng.uniform(0, h)
        r = float(rng.uniform(10, 60))
        if k % 3 == 2:
            b = tk.Brush.linear((x - r, y), (x + r, y + r), [(0.0, (*rng.uniform(0, 1, 3), 1.0)),
                                                            (1.0, (*rng.uniform(0, 1, 3), 0.6))])
        else:
            b = tk.Brush.solid(*rng.uniform(0, 1, 3), float(rng.choice([1.0, rng.uniform(0.3, 1)])))
        c.push_path(blob(rng, x, y, r), b, fill_rule=int(k % 2))

    for k in range(4):
        fill(k)
    # an opacity layer over one stack of draws
    c.push_opacity_layer(blob(rng, w * 0.5, h * 0.5, min(w, h) * 0.45), 0.6)
    for k in range(6):
        fill(k)
    c.pop_layer()
    # clip > opacity (covers every tile: no segments) > SDF clip > draws
    c.push_clip_layer(blob(rng, w * 0.4, h * 0.45, min(w, h) * 0.35))
    c.push_opacity_layer(tk.BezPath().move_to(-5, -5).line_to(w + 5, -5).line_to(w + 5, h + 5)
                         .line_to(-5, h + 5).close(), 0.35)
    c.push_clip_sdf_circle_layer(w * 0.55, h * 0.5, min(w, h) * 0.3)
    for k in range(5):
        fill(k)
    c.pop_layer()
    c.pop_layer()
    c.pop_layer()
    # a clip with draws beside an opacity layer (the clip fuses, the batches split)
    c.push_clip_layer(blob(rng, w * 0.6, h * 0.6, min(w, h) * 0.4))
    fill(0)
    c.push_opacity_layer(blob(rng, w * 0.65, h * 0.55, min(w, h) * 0.3), 0.5)
    for k in range(3):
        fill(k)
    c.pop_layer()
    fill(2)
    c.pop_layer()
    # nested opacity layers, the inner one fully transparent
    c.push_opacity_layer(blob(rng, w * 0.7, h * 0.3, 40), 1.0)
    c.push_opacity_layer(blob(rng, w * 0.72, h * 0.32, 45), 0.0)
    fill(1)
    c.pop_layer()
    c.pop_layer()
    for k in range(4):
        fill(k)
    return c


def sampled_blur_scene(seed, factor, down, up, w=200, h=150, sigma=5.0):
    """Fills inside a blur group blurred through a copy reduced by `factor`
    (BlurSampling), over fills outside it."""
    from tileink_b200 import _native as N
    rng = np.random.default_rng(seed)
    c = tk.Canvas(w, h)
    c.set_clear_color(0xFFFFFFFF)
    for _ in range(4):
        c.push_path(blob(rng, rng.uniform(0, w), rng.uniform(0, h), 30), tk.Brush.solid(*rng.uniform(0, 1, 3), 1.0))
    c.push_blur_group(sigma, factor=factor, downsample=down, upsample=up)
    for k in range(8):
        c.push_path(blob(rng, rng.uniform(10, w - 10), rng.uniform(10, h - 10), rng.uniform(8, 40)),
                    tk.Brush.solid(*rng.uniform(0, 1, 3), float(rng.uniform(0.4, 1))), fill_rule=k % 2)
    c.pop_layer()
    c.push_path(blob(rng, w * 0.5, h * 0.5, 20), tk.Brush.solid(0.1, 0.2, 0.3, 0.5))
    return c


def progressive_scene(seed, w=200, h=150, sigma=6.0, quality=0, uniform=False):
    """Fills inside a progressive blur group (Filter::ProgressiveBlur),
    sharp at one side and blurred up to `sigma` at the other, over fills
    outside it."""
    rng = np.random.default_rng(seed)
    c = tk.Canvas(w, h)
    c.set_clear_color(0xFFFFFFFF)
    for _ in range(4):
        c.push_path(blob(rng, rng.uniform(0, w), rng.uniform(0, h), 30), tk.Brush.solid(*rng.uniform(0, 1, 3), 1.0))
    start = (rng.uniform(0, w * 0.4), rng.uniform(0, h * 0.4))
    end = start if uniform else (rng.uniform(w * 0.5, w), rng.uniform(h * 0.5, h))
    c.push_progressive_blur_group(start, end, sigma, quality)
    for k in range(10):
        c.push_path(blob(rng, rng.uniform(10, w - 10), rng.uniform(10, h - 10), rng.uniform(6, 40)),
                    tk.Brush.solid(*rng.uniform(0, 1, 3), float(rng.uniform(0.4, 1))), fill_rule=k % 2)
    c.pop_layer()
    c.push_path(blob(rng, w * 0.5, h * 0.5, 20), tk.Brush.solid(0.1, 0.2, 0.3, 0.5))
    return c


def filter_scene(seed, chain, rect, fixed_region=False, w=200, h=150, children=True):
    """Fills inside a filter layer (Canvas::push_filter_layer with a chain of
    filters over a rect sample region), over fills outside it; `chain` as
    Canvas.push_filter_layer takes it. children=False leaves the layer empty
    (the same random scene otherwise)."""
    rng = np.random.default_rng(seed)
    c = tk.Canvas(w, h)
    c.set_clear_color(0xFFFFFFFF)
    for _ in range(4):
        c.push_path(blob(rng, rng.uniform(0, w), rng.uniform(0, h), 30), tk.Brush.solid(*rng.uniform(0, 1, 3), 1.0))
    c.push_filter_layer(chain, rect, fixed_region)
    for k in range(10):
        if k % 3 == 2:
            x, y, r = rng.uniform(0, w), rng.uniform(0, h), float(rng.uniform(10, 40))
            b = tk.Brush.linear((x - r, y), (x + r, y + r), [(0.0, (*rng.uniform(0, 1, 3), 1.0)),
                                                            (1.0, (*rng.uniform(0, 1, 3), 0.5))])
        else:
            b = tk.Brush.solid(*rng.uniform(0, 1, 3), float(rng.uniform(0.3, 1)))
        path = blob(rng, rng.uniform(10, w - 10), rng.uniform(10, h - 10), rng.uniform(6, 40))
        if children:
            c.push_path(path, b, fill_rule=k % 2)
    c.pop_layer()
    c.push_path(blob(rng, w * 0.5, h * 0.5, 20), tk.Brush.solid(0.1, 0.2, 0.3, 0.5))
    return c


# chains for the filter layer tests: every colour filter, the colour matrix,
# offsets, and chains mixing them
SEPIA_MATRIX = [0.393, 0.769, 0.189, 0, 0, 0.349, 0.686, 0.168, 0, 0, 0.272, 0.534, 0.131, 0, 0, 0, 0, 0, 1, 0]


def filter_chains():
    """Named chains for the filter layer tests."""
    from tileink_b200 import _native as N
    return {
        "brightness": [(N.FILTER_BRIGHTNESS, 1.6)],
        "contrast": [(N.FILTER_CONTRAST, 0.45)],
        "grayscale": [(N.FILTER_GRAYSCALE, 0.8)],
        "hue_rotate": [(N.FILTER_HUE_ROTATE, 137.0)],
        "invert": [(N.FILTER_INVERT, 0.7)],
        "opacity": [(N.FILTER_OPACITY, 0.55)],
        "saturate": [(N.FILTER_SATURATE, 2.3)],
        "sepia": [(N.FILTER_SEPIA, 1.0)],
        "matrix": [(N.FILTER_COLOR_MATRIX, SEPIA_MATRIX)],
        "matrix_alpha": [(N.FILTER_COLOR_MATRIX, [1, 0, 0, 0, 0.1, 0, 0.5, 0.5, 0, 0, 0, 0, 1, 0, -0.2,
                                                  0, 0, 0, 0.6, 0.1])],
        "offset": [(N.FILTER_OFFSET, (7.5, -4.2))],
        "chain": [(N.FILTER_GRAYSCALE, 0.5), (N.FILTER_OFFSET, (-3.0, 5.6)), (N.FILTER_HUE_ROTATE, -60.0),
                  (N.FILTER_CONTRAST, 1.4), (N.FILTER_OPACITY, 0.8)],
        "erode": [(N.FILTER_ERODE, (2.5, 1.0))],
        "dilate": [(N.FILTER_DILATE, (3.0, 4.2))],
        "morphology_chain": [(N.FILTER_DILATE, (2.0, 0.0)), (N.FILTER_SEPIA, 0.6), (N.FILTER_ERODE, (0.0, 1.5)),
                             (N.FILTER_OFFSET, (2.0, 2.0))],
        "flood": [(N.FILTER_FLOOD, (0.2, 0.6, 0.9, 0.7))],
        "drop_shadow": [(N.FILTER_DROP_SHADOW, (4.5, -3.0, 3.0, (0.0, 0.0, 0.2, 0.8)))],
        "drop_shadow_sharp": [(N.FILTER_DROP_SHADOW, (-6.0, 5.0, 0.0, (0.9, 0.1, 0.1, 1.0))),
                              (N.FILTER_GRAYSCALE, 0.3)],
        "drop_shadow_wide": [(N.FILTER_DROP_SHADOW, (2.0, 2.0, 7.5, (0.1, 0.1, 0.1, 0.6)))],
        "component_transfer": [(N.FILTER_COMPONENT_TRANSFER,
                                np.concatenate([255 - np.arange(256), (np.arange(256) ** 2) // 255,
                                                np.minimum(np.arange(256) * 2, 255), np.arange(256)])),
                               (N.FILTER_SATURATE, 1.5)],
        "convolve_box": [(N.FILTER_CONVOLVE, {"kernel": np.ones((3, 3)), "edge_mode": N.CONVOLVE_EDGE_DUPLICATE})],
        "convolve_edges": [(N.FILTER_CONVOLVE, {"kernel": [[0, -1, 0], [-1, 4, -1], [0, -1, 0]], "divisor": 1.0,
                                                "bias": 0.3, "edge_mode": N.CONVOLVE_EDGE_WRAP})],
        "convolve_preserve": [(N.FILTER_CONVOLVE, {"kernel": [[1, 2, 0.5, -1, 3], [0, 1, 0, 2, 1]],
                                                   "target": (3, 0), "divisor": 6.5, "bias": -0.1,
                                                   "edge_mode": N.CONVOLVE_EDGE_NONE, "preserve_alpha": True}),
                              (N.FILTER_OPACITY, 0.9)],
        "blur_xy": [(N.FILTER_BLUR, (2.5, 6.0)), (N.FILTER_CONTRAST, 1.3)],
        "blur_x_only": [(N.FILTER_SATURATE, 0.4), (N.FILTER_BLUR, (7.0, 0.0))],
    }
