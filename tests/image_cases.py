"""Image pattern scenes (Canvas::push_image, canvas/primitives/images.rs:9-26):
registered images of random premultiplied texels drawn into rects with every
extend and sampling mode, at full and partial opacity, over and under clips."""
from __future__ import annotations

import numpy as np

import tileink_b200 as tk
from tileink_b200 import _native as N


def premul_image(rng, w, h, opaque=False):
    """(h, w) uint32 premultiplied RGBA8 texels, red in the low byte."""
    rgb = rng.integers(0, 256, (h, w, 3))
    a = np.full((h, w), 255) if opaque else rng.integers(0, 256, (h, w))
    pm = (rgb * a[..., None] + 127) // 255
    return (pm[..., 0] | (pm[..., 1] << 8) | (pm[..., 2] << 16) | (a << 24)).astype(np.uint32)


def image_scene(seed, w=320, h=240, scale=1.0, opaque=False, clip=True):
    """opaque: every image opaque, so that the analytic route of full-tile
    images (fine/specialized.hlsli:84-90) gives the interpreter's bits."""
    rng = np.random.default_rng(seed)
    c = tk.Canvas(w, h, scale=scale)
    c.set_clear_color(0xFF302820)
    ims = [c.add_image(premul_image(rng, 7, 5, opaque=True)), c.add_image(premul_image(rng, 33, 20, opaque=opaque)),
           c.add_image(premul_image(rng, 1, 1, opaque=True)), c.add_image(premul_image(rng, 64, 64, opaque=True))]
    # a full-canvas opaque image: PTCL_IMAGE in every tile it covers
    c.push_image(0, 0, w / scale, h / scale, ims[3], tk.canvas.EXTEND_PAD, N.PATTERN_NEAREST)
    for k in range(36):
        x0, y0 = rng.uniform(-40, w / scale - 20), rng.uniform(-40, h / scale - 20)
        x1, y1 = x0 + rng.uniform(3, 150), y0 + rng.uniform(3, 120)
        c.push_image(x0, y0, x1, y1, ims[k % len(ims)], k % 3, (k // 3) % 2, 255 if k % 4 else int(rng.integers(0, 256)))
    if clip:
        c.push_clip_sdf_rect_layer(20.5, 15.25, w / scale - 30, h / scale - 25, radius=12.0)
    for k in range(8):
        x0, y0 = rng.uniform(0, w / scale - 60), rng.uniform(0, h / scale - 60)
        c.push_image(x0, y0, x0 + rng.uniform(40, 200), y0 + rng.uniform(40, 160), ims[(k + 1) % 4], k % 3, k % 2)
    if clip:
        c.pop_layer()
    c.push_rect(50, 40, 90, 70, tk.Brush.solid(0.2, 0.7, 0.4, 0.8))
    return c
