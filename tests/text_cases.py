"""Seeded text scenes for the glyph tests: glyph outline fills (PathGlyph
draws) and glyph runs over rasterized glyph images of every content kind."""
from __future__ import annotations

import numpy as np

import tileink_b200 as tk
from tileink_b200 import _native as N


def glyph_scene(seed, width=320, height=200, runs=40, sdf=False, clip=False):
    """Glyph outline fills with solid and gradient brushes, optional SDF
    shapes beside them and a clip layer around them."""
    rng = np.random.default_rng(seed)
    c = tk.Canvas(width, height)
    c.set_clear_color(int(rng.choice([0xFFFFFFFF, 0xFF202020, 0x00000000, 0xFF3366CC])))
    if clip:
        c.push_clip_layer(tk.BezPath().move_to(10, 5).line_to(width - 20, 15).line_to(width - 5, height - 10)
                          .line_to(15, height - 25).close())
    for k in range(runs):
        x, y = rng.uniform(0, width - 40), rng.uniform(20, height)
        em = rng.uniform(6, 48)
        p = tk.BezPath()
        for g in range(int(rng.integers(1, 4))):  # a few glyph contours per run
            gx = x + g * 0.7 * em
            p.move_to(gx, y)
            p.quad_to(gx + 0.3 * em, y - 1.1 * em, gx + 0.6 * em, y)
            p.line_to(gx + 0.45 * em, y)
            p.quad_to(gx + 0.3 * em, y - 0.6 * em, gx + 0.15 * em, y)
            p.close()
        c.push_glyph_outlines(p, random_brush(rng, x, y, em))
        if sdf and k % 5 == 0:
            c.push_rect(x, y - em, x + em, y, tk.Brush.solid(0.9, 0.6, 0.1, 0.6), radius=2.0)
    if clip:
        c.pop_layer()
    return c


def random_brush(rng, x, y, em):
    kind = rng.uniform()
    if kind < 0.5:
        return tk.Brush.solid(*rng.uniform(0, 1, 3), float(rng.choice([1.0, rng.uniform(0.2, 1.0)])))
    if kind < 0.8:
        return tk.Brush.linear((x, y - em), (x + 2 * em, y), [(0.0, (1, 0, 0, 1)), (1.0, (0, 0, 1, 0.7))])
    return tk.Brush.radial((x + em, y - em / 2), 1.0, (x + em, y - em / 2), 1.5 * em,
                           [(0.0, (1, 1, 1, 1)), (0.6, (0.2, 0.8, 0.3, 1)), (1.0, (0, 0, 0, 0.5))])


def glyph_image(rng, content, w, h):
    """A blob-shaped mask (or colour glyph) of w x h texels for `content`."""
    yy, xx = np.mgrid[0:h, 0:w]
    r = np.hypot((xx + 0.5 - w / 2) / (w / 2), (yy + 0.5 - h / 2) / (h / 2))
    cov = np.clip((1.1 - r) * 255 * rng.uniform(1.5, 4.0), 0, 255).astype(np.uint32)
    if content in (N.GLYPH_MASK, N.GLYPH_LINEAR_MASK):
        return cov
    if content in (N.GLYPH_SUBPIXEL_MASK, N.GLYPH_LINEAR_SUBPIXEL_MASK):
        shift = [np.clip(np.roll(cov, s, axis=1), 0, 255) for s in (-1, 0, 1)]
        return shift[0] | (shift[1] << 8) | (shift[2] << 16)
    rgb = rng.integers(0, 256, 3)
    a = cov
    return ((rgb[0] * a // 255) | ((rgb[1] * a // 255) << 8) | ((rgb[2] * a // 255) << 16) | (a << 24)).astype(np.uint32)


def glyph_run_scene(seed, width=256, height=160, runs=24, contents=None, clip=False, outlines=False):
    """Glyph runs over rasterized glyph images of the given contents (all
    six by default) at integer pen positions, some glyphs without an image,
    some runs clipped, translucent and gradient brushes, clip layers."""
    rng = np.random.default_rng(seed)
    contents = list(range(6)) if contents is None else contents
    c = tk.Canvas(width, height)
    c.set_clear_color(int(rng.choice([0xFFFFFFFF, 0xFF181818, 0x00000000, 0x80402010])))
    images = []
    for k in range(12):
        content = contents[k % len(contents)]
        w, h = int(rng.integers(3, 18)), int(rng.integers(4, 22))
        images.append(c.add_glyph_image(int(rng.integers(-2, 3)), int(h - rng.integers(0, 4)),
                                         glyph_image(rng, content, w, h), content))
    if clip:
        c.push_clip_layer(tk.BezPath().move_to(5, 8).line_to(width - 10, 2).line_to(width - 20, height - 5)
                          .line_to(8, height - 12).close())
    for k in range(runs):
        x, y = int(rng.integers(-10, width - 30)), int(rng.integers(10, height + 10))
        glyphs = []
        for g in range(int(rng.integers(1, 9))):
            img = None if rng.uniform() < 0.1 else images[int(rng.integers(0, len(images)))]
            glyphs.append((img, x, y))
            x += int(rng.integers(4, 14))
        cl = None
        if rng.uniform() < 0.25:
            cl = (int(rng.integers(0, width // 2)), int(rng.integers(0, height // 2)), width, height)
        try:
            c.push_glyph_run(glyphs, random_brush(rng, x, y, 12.0), clip=cl)
        except ValueError:  # an empty run (no image, or clipped away)
            pass
        if outlines and k % 4 == 0:
            c.push_glyph_outlines(tk.BezPath().move_to(x, y).line_to(x + 12, y - 3).line_to(x + 4, y - 14).close(),
                                  tk.Brush.solid(0.1, 0.1, 0.1, 1))
    if clip:
        c.pop_layer()
    return c
