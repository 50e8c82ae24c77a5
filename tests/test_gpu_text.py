"""Glyph outline fills (DrawTag::PathGlyph -> PTCL_PATH_GLYPH) on the GPU:
coverage as a fill, composited by src_over_mask_linear_auto_u8
(fine/interpreter.hlsli:205-206, fine/text/auto.hlsli:28-33), bit-exact
against the oracle at every stage and against the fine-only oracle, with
solid and gradient brushes, translucent text, clip layers, text beside SDF
shapes (the SDF kernel instance) and the C3 glyph workload."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import tileink_b200 as tk
from tileink_b200 import _native as N

from test_gpu_parity import compare_frame

pytestmark = pytest.mark.gpu


def glyph_scene(seed, width=320, height=200, runs=40, sdf=False, clip=False):
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
        kind = rng.uniform()
        if kind < 0.5:
            b = tk.Brush.solid(*rng.uniform(0, 1, 3), float(rng.choice([1.0, rng.uniform(0.2, 1.0)])))
        elif kind < 0.8:
            b = tk.Brush.linear((x, y - em), (x + 2 * em, y), [(0.0, (1, 0, 0, 1)), (1.0, (0, 0, 1, 0.7))])
        else:
            b = tk.Brush.radial((x + em, y - em / 2), 1.0, (x + em, y - em / 2), 1.5 * em,
                                [(0.0, (1, 1, 1, 1)), (0.6, (0.2, 0.8, 0.3, 1)), (1.0, (0, 0, 0, 0.5))])
        c.push_glyph_outlines(p, b)
        if sdf and k % 5 == 0:
            c.push_rect(x, y - em, x + em, y, tk.Brush.solid(0.9, 0.6, 0.1, 0.6), radius=2.0)
    if clip:
        c.pop_layer()
    return c


@pytest.mark.parametrize("seed, sdf, clip", [(1, False, False), (2, False, True), (3, True, False), (4, True, True)])
def test_gpu_glyph_outlines_match_oracle(renderer, seed, sdf, clip):
    c = glyph_scene(seed, sdf=sdf, clip=clip)
    img, ref = compare_frame(renderer, c)
    tags = renderer.debug(N.STAGE_PTCL, 0)["tag"]
    assert (tags == N.PTCL_PATH_GLYPH).sum() > 50
    want = oracle.interpret_path_draws(c.scene_desc(), threads=8)
    assert np.array_equal(img, want), int((img != want).any(axis=2).sum())


def test_gpu_glyph_outlines_differ_from_plain_fills_only_at_edges(renderer):
    """The same outlines as plain fills: pixels the outline covers fully or
    not at all are identical; the partly covered ones carry the correction."""
    c = glyph_scene(5, runs=30)
    a = c.scene_arrays()
    a2 = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in a.items()}
    a2["draws"]["tag"][a2["draws"]["tag"] == N.DRAW_PATH_GLYPH] = N.DRAW_BRUSH
    glyphs = renderer.render_to_image(c).copy()
    fills = renderer.render_to_image(N.ArrayScene(a2)).copy()
    differ = (glyphs != fills).any(axis=2)
    assert differ.any() and differ.mean() < 0.25
