"""Text on the GPU, bit-exact against the oracle at every stage and against
the fine-only oracle:

* glyph outline fills (DrawTag::PathGlyph -> PTCL_PATH_GLYPH): coverage as a
  fill, composited by src_over_mask_linear_auto_u8 (fine/interpreter.hlsli:
  205-206, fine/text/auto.hlsli:28-33), with solid and gradient brushes,
  translucent text, clip layers and text beside SDF shapes (the SDF kernel
  instance);
* glyph runs (PTCL_GLYPH): coarse glyph lists per tile (coarse/text.hlsli),
  fine composite_glyphs_at over glyph images of all six contents
  (fine/glyph.hlsli), clipped runs, runs under clip layers."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import tileink_b200 as tk
from tileink_b200 import _native as N

from test_gpu_parity import compare_frame
from text_cases import glyph_run_scene, glyph_scene

pytestmark = pytest.mark.gpu


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


@pytest.mark.parametrize("seed, clip, outlines", [(1, False, False), (2, True, False), (3, False, True), (4, True, True)])
def test_gpu_glyph_runs_match_oracle(renderer, seed, clip, outlines):
    c = glyph_run_scene(seed, clip=clip, outlines=outlines)
    img, ref = compare_frame(renderer, c)
    assert np.array_equal(renderer.debug(N.STAGE_GLYPHS, 0), ref.get(oracle.OR_PASS_GLYPHS, np.uint32, 0))
    tags = renderer.debug(N.STAGE_PTCL, 0)["tag"]
    assert (tags == N.PTCL_GLYPH).sum() > 20
    tiles = renderer.debug(N.STAGE_TILES, 0)
    assert tiles["glyph_count"].sum() == len(renderer.debug(N.STAGE_GLYPHS, 0)) > 0
    want = oracle.interpret_path_draws(c.scene_desc(), threads=8)
    assert np.array_equal(img, want), int((img != want).any(axis=2).sum())


@pytest.mark.parametrize("content", range(6))
def test_gpu_glyph_run_contents(renderer, content):
    c = glyph_run_scene(10 + content, contents=[content], runs=30)
    img, _ = compare_frame(renderer, c)
    want = oracle.interpret_path_draws(c.scene_desc(), threads=8)
    assert np.array_equal(img, want)


def test_gpu_glyph_runs_in_incremental_frames(renderer):
    """Damage-driven frames of a text scene equal full frames (the glyph
    lists of the redrawn tiles only)."""
    c = glyph_run_scene(21, runs=30)
    renderer.upload(c)
    renderer.render_incremental(None)
    full = renderer.readback().copy()
    st = renderer.render_incremental({"full": False, "rects": [[20, 10, 140, 90]]})
    assert st["full_redraw"] == 0
    assert np.array_equal(renderer.readback(), full)


def test_gpu_rejects_bad_glyph_runs(renderer):
    c = glyph_run_scene(5, runs=6)
    a = c.scene_arrays()
    bad = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in a.items()}
    bad["glyphs"]["image"][0] = len(a["glyph_images"]) + 3
    with pytest.raises(tk.TileinkError):
        renderer.upload(N.ArrayScene(bad))
    bad = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in a.items()}
    bad["glyph_images"]["data_offset"][0] = len(a["glyph_texels"])
    with pytest.raises(tk.TileinkError):
        renderer.upload(N.ArrayScene(bad))
    renderer.render_to_image(c)  # the context stays usable
