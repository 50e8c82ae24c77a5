"""Image patterns on the CPU: the pattern brush words of Canvas::push_image
(Brush::for_rect_resource, shared/brush.rs:557-580, under physical_brush's
scale, canvas/surface.rs:395-400), the oracle's sampler on exact placements,
and the scene arrays carrying the texture table."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import tileink_b200 as tk
from tileink_b200 import _native as N

from image_cases import image_scene, premul_image


def brush_words(c, draw):
    a = c.scene_arrays()
    bo = int(a["draws"]["brush_offset"][draw])
    return a["brush"][bo:bo + 21], a


@pytest.mark.parametrize("scale", [1.0, 1.5, 0.75])
def test_push_image_brush_words(scale):
    rng = np.random.default_rng(1)
    c = tk.Canvas(200, 150, scale=scale)
    ix = c.add_image(premul_image(rng, 13, 7))
    x0, y0, x1, y1 = 10.3, 20.7, 77.1, 61.9
    d = c.push_image(x0, y0, x1, y1, ix, tk.canvas.EXTEND_REFLECT, N.PATTERN_BILINEAR, 200)
    w, a = brush_words(c, d)
    assert list(w[:9]) == [7, 2, 0, 0,
                           0x80000000 | ix, 13, 7, 200, 1]
    f32 = np.float32
    sx, sy = f32(1.0) / f32(x1 - x0), f32(1.0) / f32(y1 - y0)
    inv = f32(1.0) / f32(scale)
    want = np.array([sx * inv, f32(0) * inv, f32(0) * inv, sy * inv, -f32(x0) * sx, -f32(y0) * sy], np.float32)
    assert w[9:15].view(np.float32).tobytes() == want.tobytes()
    assert len(a["images"]) == 1 and a["images"][0].shape == (7, 13)


def test_push_image_rejects_bad_rects_and_images():
    c = tk.Canvas(64, 64)
    ix = c.add_image(np.ones((2, 2), np.uint32))
    for rect in [(0, 0, 0, 10), (5, 5, 4, 10), (0, 0, float("nan"), 3), (0, 0, float("inf"), 3)]:
        with pytest.raises(ValueError):
            c.push_image(*rect, ix)
    with pytest.raises(ValueError):
        c.push_image(0, 0, 4, 4, ix + 1)
    with pytest.raises(ValueError):
        c.add_image(np.zeros((0, 3), np.uint32))
    # sides above the 2D texture limit
    for shape in [(1, N.MAX_IMAGE_DIMENSION + 1), (N.MAX_IMAGE_DIMENSION + 1, 1)]:
        with pytest.raises(ValueError):
            c.add_image(np.zeros(shape, np.uint32))
    assert c.add_image(np.zeros((1, N.MAX_IMAGE_DIMENSION), np.uint32)) >= 0


def test_oracle_exact_placement_reproduces_texels():
    rng = np.random.default_rng(2)
    img = premul_image(rng, 40, 24, opaque=True)
    for sampling in (N.PATTERN_NEAREST, N.PATTERN_BILINEAR):
        for extend in (0, 1, 2):
            c = tk.Canvas(48, 32)
            c.push_image(0, 0, 40, 24, c.add_image(img), extend, sampling)
            got = oracle.OracleRun(c.scene_desc()).get(oracle.OR_IMAGE, np.uint32).reshape(32, 48)
            assert np.array_equal(got[:24, :40], img), (sampling, extend)


def test_oracle_image_pipeline_equals_fine_only():
    """Coarse's PTCL_IMAGE promotion (full_tile_image) changes no pixel."""
    c = image_scene(4, 160, 128, opaque=True, clip=False)
    want = oracle.interpret_sdf_draws(c.scene_desc())
    got = oracle.OracleRun(c.scene_desc(), threads=4).get(oracle.OR_IMAGE, np.uint32)
    assert np.array_equal(got.view(np.uint8).reshape(want.shape), want)


def test_image_replay_under_translation():
    """A retained node's image replays under a translation as the same image
    pushed at the translated rect (the brush maps the image into the rect)."""
    rng = np.random.default_rng(3)
    img = premul_image(rng, 9, 6)
    src = tk.Canvas(96, 64)
    src.keep_commands(True)
    src.push_image(3.5, 2.25, 40, 33, src.add_image(img), 1, 1, 180)
    got = tk.Canvas(96, 64)
    got.replay(src, (1, 0, 0, 1, 10, 5))
    want = tk.Canvas(96, 64)
    want.push_image(13.5, 7.25, 50, 38, want.add_image(img), 1, 1, 180)
    a, b = got.scene_arrays(), want.scene_arrays()
    assert np.array_equal(a["brush"], b["brush"]) and np.array_equal(a["sdf"], b["sdf"])
    assert np.array_equal(a["images"][0], b["images"][0])
    with pytest.raises(ValueError):
        tk.Canvas(96, 64).replay(src, (2, 0, 0, 1, 0, 0))
