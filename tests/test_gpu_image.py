"""GPU parity of image patterns (BRUSH_PATTERN_RESOURCE sampled in fine,
shared/brush/texture.hlsli:7-31; PTCL_IMAGE from coarse's full_tile_image,
coarse/paint.hlsli:30-34): PTCL, tile records and pixels of the sm_100a path
equal the oracle's bit for bit; the full-tile promotion gives the pixels of
fine interpreting every draw in every tile."""
from __future__ import annotations

import numpy as np
import pytest

import tileink_b200 as tk
from tileink_b200 import _native as N

from image_cases import image_scene, premul_image
from test_gpu_parity import compare_frame

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed,scale", [(1, 1.0), (2, 1.5), (3, 0.8)])
def test_gpu_image_patterns(renderer, seed, scale):
    c = image_scene(seed, scale=scale)
    compare_frame(renderer, c)
    ptcl = renderer.debug(N.STAGE_PTCL, 0)
    assert (ptcl["tag"] == N.PTCL_IMAGE).any()


def test_gpu_image_promotion_matches_fine_only_oracle(renderer):
    import oracle
    c = image_scene(5, opaque=True, clip=False)
    want = oracle.interpret_sdf_draws(c.scene_desc())
    renderer.upload(c)
    renderer.render()
    got = renderer.readback().view(np.uint8).reshape(want.shape)
    assert np.array_equal(got, want), int((got != want).any(axis=2).sum())


def test_gpu_image_exact_placement(renderer):
    """An opaque image drawn at its own size on the pixel grid with nearest
    sampling reproduces its texels."""
    rng = np.random.default_rng(9)
    img = premul_image(rng, 48, 40, opaque=True)
    c = tk.Canvas(64, 48)
    ix = c.add_image(img)
    c.push_image(0, 0, 48, 40, ix)
    renderer.upload(c)
    renderer.render()
    got = renderer.readback().reshape(48, 64)
    assert np.array_equal(got[:40, :48], img)


def test_gpu_rejects_bad_image_brushes(renderer):
    rng = np.random.default_rng(3)
    c = tk.Canvas(64, 64)
    ix = c.add_image(premul_image(rng, 8, 8))
    c.push_image(4, 4, 40, 40, ix)
    a = c.scene_arrays()
    a["brush"] = a["brush"].copy()
    a["brush"][int(a["draws"]["brush_offset"][0]) + 5] = 9  # width differs from the image's
    with pytest.raises(Exception):
        renderer.upload(N.ArrayScene(a))
    b = c.scene_arrays()
    b["images"] = []
    with pytest.raises(Exception):
        renderer.upload(N.ArrayScene(b))
    # one side above the 2D texture limit (a reflect period of 2^32 would
    # wrap the sampler's index arithmetic)
    wide = c.scene_arrays()
    wide["images"] = [np.zeros((1, N.MAX_IMAGE_DIMENSION + 1), np.uint32)]
    with pytest.raises(Exception, match="texture limit"):
        renderer.upload(N.ArrayScene(wide))
