"""The library's multi-GPU splits, run rank after rank on one GPU (ranks
whose kernels would wait on one another never share a GPU here; these ranks
do not wait on one another at all):

* band split (tk_set_band): each band's context clamps the paths to its tile
  rows at upload and renders only them; the bands' pixel rows, assembled,
  equal the whole frame bit for bit, at 768x512 and at the benchmarked
  4096x4096 / 50,000-path frame;
* row-split objective (tk_diff_scene.loss_row0/1): the per-rank losses and
  gradients sum to the whole image's."""
from __future__ import annotations

import numpy as np
import pytest

import tileink_b200 as tk
from tileink_b200 import _native as N
from tileink_b200 import diff
from tileink_b200 import shard

pytestmark = pytest.mark.gpu


def band_frames(canvas, world, device_flatten=False):
    """(full frame, assembled bands, per-band segment counts)."""
    a = canvas.scene_arrays()
    full_r = tk.NativeRenderer(0)
    full = full_r.render_to_image(canvas).reshape(-1).view(np.uint32).copy()
    h, w = full_r.height, full_r.width
    full_segments = full_r.stats()["segments"]
    full_r.close()
    bands = shard.band_partition(shard.row_weights(a["paths"], (h + 15) // 16), world)
    out = np.zeros((h, w), np.uint32)
    segs = []
    r = tk.NativeRenderer(0)
    try:
        for y0, y1 in bands:
            r.set_band(y0, y1)
            r.upload(canvas)
            r.render()
            p0, p1 = shard.pixel_rows((y0, y1), h)
            out[p0:p1] = r.readback_rows(p0, p1)
            segs.append(r.stats()["segments"])
    finally:
        r.close()
    return full.reshape(h, w), out, segs, full_segments, bands


@pytest.mark.parametrize("config, kw, world", [
    (2, dict(width=768, height=512, paths=600), 3),
    (1, dict(), 2),
    (3, dict(width=480, height=270, paths=1500), 4),
    (4, dict(variant=2), 2),
])
def test_gpu_band_split_assembles_the_frame(config, kw, world):
    c = tk.generate(config, 7, **kw)
    full, bands_img, segs, full_segs, bands = band_frames(c, world)
    assert np.array_equal(full, bands_img), int((full != bands_img).sum())
    # each rank scanned only its band's segments, and together exactly the frame's
    assert sum(segs) == full_segs and max(segs) < full_segs


def test_gpu_band_split_of_the_benchmarked_frame():
    """4096x4096, 50,000 paths (seed 2, device segment plan): four bands."""
    c = tk.generate(2, 2, device_segment_plan=True)
    full, bands_img, segs, full_segs, bands = band_frames(c, 4)
    assert np.array_equal(full, bands_img), int((full != bands_img).sum())
    assert sum(segs) == full_segs


def test_gpu_band_mode_rejects_blur_layers_and_returns_to_frames(renderer):
    c = tk.generate(5, 5, width=256, height=192, paths=24)
    renderer.set_band(2, 5)
    with pytest.raises(tk.TileinkError):
        renderer.upload(c)
    renderer.set_band(0, 0)
    renderer.render_to_image(c)


def test_gpu_row_split_loss_and_gradients_sum_to_the_whole(renderer):
    sc = diff.blur_group_scene(5, width=256, height=192, paths=16)
    tg = diff.blur_group_scene(5, width=256, height=192, paths=16, jitter=3.0)
    _, target = renderer.diff_forward(tg, np.zeros((192, 256, 4), np.float32), return_image=True)
    loss = renderer.diff_forward(sc, target)
    dp, dc, ds = renderer.diff_backward()
    parts = []
    for rows in [(0, 70), (70, 150), (150, 192)]:
        part = sc.with_params()
        part.loss_rows = rows
        lr = renderer.diff_forward(part, target)
        parts.append((lr,) + renderer.diff_backward())
    sums = [sum(p[k] for p in parts) for k in range(4)]
    assert abs(sums[0] - loss) <= 1e-9 * abs(loss)
    for got, want in ((sums[1], dp), (sums[2], dc)):
        assert np.linalg.norm(got - want) <= 1e-5 * np.linalg.norm(want)
    assert abs(sums[3] - ds) <= 1e-5 * abs(ds)
    assert all(np.abs(p[1]).sum() > 0 for p in parts)
