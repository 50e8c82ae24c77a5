"""Batched mode: independent scenes of uneven size rendered together by one
CUDA graph launch, against the same scenes rendered one by one. Every
scene's PTCL must be bit-identical to its serial PTCL once the batch offsets
(tk_batch_info) are taken off, and every image identical."""
from __future__ import annotations

import numpy as np
import pytest

import tileink_b200 as tk
from tileink_b200 import _native as N

pytestmark = pytest.mark.gpu

FILL_LIKE = (N.PTCL_FILL, N.PTCL_BEGIN_CLIP)


def uneven_scenes(n, seed):
    """Scenes like the batched workload (log-uniform sizes and path counts,
    solid fills) plus a few mixed scenes with strokes, gradients and clips."""
    scenes = [tk.generate(4, seed + i) for i in range(n)]
    scenes += [tk.generate(2, seed + 100 + i, width=160 + 48 * i, height=96 + 40 * i, paths=60 + 30 * i)
               for i in range(3)]
    return scenes


def serial_outputs(renderer, canvas):
    img = renderer.render_to_image(canvas)
    return img, renderer.debug(N.STAGE_TILES, 0), renderer.debug(N.STAGE_PTCL, 0)


def unoffset(records, info):
    r = records.copy()
    fill_like = np.isin(r["tag"], FILL_LIKE)
    r["segment_start"][fill_like] -= np.uint32(info.segment_base)
    r["segment_end"][fill_like] -= np.uint32(info.segment_base)
    fill = r["tag"] == N.PTCL_FILL
    r["color"][fill] -= np.uint32(info.draw_base)
    sdf = r["tag"] == N.PTCL_SDF  # SDF records name their draw in segment_start and color
    r["segment_start"][sdf] -= np.uint32(info.draw_base)
    r["color"][sdf] -= np.uint32(info.draw_base)
    bb = r["tag"] == N.PTCL_BATCH_BEGIN
    r["segment_start"][bb] -= np.uint32(info.batch_base)
    return r


def check_batch_against_serial(renderer, scenes, serial):
    imgs = renderer.batch_readback()
    tiles = renderer.debug(N.STAGE_TILES, 0)
    ptcl = renderer.debug(N.STAGE_PTCL, 0)
    for k, (img_s, tiles_s, ptcl_s) in enumerate(serial):
        info = renderer.batch_info(k)
        assert np.array_equal(imgs[k], img_s), k
        bt = tiles[info.tile_base:info.tile_base + info.tile_count]
        assert len(bt) == len(tiles_s)
        assert np.array_equal(bt["ptcl_count"], tiles_s["ptcl_count"]), k
        # each tile's stream, offsets removed, equals the serial stream
        starts = bt["ptcl_start"].astype(np.int64)
        ends = bt["ptcl_end"].astype(np.int64)
        if len(bt):
            lo, hi = starts.min(), ends.max()
            got = unoffset(ptcl[lo:hi], info)
            assert np.array_equal(starts - lo, tiles_s["ptcl_start"].astype(np.int64) - tiles_s["ptcl_start"].min())
            assert got.tobytes() == ptcl_s[tiles_s["ptcl_start"].min():tiles_s["ptcl_end"].max()].tobytes(), k


def test_gpu_batch_matches_serial_scenes(renderer):
    scenes = uneven_scenes(12, 40)
    serial = [serial_outputs(renderer, c) for c in scenes]
    r = tk.NativeRenderer(0)
    try:
        r.batch_upload(scenes)
        r.batch_render()
        check_batch_against_serial(r, scenes, serial)
        # graph replays give the same frame
        first = [im.copy() for im in r.batch_readback()]
        r.batch_render()
        r.batch_render()
        assert all(np.array_equal(a, b) for a, b in zip(first, r.batch_readback()))
    finally:
        r.close()


def test_gpu_autotune_keeps_output_identical(renderer):
    scenes = uneven_scenes(6, 77)
    serial = [serial_outputs(renderer, c) for c in scenes]
    r = tk.NativeRenderer(0)
    try:
        r.batch_upload(scenes)
        res = r.autotune(2)
        assert res.candidates == 4 and res.scan_item_elems in (512, 1024, 2048, 4096)
        assert res.tile_width == 16 and res.tile_height == 16
        assert all(res.candidate_ms[i] > 0 for i in range(4))
        r.batch_render()
        check_batch_against_serial(r, scenes, serial)
    finally:
        r.close()


def test_gpu_autotune_single_scene_keeps_output_identical(renderer):
    canvas = tk.generate(2, 5, width=320, height=240, paths=200)
    img0 = renderer.render_to_image(canvas)
    ptcl0 = renderer.debug(N.STAGE_PTCL, 0)
    res = renderer.autotune(2)
    assert res.scan_item_elems in (512, 1024, 2048, 4096)
    renderer.render()
    assert np.array_equal(renderer.readback().view(np.uint8).reshape(img0.shape), img0)
    assert renderer.debug(N.STAGE_PTCL, 0).tobytes() == ptcl0.tobytes()


def test_gpu_batch_rejects_blur_groups():
    r = tk.NativeRenderer(0)
    try:
        with pytest.raises(tk.TileinkError):
            r.batch_upload([tk.generate(4, 1), tk.generate(5, 1, width=64, height=64, paths=4)])
    finally:
        r.close()
