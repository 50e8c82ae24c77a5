"""Parity at the full sizes of the measured workloads.

* The full 1920x1080 glyph frame (20,000 glyphs) and the full 1024x1024
  blur-group frame (256 paths, sigma 4): every stage bit-exact against the
  oracle, as in test_gpu_parity.
* The benchmarked 4096x4096, 50,000-path frame (seed 2, device segment plan,
  as bench.py renders it): the whole scan (counts, backdrops, ranges and all
  335 M segments, compared in chunks) and the device's segment plan against
  the oracle's per-path totals, then three tile-row bands of 16 rows (top,
  middle, bottom) through coarse and fine: tile records, PTCL and pixels of
  those rows bit-exact. The oracle scans once and rasters each band
  (OracleRun.prepare / raster); the GPU renders the full frame once.

Stage buffers are compared in the reference's guard-word spirit
(src/native/runtime/tests/scan_cases.rs:8-157): every element, including
the ones that must stay untouched, is compared."""
from __future__ import annotations

import os

import numpy as np
import pytest

import oracle
import tileink_b200 as tk
from tileink_b200 import _native as N

from test_gpu_parity import compare_frame

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 8
CHUNK = 1 << 24  # elements per compared slice of the large buffers
BANDS = [(0, 16), (120, 136), (240, 256)]


def test_gpu_full_glyph_frame(renderer):
    """1920x1080, 20,000 glyphs of 2-4 quadratic contours (seed 3)."""
    img, ref = compare_frame(renderer, tk.generate(3, 3), threads=THREADS)
    assert img.shape == (1080, 1920, 4)


def test_gpu_full_blur_group_frame(renderer):
    """1024x1024, 256 closed paths x 12 cubics, blur group sigma 4 (seed 5)."""
    img, ref = compare_frame(renderer, tk.generate(5, 5), threads=THREADS)
    assert img.shape == (1024, 1024, 4)


def compare_chunked(renderer, ref, stage, what, dtype):
    n = renderer.debug_size(stage)
    assert n == ref.size(what), (stage, n, ref.size(what))
    for first in range(0, n, CHUNK):
        got = renderer.debug_range(stage, first, CHUNK)
        want = ref.get_range(what, dtype, first, CHUNK)
        assert got.tobytes() == want.tobytes(), (stage, first)
    return n


@pytest.fixture(scope="module")
def c2_frame():
    """The benchmarked frame on the GPU and its oracle scan."""
    r = tk.NativeRenderer(0)
    c = tk.generate(2, 2, device_segment_plan=True)
    r.upload(c)
    r.render()
    img = r.readback().copy()
    gpu_paths = r.debug(N.STAGE_PATHS)
    # the oracle scans the same records, placed by the device's segment plan
    a = c.scene_arrays()
    a["paths"] = gpu_paths.copy()
    scene = N.ArrayScene(a)
    ref = oracle.OracleRun.prepare(scene.desc, threads=THREADS)
    yield r, c, scene, ref, img, gpu_paths
    del ref
    r.close()


def test_gpu_full_c2_scan_and_device_segment_plan(c2_frame):
    r, c, scene, ref, img, gpu_paths = c2_frame
    stats = r.stats()
    assert stats["lines"] > 190_000_000 and stats["segments"] > 300_000_000
    # device plan = the host planner's plan: capacity = the path's scanned
    # segment total, starts = their exclusive prefix
    bumps = ref.get(oracle.OR_BUMPS, np.uint32)
    assert np.array_equal(gpu_paths["segment_capacity"], bumps)
    starts = np.concatenate([[0], np.cumsum(bumps.astype(np.uint64))[:-1]])
    assert np.array_equal(gpu_paths["segment_start"].astype(np.uint64), starts)
    assert int(starts[-1]) + int(bumps[-1]) > 1 << 28  # offsets past 2^28 are exercised
    compare_chunked(r, ref, N.STAGE_COUNTS, oracle.OR_COUNTS, np.uint32)
    compare_chunked(r, ref, N.STAGE_BACKDROPS, oracle.OR_BACKDROPS, np.int32)
    compare_chunked(r, ref, N.STAGE_RANGES, oracle.OR_RANGES, N.RANGE_DTYPE)
    s = compare_chunked(r, ref, N.STAGE_SEGMENTS, oracle.OR_SEGMENTS, N.SEGMENT_DTYPE)
    assert s == stats["segments"]


@pytest.mark.parametrize("band", BANDS)
def test_gpu_full_c2_tile_row_band(c2_frame, band):
    r, c, scene, ref, img, gpu_paths = c2_frame
    y0, y1 = band
    ref.raster(y0, y1, threads=THREADS)
    assert ref.pass_count == 1
    tw = (r.width + 15) // 16
    tiles = r.debug(N.STAGE_TILES, 0)
    rtiles = ref.get(oracle.OR_PASS_TILES, N.TILE_DTYPE, 0)
    band_tiles = slice(y0 * tw, y1 * tw)
    assert np.array_equal(tiles["ptcl_count"][band_tiles], rtiles["ptcl_count"][band_tiles])
    assert not rtiles["ptcl_count"][:y0 * tw].any() and not rtiles["ptcl_count"][y1 * tw:].any()
    # the band's PTCL records are contiguous on the device (row-major tiles)
    first, last = int(tiles["ptcl_start"][y0 * tw]), int(tiles["ptcl_end"][y1 * tw - 1])
    assert first > 0 or y0 == 0
    got = r.debug_range(N.STAGE_PTCL, first, last - first)
    want = ref.get(oracle.OR_PASS_PTCL, N.PTCL_DTYPE, 0)
    assert len(got) == len(want) > 0
    assert got.tobytes() == want.tobytes()
    # pixels of the band's rows
    h, w = r.height, r.width
    rows = slice(y0 * 16, min(y1 * 16, h))
    rimg = ref.get(oracle.OR_IMAGE, np.uint32).reshape(h, w)
    assert np.array_equal(img.reshape(h, w)[rows], rimg[rows])
