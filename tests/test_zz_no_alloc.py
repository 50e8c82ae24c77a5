"""The allocation-free pool scan (tk_pool_scan_noalloc) against the allocating
stage harness (tk_stage_scan_prefix) on the same inputs, several calls in a
row on one device, with caller-owned device buffers.

Collected last on purpose: it must also pass after every other GPU test has
used the same context and device."""
from __future__ import annotations

import numpy as np
import pytest

from tileink_b200 import _native as N
from tileink_b200.renderer import TileinkError

from helpers import prefix_case

pytestmark = pytest.mark.gpu

NO_ALLOC_TOLERANCE = 0  # integer outputs: bit-exact


def long_paths_case(seed):
    """Paths whose bboxes span several scan work items (wide, tall and one
    4096-tile row stride), with random backdrop deltas."""
    rng = np.random.default_rng(seed)
    dims = [(37, 400), (1, 9000), (4096, 3), (5, 0), (300, 61)]
    paths = np.zeros(len(dims), dtype=N.PATH_DTYPE)
    off = 5
    for k, (w, h) in enumerate(dims):
        paths[k]["path_id"] = k
        paths[k]["data_offset"] = off
        paths[k]["data_len"] = w * h
        paths[k]["tile_x1"], paths[k]["tile_y1"] = w, h
        paths[k]["segment_start"] = 1000 * k + 7
        off += w * h + 11
    counts = rng.integers(0, 5, off).astype(np.uint32)
    backdrops = rng.integers(-3, 4, off).astype(np.int32)
    return counts, paths, backdrops


def guard_case():
    case = prefix_case([256, 0, 17, 1, 255], 19)
    rng = np.random.default_rng(11)
    backdrops = rng.integers(-2, 3, len(case["counts"])).astype(np.int32)
    return case["counts"], case["paths"], backdrops


def rowwise_cumsum(backdrops, paths):
    out = backdrops.copy()
    for p in paths:
        w = int(p["tile_x1"]) - int(p["tile_x0"])
        n = int(p["data_len"])
        if n == 0:
            continue
        o = int(p["data_offset"])
        out[o:o + n] = np.cumsum(out[o:o + n].reshape(-1, w), axis=1, dtype=np.int64).astype(np.int32).ravel()
    return out


def run_noalloc(renderer, counts, paths, backdrops, init_ranges, init_cursors):
    import torch
    dev = torch.device("cuda", 0)
    d_counts = torch.from_numpy(counts.view(np.int32).copy()).to(dev)
    d_bd = torch.from_numpy(backdrops.copy()).to(dev)
    d_ranges = torch.from_numpy(init_ranges.view(np.int32).copy()).to(dev)
    d_cursors = torch.from_numpy(init_cursors.view(np.int32).copy()).to(dev)
    d_bumps = torch.full((max(len(paths), 1),), 0x1234, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()  # the library's stream does not wait for torch's
    renderer.pool_scan_noalloc(paths, d_counts.data_ptr(), d_bd.data_ptr(), d_ranges.data_ptr(),
                               d_cursors.data_ptr(), len(counts), d_bumps.data_ptr())
    ranges = d_ranges.cpu().numpy().view(N.RANGE_DTYPE).reshape(-1)
    cursors = d_cursors.cpu().numpy().view(np.uint32)
    bumps = d_bumps.cpu().numpy().view(np.uint32)[:len(paths)]
    return ranges, cursors, bumps, d_bd.cpu().numpy()


def check_against_stage_harness(renderer, counts, paths, backdrops):
    init_r = np.zeros(len(counts), dtype=N.RANGE_DTYPE)
    init_r["start"] = 0x55555555
    init_r["end"] = 0xAAAAAAAA
    init_c = np.full(len(counts), 0x55555555, dtype=np.uint32)
    er, ec, eb = renderer.stage_scan_prefix(counts, paths, init_r, init_c)
    ranges, cursors, bumps, bd = run_noalloc(renderer, counts, paths, backdrops, init_r, init_c)
    assert np.abs(ranges["start"].astype(np.int64) - er["start"]).max() <= NO_ALLOC_TOLERANCE
    assert np.abs(ranges["end"].astype(np.int64) - er["end"]).max() <= NO_ALLOC_TOLERANCE
    assert np.abs(cursors.astype(np.int64) - ec).max() <= NO_ALLOC_TOLERANCE
    assert np.abs(bumps.astype(np.int64) - eb).max() <= NO_ALLOC_TOLERANCE
    assert np.array_equal(bd, rowwise_cumsum(backdrops, paths))


def test_noalloc_pool_scan_matches_stage_harness_on_consecutive_calls(renderer):
    big = long_paths_case(5)
    small = guard_case()
    # large, then smaller (the first call's per-item sums and prefixes stay
    # beyond the second call's items), then the large case again
    for counts, paths, backdrops in (big, small, big, long_paths_case(6)):
        check_against_stage_harness(renderer, counts, paths, backdrops)


def test_noalloc_pool_scan_rejects_sizes_over_its_limits(renderer):
    import torch
    paths = np.zeros(16385, dtype=N.PATH_DTYPE)  # all empty: no pool needed
    d_bumps = torch.zeros(16385, dtype=torch.int32, device="cuda:0")
    torch.cuda.synchronize()
    with pytest.raises(TileinkError) as e:
        renderer.pool_scan_noalloc(paths, 0, 0, 0, 0, 0, d_bumps.data_ptr())
    assert "allocation-free limit" in str(e.value)
    assert int(d_bumps.abs().sum().item()) == 0  # nothing launched
    # the context stays usable after the rejection
    counts, p, bd = guard_case()
    check_against_stage_harness(renderer, counts, p, bd)
