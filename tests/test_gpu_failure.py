"""Failure detection without a GPU fault: the tile prefix's look-back wait is
bounded, and when it runs out the call reports TK_E_TIMEOUT and the context
stays usable. The wait is made to run out by a predecessor that never
publishes (the block tickets start at 1, so nothing publishes block 0); every
wait in the kernel still ends after `poll_limit` polls.

The reference latches a failed submission on its context
(src/native/runtime/adapter.rs:8-15); here the failure is an error status
that the host reads, and the next call on the same context works."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import tileink_b200 as tk
from tileink_b200 import _native as N
from tileink_b200.renderer import TileinkError

pytestmark = pytest.mark.gpu

TK_E_TIMEOUT = -4


def tiles_with_counts(n, seed):
    rng = np.random.default_rng(seed)
    t = np.zeros(n, dtype=N.TILE_DTYPE)
    t["ptcl_count"] = rng.integers(0, 40, n)
    t["ptcl_start"] = 0xDEADBEEF
    t["glyph_count"] = 7
    return t


@pytest.mark.parametrize("n", [0, 1, 4095, 4096, 4097, 70001])
def test_gpu_tile_prefix_harness_matches_exclusive_scan(renderer, n):
    """coarse/prefix.hlsl:11-63: ptcl_start is the exclusive prefix of
    ptcl_count, ptcl_end = start + count; this is the PTCL component of the
    scan, so glyph_count stays as given and the glyph range is cleared (text
    scenes run the glyph component after it)."""
    t = tiles_with_counts(n, n)
    got, total = renderer.stage_tile_prefix(t)
    excl = np.concatenate([[0], np.cumsum(t["ptcl_count"].astype(np.uint64))[:-1]]) if n else np.zeros(0)
    assert np.array_equal(got["ptcl_count"], t["ptcl_count"])
    assert np.array_equal(got["ptcl_start"], excl.astype(np.uint32))
    assert np.array_equal(got["ptcl_end"], (excl + t["ptcl_count"]).astype(np.uint32))
    assert np.array_equal(got["glyph_count"], t["glyph_count"])
    assert not got["glyph_start"].any() and not got["glyph_end"].any()
    assert total == int(t["ptcl_count"].astype(np.uint64).sum())


def test_gpu_lookback_wait_gives_up_and_context_stays_usable(renderer):
    t = tiles_with_counts(70001, 3)  # 18 blocks of 4096 tiles
    with pytest.raises(TileinkError) as e:
        renderer.stage_tile_prefix(t, poll_limit=4096, withhold_first=True)
    assert e.value.code == TK_E_TIMEOUT
    assert "look-back wait gave up after 4096 polls" in str(e.value)
    # the same context: the same harness without the withheld block, then a
    # full frame, both exact
    got, total = renderer.stage_tile_prefix(t)
    assert total == int(t["ptcl_count"].astype(np.uint64).sum())
    c = tk.generate(1, 1)
    img = renderer.render_to_image(c)
    ref = oracle.OracleRun(c.scene_desc(), threads=4)
    want = ref.get(oracle.OR_IMAGE, np.uint32).view(np.uint8).reshape(img.shape)
    assert np.array_equal(img, want)
    assert np.array_equal(renderer.debug(N.STAGE_PTCL, 0), ref.get(oracle.OR_PASS_PTCL, N.PTCL_DTYPE, 0))
