"""Multi-rank partitions of the path on CPU (gloo, world size 2, ranks as
spawned processes; the oracle renders each rank's share):

* the band split of one scene: tile-row bands cover every row once; each rank
  rasters its band scene (the path records tk_set_band uploads: bboxes
  clamped to the band, slices repacked, segments planned from the scanned
  totals) and the gathered bands equal the single-rank frame bit for bit;
* the scene split of a batch: every scene on exactly one rank, the gathered
  images equal the single-rank images;
* the split objective: the per-rank partial sums all-reduced equal the
  whole sum."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from tileink_b200 import shard  # noqa: E402


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("rows, world", [(256, 2), (256, 8), (23, 4), (3, 4), (1, 1), (68, 3)])
def test_band_partition_covers_rows_once(rows, world):
    rng = np.random.default_rng(rows + world)
    w = rng.integers(0, 1000, rows) * (rng.uniform(size=rows) < 0.7)
    bands = shard.band_partition(w, world)
    assert len(bands) == world
    assert bands[0][0] == 0 and bands[-1][1] == rows
    for (a0, a1), (b0, b1) in zip(bands, bands[1:]):
        assert a1 == b0 and a0 <= a1
    if rows >= world:
        assert all(y1 > y0 for y0, y1 in bands)
    # balance: no band heavier than its share plus the heaviest row
    tot = (w + 1).sum()
    heaviest = (w + 1).max()
    for y0, y1 in bands:
        assert (w[y0:y1] + 1).sum() <= tot / world + heaviest + 1e-9


def test_row_weights_are_backdrop_tiles_per_row():
    import tileink_b200 as tk
    c = tk.generate(2, 7, width=512, height=256, paths=200)
    paths = c.scene_arrays()["paths"]
    w = shard.row_weights(paths, 16)
    assert w.sum() == paths["data_len"].astype(np.int64).sum()


def test_band_paths_clamp_and_repack():
    import tileink_b200 as tk
    c = tk.generate(2, 3, width=640, height=400, paths=300)
    p = c.scene_arrays()["paths"]
    b = shard.band_paths(p, 7, 13)
    assert np.all((b["tile_y0"] >= 7) & (b["tile_y1"] <= 13) & (b["tile_y0"] <= b["tile_y1"]))
    assert np.array_equal(b["data_len"], (b["tile_x1"] - b["tile_x0"]) * (b["tile_y1"] - b["tile_y0"]))
    assert np.array_equal(b["data_offset"], np.concatenate([[0], np.cumsum(b["data_len"])[:-1]]))
    assert not b["segment_start"].any() and not b["segment_capacity"].any()
    assert np.array_equal(b["line_start"], p["line_start"]) and np.array_equal(b["line_count"], p["line_count"])


def test_scene_partition_covers_scenes_once():
    rng = np.random.default_rng(5)
    costs = rng.integers(10, 100000, 37)
    parts = shard.scene_partition(costs, 4)
    assert sorted(i for p in parts for i in p) == list(range(37))
    loads = [costs[p].sum() for p in parts]
    assert max(loads) - min(loads) <= costs.max()


def _band_worker(rank, world, port, results, spec):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        import oracle
        import tileink_b200 as tk
        from tileink_b200 import _native as N
        from tileink_b200 import shard as S
        config, seed, kw = spec
        c = tk.generate(config, seed, **kw)
        a = c.scene_arrays()
        d = c.scene_desc()
        th = (d.height + 15) // 16
        bands = S.band_partition(S.row_weights(a["paths"], th), world)
        y0, y1 = bands[rank]
        # this rank's scene: the band's path records, segments planned from
        # the scanned totals
        a["paths"] = S.band_paths(a["paths"], y0, y1)
        scene = N.ArrayScene(a)
        scene.desc.flags |= N.SCENE_SEGMENTS_FROM_DEVICE
        run = oracle.OracleRun(scene.desc, threads=4, tile_rows=(y0, y1))
        img = run.get(oracle.OR_IMAGE, np.uint32).reshape(d.height, d.width)
        r0, r1 = S.pixel_rows((y0, y1), d.height)
        full = S.gather_bands(img[r0:r1], [S.pixel_rows(b, d.height) for b in bands], d.width)
        results[rank] = (bands, full.tobytes())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("spec", [
    (2, 7, dict(width=768, height=512, paths=600)),   # fills, strokes, gradients, clip layers
    (1, 1, dict()),                                   # 640x360 cubic fills
    (3, 3, dict(width=480, height=270, paths=800)),   # glyphs
])
def test_band_split_gathers_the_single_rank_frame(spec):
    import oracle
    import tileink_b200 as tk
    config, seed, kw = spec
    canvas = tk.generate(config, seed, **kw)  # owns the records the descriptor points at
    d = canvas.scene_desc()
    want = oracle.OracleRun(d, threads=8).get(oracle.OR_IMAGE, np.uint32).reshape(d.height, d.width)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        results = m.dict()
        mp.start_processes(_band_worker, args=(2, free_port(), results, spec), nprocs=2, join=True,
                           start_method="spawn")
        bands0, img0 = results[0]
        bands1, img1 = results[1]
    assert bands0 == bands1 and bands0[0][1] == bands0[1][0]
    assert img0 == img1
    got = np.frombuffer(img0, np.uint32).reshape(d.height, d.width)
    assert np.array_equal(got, want), int((got != want).sum())


def _scene_worker(rank, world, port, results, n):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        import oracle
        import tileink_b200 as tk
        from tileink_b200 import shard as S
        scenes = [tk.generate(4, 1000 + i) for i in range(n)]
        costs = [int(s.scene_desc().line_count) for s in scenes]
        parts = S.scene_partition(costs, world)
        mine = {}
        for i in parts[rank]:
            mine[i] = oracle.OracleRun(scenes[i].scene_desc(), threads=2).get(oracle.OR_IMAGE, np.uint32).tobytes()
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        merged = {}
        for g in gathered:
            merged.update(g)
        results[rank] = (parts, merged)
    finally:
        dist.destroy_process_group()


def test_scene_split_gathers_every_scene_once():
    import oracle
    import tileink_b200 as tk
    n = 10
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        results = m.dict()
        mp.start_processes(_scene_worker, args=(2, free_port(), results, n), nprocs=2, join=True,
                           start_method="spawn")
        parts, merged = results[0]
    assert sorted(parts[0] + parts[1]) == list(range(n)) and not set(parts[0]) & set(parts[1])
    for i in range(n):
        canvas = tk.generate(4, 1000 + i)
        d = canvas.scene_desc()
        assert merged[i] == oracle.OracleRun(d, threads=2).get(oracle.OR_IMAGE, np.uint32).tobytes()


def _sum_worker(rank, world, port, results):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from tileink_b200 import shard as S
        rng = np.random.default_rng(rank)
        parts = [rng.normal(size=(40, 2)).astype(np.float32), rng.normal(size=7).astype(np.float64)]
        results[rank] = [p.tobytes() for p in parts] + [x.tobytes() for x in S.allreduce_sum(parts)]
    finally:
        dist.destroy_process_group()


def test_allreduce_sum_of_partial_gradients():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        results = m.dict()
        mp.start_processes(_sum_worker, args=(2, free_port(), results), nprocs=2, join=True, start_method="spawn")
        r0, r1 = results[0], results[1]
    a = np.frombuffer(r0[0], np.float32) + np.frombuffer(r1[0], np.float32)
    b = np.frombuffer(r0[1], np.float64) + np.frombuffer(r1[1], np.float64)
    for r in (r0, r1):
        assert np.array_equal(np.frombuffer(r[2], np.float32), a)
        assert np.array_equal(np.frombuffer(r[3], np.float64), b)
