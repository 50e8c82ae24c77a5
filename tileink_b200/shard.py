"""Work partitions for one process per GPU (torch.distributed), after the
reference's own independence structure: tile rows are independent after the
scan (a backdrop is the row-wise cumsum of its row's deltas), and scenes are
independent. The reference itself renders on one device
(src/native/runtime/adapter.rs:159); these are the splits its path admits.

* band_partition: one scene's tile rows in contiguous bands, balanced by the
  backdrop tiles each row holds (the per-row share of the scan's pool and of
  coarse and fine's candidates). Each rank renders its band
  (NativeRenderer.set_band) and the bands are gathered (gather_bands).
* scene_partition: independent scenes over ranks, balanced by their line
  counts (longest first onto the least loaded rank).
* allreduce_sum: the exchange of a split objective's partial gradients.
"""
from __future__ import annotations

import numpy as np

from . import _native as N


def row_weights(paths: np.ndarray, tile_rows: int) -> np.ndarray:
    """Backdrop tiles per tile row: every path adds its bbox width to each of
    its bbox rows."""
    paths = np.asarray(paths, dtype=N.PATH_DTYPE)
    stride = (paths["tile_x1"].astype(np.int64) - paths["tile_x0"]).clip(min=0)
    y0 = np.minimum(paths["tile_y0"].astype(np.int64), tile_rows)
    y1 = np.minimum(paths["tile_y1"].astype(np.int64), tile_rows)
    ok = (y1 > y0) & (stride > 0)
    diff = np.zeros(tile_rows + 1, np.int64)
    np.add.at(diff, y0[ok], stride[ok])
    np.add.at(diff, y1[ok], -stride[ok])
    return np.cumsum(diff[:-1])


def band_partition(weights: np.ndarray, world: int) -> list[tuple[int, int]]:
    """Contiguous tile-row bands [y0, y1), one per rank, covering every row
    exactly once, with about equal total weight (a row of weight 0 still
    counts 1, so empty rows spread too). Every band holds at least one row
    when there are at least `world` rows."""
    rows = len(weights)
    if world < 1:
        raise ValueError("world must be >= 1")
    w = np.asarray(weights, dtype=np.float64) + 1.0
    c = np.concatenate([[0.0], np.cumsum(w)])
    cuts = [0]
    for k in range(1, world):
        y = int(np.searchsorted(c, c[-1] * k / world, side="left"))
        lo = cuts[-1] + (1 if rows >= world else 0)
        hi = rows - (world - k if rows >= world else 0)
        cuts.append(min(max(y, lo), max(hi, lo)))
    cuts.append(rows)
    return [(cuts[k], cuts[k + 1]) for k in range(world)]


def scene_partition(costs, world: int) -> list[list[int]]:
    """Scene indices per rank: longest first onto the least loaded rank;
    every scene on exactly one rank, each rank's list in scene order."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(costs[i])
    return [sorted(v) for v in out]


def pixel_rows(band: tuple[int, int], height: int) -> tuple[int, int]:
    """Pixel rows [r0, r1) of a tile-row band on a canvas `height` pixels tall."""
    return min(band[0] * 16, height), min(band[1] * 16, height)


def band_paths(paths: np.ndarray, tile_y0: int, tile_y1: int) -> np.ndarray:
    """The path records of one band as tk_set_band uploads them
    (tk_band_paths): bboxes clamped to the band's rows, backdrop slices
    repacked, segments left to the device plan."""
    paths = np.ascontiguousarray(paths, dtype=N.PATH_DTYPE)
    out = np.zeros_like(paths)
    N.library().tk_band_paths(N.ptr(paths), len(paths), int(tile_y0), int(tile_y1), N.ptr(out))
    return out


def gather_bands(local, pixel_bands, width: int, device="cpu"):
    """All-gather the ranks' band images (each (rows, width) uint32, its
    pixel rows) into the full image on every rank; bands are padded to the
    tallest for the collective. Returns a (H, W) uint32 numpy array."""
    import torch
    import torch.distributed as dist
    bands = pixel_bands
    heights = [(y1 - y0) for (y0, y1) in bands]
    tallest = max(heights)
    buf = torch.zeros((tallest, width), dtype=torch.int32, device=device)
    mine = torch.as_tensor(np.ascontiguousarray(local).view(np.int32))
    buf[:mine.shape[0]] = mine.to(device)
    parts = [torch.empty_like(buf) for _ in bands]
    dist.all_gather(parts, buf)
    rows = [p[:h].cpu().numpy().view(np.uint32) for p, h in zip(parts, heights)]
    return np.concatenate(rows, axis=0)


def allreduce_sum(arrays, device="cpu"):
    """Sum each numpy array over all ranks (one collective per array)."""
    import torch
    import torch.distributed as dist
    out = []
    for a in arrays:
        t = torch.as_tensor(np.ascontiguousarray(a)).to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        out.append(t.cpu().numpy())
    return out
