"""Shared test helpers: the reference's own test inputs restated."""
from __future__ import annotations

import math

import numpy as np

from tileink_b200 import _native as N

LCG_A, LCG_C = 1_664_525, 1_013_904_223
M32 = 0xFFFFFFFF


def lcg(x: int) -> int:
    return (x * LCG_A + LCG_C) & M32


def prefix_case(lengths, seed):
    """The reference's scan prefix acceptance case (src/native/runtime/tests/
    scan_cases.rs:8-157): LCG counts in chunks separated by 0x98765432 guard
    words, ranges starting at segment_start 19, wrapping u32 arithmetic.

    In this build a path's backdrop slice is scanned whole, so every chunk is
    one path (1 row, stride = len) whose segment_start is the running offset
    the reference carries across chunks; the guard words lie outside every
    slice. Returns inputs and the expected outputs of the reference harness."""
    counts = [0x98765432] * 7
    chunks = []
    rng = seed
    for ln in lengths:
        chunks.append((len(counts), ln))
        for _ in range(ln):
            rng = lcg(rng)
            counts.append(rng)
        counts.extend([0x98765432] * 3)
    ranges = [(0x55555555, 0x55555555)] * len(counts)
    cursors = [0x55555555] * len(counts)
    totals, offsets = [], []
    nxt = 19
    paths = np.zeros(len(chunks), dtype=N.PATH_DTYPE)
    for k, (off, ln) in enumerate(chunks):
        offsets.append(nxt)
        total = 0
        for i in range(off, off + ln):
            c = counts[i]
            start = (nxt + total) & M32
            total = (total + c) & M32
            ranges[i] = (start, (nxt + total) & M32)
            cursors[i] = start
        totals.append(total)
        paths[k]["path_id"] = k
        paths[k]["data_offset"] = off
        paths[k]["data_len"] = ln
        paths[k]["tile_x0"], paths[k]["tile_x1"] = 0, max(ln, 0)
        paths[k]["tile_y0"], paths[k]["tile_y1"] = 0, 1 if ln else 0
        paths[k]["segment_start"] = nxt
        nxt = (nxt + total) & M32
    r = np.zeros(len(counts), dtype=N.RANGE_DTYPE)
    r["start"] = [a for a, _ in ranges]
    r["end"] = [b for _, b in ranges]
    init_ranges = np.zeros(len(counts), dtype=N.RANGE_DTYPE)
    init_ranges["start"] = 0x55555555
    init_ranges["end"] = 0x55555555
    return {
        "counts": np.array(counts, dtype=np.uint32),
        "paths": paths,
        "init_ranges": init_ranges,
        "init_cursors": np.full(len(counts), 0x55555555, dtype=np.uint32),
        "ranges": r,
        "cursors": np.array(cursors, dtype=np.uint32),
        "totals": np.array(totals, dtype=np.uint32),
        "offsets": np.array(offsets, dtype=np.uint32),
    }


PREFIX_LENGTHS = [[0], [1], [255], [256], [256, 1], [256, 0, 17, 1, 255]]
PREFIX_SEEDS = [0, 19, M32]


def count_segments():
    """Single-line scan_count inputs (src/native/runtime/metal/scan_tests.rs:29-48)."""
    segs = [
        ([8.0, 0.0], [8.0, 48.0]),
        ([0.0, 8.0], [48.0, 8.0]),
        ([-8.0, 0.0], [-8.0, 48.0]),
        ([0.0, 0.0], [48.0, 48.0]),
        ([16.0, 16.0], [16.0, 16.0]),
        ([0.0, 16.0], [128.0, 16.0]),
        ([-16.0, -16.0], [144.0, 128.0]),
        ([0.0, 0.000_001], [128.0, 0.000_001]),
    ]
    seed = 127

    def point():
        nonlocal seed
        out = []
        for _ in range(2):
            seed = lcg(seed)
            out.append(np.float32(seed % 3073) / np.float32(16.0) - np.float32(32.0))
        return [float(v) for v in out]

    for _ in range(120):
        segs.append((point(), point()))
    return segs


def count_case_inputs(p0, p1):
    """count_case (scan_cases.rs:159-213): one line, an 8x8-tile path at
    data_offset 7, guard words 0x12345678 around the 64 tile words."""
    line = np.zeros(1, dtype=N.LINE_DTYPE)
    line[0]["path_id"] = 0
    line[0]["p0"] = p0
    line[0]["p1"] = p1
    path = np.zeros(1, dtype=N.PATH_DTYPE)
    path[0]["line_count"] = 1
    path[0]["data_offset"] = 7
    path[0]["data_len"] = 64
    path[0]["tile_x1"] = 8
    path[0]["tile_y1"] = 8
    path[0]["transform"] = (1.0, 0.0, 0.0, 1.0, 0.0, 0.0)
    init = np.array([0x12345678] * 7 + [0] * 64 + [0x12345678] * 7, dtype=np.uint32)
    return line, path, init


BLUR_SIZES = [(1, 1), (17, 15), (49, 35)]
BLUR_SIGMAS = [0.0, 0.01, 1.0 / 3.0, 0.5, 1.0, 3.25, 5.0, 16.0 / 3.0, 5.5]


def blur_source(width, height):
    """Source texture of tests/shared_blur_gpu.rs:31-43."""
    out = np.zeros((width * height, 4), dtype=np.uint8)
    for i in range(width * height):
        alpha = (i * 43) % 256
        mod = alpha + 1
        out[i] = ((i * 11) % mod, (i * 37) % mod, (i * 71) % mod, alpha)
    return out.view(np.uint32).reshape(-1)


def blur_config(width, height, inset):
    region = (width // 3 if inset else 0, height // 3 if inset else 0,
              width - (2 * (width // 3) if inset else 0), height - (2 * (height // 3) if inset else 0))
    source = (width // 5, height // 5, width, height)
    return region, source


def gaussian_f64(src_u32, width, height, source, x, y, sigma, axis):
    """Independent f64 Gaussian of tests/shared_blur_gpu.rs:125-155."""
    src = src_u32.view(np.uint8).reshape(-1, 4)
    if sigma <= 0.0:
        return src[y * width + x].copy()
    radius = max(math.ceil(np.float32(sigma) * np.float32(3.0)), 1)
    s = [0.0] * 4
    total = 0.0
    for d in range(-radius, radius + 1):
        w = math.exp(-(d * d) / (2.0 * sigma * sigma))
        total += w
        sx = x + (d if axis == 0 else 0)
        sy = y + (d if axis == 1 else 0)
        if sx < source[0] or sy < source[1] or sx >= source[2] or sy >= source[3]:
            continue
        for c in range(4):
            s[c] += w * float(src[sy * width + sx][c])
    return np.array([min(max(round(v / total), 0), 255) for v in s], dtype=np.uint8)


def circle_path(cx, cy, r):
    """Circle as four cubic quarter arcs (kappa = 4/3 (sqrt(2) - 1))."""
    from tileink_b200 import BezPath
    k = 4.0 / 3.0 * (math.sqrt(2.0) - 1.0) * r
    p = BezPath().move_to(cx + r, cy)
    p.cubic_to(cx + r, cy + k, cx + k, cy + r, cx, cy + r)
    p.cubic_to(cx - k, cy + r, cx - r, cy + k, cx - r, cy)
    p.cubic_to(cx - r, cy - k, cx - k, cy - r, cx, cy - r)
    p.cubic_to(cx + k, cy - r, cx + r, cy - k, cx + r, cy)
    return p.close()
