"""Progressive blur (Filter::ProgressiveBlur) on CPU: the oracle's pyramid
plan against the reference's pyramid tests
(native/runtime/program/filter/progressive/tests.rs:3-79), its output against
the reference's quality bounds for shallow edges and integer translations
(progressive/quality_tests.rs:7-67), and the Canvas records of a progressive
blur group."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

import oracle
import tileink_b200 as tk
from tileink_b200 import _native as N


def plan(w, h, sigma, quality):
    lib = oracle.lib()
    out = np.zeros(7 * 80, np.float32)
    n = lib.or_progressive_levels(w, h, float(sigma), quality, out.ctypes.data, 80)
    return out[: 7 * min(n, 80)].reshape(-1, 7), n


@pytest.mark.parametrize("quality", [N.PROGRESSIVE_BALANCED, N.PROGRESSIVE_HIGH])
def test_pyramid_delays_downsampling_and_bounds_resources(quality):
    lv, n = plan(511, 257, 32.0, quality)
    w, h, scale, var, step, wsum = lv[:, 0], lv[:, 1], lv[:, 2], lv[:, 3], lv[:, 4], lv[:, 5]
    assert all(scale[k] == 1.0 for k in range(1, n) if var[k] < 8.0)
    assert var[-1] >= 1024.0 and var[-2] < 1024.0
    for k in range(1, n):
        assert var[k] > var[k - 1]
        assert w[k] == math.ceil(w[k - 1] / step[k]) and h[k] == math.ceil(h[k - 1] / step[k])
        assert abs(wsum[k] - 1.0) < 1e-5
    assert plan(1, 1, 65536.0, quality)[1] <= 64
    assert plan(1, 7, 1.0, quality)[1] == 1


def test_high_quality_has_more_levels():
    assert plan(511, 257, 32.0, N.PROGRESSIVE_HIGH)[1] > plan(511, 257, 32.0, N.PROGRESSIVE_BALANCED)[1]


@pytest.mark.parametrize("quality", [N.PROGRESSIVE_BALANCED, N.PROGRESSIVE_HIGH])
def test_source_halo_contains_every_kernel_sample(quality):
    """sample_outset = ceil(20 sigma + 8) covers the pyramid's support."""
    for exponent in range(-4, 65):
        sigma = min(2.0 ** (exponent / 4.0), 65536.0)
        lv, n = plan(511, 257, sigma, quality)
        support = 0.0
        for k in range(1, n):
            support += lv[k - 1, 2] * lv[k, 6]
        support = max(support + lv[-1, 2], 3.0)
        assert support <= math.ceil(20.0 * np.float32(sigma) + 8.0), (sigma, support)


def oracle_progressive(img, rect, start, end, sigma, quality):
    h, w = img.shape
    out = np.ascontiguousarray(img.copy())
    sx, sy, ex, ey = map(float, (*start, *end))
    dx, dy = ex - sx, ey - sy
    l2 = dx * dx + dy * dy
    blur = N.PROGRESSIVE_DTYPE.type(0) if False else np.zeros(1, N.PROGRESSIVE_DTYPE)
    blur[0] = (sx, sy, dx / l2 if l2 else 0.0, dy / l2 if l2 else 0.0, sigma, quality)
    r = (C.c_int32 * 4)(*rect)
    assert oracle.lib().or_progressive_blur(out.ctypes.data, w, h, r, blur.ctypes.data) == 0
    return out


@pytest.mark.parametrize("quality", [N.PROGRESSIVE_BALANCED, N.PROGRESSIVE_HIGH])
def test_shallow_edges_match_gaussian_and_stay_when_moving(quality):
    """The reference's acceptance bounds: a vertical edge under a blur growing
    from 0 (y = 8) to sigma 4 (y = 56) stays within 4/255 of the exact 1-D
    Gaussian of the edge, and moving the edge by whole pixels changes the
    profile by at most 3/255."""
    W, H = 97, 65
    worst, profiles = 0.0, []
    for edge in range(44, 52):
        v = np.where(np.arange(W) >= edge, 255, 0).astype(np.uint32)
        img = np.tile(v | (v << 8) | (v << 16) | (255 << 24), (H, 1)).astype(np.uint32)
        out = oracle_progressive(img, (0, 0, W, H), (0.0, 8.0), (0.0, 56.0), 4.0, quality)
        prof = []
        for y in range(12, 52):
            t = (y + 0.5 - 8.0) / 48.0
            s = 4.0 * t * t * (3.0 - 2.0 * t)
            rad = math.ceil(4.0 * s)
            for x in range(edge - 8, edge + 8):
                num = den = 0.0
                for dx in range(-rad, rad + 1):
                    wt = math.exp(-(dx * dx) / (2.0 * s * s))
                    num += 255.0 * wt if x + dx >= edge else 0.0
                    den += wt
                actual = float(out[y, x] & 255)
                worst = max(worst, abs(actual - num / den))
                prof.append(actual)
        profiles.append(np.array(prof))
    movement = max(float(np.abs(p - profiles[0]).max()) for p in profiles[1:])
    assert worst < 4.0 and movement <= 3.0, (worst, movement)


def test_before_start_unchanged_and_uniform_blur_is_smooth():
    rng = np.random.default_rng(3)
    img = (rng.integers(0, 256, (48, 64)).astype(np.uint32) * 0x01010101).astype(np.uint32)
    out = oracle_progressive(img, (0, 0, 64, 48), (0.0, 20.0), (0.0, 40.0), 6.0, N.PROGRESSIVE_BALANCED)
    assert np.array_equal(out[:20], img[:20])  # t = 0 above the start: sigma 0, pixels kept
    assert not np.array_equal(out[40:], img[40:])
    uni = oracle_progressive(img, (0, 0, 64, 48), (5.0, 5.0), (5.0, 5.0), 6.0, N.PROGRESSIVE_BALANCED)
    g = (uni[8:40, 8:56] & 255).astype(float)
    assert g.std() < (img[8:40, 8:56] & 255).astype(float).std() / 4


def test_canvas_records_progressive_blur_groups():
    c = tk.Canvas(128, 96)
    c.push_progressive_blur_group((10, 20), (30, 40), 8.0, N.PROGRESSIVE_HIGH)
    c.push_path(tk.BezPath().move_to(40, 30).line_to(80, 35).line_to(60, 70).close(), tk.Brush.solid(1, 0, 0, 1))
    c.pop_layer()
    a = c.scene_arrays()
    ops = a["ops"]
    assert list(ops["kind"]) == [N.OP_PROGRESSIVE_BEGIN, N.OP_DRAW_BATCH, N.OP_BLUR_END]
    p = a["progressive"][ops["batch_id"][0]]
    assert (p["start_x"], p["start_y"], p["max_std_dev"], p["quality"]) == (10.0, 20.0, 8.0, N.PROGRESSIVE_HIGH)
    assert p["dir_x"] == np.float32(20.0 / 800.0) and p["dir_y"] == np.float32(20.0 / 800.0)
    outset = math.ceil(20.0 * 8.0 + 8.0)
    assert list(ops["bounds"][0]) == [0, 0, 128, 96]  # the path's bounds outset by 168, clipped
    with pytest.raises(ValueError):
        c.push_progressive_blur_group((0, 0), (1, 1), float("nan"))
    with pytest.raises(ValueError):
        c.push_progressive_blur_group((0, 0), (1, 1), 70000.0)


def test_progressive_scene_renders_in_the_oracle():
    from layer_cases import progressive_scene
    c = progressive_scene(1)
    d = c.scene_desc()
    img = oracle.OracleRun(d, threads=4).get(oracle.OR_IMAGE, np.uint32)
    assert img.any()
