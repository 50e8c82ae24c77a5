"""Stroking with round joins and caps (kurbo::stroke's contract,
src/canvas/primitives/paths.rs:24-48): the outline's nonzero fill covers
exactly the points within half the width of the flattened centerline, up to
the tolerance. The outline lines come from the shared host/device stroker, so
this pins the geometry the GPU stroker reproduces bit for bit (the GPU
comparison is in test_gpu_flatten.py)."""
from __future__ import annotations

import numpy as np
import pytest

import tileink_b200 as tk
from tileink_b200 import _native as N


def winding(lines, px, py):
    """Nonzero winding number of the line set at each sample point."""
    w = np.zeros(px.shape, np.int32)
    for ln in lines:
        x0, y0 = float(ln["p0"][0]), float(ln["p0"][1])
        x1, y1 = float(ln["p1"][0]), float(ln["p1"][1])
        up = (y0 <= py) & (y1 > py)
        dn = (y1 <= py) & (y0 > py)
        t = (py - y0) / (y1 - y0 if y1 != y0 else 1.0)
        right = x0 + t * (x1 - x0) > px
        w += (up & right).astype(np.int32) - (dn & right).astype(np.int32)
    return w


def polyline_distance(px, py, pts, closed):
    pts = list(pts) + ([pts[0]] if closed and len(pts) > 1 else [])
    if len(pts) == 1:
        return np.hypot(px - pts[0][0], py - pts[0][1])
    d = np.full(px.shape, np.inf)
    for (ax, ay), (bx, by) in zip(pts[:-1], pts[1:]):
        dx, dy = bx - ax, by - ay
        l2 = dx * dx + dy * dy
        if l2 == 0.0:
            continue
        t = np.clip(((px - ax) * dx + (py - ay) * dy) / l2, 0.0, 1.0)
        d = np.minimum(d, np.hypot(px - (ax + t * dx), py - (ay + t * dy)))
    return d


def bezier(ctrl, n=2000):
    t = np.linspace(0.0, 1.0, n + 1)[:, None]
    c = np.asarray(ctrl, float)
    if len(c) == 3:
        return (1 - t) ** 2 * c[0] + 2 * (1 - t) * t * c[1] + t * t * c[2]
    return (1 - t) ** 3 * c[0] + 3 * (1 - t) ** 2 * t * c[1] + 3 * (1 - t) * t * t * c[2] + t ** 3 * c[3]


def stroke_lines(build, width, tol, transform=None, size=200):
    c = tk.Canvas(size, size)
    p = tk.BezPath()
    build(p)
    c.push_stroke(p, tk.Brush.solid(0, 0, 0, 1), width, transform=transform, tolerance=tol)
    return c.scene_arrays()


def assert_band(lines, subpaths, half, tol, size=200, step=0.43):
    """Covered where the distance to a centerline is below half - tol, not
    covered above half + tol (the band between is the flattening error)."""
    ys, xs = np.mgrid[0:size:step, 0:size:step]
    w = winding(lines, xs, ys)
    d = np.full(xs.shape, np.inf)
    for pts, closed in subpaths:
        d = np.minimum(d, polyline_distance(xs, ys, pts, closed))
    assert np.count_nonzero((w == 0) & (d < half - tol - 1e-3)) == 0
    assert np.count_nonzero((w != 0) & (d > half + tol + 1e-3)) == 0
    assert np.count_nonzero(w != 0) > 0


CASES = {
    "polyline": (lambda p: (p.move_to(20, 30), p.line_to(150, 60), p.line_to(60, 170), p.line_to(180, 180)),
                 [([(20, 30), (150, 60), (60, 170), (180, 180)], False)], 16.0),
    "closed_square": (lambda p: (p.move_to(40, 40), p.line_to(160, 40), p.line_to(160, 160), p.line_to(40, 160),
                                 p.close()),
                      [([(40, 40), (160, 40), (160, 160), (40, 160)], True)], 20.0),
    "closed_triangle_reversed": (lambda p: (p.move_to(100, 20), p.line_to(30, 170), p.line_to(175, 150), p.close()),
                                 [([(100, 20), (30, 170), (175, 150)], True)], 9.0),
    "dot": (lambda p: (p.move_to(100, 100), p.line_to(100, 100)), [([(100, 100)], False)], 30.0),
    "single_segment": (lambda p: (p.move_to(30, 100), p.line_to(170, 100)), [([(30, 100), (170, 100)], False)], 41.0),
    "hairpin": (lambda p: (p.move_to(20, 100), p.line_to(180, 100), p.line_to(20, 101)),
                [([(20, 100), (180, 100), (20, 101)], False)], 6.0),
    "two_subpaths": (lambda p: (p.move_to(20, 20), p.line_to(80, 60), p.move_to(120, 150), p.line_to(180, 40)),
                     [([(20, 20), (80, 60)], False), ([(120, 150), (180, 40)], False)], 10.0),
    "close_then_continue": (lambda p: (p.move_to(50, 50), p.line_to(150, 50), p.line_to(100, 120), p.close(),
                                       p.line_to(60, 180)),
                            [([(50, 50), (150, 50), (100, 120)], True), ([(50, 50), (60, 180)], False)], 8.0),
    "curves": (lambda p: (p.move_to(20, 180), p.cubic_to(20, 0, 180, 200, 180, 20), p.quad_to(100, 100, 40, 60)),
               [(list(map(tuple, np.vstack([bezier([(20, 180), (20, 0), (180, 200), (180, 20)]),
                                            bezier([(180, 20), (100, 100), (40, 60)])]))), False)], 12.0),
    "cusp": (lambda p: (p.move_to(30, 150), p.cubic_to(170, 20, 30, 20, 170, 150)),
             [(list(map(tuple, bezier([(30, 150), (170, 20), (30, 20), (170, 150)]))), False)], 7.0),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_stroke_outline_covers_the_distance_band(name):
    build, subpaths, width = CASES[name]
    tol = 0.05
    a = stroke_lines(build, width, tol)
    assert len(a["lines"]) > 0 and np.all(a["lines"]["path_id"] == 0)
    assert_band(a["lines"], subpaths, width / 2, tol)


def test_stroke_is_outlined_in_local_space_then_transformed():
    # a rotation by 30 degrees and scale 1.5 about (100, 100): round caps and
    # joins stay round, the width scales with the transform
    ang, s = np.deg2rad(30.0), 1.5
    ca, sa = s * np.cos(ang), s * np.sin(ang)
    t = (ca, sa, -sa, ca, 100 - (ca * 50 - sa * 50), 100 - (sa * 50 + ca * 50))
    local = [(10.0, 20.0), (90.0, 30.0), (50.0, 95.0)]
    a = stroke_lines(lambda p: (p.move_to(*local[0]), p.line_to(*local[1]), p.line_to(*local[2])), 8.0, 0.05,
                     transform=t)
    dev = [(t[0] * x + t[2] * y + t[4], t[1] * x + t[3] * y + t[5]) for x, y in local]
    assert_band(a["lines"], [(dev, False)], 8.0 * s / 2, 0.05 * s)
    # the stroke's bounds hold every outline line
    d = a["draws"][0]["pixel_bounds"]
    ln = a["lines"]
    xs = np.concatenate([ln["p0"][:, 0], ln["p1"][:, 0]])
    ys = np.concatenate([ln["p0"][:, 1], ln["p1"][:, 1]])
    assert d["x0"] <= xs.min() and xs.max() <= d["x1"] and d["y0"] <= ys.min() and ys.max() <= d["y1"]


def test_stroke_degenerate_inputs():
    # a lone move_to strokes nothing; a repeated point is one point (a dot)
    a = stroke_lines(lambda p: p.move_to(50, 50), 10.0, 0.1)
    assert len(a["lines"]) == 0
    b = stroke_lines(lambda p: (p.move_to(50, 50), p.line_to(50, 50), p.line_to(50, 50 + 1e-12)), 10.0, 0.1)
    c = stroke_lines(lambda p: (p.move_to(50, 50), p.line_to(50, 50)), 10.0, 0.1)
    assert b["lines"].tobytes() == c["lines"].tobytes()
    # a hair-thin stroke still makes a closed outline (every vertex has two edges)
    d = stroke_lines(lambda p: (p.move_to(10, 10), p.line_to(100, 120)), 1e-4, 0.1)
    pts = np.concatenate([d["lines"]["p0"], d["lines"]["p1"]])
    _, counts = np.unique(pts, axis=0, return_counts=True)
    assert len(d["lines"]) >= 3 and np.all(counts % 2 == 0)


def test_device_stroke_records_match_the_canvas_contract():
    c = tk.Canvas(256, 256)
    c.set_device_flatten(True)
    p = tk.BezPath()
    p.move_to(10, 10)
    p.line_to(100, 20)
    p.close()
    p.quad_to(50, 50, 80, 90)
    p.move_to(200, 200)
    p.move_to(150, 150)
    p.cubic_to(160, 140, 170, 170, 180, 150)
    c.push_stroke(p, tk.Brush.solid(1, 0, 0, 1), 3.0, transform=(2, 0, 0, 2, 5, 7), tolerance=0.2)
    a = c.flatten_arrays()
    assert len(a["strokes"]) == 1 and len(a["polylines"]) == 3
    s = a["strokes"][0]
    assert s["path"] == 0 and s["polyline0"] == 0 and s["polyline_count"] == 3
    assert s["half_width"] == 1.5 and s["tolerance"] == 0.2
    assert list(s["transform"]) == [2, 0, 0, 2, 5, 7]
    pl = a["polylines"]
    assert list(pl["closed"]) == [1, 0, 0] and list(pl["element_count"]) == [2, 2, 2]
    els = a["stroke_elements"]
    for k, P in enumerate(pl):
        e = els[P["element0"]:P["element0"] + P["element_count"]]
        assert e["verb"][0] == N.EL_MOVE and np.all(e["path"] == k) and np.all(e["tolerance"] == 0.2)
    # after the close the next polyline starts at the closed one's start
    assert tuple(els[pl["element0"][1]]["p"][0]) == (10.0, 10.0)
    # no host lines: the device makes the stroke's lines
    assert c.scene_desc().line_count == 0 and len(a["elements"]) == 0
