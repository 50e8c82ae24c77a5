"""Analytic SDF shapes on the host: their physical records and pixel bounds
(Sdf::bounds / SdfShadow::bounds, src/shared/sdf/{rect,circle,line,shadow}.rs;
encode_sdf, src/shared/gpu_sdf.rs:48-260), the oracle's coverage
(shared/sdf/coverage.hlsli) against closed-form distances, and the coarse
particles SDF draws give (coarse/emit_draw.hlsli:22-30,
coarse/sdf_clip.hlsli:8-56, coarse/tile_classification.hlsli). The device
path is compared with the oracle in test_gpu_sdf.py."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

import oracle
import tileink_b200 as tk
from tileink_b200 import _native as N

SOLID = tk.Brush.solid(0.2, 0.5, 0.9, 1.0)


def record(canvas, draw):
    a = canvas.scene_arrays()
    d = a["draws"][draw]
    if d["sdf_offset"] != 0xFFFFFFFF:
        w = a["sdf"][d["sdf_offset"]:d["sdf_offset"] + d["sdf_len"]]
    else:
        w = a["sdf_shadow"][d["sdf_shadow_offset"]:d["sdf_shadow_offset"] + d["sdf_shadow_len"]]
    return int(w[0]), w[1:].view(np.float32), tuple(int(v) for v in d["pixel_bounds"])


def test_sdf_records_and_bounds():
    c = tk.Canvas(320, 240)
    # src/shared/sdf.rs:126-142: Rect (12, 24)-(28, 40), radius 3 -> bounds (12, 24, 28, 40)
    kind, f, pb = record(c, c.push_rect(12, 24, 28, 40, SOLID, radius=3))
    assert kind == N.SDF_RECT and pb == (12, 24, 28, 40)
    assert list(f[:8]) == [12, 24, 28, 40, 3, 3, 3, 3] and not f[8:].any()
    # corners are stored sorted; radii in top-left, top-right, bottom-left, bottom-right order
    kind, f, pb = record(c, c.push_rect(28.5, 40.25, 12.75, 24, SOLID, radius=(1, 2, 3, 4)))
    assert list(f[:8]) == [12.75, 24, 28.5, 40.25, 1, 2, 3, 4] and pb == (12, 24, 29, 41)
    # src/shared/gpu_sdf/tests.rs:86-101: side widths top 2, right 4, bottom 6, left 8 are
    # stored as half widths; the bounds are the outer rectangle
    kind, f, pb = record(c, c.push_rect_stroke(4, 5, 40, 41, (2, 4, 6, 8), SOLID, radius=(1, 2, 4, 3)))
    assert kind == N.SDF_RECT_STROKE
    assert list(f[:12]) == [4, 5, 40, 41, 1, 2, 4, 3, 1, 2, 3, 4]
    assert pb == (4 - 4, 5 - 1, 40 + 2, 41 + 3)
    # circles: bounds in f32 (src/shared/sdf/circle.rs:13-20)
    kind, f, pb = record(c, c.push_circle(100.5, 120.25, 30, SOLID))
    assert kind == N.SDF_CIRCLE and list(f[:4]) == [100.5, 120.25, 30, 0] and pb == (70, 90, 131, 151)
    kind, f, pb = record(c, c.push_circle_stroke(100, 100, 20, 5, SOLID))
    assert kind == N.SDF_CIRCLE_STROKE and list(f[8:12]) == [2.5] * 4 and pb == (77, 77, 123, 123)
    # lines: width and cap in the radius words; square caps extend the bounds along the axis
    kind, f, pb = record(c, c.push_line(10, 150, 300, 150, 3, SOLID, cap=N.CAP_SQUARE))
    assert kind == N.SDF_LINE and list(f[:6]) == [10, 150, 300, 150, 3, N.CAP_SQUARE]
    assert pb == (7, 148, 303, 152)
    kind, f, pb = record(c, c.push_line(10, 150, 300, 180, 3, SOLID, cap=N.CAP_ROUND))
    assert pb == (8, 148, 302, 182)
    # shadows: the shape's bounds outset by 4 expand + 1 and moved by the offset (shadow.rs:35-43)
    kind, f, pb = record(c, c.push_rect_shadow(50, 50, 150, 120, SOLID, offset=(3, 4), expand=6, intensity=0.7,
                                                 radius=10))
    assert kind == N.SDF_RECT_SHADOW and list(f[12:16]) == [3, 4, 6, np.float32(0.7)]
    assert pb == (50 + 3 - 25, 50 + 4 - 25, 150 + 3 + 25, 120 + 4 + 25)
    kind, f, pb = record(c, c.push_circle_shadow(60, 60, 10, SOLID, expand=-2, intensity=3))
    assert kind == N.SDF_CIRCLE_SHADOW and list(f[12:16]) == [0, 0, 0, 1]  # normalized options
    assert pb == (49, 49, 71, 71)
    # shapes that draw nothing: the reference's None
    assert c.push_rect_stroke(0, 0, 10, 10, 0, SOLID) is None
    assert c.push_circle_stroke(0, 0, 10, -1, SOLID) is None
    assert c.push_line(5, 5, 5, 5, 2, SOLID) is None  # butt-capped point
    assert c.push_line(5, 5, 9, 5, 0, SOLID) is None
    assert c.push_rect_shadow(0, 0, 10, 10, SOLID, intensity=0) is None
    assert c.push_line(5, 5, 5, 5, 2, SOLID, cap=N.CAP_ROUND) is not None  # a round dot
    with pytest.raises(ValueError):
        c.push_rect(0, 0, 1, 1, SOLID, radius=(1, 2))


def test_sdf_physical_scale():
    c = tk.Canvas(100, 80, scale=2.0)
    kind, f, pb = record(c, c.push_rect_stroke(10, 10, 30, 20, 3, SOLID, radius=2))
    assert list(f[:12]) == [20, 20, 60, 40, 4, 4, 4, 4, 3, 3, 3, 3] and pb == (17, 17, 63, 43)
    kind, f, pb = record(c, c.push_circle_shadow(20, 20, 5, SOLID, offset=(1, -1), expand=2, intensity=0.5))
    assert list(f[:3]) == [40, 40, 10] and list(f[12:16]) == [2, -2, 4, 0.5]
    kind, f, pb = record(c, c.push_line(0, 0, 10, 0, 1.5, SOLID))
    assert list(f[:5]) == [0, 0, 20, 0, 3]


def test_oracle_exp_is_correctly_rounded():
    lib = oracle.lib()
    xs = np.concatenate([-np.logspace(-8, 2, 4001), [0.0, -1e-30, -87.0, -103.0]]).astype(np.float32)
    got = np.array([lib.or_exp_nonpos(float(x)) for x in xs], np.float64)
    ref = np.exp(xs.astype(np.float64))
    ulp = np.spacing(ref.astype(np.float32)).astype(np.float64)
    normal = ref > np.finfo(np.float32).tiny
    assert (np.abs(got - ref)[normal] <= 0.5 * ulp[normal] * (1 + 1e-6)).all()
    assert lib.or_exp_nonpos(-200.0) == 0.0 and lib.or_exp_nonpos(0.0) == 1.0


def sdf_words(kind, coords=(0, 0, 0, 0), radii=(0, 0, 0, 0), stroke=(0, 0, 0, 0), shadow=(0, 0, 0, 0)):
    w = np.zeros(N.SDF_RECORD_WORDS, np.uint32)
    w[0] = kind
    pad = lambda v: list(v) + [0] * (4 - len(v))
    w[1:].view(np.float32)[:] = np.float32(pad(coords) + pad(radii) + pad(stroke) + pad(shadow))
    return w


def coverage(words, x, y, inv=(1, 0, 0, 1, 0, 0)):
    m = (C.c_float * 6)(*inv)
    return oracle.lib().or_sdf_coverage(words.ctypes.data, float(x), float(y), C.cast(m, C.c_void_p))


# The oracle evaluates in f32: a few ulps of coordinates near 50-100.
TOL = 2e-5


def test_oracle_sdf_coverage_against_closed_forms():
    rect = sdf_words(N.SDF_RECT, (10, 10, 20, 30))
    for x, y, d in [(15, 20, -5), (10, 20, 0), (9.75, 20, 0.25), (10.25, 20, -0.25), (21, 20, 1), (15, 30.4, 0.4)]:
        assert coverage(rect, x, y) == pytest.approx(min(max(0.5 - d, 0), 1), abs=TOL)
    # rounded corner: distance to the corner circle
    rr = sdf_words(N.SDF_RECT, (0, 0, 40, 40), (8, 8, 8, 8))
    d = math.hypot(2 - 8, 2 - 8) - 8
    assert coverage(rr, 2, 2) == pytest.approx(min(max(0.5 - d, 0), 1), abs=TOL)
    circle = sdf_words(N.SDF_CIRCLE, (50, 60, 10))
    for x, y in [(50, 60), (60.2, 60), (57, 67.3), (49.5, 49.8)]:
        d = math.hypot(x - 50, y - 60) - 10
        assert coverage(circle, x, y) == pytest.approx(min(max(0.5 - d, 0), 1), abs=TOL)
    # a circle stroke covers the ring: outer minus inner coverage
    ring = sdf_words(N.SDF_CIRCLE_STROKE, (0, 0, 20), stroke=(3, 3, 3, 3))
    assert coverage(ring, 20, 0) == 1.0 and coverage(ring, 0, 0) == 0.0
    assert coverage(ring, 23.2, 0) == pytest.approx(0.3, abs=TOL)
    # a rect stroke's hole is empty, its band full
    band = sdf_words(N.SDF_RECT_STROKE, (0, 0, 100, 60), stroke=(2, 2, 2, 2))
    assert coverage(band, 50, 30) == 0.0 and coverage(band, 50, 0) == 1.0
    # lines: butt ends stop at the end points, square ends reach half the width further
    for cap, reach in [(N.CAP_BUTT, 0.0), (N.CAP_SQUARE, 2.0)]:
        line = sdf_words(N.SDF_LINE, (10, 10, 50, 10), (4, cap))
        assert coverage(line, 30, 10) == 1.0 and coverage(line, 30, 12.25) == pytest.approx(0.25, abs=TOL)
        assert coverage(line, 50 + reach + 0.3, 10) == pytest.approx(0.2, abs=TOL)
    line = sdf_words(N.SDF_LINE, (10, 10, 50, 10), (4, N.CAP_ROUND))
    d = math.hypot(1.5, 1.5) - 2  # past the end: distance to the end point
    assert coverage(line, 51.5, 11.5) == pytest.approx(min(max(0.5 - d, 0), 1), abs=TOL)
    # shadows: exp(-max(d, 0) / expand) * intensity outside, intensity inside
    sh = sdf_words(N.SDF_RECT_SHADOW, (0, 0, 20, 20), shadow=(2, 3, 4, 0.5))
    assert coverage(sh, 12, 13) == pytest.approx(0.5)
    assert coverage(sh, 22 + 6, 13) == pytest.approx(0.5 * math.exp(-6 / 4), rel=1e-6)
    # an anisotropic inverse transform scales the distance by the normal's footprint
    inv = (0.5, 0, 0, 2, 0, 0)
    assert coverage(rect, 20.25, 20, inv) == pytest.approx(0.5 - 0.25 / 0.5, abs=TOL)


def ptcl_of(canvas):
    run = oracle.OracleRun(canvas.scene_desc(), threads=4)
    return (run.get(oracle.OR_PASS_PTCL, N.PTCL_DTYPE, 0), run.get(oracle.OR_PASS_TILES, N.TILE_DTYPE, 0),
            run.get(oracle.OR_PASS_KINDS, np.uint32, 0))


def tile_stream(ptcl, tiles, t):
    r = tiles[t]
    return ptcl[r["ptcl_start"]:r["ptcl_end"]]


def test_oracle_sdf_particles_and_tile_kinds():
    W, H = 384, 128
    tw = W // 16
    c = tk.Canvas(W, H)
    c.push_rect(20, 20, 200, 108, tk.Brush.solid(0.9, 0.1, 0.1, 1.0))            # draw 0: solid rect
    c.push_rect_stroke(208, 8, 376, 120, 4, tk.Brush.solid(0.1, 0.8, 0.1, 1.0))  # draw 1: hollow stroke
    c.push_circle(64, 64, 20, tk.Brush.solid(0.1, 0.1, 0.9, 0.5))               # draw 2: circle
    ptcl, tiles, kinds = ptcl_of(c)

    def draws_in(tx, ty):
        s = tile_stream(ptcl, tiles, ty * tw + tx)
        return [(int(p["tag"]), int(p["color"])) for p in s if p["tag"] not in (N.PTCL_BATCH_BEGIN, N.PTCL_END)]

    def kind_of(tx, ty):
        return int(tile_stream(ptcl, tiles, ty * tw + tx)[0]["color"]) & 7

    a = c.scene_arrays()
    color = int(a["brush"][a["draws"][0]["brush_offset"] + 4])
    # every pixel centre of the tile at least half a pixel inside the solid rect:
    # one colour particle (full_tile_solid), a COLOR tile
    assert draws_in(8, 3) == [(N.PTCL_COLOR, color)] and kind_of(8, 3) == N.TILE_KIND_COLOR
    # on the rect's edge it is an SDF particle of draw 0; solid rects are
    # solid-supported SDFs, so the tile is an SDF tile
    assert draws_in(1, 1) == [(N.PTCL_SDF, 0)] and kind_of(1, 1) == N.TILE_KIND_SDF
    assert draws_in(8, 6) == [(N.PTCL_SDF, 0)]
    # the circle's tiles: the rect as a colour, the circle (not solid-supported) interpreted
    assert draws_in(3, 3) == [(N.PTCL_COLOR, color), (N.PTCL_SDF, 2)]
    assert kind_of(3, 3) == N.TILE_KIND_INTERPRETER
    # tiles at least a pixel inside the stroke's hole have no particle (sdf_stroke_empty)
    for tx in range(14, 23):
        for ty in range(1, 7):
            assert draws_in(tx, ty) == [], (tx, ty)
    assert draws_in(13, 3) == [(N.PTCL_SDF, 1)] and draws_in(23, 3) == [(N.PTCL_SDF, 1)]
    # MIXED: a colour particle and a solid-supported SDF particle in one tile
    m = tk.Canvas(64, 64)
    m.push_rect(0, 0, 64, 64, tk.Brush.solid(1, 1, 1, 1))
    m.push_rect(5.5, 5.5, 40, 40, tk.Brush.solid(0, 0, 0, 1))
    p2, t2, k2 = ptcl_of(m)
    assert int(tile_stream(p2, t2, 0)[0]["color"]) & 7 == N.TILE_KIND_MIXED


def test_sdf_nodes_replay_under_translations_only():
    node = tk.Canvas(200, 100)
    node.keep_commands()
    node.push_rect(10, 10, 50, 40, SOLID, radius=4)
    node.push_line(0, 0, 30, 20, 2, SOLID, cap=N.CAP_ROUND)
    moved = tk.Canvas(200, 100)
    moved.replay(node, (1, 0, 0, 1, 7.5, -3))
    direct = tk.Canvas(200, 100)
    direct.push_rect(17.5, 7, 57.5, 37, SOLID, radius=4)
    direct.push_line(7.5, -3, 37.5, 17, 2, SOLID, cap=N.CAP_ROUND)
    a, b = moved.scene_arrays(), direct.scene_arrays()
    for k in ("draws", "sdf", "brush", "draw_order"):
        assert a[k].tobytes() == b[k].tobytes(), k
    with pytest.raises(ValueError):
        tk.Canvas(200, 100).replay(node, (0.9, 0.1, -0.1, 0.9, 0, 0))
    # a retained scene reports the shapes' pixel bounds as damage when a node moves
    rs = tk.RetainedScene(200, 100)
    rs.insert(1, node)
    rs.materialize()
    rs.set_transform(1, (1, 0, 0, 1, 20, 0))
    canvas, damage = rs.materialize()
    rects = {tuple(r) for r in damage["rects"].tolist()}
    assert (10, 10, 50, 40) in rects and (30, 10, 70, 40) in rects


def test_oracle_coarse_proofs_match_fine_only_oracle():
    """The oracle's full pipeline (coarse with its full-tile colour,
    hollow-stroke and occlusion proofs, then fine) gives the fine-only
    oracle's pixels on the reference's rect known-answer scenes."""
    from sdf_cases import all_cases, desc_of
    for name, scene in all_cases():
        keep, d = desc_of(scene)
        want = oracle.interpret_sdf_draws(d)
        run = oracle.OracleRun(d, threads=4)
        got = run.get(oracle.OR_IMAGE, np.uint32).view(np.uint8).reshape(want.shape)
        assert np.array_equal(got, want), (name, int((got != want).any(axis=2).sum()))


def test_extended_sdf_kinds_records_and_bounds():
    c = tk.Canvas(200, 120)
    # src/shared/sdf/triangle.rs:95-105 and candlestick.rs:97-102
    kind, f, pb = record(c, c.push_triangle((8, 4), (20, 16), (8, 28), SOLID, corner_radius=2.0))
    assert kind == N.SDF_TRIANGLE and list(f[:7]) == [8, 4, 20, 16, 8, 28, 2] and pb == (6, 2, 22, 30)
    kind, f, pb = record(c, c.push_candlestick(16.5, 4.0, 28.0, 10.0, 22.0, 7, 1, SOLID))
    assert kind == N.SDF_CANDLESTICK and list(f[:7]) == [16.5, 4, 28, 10, 22, 7, 1] and pb == (13, 4, 20, 28)
    kind, f, pb = record(c, c.push_dash_line(10, 100, 190, 100, 3, 6, 4, SOLID, cap=N.CAP_ROUND, dash_offset=2))
    assert kind == N.SDF_DASH_LINE and list(f[:9]) == [10, 100, 190, 100, 3, N.CAP_ROUND, 6, 4, 2]
    base, cells = c.push_checkerboard(100, 10, 180, 70, 8, SOLID, tk.Brush.solid(1, 1, 1, 1))
    kind, f, pb = record(c, cells)
    assert kind == N.SDF_CHECKERBOARD and list(f[:5]) == [100, 10, 180, 70, 8] and record(c, base)[0] == N.SDF_RECT
    # the reference's None: collinear triangle, no visible dash, empty checkerboard
    assert c.push_triangle((0, 0), (1, 1), (2, 2), SOLID) is None
    assert c.push_dash_line(0, 0, 1, 0, 1, 1, 10, SOLID, dash_offset=2) is None
    assert c.push_checkerboard(0, 0, 0, 10, 2, SOLID, SOLID) is None
    with pytest.raises(ValueError):
        c.push_candlestick(1, 2, 3, 4, 5, 0, 1, SOLID)  # CandleStick::new rejects a zero width


def test_oracle_extended_kinds_against_closed_forms():
    # triangle: inside, the distance to the nearest edge, negated
    tri = sdf_words(N.SDF_TRIANGLE, (0, 0, 40, 0), (0, 40, 0))
    assert coverage(tri, 10, 10) == 1.0 and coverage(tri, 30, 30) == 0.0
    d = (25.0 + 25.0 - 40.0) / math.sqrt(2.0)  # (25, 25) lies outside the hypotenuse x + y = 40
    assert coverage(tri, 25, 25) == pytest.approx(min(max(0.5 - d, 0), 1), abs=TOL)
    assert coverage(tri, 0.25, 20) == pytest.approx(0.75, abs=TOL)
    # checkerboard: even cells (cell x + cell y even) covered, odd ones not
    cb = sdf_words(N.SDF_CHECKERBOARD, (0, 0, 64, 64), (8,))
    assert coverage(cb, 4, 4) == 1.0 and coverage(cb, 12, 4) == 0.0 and coverage(cb, 12, 12) == 1.0
    assert coverage(cb, 8.25, 4) == pytest.approx(0.25, abs=TOL)  # a quarter pixel into the odd cell
    # dash line: dashes of 6 with gaps of 4 from x = 0; a gap's middle is empty
    dash = sdf_words(N.SDF_DASH_LINE, (0, 10, 100, 10), (2, N.CAP_BUTT, 6, 4))
    assert coverage(dash, 3, 10) == 1.0 and coverage(dash, 8, 10) == 0.0 and coverage(dash, 13, 10) == 1.0
    assert coverage(dash, 6.25, 10) == pytest.approx(0.25, abs=TOL)
    # candlestick: wick or body, whichever covers more
    candle = sdf_words(N.SDF_CANDLESTICK, (20, 0, 60, 20), (40, 9, 1))
    assert coverage(candle, 20, 5) == pytest.approx(1.0) and coverage(candle, 24, 30) == pytest.approx(1.0)
    assert coverage(candle, 24.75, 30) == pytest.approx(0.25, abs=TOL) and coverage(candle, 24, 5) == 0.0


def test_callout_bounds_match_the_reference():
    """src/shared/sdf/callout.rs:279-340: a 100 x 40 body with radius 8 and a
    tail (offset 50, width 10, length 6, radius 1.5) on each side, its stroke
    and shadow, and the hidden tail."""
    c = tk.Canvas(200, 120)
    body, tail = (10, 20, 110, 60), (50.0, 10.0, 6.0, 1.5)
    want = [(10, 14, 110, 60), (10, 20, 116, 60), (10, 20, 110, 66), (4, 20, 110, 60)]
    for side in range(4):
        assert record(c, c.push_callout(body, 8.0, (side,) + tail, SOLID))[2] == want[side]
    assert record(c, c.push_callout_stroke(body, 8.0, (N.SIDE_BOTTOM,) + tail, 2.0, SOLID))[2] == (9, 19, 111, 67)
    kind, f, pb = record(c, c.push_callout_shadow(body, 8.0, (N.SIDE_BOTTOM,) + tail, SOLID, offset=(0, 2), expand=4,
                                                  intensity=0.5))
    assert kind == N.SDF_CALLOUT_SHADOW and pb == (-7, 5, 127, 85)
    assert list(f[:12]) == [10, 20, 110, 60, 8, 50, 10, 6, 1.5, 2, 0, 1]
    assert record(c, c.push_callout(body, 8.0, None, SOLID))[2] == (10, 20, 110, 60)
    assert record(c, c.push_callout_stroke(body, 8.0, None, 2.0, SOLID))[2] == (9, 19, 111, 61)
    # empty: a flat body, a zero tail width, a zero stroke
    assert c.push_callout((0, 0, 10, 0), 1.0, None, SOLID) is None
    assert c.push_callout(body, 8.0, (0, 50.0, 0.0, 6.0, 1.5), SOLID) is None
    assert c.push_callout_stroke(body, 8.0, None, 0.0, SOLID) is None


def test_oracle_callout_coverage():
    # body (0, 0)-(100, 40) radius 0, tail on the bottom: offset 50, width 20, length 10
    w = sdf_words(N.SDF_CALLOUT, (0, 0, 100, 40), (0, 50, 20, 10), (0, N.SIDE_BOTTOM, 0, 1))
    assert coverage(w, 20, 20) == 1.0 and coverage(w, 20, 45) == 0.0
    assert coverage(w, 50, 44) == 1.0  # inside the tail
    assert coverage(w, 50, 50.25) == pytest.approx(0.25, abs=TOL)  # just past the tail's tip
    hidden = sdf_words(N.SDF_CALLOUT, (0, 0, 100, 40), (0, 50, 20, 10), (0, N.SIDE_BOTTOM, 0, 0))
    assert coverage(hidden, 50, 44) == 0.0
    stroke = sdf_words(N.SDF_CALLOUT_STROKE, (0, 0, 100, 40), (0, 50, 20, 10), (0, N.SIDE_BOTTOM, 1.5, 1))
    assert coverage(stroke, 20, 20) == 0.0 and coverage(stroke, 0, 20) == 1.0


def test_arc_and_star_bounds_match_the_reference():
    c = tk.Canvas(100, 100)
    # src/shared/sdf/arc.rs (tests): radius 10 at (20, 20), sweep pi, width 4 -> (7, 17, 33, 33)
    kind, f, pb = record(c, c.push_sdf_arc(20, 20, 10, 0.0, math.pi, 4, SOLID))
    assert kind == N.SDF_ARC and pb == (7, 17, 33, 33)
    assert list(f[:7]) == [20, 20, 10, 4, 0, np.float32(math.pi), N.CAP_BUTT]
    # src/shared/sdf/star.rs (tests): star at (16, 20), radii 8 / 3.5, corner 1.25, rotation -pi/2
    kind, f, pb = record(c, c.push_star(16, 20, 8, 3.5, SOLID, corner_radius=1.25, rotation=-math.pi / 2))
    assert kind == N.SDF_STAR and pb == (7, 10, 25, 28)
    assert record(c, c.push_star_stroke(16, 20, 8, 3.5, 2.5, SOLID, corner_radius=1.25,
                                        rotation=-math.pi / 2))[2] == (5, 9, 27, 29)
    kind, f, pb = record(c, c.push_arc_shadow(50, 50, 20, 1.0, -2.0, 3, SOLID, offset=(1, 2), expand=2,
                                              intensity=0.5, cap=N.CAP_ROUND))
    assert kind == N.SDF_ARC_SHADOW and list(f[12:16]) == [1, 2, 2, 0.5]
    # the reference's None: zero sweep, inner radius not below outer
    assert c.push_sdf_arc(20, 20, 10, 0.0, 0.0, 4, SOLID) is None
    assert c.push_star(16, 20, 3, 3, SOLID) is None


def test_oracle_trig_is_correctly_rounded():
    lib = oracle.lib()
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.uniform(-30, 30, 3000), [0.0, math.pi, -math.pi / 2, 1e-7, 700.25]]).astype(np.float32)
    s, c = C.c_float(), C.c_float()
    for x in xs:
        lib.or_sincos(float(x), C.byref(s), C.byref(c))
        for got, ref in ((s.value, math.sin(float(x))), (c.value, math.cos(float(x)))):
            assert abs(got - ref) <= 0.5 * abs(float(np.spacing(np.float32(ref)))) * (1 + 1e-6), (x, got, ref)
    for y, x in rng.uniform(-50, 50, (3000, 2)).astype(np.float32):
        ref = math.atan2(float(y), float(x))
        assert abs(lib.or_atan2(float(y), float(x)) - ref) <= 0.5 * abs(float(np.spacing(np.float32(ref)))) * (1 + 1e-6)


def test_oracle_arc_and_star_coverage():
    # a half ring of radius 20, width 4, from angle 0 over pi (y grows downwards: the lower half)
    arc = sdf_words(N.SDF_ARC, (0, 0, 20, 4), (0, math.pi, N.CAP_BUTT))
    assert coverage(arc, 0, 20) == 1.0 and coverage(arc, 0, -20) == 0.0 and coverage(arc, 0, 0) == 0.0
    assert coverage(arc, 0, 22.25) == pytest.approx(0.25, abs=TOL)
    # a round cap reaches half the width past the end at (20, 0)
    round_arc = sdf_words(N.SDF_ARC, (0, 0, 20, 4), (0, math.pi, N.CAP_ROUND))
    assert coverage(round_arc, 20, -1.75) == pytest.approx(0.75, abs=1e-4) and coverage(arc, 20, -1.75) == 0.0
    # a star of outer radius 30, inner 12: its centre inside, far points outside
    star = sdf_words(N.SDF_STAR, (50, 50, 30, 12), (0, 0))
    assert coverage(star, 50, 50) == 1.0 and coverage(star, 50, 10) == 0.0
    # a quarter pixel inside the tip at angle 0: the edges meet there at +-h from the axis, so
    # the nearest edge is 0.25 sin(h) away
    ix, iy = 12 * math.cos(math.pi / 5), 12 * math.sin(math.pi / 5)
    h = math.atan2(iy, 30 - ix)
    assert coverage(star, 79.75, 50) == pytest.approx(0.5 + 0.25 * math.sin(h), abs=1e-4)


def test_oracle_partial_sdf_clip_matches_fine_only_oracle():
    """occlusion_pixels.rs:48-83 on the oracle: coarse's SDF clip wrappers
    (dropped where the clip rect covers the tile) and the occlusion skip give
    the pixels of the explicit clip stream interpreted in every tile."""
    from sdf_cases import partial_clip_cases
    for name, canvas, stream in partial_clip_cases():
        d = canvas.scene_desc()
        want = oracle.interpret_particles(d, stream)
        got = oracle.OracleRun(d, threads=4).get(oracle.OR_IMAGE, np.uint32).view(np.uint8).reshape(want.shape)
        assert np.array_equal(got, want), name
