"""CPU tests: the oracle pinned against the reference's own test algorithms and
known answers, the host planner, flattening structure, and the canvas compile.

No GPU is used here.
"""
import math

import numpy as np
import pytest

import oracle
import tileink_b200 as tk
from tileink_b200 import _native as N

from helpers import (BLUR_SIGMAS, BLUR_SIZES, PREFIX_LENGTHS, PREFIX_SEEDS, blur_config, blur_source, circle_path,
                     count_case_inputs, count_segments, gaussian_f64, prefix_case)


# --- scan prefix (scan_cases.rs:8-157) ------------------------------------------------
@pytest.mark.parametrize("lengths", PREFIX_LENGTHS)
@pytest.mark.parametrize("seed", PREFIX_SEEDS)
def test_oracle_prefix_matches_reference_case(lengths, seed):
    case = prefix_case(lengths, seed)
    ranges = case["init_ranges"].copy()
    cursors = case["init_cursors"].copy()
    bumps = np.zeros(len(case["paths"]), dtype=np.uint32)
    oracle.lib().or_scan_prefix(N.ptr(case["counts"]), N.ptr(case["paths"]), len(case["paths"]),
                                N.ptr(ranges), N.ptr(cursors), N.ptr(bumps))
    assert np.array_equal(ranges, case["ranges"])
    assert np.array_equal(cursors, case["cursors"])
    assert np.array_equal(bumps, case["totals"])


# --- single-line scan_count (metal/scan_tests.rs:24-95) -------------------------------
def test_oracle_count_matches_cpu_planner_and_keeps_guards():
    mismatches = []
    for a, b in count_segments():
        for p0, p1 in ((a, b), (b, a)):
            line, path, init = count_case_inputs(p0, p1)
            bd = init.view(np.int32).copy()
            cnt = init.copy()
            oracle.lib().or_scan_count(N.ptr(line), 1, N.ptr(path), 1, N.ptr(bd), N.ptr(cnt))
            for arr in (bd.view(np.uint32), cnt):
                assert np.all(arr[:7] == 0x12345678) and np.all(arr[71:] == 0x12345678)
            total = int(cnt[7:71].sum())
            planned = oracle.lib().or_line_scanned_tile_count(N.ptr(line), 0, 0, 8, 8)
            host = tk.plan_line_tile_count(line[0], (0, 0, 8, 8))
            assert planned == host
            if total != planned:
                mismatches.append((p0, p1, total, planned))
    assert not mismatches, mismatches


def test_host_planner_matches_oracle_planner_on_random_lines():
    rng = np.random.default_rng(5)
    lines = np.zeros(4000, dtype=N.LINE_DTYPE)
    lines["p0"] = rng.uniform(-40, 200, (4000, 2)).astype(np.float32)
    lines["p1"] = rng.uniform(-40, 200, (4000, 2)).astype(np.float32)
    lines["p1"][::7] = lines["p0"][::7] + rng.integers(-3, 4, (len(lines[::7]), 2)) * 16  # tile-aligned deltas
    for ln in lines:
        l1 = np.array([ln], dtype=N.LINE_DTYPE)
        for bbox in ((0, 0, 8, 8), (2, 1, 9, 12), (3, 3, 4, 4)):
            assert tk.plan_line_tile_count(ln, bbox) == oracle.lib().or_line_scanned_tile_count(N.ptr(l1), *bbox)


# --- flattening structure (src/shared/path_flatten.rs:90-173) --------------------------
def test_flatten_line_after_move_to_is_not_skipped():
    lines = tk.BezPath().move_to(1, 2).line_to(5, 2).flatten(0.1)
    assert len(lines) == 2
    assert list(lines[0]["p0"]) == [1, 2] and list(lines[0]["p1"]) == [5, 2]
    assert list(lines[1]["p0"]) == [5, 2] and list(lines[1]["p1"]) == [1, 2]


def test_flatten_final_open_contour_is_closed():
    lines = tk.BezPath().move_to(0, 0).line_to(10, 0).line_to(10, 10).flatten(0.1)
    assert len(lines) == 3
    assert list(lines[2]["p0"]) == [10, 10] and list(lines[2]["p1"]) == [0, 0]


def test_flatten_closed_rect_keeps_all_edges():
    lines = tk.BezPath().move_to(0, 0).line_to(10, 0).line_to(10, 10).line_to(0, 10).close().flatten(0.1)
    assert len(lines) == 4


def test_flatten_duplicate_points_and_repeated_close():
    p = tk.BezPath().move_to(0, 0).line_to(0, 0).line_to(10, 0).line_to(10, 0).close().close()
    lines = p.flatten(0.1, path_id=7)
    assert len(lines) == 2
    assert list(lines[0]["p0"]) == [0, 0] and list(lines[0]["p1"]) == [10, 0]
    assert list(lines[1]["p0"]) == [10, 0] and list(lines[1]["p1"]) == [0, 0]
    assert np.all(lines["path_id"] == 7)


def test_flatten_circle_many_small_lines_within_bounds():
    lines = circle_path(20, 20, 10).flatten(0.1)
    assert len(lines) > 16
    pts = np.concatenate([lines["p0"], lines["p1"]])
    assert np.all(pts >= 9.0) and np.all(pts <= 31.0)


def _cubic(c, t):
    mt = 1 - t
    return (mt ** 3) * c[0] + 3 * mt * mt * t * c[1] + 3 * mt * t * t * c[2] + t ** 3 * c[3]


@pytest.mark.parametrize("tol", [0.1, 0.25, 1.0])
def test_flatten_cubic_stays_within_tolerance(tol):
    rng = np.random.default_rng(11)
    for _ in range(40):
        c = rng.uniform(0, 600, (4, 2))
        p = tk.BezPath().move_to(*c[0]).cubic_to(*c[1], *c[2], *c[3])
        lines = p.flatten(tol)[:-1]  # drop the closing edge
        ts = np.linspace(0, 1, 4001)
        curve = np.array([_cubic(c, t) for t in ts])
        # every curve sample lies within tol (plus f32 rounding) of the polyline
        a = lines["p0"].astype(np.float64)
        b = lines["p1"].astype(np.float64)
        ab = b - a
        worst = 0.0
        for q in curve[::8]:
            t = np.clip(((q - a) * ab).sum(1) / np.maximum((ab * ab).sum(1), 1e-30), 0, 1)
            d = np.sqrt((((a + t[:, None] * ab) - q) ** 2).sum(1)).min()
            worst = max(worst, d)
        assert worst <= tol * 1.01 + 1e-3, worst


# --- blur (tests/shared_blur_gpu.rs:9-155) ---------------------------------------------
@pytest.mark.parametrize("size", BLUR_SIZES)
def test_oracle_blur_within_one_lsb_of_f64_gaussian(size):
    width, height = size
    src = blur_source(width, height)
    untouched = np.full(width * height, int.from_bytes(bytes([29, 31, 37, 113]), "little"), dtype=np.uint32)
    for sigma in BLUR_SIGMAS:
        s32 = float(np.float32(sigma))
        for axis in (0, 1):
            for inset in (False, True):
                region, source = blur_config(width, height, inset)
                dst = untouched.copy()
                reg = np.array(region, dtype=np.uint32)
                srcb = np.array(source, dtype=np.uint32)
                oracle.lib().or_blur_pass(N.ptr(src), N.ptr(dst), width, height, N.ptr(reg), N.ptr(srcb),
                                          np.float32(sigma), axis)
                out = dst.view(np.uint8).reshape(-1, 4)
                for y in range(height):
                    for x in range(width):
                        inside = region[0] <= x < region[0] + region[2] and region[1] <= y < region[1] + region[3]
                        if not inside:
                            assert dst[y * width + x] == untouched[0]
                            continue
                        exp = gaussian_f64(src, width, height, source, x, y, s32, axis)
                        diff = np.abs(out[y * width + x].astype(int) - exp.astype(int)).max()
                        assert diff <= 1, (size, sigma, axis, inset, x, y, out[y * width + x], exp)


# --- coverage: f32 restatement vs an f64 evaluation of the same formula ---------------
def _fill_value_f64(segs, backdrop, x, y):
    base, running, partial = float(backdrop), 0.0, 0.0
    for s in segs:
        p0x, p0y, p1x, p1y, ye = (float(v) for v in s)
        dxx, dyy = p1x - p0x, p1y - p0y
        ly = p0y - y
        y0, y1 = min(max(ly, 0), 1), min(max(p1y - y, 0), 1)
        dy = y0 - y1
        base += (-1.0 if dxx < 0 else 1.0) * min(max(y - ye + 1, 0), 1)
        if dy == 0:
            continue
        slope = dxx / dyy
        near = abs(ly - 0.5) <= abs(p1y - y - 0.5)
        ax, ay = (p0x, ly) if near else (p1x, p1y - y)
        sx0, sx1 = (y0 - ay) * slope + ax, (y1 - ay) * slope + ax
        lo_x, hi_x = min(sx0, sx1), max(sx0, sx1)
        fs = min(max(math.ceil(hi_x), 0), 16)
        if fs < 16 and x >= fs:
            running += dy
        ps = min(max(math.floor(lo_x), 0), 16)
        if ps <= x < fs:
            xmin, xmax = lo_x - x, hi_x - x
            w = xmax - xmin
            if w == 0:
                a = min(max(1 - xmin, 0), 1)
            elif xmin >= 0 and xmax <= 1:
                a = 1 - 0.5 * (xmin + xmax)
            else:
                l, r = min(max(xmin, 0), 1), min(max(xmax, 0), 1)
                a = ((r - l) * (1 - 0.5 * (l + r)) + min(max(-xmin, 0), w)) / w
            partial += a * dy
    return base + running + partial


def test_fp32_coverage_within_2e5_of_fp64():
    c = tk.generate(1, 3, width=160, height=96, paths=20)
    d = c.scene_desc()
    run = oracle.OracleRun(d, threads=4)
    segs = run.get(oracle.OR_SEGMENTS, N.SEGMENT_DTYPE)
    ptcl = run.get(oracle.OR_PASS_PTCL, N.PTCL_DTYPE, 0)
    fills = ptcl[(ptcl["tag"] == N.PTCL_FILL) & (ptcl["segment_end"] > ptcl["segment_start"])]
    rng = np.random.default_rng(0)
    worst = 0.0
    for rec in fills[rng.choice(len(fills), size=min(200, len(fills)), replace=False)]:
        s = np.ascontiguousarray(segs[rec["segment_start"]:rec["segment_end"]])
        for (x, y) in rng.integers(0, 16, (8, 2)):
            v32 = oracle.lib().or_fill_value(N.ptr(s), len(s), int(rec["backdrop"]), int(x), int(y))
            v64 = _fill_value_f64(s, rec["backdrop"], int(x), int(y))
            worst = max(worst, abs(float(v32) - v64))
    assert worst <= 2e-5, worst


# --- merged PTCL layout is a pure relayout of the per-batch reference streams ----------
def test_merged_pass_stream_relayouts_batch_streams():
    c = tk.generate(2, 9, width=512, height=384, paths=300)
    run = oracle.OracleRun(c.scene_desc(), threads=8)
    assert run.pass_count == 1 and run.batch_count > 3
    merged = run.get(oracle.OR_PASS_PTCL, N.PTCL_DTYPE, 0)
    tiles = run.get(oracle.OR_PASS_TILES, N.TILE_DTYPE, 0)
    per_batch = [(run.get(oracle.OR_BATCH_PTCL, N.PTCL_DTYPE, b), run.get(oracle.OR_BATCH_TILES, N.TILE_DTYPE, b),
                  run.get(oracle.OR_BATCH_KINDS, np.uint32, b)) for b in range(run.batch_count)]
    for t in range(len(tiles)):
        stream = merged[tiles[t]["ptcl_start"]:tiles[t]["ptcl_end"]]
        rebuilt = []
        for b, (bp, bt, bk) in enumerate(per_batch):
            rec = bt[t]
            if rec["ptcl_count"] == 0:
                continue
            rebuilt.append(np.array([(N.PTCL_BATCH_BEGIN, 0, 0, b, rec["ptcl_count"] - 1, bk[t])], dtype=N.PTCL_DTYPE))
            seg = bp[rec["ptcl_start"]:rec["ptcl_end"]]
            assert seg[-1]["tag"] == N.PTCL_END
            rebuilt.append(seg[:-1])
        if rebuilt:
            rebuilt.append(np.zeros(1, dtype=N.PTCL_DTYPE))
            assert np.array_equal(np.concatenate(rebuilt), stream)
        else:
            assert len(stream) == 0


# --- canvas compile (src/canvas/compile.rs, src/shared/execution/batches.rs) -----------
def _square(x, y, s):
    return tk.BezPath().move_to(x, y).line_to(x + s, y).line_to(x + s, y + s).line_to(x, y + s).close()


def test_canvas_compile_splits_batches_at_clip_layers_and_assigns_ids_in_op_order():
    cv = tk.Canvas(64, 64)
    red = tk.Brush.solid(1, 0, 0, 1)
    a = cv.push_path(_square(1, 1, 10), red)
    cv.push_clip_layer(_square(0, 0, 30))
    b = cv.push_path(_square(5, 5, 10), red)
    cv.push_clip_layer(_square(2, 2, 20), fill_rule=tk.FILL_EVEN_ODD)
    c = cv.push_path(_square(6, 6, 4), red)
    cv.pop_layer()
    cv.pop_layer()
    d = cv.push_path(_square(40, 40, 10), red)
    s = cv.scene_arrays()
    ops = s["ops"]
    assert list(ops["kind"]) == [N.OP_DRAW_BATCH] * 4
    assert list(ops["batch_id"]) == [0, 1, 2, 3]
    stacks = [s["layers"][o["layer_start"]:o["layer_end"]] for o in ops]
    assert [len(x) for x in stacks] == [0, 1, 2, 0]
    clip_draws = [int(x["draw"]) for x in stacks[2]]
    assert s["draws"][clip_draws[0]]["tag"] == 1 and s["draws"][clip_draws[1]]["fill_rule"] == 1
    assert list(s["draw_order"]) == [a, b, c, d]
    assert [s["draw_batch_ids"][i] for i in (a, b, c, d)] == [0, 1, 2, 3]
    assert s["draw_batch_ids"][clip_draws[0]] == N.INVALID
    # record allocation rules (canvas/paths.rs:115-130)
    p = s["paths"]
    assert np.all(p["data_offset"][1:] == p["data_offset"][:-1] + p["data_len"][:-1])
    assert np.all(p["segment_start"][1:] == p["segment_start"][:-1] + p["segment_capacity"][:-1])
    assert np.all(p["data_len"] == (p["tile_x1"] - p["tile_x0"]) * (p["tile_y1"] - p["tile_y0"]))


def test_canvas_blur_group_is_an_offscreen_op_with_outset_bounds():
    cv = tk.Canvas(200, 100)
    cv.push_blur_group(4.0)
    cv.push_path(_square(50, 30, 20), tk.Brush.solid(0, 0, 1, 1))
    cv.pop_layer()
    s = cv.scene_arrays()
    kinds = list(s["ops"]["kind"])
    assert kinds == [N.OP_BLUR_BEGIN, N.OP_DRAW_BATCH, N.OP_BLUR_END]
    assert list(s["ops"][0]["bounds"]) == [50 - 12, 30 - 12, 70 + 12, 50 + 12]
    assert s["ops"][0]["sigma"] == np.float32(4.0)


def test_segment_capacity_plan_equals_oracle_count_totals():
    c = tk.generate(1, 2, width=200, height=120, paths=30)
    run = oracle.OracleRun(c.scene_desc(), threads=4)
    paths = c.scene_arrays()["paths"]
    bumps = run.get(oracle.OR_BUMPS, np.uint32)
    assert np.array_equal(bumps, paths["segment_capacity"])
    ranges = run.get(oracle.OR_RANGES, N.RANGE_DTYPE)
    counts = run.get(oracle.OR_COUNTS, np.uint32)
    assert np.array_equal(ranges["end"] - ranges["start"], counts)


def test_brush_encoding_layout():
    cv = tk.Canvas(32, 32)
    cv.push_path(_square(1, 1, 4), tk.Brush.solid(1.0, 0.5, 0.0, 0.5))
    cv.push_path(_square(1, 1, 4), tk.Brush.linear((0, 0), (100, 0), [(0, (1, 0, 0, 1)), (1, (0, 0, 1, 1))]))
    s = cv.scene_arrays()
    w = s["brush"]
    # solid: header kind 1, premultiplied RGBA8 (pixel.rs:14-21) at word 4
    assert w[0] == 1 and w[4] == (int(0.5 * 255 + 0.5) | (int(0.25 * 255 + 0.5) << 8) | (0 << 16) | (128 << 24))
    lin = s["draws"][1]["brush_offset"]
    assert w[lin] == 2 and w[lin + 2] == 21 and w[lin + 3] >= 64
    params = w[lin + 9: lin + 21].view(np.float32)
    assert list(params[:4]) == [0, 0, 100, 0] and list(params[4:10]) == [1, 0, 0, 1, 0, 0]
    ramp = w[lin + 21: lin + 21 + w[lin + 3]]
    assert ramp[0] == 0xFF0000FF and ramp[-1] == 0xFFFF0000


# --- C ABI: the library loads and exports every declared entry point -------------------
def test_library_exports_every_declared_symbol():
    import re
    from pathlib import Path
    lib = N.library()
    names = set()
    for h in (Path(__file__).resolve().parents[1] / "include").glob("*.h"):
        text = h.read_text()
        names |= set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(tk_\w+)\s*\(", text, re.M))
    assert len(names) > 30
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string():
    assert b"sm_100a" in N.library().tk_version()


# --- differentiable path: flattening structure and the FP64 oracle -------------------
def test_diff_flatten_matches_canvas_flattening_bitwise():
    from tileink_b200 import diff
    sc = diff.blur_group_scene(11, width=320, height=200, paths=12)
    lines, ep, w = diff.flatten(sc)
    canvas_lines = tk.generate(5, 11, width=320, height=200, paths=12).scene_arrays()["lines"]
    assert len(lines) == len(canvas_lines)
    assert lines.tobytes() == canvas_lines.tobytes()


def test_diff_flatten_weights_reconstruct_line_endpoints():
    from tileink_b200 import diff
    sc = diff.blur_group_scene(12, width=256, height=256, paths=8)
    lines, ep, w = diff.flatten(sc)
    P = sc.points.reshape(-1, 2).astype(np.float64)
    for e, key in ((0, "p0"), (1, "p1")):
        pts = np.stack([P[ep[:, e] + i] for i in range(4)], axis=1)  # [L, 4, 2]
        rec = np.einsum("li,lid->ld", w[:, e, :].astype(np.float64), pts)
        assert np.abs(rec - lines[key]).max() < 1e-4
    # weights of each endpoint sum to one (affine combinations of control points)
    assert np.abs(w.sum(axis=2) - 1.0).max() < 1e-5
    # consecutive lines share endpoints
    assert np.array_equal(lines["p1"][:-1][lines["path_id"][:-1] == lines["path_id"][1:]],
                          lines["p0"][1:][lines["path_id"][:-1] == lines["path_id"][1:]])


def test_diff_oracle_exact_area_of_a_square():
    # a 10x10 square with corners at half pixels, drawn as 4 straight cubics:
    # interior pixels are fully covered, edge pixels half, corners a quarter
    from tileink_b200 import diff
    corners = [(3.5, 3.5), (13.5, 3.5), (13.5, 13.5), (3.5, 13.5)]
    pts = [corners[0]]
    for k in range(4):
        a, b = np.array(corners[k]), np.array(corners[(k + 1) % 4])
        pts += [tuple(a + (b - a) / 3), tuple(a + 2 * (b - a) / 3), tuple(b)]
    sc = diff.DiffScene(20, 20, np.array([pts], np.float32), np.array([[1.0, 0.0, 0.0, 1.0]], np.float32),
                        sigma=0.0, background=(0.0, 0.0, 0.0, 0.0))
    lines, ep, w = diff.flatten(sc)
    _, img = oracle.diff_loss(sc, lines, ep, w, sc.points, sc.colors, 0.0, np.zeros((20, 20, 4), np.float32),
                              return_image=True)
    a = img[..., 3]
    assert abs(a[8, 8] - 1.0) < 1e-12 and abs(a[3, 8] - 0.5) < 1e-12 and abs(a[3, 3] - 0.25) < 1e-12
    assert abs(a.sum() - 100.0) < 1e-9 and a[0, 0] == 0.0


def test_oracle_band_rasters_compose_the_full_frame():
    """One scan, then interleaved tile-row sets rastered one after another:
    each set's rows, tile records and PTCL equal the full frame's."""
    c = tk.generate(2, 7, width=320, height=272, paths=120)
    d = c.scene_desc()
    from oracle import OracleRun, OR_IMAGE, OR_PASS_TILES, OR_PASS_PTCL, OR_SEGMENTS
    full = OracleRun(d, threads=4)
    img = full.get(OR_IMAGE, np.uint32).reshape(272, 320)
    tiles = full.get(OR_PASS_TILES, N.TILE_DTYPE, 0)
    ptcl = full.get(OR_PASS_PTCL, N.PTCL_DTYPE, 0)
    tw, th = 20, 17
    part = OracleRun.prepare(d, threads=4)
    assert np.array_equal(part.get(OR_SEGMENTS, N.SEGMENT_DTYPE), full.get(OR_SEGMENTS, N.SEGMENT_DTYPE))
    seen = np.zeros(th, bool)
    for k in range(3):
        part.raster(k, 0, 3, threads=4)
        rows = np.arange(k, th, 3)
        seen[rows] = True
        pimg = part.get(OR_IMAGE, np.uint32).reshape(272, 320)
        ptiles = part.get(OR_PASS_TILES, N.TILE_DTYPE, 0)
        pptcl = part.get(OR_PASS_PTCL, N.PTCL_DTYPE, 0)
        for ty in range(th):
            px = slice(ty * 16, ty * 16 + 16)
            t = slice(ty * tw, ty * tw + tw)
            if ty in rows:
                assert np.array_equal(pimg[px], img[px])
                assert np.array_equal(ptiles["ptcl_count"][t], tiles["ptcl_count"][t])
                for i in range(ty * tw, ty * tw + tw):
                    a, b = int(ptiles["ptcl_start"][i]), int(ptiles["ptcl_end"][i])
                    e, f = int(tiles["ptcl_start"][i]), int(tiles["ptcl_end"][i])
                    assert pptcl[a:b].tobytes() == ptcl[e:f].tobytes()
            else:
                assert not ptiles["ptcl_count"][t].any()
                assert np.all(pimg[px] == c.scene_desc().clear_color)
    assert seen.all()


@pytest.mark.parametrize("config, kw", [
    (1, dict(width=640, height=360)),
    (2, dict(width=768, height=512, paths=600)),
    (2, dict(width=333, height=210, paths=150, variant=0)),
    (3, dict(width=480, height=270, paths=600)),
])
def test_oracle_pipeline_equals_fine_only_path_oracle(config, kw):
    """coarse_count/rect_pixels.rs:3-13's method for path fills: the oracle's
    full pipeline (bins, coarse elision, colour promotion, occlusion skip)
    gives the pixels of interpreting every draw in every tile."""
    from oracle import OracleRun, OR_IMAGE, interpret_path_draws
    c = tk.generate(config, 7, **kw)
    d = c.scene_desc()
    full = OracleRun(d, threads=8).get(OR_IMAGE, np.uint32).view(np.uint8).reshape(d.height, d.width, 4)
    only = interpret_path_draws(d, threads=8)
    assert np.array_equal(full, only), int((full != only).any(axis=2).sum())


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_opacity_layers_equal_fine_only_oracle(seed):
    """Fused opacity layers (BEGIN_OPACITY / END_OPACITY) nested with path
    and SDF clips: the full pipeline equals interpreting every layer and draw
    in every tile."""
    from oracle import OracleRun, OR_IMAGE, OR_PASS_PTCL, interpret_path_draws
    from layer_cases import opacity_scene
    c = opacity_scene(seed)
    d = c.scene_desc()
    assert (c.scene_arrays()["layers"]["tag"] == N.LAYER_OPACITY).sum() >= 4
    run = OracleRun(d, threads=8)
    tags = run.get(OR_PASS_PTCL, N.PTCL_DTYPE, 0)["tag"]
    assert (tags == N.PTCL_BEGIN_OPACITY).any() and (tags == N.PTCL_END_OPACITY).any()
    full = run.get(OR_IMAGE, np.uint32).view(np.uint8).reshape(d.height, d.width, 4)
    only = interpret_path_draws(d, threads=8)
    assert np.array_equal(full, only), int((full != only).any(axis=2).sum())


def test_opacity_layer_payload_and_fusion_rules():
    c = tk.Canvas(64, 64)
    sq = tk.BezPath().move_to(0, 0).line_to(64, 0).line_to(64, 64).line_to(0, 64).close()
    for op, want in [(0.6, 153), (1.0, 255), (0.0, 0), (-2.0, 0), (7.0, 255), (0.5, 128)]:
        c.push_opacity_layer(sq, op)
        c.push_path(sq, tk.Brush.solid(1, 0, 0, 1))
        c.pop_layer()
        layers = c.scene_arrays()["layers"]
        assert layers[-1]["tag"] == N.LAYER_OPACITY and layers[-1]["payload"] == want
    with pytest.raises(ValueError):
        c.push_opacity_layer(sq, float("nan"))
    # draws beside and inside a nested layer: the reference needs an
    # offscreen group there (Canvas::can_fuse is false)
    bad = tk.Canvas(64, 64)
    bad.push_opacity_layer(sq, 0.5)
    bad.push_path(sq, tk.Brush.solid(1, 0, 0, 1))
    bad.push_clip_layer(sq)
    bad.push_path(sq, tk.Brush.solid(0, 1, 0, 1))
    bad.pop_layer()
    bad.pop_layer()
    with pytest.raises(RuntimeError, match="offscreen group"):
        bad.scene_desc()
    # a nested layer alone under the opacity layer is one stack: fused
    ok = tk.Canvas(64, 64)
    ok.push_opacity_layer(sq, 0.5)
    ok.push_clip_layer(sq)
    ok.push_path(sq, tk.Brush.solid(0, 1, 0, 1))
    ok.pop_layer()
    ok.pop_layer()
    assert list(ok.scene_arrays()["layers"]["tag"]) == [N.LAYER_OPACITY, N.LAYER_CLIP]


def test_sampled_blur_factor_one_records_a_full_resolution_blur():
    from layer_cases import sampled_blur_scene
    a = sampled_blur_scene(3, 1, N.BLUR_DOWNSAMPLE_BOX, N.BLUR_UPSAMPLE_BILINEAR)
    ops = a.scene_arrays()["ops"]
    assert ops[ops["kind"] == N.OP_BLUR_BEGIN]["batch_id"].tolist() == [0]


@pytest.mark.parametrize("factor, down, up", [(2, 1, 1), (4, 1, 1), (3, 0, 0), (4, 1, 0), (8, 0, 1)])
def test_oracle_sampled_blur_stays_near_the_full_resolution_blur(factor, down, up):
    """A reduced-resolution blur (BlurSampling, filter/resample.hlsli)
    approximates the full-resolution Gaussian of the same group: uniform
    regions stay uniform and the images differ by a few levels at most."""
    from oracle import OracleRun, OR_IMAGE
    from layer_cases import sampled_blur_scene
    full = sampled_blur_scene(5, 1, 1, 1, sigma=8.0)
    red = sampled_blur_scene(5, factor, down, up, sigma=8.0)
    ops = red.scene_arrays()["ops"]
    assert ops[ops["kind"] == N.OP_BLUR_BEGIN]["batch_id"].tolist() == [N.blur_sampling(factor, down, up)]
    a = OracleRun(full.scene_desc(), threads=4).get(OR_IMAGE, np.uint32).view(np.uint8).reshape(150, 200, 4)
    b = OracleRun(red.scene_desc(), threads=4).get(OR_IMAGE, np.uint32).view(np.uint8).reshape(150, 200, 4)
    diff = np.abs(a.astype(int) - b.astype(int))
    assert np.median(diff) <= 1
    assert diff.max() <= (40 if up == 0 else 24)


def test_sampled_blur_rejects_bad_sampling():
    c = tk.Canvas(64, 64)
    for f, d, u in [(65, 1, 1), (2, 2, 1), (2, 1, 2)]:
        with pytest.raises(ValueError):
            c.push_blur_group(4.0, factor=f, downsample=d, upsample=u)
