"""GPU parity: the sm_100a path against the oracle through the C ABI.

Integer and index buffers (counts, backdrops, ranges, segments in their
canonical order, PTCL, tile records) must be bit-exact; pixels must match the
oracle within 1/255 per channel (the oracle and the kernels evaluate the same
f32 operations, so exact equality is expected and asserted separately).
"""
import numpy as np
import pytest

import oracle
import tileink_b200 as tk
from tileink_b200 import _native as N

from helpers import (BLUR_SIGMAS, BLUR_SIZES, PREFIX_LENGTHS, PREFIX_SEEDS, blur_config, blur_source,
                     count_case_inputs, count_segments, gaussian_f64, prefix_case)

pytestmark = pytest.mark.gpu

PIXEL_TOLERANCE = 1  # RGBA8 units


def compare_frame(renderer, canvas, threads=8, exact_pixels=True):
    d = canvas.scene_desc()
    img = renderer.render_to_image(canvas)
    ref = oracle.OracleRun(d, threads=threads)
    a = canvas.scene_arrays()
    # scan stage
    assert np.array_equal(renderer.debug(N.STAGE_COUNTS), ref.get(oracle.OR_COUNTS, np.uint32))
    assert np.array_equal(renderer.debug(N.STAGE_BACKDROPS), ref.get(oracle.OR_BACKDROPS, np.int32))
    assert np.array_equal(renderer.debug(N.STAGE_RANGES), ref.get(oracle.OR_RANGES, N.RANGE_DTYPE))
    segs = renderer.debug(N.STAGE_SEGMENTS)
    rsegs = ref.get(oracle.OR_SEGMENTS, N.SEGMENT_DTYPE)
    assert len(segs) == len(rsegs)
    assert segs.tobytes() == rsegs.tobytes()
    # coarse stage, per target pass
    for p in range(ref.pass_count):
        assert np.array_equal(renderer.debug(N.STAGE_TILES, p), ref.get(oracle.OR_PASS_TILES, N.TILE_DTYPE, p))
        assert np.array_equal(renderer.debug(N.STAGE_PTCL, p), ref.get(oracle.OR_PASS_PTCL, N.PTCL_DTYPE, p))
        assert np.array_equal(renderer.debug(N.STAGE_KINDS, p), ref.get(oracle.OR_PASS_KINDS, np.uint32, p))
    # pixels
    rimg = ref.get(oracle.OR_IMAGE, np.uint32).view(np.uint8).reshape(img.shape)
    diff = np.abs(img.astype(np.int16) - rimg.astype(np.int16))
    assert diff.max() <= PIXEL_TOLERANCE, diff.max()
    if exact_pixels:
        assert np.array_equal(img, rimg), int((diff > 0).sum())
    return img, ref


# --- stage harnesses: the reference's kernel acceptance cases ---------------------------
@pytest.mark.parametrize("lengths", PREFIX_LENGTHS)
@pytest.mark.parametrize("seed", PREFIX_SEEDS)
def test_gpu_prefix_matches_reference_case(renderer, lengths, seed):
    case = prefix_case(lengths, seed)
    ranges, cursors, bumps = renderer.stage_scan_prefix(case["counts"], case["paths"], case["init_ranges"],
                                                         case["init_cursors"])
    assert np.array_equal(ranges, case["ranges"])
    assert np.array_equal(cursors, case["cursors"])
    assert np.array_equal(bumps, case["totals"])


def test_gpu_prefix_long_paths_chain_across_items(renderer):
    rng = np.random.default_rng(3)
    paths = np.zeros(3, dtype=N.PATH_DTYPE)
    dims = [(37, 400), (1, 9000), (4096, 3)]  # stride, rows: several items per path
    off = 5
    for k, (w, h) in enumerate(dims):
        paths[k]["data_offset"] = off
        paths[k]["data_len"] = w * h
        paths[k]["tile_x1"], paths[k]["tile_y1"] = w, h
        paths[k]["segment_start"] = 1000 * k + 7
        off += w * h + 11
    counts = rng.integers(0, 5, off).astype(np.uint32)
    init_r = np.zeros(off, dtype=N.RANGE_DTYPE)
    init_r["start"] = 0xABCD
    init_c = np.full(off, 0xABCD, dtype=np.uint32)
    ranges, cursors, bumps = renderer.stage_scan_prefix(counts, paths, init_r, init_c)
    er, ec, eb = init_r.copy(), init_c.copy(), np.zeros(3, dtype=np.uint32)
    oracle.lib().or_scan_prefix(N.ptr(counts), N.ptr(paths), 3, N.ptr(er), N.ptr(ec), N.ptr(eb))
    assert np.array_equal(ranges, er) and np.array_equal(cursors, ec) and np.array_equal(bumps, eb)


def test_gpu_count_matches_oracle_and_planner_with_guards(renderer):
    for a, b in count_segments():
        for p0, p1 in ((a, b), (b, a)):
            line, path, init = count_case_inputs(p0, p1)
            bd, cnt = renderer.stage_scan_count(line, path, init.view(np.int32), init)
            ebd, ecnt = init.view(np.int32).copy(), init.copy()
            oracle.lib().or_scan_count(N.ptr(line), 1, N.ptr(path), 1, N.ptr(ebd), N.ptr(ecnt))
            assert np.array_equal(bd, ebd) and np.array_equal(cnt, ecnt), (p0, p1)
            assert int(cnt[7:71].sum()) == tk.plan_line_tile_count(line[0], (0, 0, 8, 8))


@pytest.mark.parametrize("size", BLUR_SIZES)
def test_gpu_blur_matches_oracle_and_f64_gaussian(renderer, size):
    width, height = size
    src = blur_source(width, height)
    untouched = np.full(width * height, int.from_bytes(bytes([29, 31, 37, 113]), "little"), dtype=np.uint32)
    for sigma in BLUR_SIGMAS:
        for axis in (0, 1):
            for inset in (False, True):
                region, source = blur_config(width, height, inset)
                out = renderer.stage_blur(src, untouched, width, height, region, source, sigma, axis)
                exp = untouched.copy()
                reg = np.array(region, dtype=np.uint32)
                srcb = np.array(source, dtype=np.uint32)
                oracle.lib().or_blur_pass(N.ptr(src), N.ptr(exp), width, height, N.ptr(reg), N.ptr(srcb),
                                          np.float32(sigma), axis)
                assert np.array_equal(out, exp), (size, sigma, axis, inset)
                o8 = out.view(np.uint8).reshape(-1, 4)
                s32 = float(np.float32(sigma))
                for y in range(region[1], region[1] + region[3]):
                    for x in range(region[0], region[0] + region[2]):
                        g = gaussian_f64(src, width, height, source, x, y, s32, axis)
                        assert np.abs(o8[y * width + x].astype(int) - g.astype(int)).max() <= 1


# --- whole frames ---------------------------------------------------------------------
def test_gpu_frame_small_cubic_fills(renderer):
    """640x360, 240 closed cubic paths, nonzero, alpha 0.3-1 over white."""
    compare_frame(renderer, tk.generate(1, 1))


def test_gpu_frame_mixed_clips_gradients_strokes(renderer):
    c = tk.generate(2, 7, width=768, height=512, paths=600)
    img, ref = compare_frame(renderer, c)
    assert ref.batch_count > 3


def test_gpu_frame_glyphs(renderer):
    compare_frame(renderer, tk.generate(3, 3, width=480, height=270, paths=1500))


def test_gpu_frame_blur_group(renderer):
    compare_frame(renderer, tk.generate(5, 5, width=256, height=192, paths=24))


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
def test_gpu_frame_uneven_scenes(renderer, variant):
    compare_frame(renderer, tk.generate(4, 11, variant=variant))


def test_gpu_device_segment_plan_equals_host_plan(renderer):
    host = tk.generate(1, 4, width=300, height=200, paths=40)
    dev = tk.generate(1, 4, width=300, height=200, paths=40, device_segment_plan=True)
    ha, da = host.scene_arrays(), dev.scene_arrays()
    assert np.all(da["paths"]["segment_capacity"] == 0)
    img_h = renderer.render_to_image(host).copy()
    segs_h = renderer.debug(N.STAGE_SEGMENTS).copy()
    img_d = renderer.render_to_image(dev).copy()
    paths_d = renderer.debug(N.STAGE_PATHS)
    assert np.array_equal(paths_d["segment_start"], ha["paths"]["segment_start"])
    assert np.array_equal(paths_d["segment_capacity"], ha["paths"]["segment_capacity"])
    assert renderer.debug(N.STAGE_SEGMENTS).tobytes() == segs_h.tobytes()
    assert np.array_equal(img_h, img_d)


def test_gpu_render_is_deterministic_across_frames(renderer):
    c = tk.generate(2, 8, width=512, height=512, paths=400)
    renderer.upload(c)
    renderer.render()
    a = renderer.readback().copy()
    sa = renderer.debug(N.STAGE_SEGMENTS).copy()
    renderer.render()
    b = renderer.readback().copy()
    assert np.array_equal(a, b)
    assert renderer.debug(N.STAGE_SEGMENTS).tobytes() == sa.tobytes()


# --- edge cases -------------------------------------------------------------------------
def test_gpu_empty_scene_is_clear_color(renderer):
    c = tk.Canvas(37, 19)
    c.set_clear_color(0x80402010)
    img = renderer.render_to_image(c)
    assert np.all(img.reshape(-1, 4).view(np.uint32) == 0x80402010)


def test_gpu_paths_outside_and_on_tile_edges(renderer):
    cv = tk.Canvas(100, 70)
    cv.set_clear_color(0xFFFFFFFF)
    b = tk.Brush.solid(0.2, 0.4, 0.9, 0.8)
    cv.push_path(tk.BezPath().move_to(-50, -50).line_to(-10, -50).line_to(-10, -10).close(), b)  # off canvas
    cv.push_path(tk.BezPath().move_to(16, 16).line_to(48, 16).line_to(48, 48).line_to(16, 48).close(), b)
    cv.push_path(tk.BezPath().move_to(-20, 30).line_to(130, 31).line_to(120, 90).close(), b,
                 fill_rule=tk.FILL_EVEN_ODD)
    cv.push_path(tk.BezPath().move_to(64, 0).line_to(64, 70).line_to(64.5, 70).line_to(64.5, 0).close(), b)
    compare_frame(renderer, cv)


def test_gpu_nested_clips_deeper_than_register_stack(renderer):
    cv = tk.Canvas(96, 96)
    cv.set_clear_color(0xFFFFFFFF)
    for k in range(7):  # clip depth 7 > 4 register slots
        s = 2 + k * 3
        cv.push_clip_layer(tk.BezPath().move_to(s, s + 1).line_to(96 - s, s).line_to(90 - s, 96 - s)
                           .line_to(s + 2, 94 - s).close())
    cv.push_path(tk.BezPath().move_to(0, 0).line_to(96, 10).line_to(80, 96).line_to(5, 90).close(),
                 tk.Brush.solid(1, 0, 0, 0.9))
    for _ in range(7):
        cv.pop_layer()
    compare_frame(renderer, cv)


def test_gpu_rejects_invalid_scenes(renderer):
    c = tk.generate(1, 1, width=64, height=64, paths=3)
    arrays = c.scene_arrays()
    bad = dict(arrays)
    bad["ops"] = arrays["ops"].copy()
    bad["ops"]["kind"] = 7
    with pytest.raises(tk.TileinkError) as e:
        renderer.upload(N.ArrayScene(bad))
    assert e.value.code == N.TK_E_INVALID
    bad = dict(arrays)
    bad["paths"] = arrays["paths"].copy()
    bad["paths"][1]["line_start"] += 1
    with pytest.raises(tk.TileinkError):
        renderer.upload(N.ArrayScene(bad))
    bad = dict(arrays)
    bad["draws"] = arrays["draws"].copy()
    bad["draws"][0]["sdf_offset"] = 0
    with pytest.raises(tk.TileinkError):
        renderer.upload(N.ArrayScene(bad))
    # a valid scene still renders after the rejections
    renderer.render_to_image(c)


def test_gpu_line_path_mismatch_is_reported(renderer):
    c = tk.generate(1, 1, width=64, height=64, paths=3)
    arrays = c.scene_arrays()
    bad = dict(arrays)
    bad["lines"] = arrays["lines"].copy()
    bad["lines"][0]["path_id"] = 2
    renderer.upload(N.ArrayScene(bad))
    renderer.render()
    with pytest.raises(tk.TileinkError):
        renderer.readback()
    renderer.render_to_image(c)
