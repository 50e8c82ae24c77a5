"""Glyph outline compositing (PTCL_PATH_GLYPH) on CPU: the oracle's pow
against the C library's, its text coverage correction and source-over
(fine/text/{gamma,auto,basic}.hlsli) against an independent float32 restatement
in numpy, and the Canvas records the reference's push_text_layout_as_path
makes (src/canvas/primitives/text.rs:107-147, src/text/tests/recording.rs:41)."""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
import tileink_b200 as tk
from tileink_b200 import _native as N

F = np.float32


def test_text_pow_is_the_correctly_rounded_pow():
    """x^2.4 and x^(1/2.4) over the ranges the sRGB transfer uses: the
    double-precision evaluation rounds to the float nearest the true power
    (within one float ulp of the C library's double pow, and equal to it
    rounded almost always)."""
    lib = oracle.lib()
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(0.0031308, 1.0, 20000), np.linspace(0.09, 1.0, 2000)]).astype(np.float32)
    exact = 0
    for y in (F(2.4), F(1.0) / F(2.4)):
        for x in xs:
            got = F(lib.or_text_pow(float(x), float(y)))
            want = F(math.pow(float(x), float(y)))
            assert abs(int(got.view(np.int32)) - int(want.view(np.int32))) <= 1, (x, y, got, want)
            exact += got == want
    assert exact >= 0.9999 * 2 * len(xs)
    assert lib.or_text_pow(1.0, 2.4) == 1.0


def np_srgb_to_linear(v):
    v = F(min(max(v, F(0)), F(1)))
    r = F(v / F(12.92))
    if v > F(0.04045):
        r = F(math.pow(float(F((v + F(0.055)) / F(1.055))), float(F(2.4))))
    return r


def np_linear_to_srgb(v):
    v = F(min(max(v, F(0)), F(1)))
    r = F(v * F(12.92))
    if v > F(0.0031308):
        r = F(F(F(1.055) * F(math.pow(float(v), float(F(1.0) / F(2.4))))) - F(0.055))
    return r


def np_glyph_over(dst, src, cov):
    """src_over_mask_linear_auto_u8 restated in numpy float32."""
    sa = src >> 24
    if sa == 0 or cov == 0:
        return dst
    alpha = F(sa)
    ch = [F(min(max(F(F((src >> s) & 255) / alpha), F(0)), F(1))) for s in (0, 8, 16)]
    fg = F(F(F(ch[0] * F(0.2126)) + F(ch[1] * F(0.7152))) + F(ch[2] * F(0.0722)))
    if cov in (0, 255):
        c = F(F(cov) * F(F(1) / F(255)))
    else:
        raw = F(F(cov) * F(F(1) / F(255)))
        bg = F(F(1) - fg)
        bgl = np_srgb_to_linear(bg)
        enh = F(raw + F(F(raw * F(F(1) - raw)) * bgl))
        diff = F(fg - bg)
        if abs(diff) < F(1) / F(256):
            c = enh
        else:
            fgl = np_srgb_to_linear(fg)
            out = np_linear_to_srgb(F(bgl + F(enh * F(fgl - bgl))))
            c = F(min(max(F(F(out - bg) / diff), F(0)), F(1)))
    if c == 0:
        return dst
    if (dst >> 24) != 255:
        c = F(F(F(c + c) + c) / F(3))
    a = F(F(sa) * F(F(1) / F(255)))
    amount = F(a * c)
    keep = F(F(1) - amount)
    out = [F(F(F((src >> s) & 255) * c) + F(F((dst >> s) & 255) * keep)) for s in (0, 8, 16)]
    oa = F(F(amount * F(255)) + F(F(dst >> 24) * keep))
    q = [int(F(v + F(0.5))) for v in out + [oa]]
    return q[0] | (q[1] << 8) | (q[2] << 16) | (q[3] << 24)


def test_glyph_composite_matches_a_float32_restatement():
    lib = oracle.lib()
    rng = np.random.default_rng(2)
    cases = 0
    for _ in range(6000):
        a = int(rng.integers(0, 256))
        src = int(rng.integers(0, a + 1)) | (int(rng.integers(0, a + 1)) << 8) | (int(rng.integers(0, a + 1)) << 16) \
            | (a << 24)
        if rng.uniform() < 0.3:
            src = (255 << 24) | int(rng.choice([0, 0x808080, 0xFFFFFF]))  # black, grey and white text
        da = int(rng.choice([255, int(rng.integers(0, 256))]))
        dst = int(rng.integers(0, da + 1)) | (int(rng.integers(0, da + 1)) << 8) | (int(rng.integers(0, da + 1)) << 16) \
            | (da << 24)
        cov = int(rng.integers(0, 256))
        got = lib.or_glyph_over(dst, src, cov)
        want = np_glyph_over(dst, src, cov)
        for s in (0, 8, 16, 24):
            assert abs(((got >> s) & 255) - ((want >> s) & 255)) <= 1, (hex(dst), hex(src), cov, hex(got), hex(want))
        cases += got == want
    assert cases >= 5900  # differences only where the two pows round apart


def test_glyph_composite_known_values():
    lib = oracle.lib()
    white, black = 0xFFFFFFFF, 0xFF000000
    assert lib.or_glyph_over(white, black, 0) == white
    assert lib.or_glyph_over(white, black, 255) == black
    assert lib.or_glyph_over(white, 0x00000000, 128) == white
    # black text on white at half coverage: the correction's coverage is
    # (1 - linear_to_srgb(1 - enhanced)) with enhanced = raw + raw (1 - raw),
    # 0.464 for raw = 128/255, so the grey is lighter than plain source-over's
    # 127: 255 - 0.464 * 255 = 136.7 -> 136
    half = lib.or_glyph_over(white, black, 128)
    assert half == 0xFF888888 == np_glyph_over(white, black, 128)


def test_canvas_records_glyph_outlines_as_path_glyph_draws():
    c = tk.Canvas(64, 32)
    p = tk.BezPath().move_to(4, 4).line_to(20, 6).quad_to(24, 20, 8, 24).close()
    d = c.push_glyph_outlines(p, tk.Brush.solid(0, 0, 0, 1))
    a = c.scene_arrays()
    assert a["draws"]["tag"][d] == N.DRAW_PATH_GLYPH
    assert a["draws"]["fill_rule"][d] == N.FILL_NONZERO
    plain = tk.Canvas(64, 32)
    plain.push_path(p, tk.Brush.solid(0, 0, 0, 1))
    b = plain.scene_arrays()
    assert np.array_equal(a["lines"], b["lines"]) and np.array_equal(a["paths"], b["paths"])
    # the oracle renders them with the text composite: partial pixels differ
    # from the plain fill, covered and uncovered pixels do not
    ia = oracle.OracleRun(c.scene_desc(), threads=1).get(oracle.OR_IMAGE, np.uint32)
    ib = oracle.OracleRun(plain.scene_desc(), threads=1).get(oracle.OR_IMAGE, np.uint32)
    differ = ia != ib
    assert differ.any() and differ.mean() < 0.2
    assert np.array_equal(ia[ib == 0xFFFFFFFF], ib[ib == 0xFFFFFFFF])


def test_retained_replay_keeps_glyph_outlines():
    c = tk.Canvas(64, 32)
    c.keep_commands()
    c.push_glyph_outlines(tk.BezPath().move_to(4, 4).line_to(20, 6).line_to(8, 24).close(), tk.Brush.solid(0, 0, 0, 1))
    rs = tk.RetainedScene(64, 32)
    rs.insert(1, c)
    m, _ = rs.materialize()
    assert list(m.scene_arrays()["draws"]["tag"]) == [N.DRAW_PATH_GLYPH]


@pytest.mark.parametrize("seed", [3])
def test_c3_glyphs_are_path_glyph_draws(seed):
    c = tk.generate(3, seed, width=240, height=135, paths=60)
    tags = c.scene_arrays()["draws"]["tag"]
    assert len(tags) == 60 and (tags == N.DRAW_PATH_GLYPH).all()


@pytest.mark.parametrize("seed, sdf, clip", [(1, False, False), (4, True, True)])
def test_oracle_glyph_pipeline_equals_fine_only(seed, sdf, clip):
    """Coarse for glyph outline draws, pinned by the fine-only method
    (src/native/runtime/tests/coarse_count/rect_pixels.rs:3-14): every draw
    as a particle in every tile of its bbox gives the pipeline's image."""
    from text_cases import glyph_scene
    c = glyph_scene(seed, sdf=sdf, clip=clip)
    d = c.scene_desc()
    run = oracle.OracleRun(d, threads=4)
    img = run.get(oracle.OR_IMAGE, np.uint32).view(np.uint8).reshape(d.height, d.width, 4)
    assert (run.get(oracle.OR_PASS_PTCL, N.PTCL_DTYPE, 0)["tag"] == N.PTCL_PATH_GLYPH).sum() > 50
    assert np.array_equal(img, oracle.interpret_path_draws(d, threads=4))


@pytest.mark.parametrize("seed, clip, outlines", [(1, False, False), (2, True, True)])
def test_oracle_glyph_run_pipeline_equals_fine_only(seed, clip, outlines):
    """Coarse glyph lists (coarse/text.hlsli: a glyph enters a tile's list when
    its image, a pixel wider, meets the tile) pinned by the fine-only method:
    every glyph of every run in every tile gives the same image."""
    from text_cases import glyph_run_scene
    c = glyph_run_scene(seed, clip=clip, outlines=outlines)
    d = c.scene_desc()
    run = oracle.OracleRun(d, threads=4)
    img = run.get(oracle.OR_IMAGE, np.uint32).view(np.uint8).reshape(d.height, d.width, 4)
    ptcl = run.get(oracle.OR_PASS_PTCL, N.PTCL_DTYPE, 0)
    glyphs = run.get(oracle.OR_PASS_GLYPHS, np.uint32, 0)
    tiles = run.get(oracle.OR_PASS_TILES, N.TILE_DTYPE, 0)
    g = ptcl[ptcl["tag"] == N.PTCL_GLYPH]
    assert len(g) > 20 and (g["segment_end"] > g["segment_start"]).all()
    assert tiles["glyph_count"].sum() == len(glyphs) and tiles["glyph_end"][-1] == len(glyphs)
    assert not np.array_equal(img, np.full_like(img, 0))
    assert np.array_equal(img, oracle.interpret_path_draws(d, threads=4))


def test_glyph_run_records():
    """push_text_layout's draw record (src/canvas/primitives/text.rs:80-96):
    a brush draw with no path, the run's glyphs and bounds from its images."""
    c = tk.Canvas(64, 48)
    im = c.add_glyph_image(1, 10, np.full((12, 6), 255, np.uint32), N.GLYPH_MASK)
    assert c.add_glyph_image(1, 10, np.full((12, 6), 255, np.uint32), N.GLYPH_MASK) == im + 1  # other texels
    d = c.push_glyph_run([(im, 10, 30), (None, 20, 30), (im, 30, 32)], tk.Brush.solid(0, 0, 0, 1))
    a = c.scene_arrays()
    r = a["draws"][d]
    assert r["path_id"] == N.INVALID and r["glyph_run_id"] == 0 and r["tag"] == N.DRAW_BRUSH
    assert tuple(r["pixel_bounds"]) == (11, 20, 37, 34)
    assert list(a["glyph_runs"][0]) == [0, 3]
    assert a["glyphs"]["image"][1] == N.INVALID
    d2 = c.push_glyph_run([(im, 10, 30)], tk.Brush.solid(0, 0, 0, 1), clip=(0, 0, 14, 100))
    assert tuple(c.scene_arrays()["draws"][d2]["pixel_bounds"]) == (11, 20, 14, 32)
    with pytest.raises(ValueError):
        c.push_glyph_run([(im, 10, 30)], tk.Brush.solid(0, 0, 0, 1), clip=(40, 0, 50, 10))
    with pytest.raises(ValueError):
        c.push_glyph_run([(im + 5, 10, 30)], tk.Brush.solid(0, 0, 0, 1))


def test_retained_replay_moves_glyph_runs_by_whole_pixels():
    c = tk.Canvas(64, 48)
    c.keep_commands()
    im = c.add_glyph_image(0, 8, np.full((8, 5), 200, np.uint32), N.GLYPH_MASK)
    c.push_glyph_run([(im, 4, 20), (im, 10, 20)], tk.Brush.solid(0, 0, 0, 1))
    rs = tk.RetainedScene(64, 48)
    rs.insert(1, c)
    rs.set_transform(1, (1, 0, 0, 1, 7, 3))
    m, _ = rs.materialize()
    a = m.scene_arrays()
    assert list(a["glyphs"]["x"]) == [11, 17] and list(a["glyphs"]["y"]) == [23, 23]
    assert len(a["glyph_images"]) == 1 and len(a["glyph_texels"]) == 40
