"""GPU parity of analytic SDF shapes (PTCL_SDF, fine/interpreter.hlsli:70-84;
coarse/emit_draw.hlsli:22-30): PTCL, tile records, tile kinds and pixels of
the sm_100a path equal the oracle's bit for bit, in single scenes next to path
fills, clips and blur groups, in batched mode and in incremental frames."""
from __future__ import annotations

import numpy as np
import pytest

import tileink_b200 as tk
from tileink_b200 import _native as N

from test_gpu_parity import compare_frame
from test_gpu_batch import check_batch_against_serial, serial_outputs

pytestmark = pytest.mark.gpu


def gradient(rng, w, h):
    stops = [(0.0, tuple(rng.uniform(0, 1, 3)) + (float(rng.uniform(0.3, 1)),)),
             (1.0, tuple(rng.uniform(0, 1, 3)) + (float(rng.uniform(0.3, 1)),))]
    if rng.uniform() < 0.5:
        return tk.Brush.linear(tuple(rng.uniform(0, w, 2)), tuple(rng.uniform(0, h, 2)), stops)
    return tk.Brush.radial(tuple(rng.uniform(0, w, 2)), 0.0, tuple(rng.uniform(0, h, 2)), float(rng.uniform(20, 200)),
                           stops)


def random_shapes(c, rng, n, w, h):
    """n seeded SDF shapes of every supported kind, solid or gradient paint,
    degenerate sizes included."""
    for k in range(n):
        b = gradient(rng, w, h) if rng.uniform() < 0.25 else tk.Brush.solid(*rng.uniform(0, 1, 3),
                                                                          float(rng.choice([1.0, rng.uniform(0.2, 1)])))
        x0, y0 = rng.uniform(-20, w), rng.uniform(-20, h)
        sw, sh = rng.choice([0.0, 0.4, rng.uniform(1, 30), rng.uniform(30, 260)], 2)
        radii = rng.choice([0.0, rng.uniform(0, 12), rng.uniform(0, 400)]) if rng.uniform() < 0.5 else \
            tuple(rng.uniform(0, 20, 4))
        kind = k % 8
        if kind == 0:
            c.push_rect(x0, y0, x0 + sw, y0 + sh, b, radius=radii)
        elif kind == 1:
            widths = rng.uniform(0, 8) if rng.uniform() < 0.5 else tuple(rng.uniform(-1, 10, 4))
            c.push_rect_stroke(x0, y0, x0 + sw, y0 + sh, widths, b, radius=radii)
        elif kind == 2:
            c.push_circle(x0, y0, float(rng.choice([0.0, rng.uniform(0.3, 3), rng.uniform(3, 120)])), b)
        elif kind == 3:
            c.push_circle_stroke(x0, y0, float(rng.uniform(0, 90)), float(rng.uniform(0.2, 12)), b)
        elif kind == 4:
            x1, y1 = (x0, y0) if rng.uniform() < 0.1 else (x0 + rng.uniform(-200, 200), y0 + rng.uniform(-200, 200))
            c.push_line(x0, y0, x1, y1, float(rng.uniform(0.3, 9)), b, cap=int(rng.integers(0, 3)))
        elif kind == 5:
            c.push_rect_shadow(x0, y0, x0 + sw, y0 + sh, b, offset=tuple(rng.uniform(-6, 6, 2)),
                               expand=float(rng.choice([0.0, rng.uniform(0.5, 12)])),
                               intensity=float(rng.uniform(0.1, 1.0)), radius=radii)
        elif kind == 6:
            c.push_circle_shadow(x0, y0, float(rng.uniform(1, 60)), b, offset=tuple(rng.uniform(-6, 6, 2)),
                                 expand=float(rng.uniform(0, 10)), intensity=float(rng.uniform(0.1, 1.0)))
        else:
            c.push_line_shadow(x0, y0, x0 + rng.uniform(-150, 150), y0 + rng.uniform(-150, 150),
                               float(rng.uniform(0.5, 8)), b, offset=tuple(rng.uniform(-6, 6, 2)),
                               expand=float(rng.uniform(0, 8)), intensity=float(rng.uniform(0.1, 1.0)),
                               cap=int(rng.integers(0, 3)))


def extended_shapes(c, rng, n, w, h):
    """n seeded shapes of the extended kinds (triangles, dash lines,
    checkerboards, candlesticks, callouts, arcs and stars, with their
    strokes and shadows), degenerate ones included."""
    for k in range(n):
        b = gradient(rng, w, h) if rng.uniform() < 0.25 else tk.Brush.solid(*rng.uniform(0, 1, 3),
                                                                          float(rng.choice([1.0, rng.uniform(0.2, 1)])))
        x0, y0 = rng.uniform(-20, w), rng.uniform(-20, h)
        kind = k % 11
        if kind >= 7:  # arcs and stars, fill, stroke and shadow
            r = float(rng.uniform(2, 80))
            if kind == 7:
                c.push_sdf_arc(x0, y0, r, float(rng.uniform(-7, 7)), float(rng.choice([rng.uniform(-7, 7), 6.3, -0.01])),
                               float(rng.uniform(0.5, 12)), b, cap=int(rng.integers(0, 3)))
            elif kind == 8:
                c.push_arc_shadow(x0, y0, r, float(rng.uniform(-7, 7)), float(rng.uniform(-7, 7)),
                                  float(rng.uniform(0.5, 12)), b, offset=tuple(rng.uniform(-5, 5, 2)),
                                  expand=float(rng.uniform(0, 6)), intensity=float(rng.uniform(0.2, 1)),
                                  cap=int(rng.integers(0, 3)))
            elif kind == 9:
                c.push_star(x0, y0, r, r * float(rng.uniform(0.2, 0.95)), b, corner_radius=float(rng.uniform(0, 4)),
                            rotation=float(rng.uniform(-4, 4)))
            else:
                c.push_star_stroke(x0, y0, r, r * float(rng.uniform(0.2, 0.95)), float(rng.uniform(0.5, 6)), b,
                                   corner_radius=float(rng.uniform(0, 4)), rotation=float(rng.uniform(-4, 4)))
        elif kind >= 4:  # callouts: fill, stroke, shadow
            rect = (x0, y0, x0 + rng.uniform(1, 160), y0 + rng.uniform(1, 120))
            tail = None if rng.uniform() < 0.2 else (int(rng.integers(0, 4)), float(rng.uniform(-20, 180)),
                                                     float(rng.uniform(0.5, 60)), float(rng.uniform(0.5, 40)),
                                                     float(rng.uniform(0, 10)))
            body_radius = float(rng.choice([0.0, rng.uniform(0, 30)]))
            if kind == 4:
                c.push_callout(rect, body_radius, tail, b)
            elif kind == 5:
                c.push_callout_stroke(rect, body_radius, tail, float(rng.uniform(0.5, 8)), b)
            else:
                c.push_callout_shadow(rect, body_radius, tail, b, offset=tuple(rng.uniform(-6, 6, 2)),
                                      expand=float(rng.uniform(0, 8)), intensity=float(rng.uniform(0.2, 1)))
        elif kind == 0:
            pts = [(x0, y0)] + [(x0 + rng.uniform(-90, 90), y0 + rng.uniform(-90, 90)) for _ in range(2)]
            if rng.uniform() < 0.1:
                pts[2] = (pts[0][0] + 1e-3, pts[0][1] + 2e-3)  # a sliver
            c.push_triangle(*pts, b, corner_radius=float(rng.choice([0.0, rng.uniform(0, 6)])))
        elif kind == 1:
            c.push_dash_line(x0, y0, x0 + rng.uniform(-250, 250), y0 + rng.uniform(-250, 250),
                             float(rng.uniform(0.5, 6)), float(rng.uniform(0.5, 20)),
                             float(rng.choice([0.0, rng.uniform(0.5, 15)])), b, cap=int(rng.integers(0, 3)),
                             dash_offset=float(rng.uniform(-30, 30)))
        elif kind == 2:
            c.push_checkerboard(x0, y0, x0 + rng.uniform(1, 200), y0 + rng.uniform(1, 200),
                                float(rng.choice([rng.uniform(0.3, 2), rng.uniform(2, 40)])), b,
                                tk.Brush.solid(*rng.uniform(0, 1, 3), 1.0))
        else:
            top, bottom = rng.uniform(y0, y0 + 120, 2)
            c.push_candlestick(x0, y0, y0 + rng.uniform(0, 160), top, float(rng.choice([bottom, top])),
                               int(rng.integers(1, 15)), int(rng.integers(1, 4)), b)


def cubic_path(rng, w, h, n=6):
    p = tk.BezPath()
    cx, cy = rng.uniform(0, w), rng.uniform(0, h)
    p.move_to(cx, cy)
    for _ in range(n):
        p.cubic_to(*(rng.uniform(-80, 80, 6) + np.tile([cx, cy], 3)))
    p.close()
    return p


def kinds_scene(rng):
    W, H = 400, 300
    c = tk.Canvas(W, H)
    c.set_clear_color(0xFFFFFFFF)
    c.push_rect(8, 8, 392, 292, tk.Brush.solid(0.95, 0.95, 0.9, 1.0))  # opaque background: COLOR tiles
    c.push_rect(30.5, 20.25, 210, 140, tk.Brush.solid(0.2, 0.3, 0.8, 1.0), radius=(0, 6, 18, 40))
    c.push_rect_stroke(220, 20, 380, 160, (2, 4, 6, 8), tk.Brush.solid(0.9, 0.2, 0.1, 0.9), radius=12)
    c.push_circle(120, 200, 60.5, gradient(rng, W, H))
    c.push_circle_stroke(300, 220, 50, 7, tk.Brush.solid(0.1, 0.6, 0.2, 0.7))
    c.push_line(10, 290, 390, 170, 5, tk.Brush.solid(0.0, 0.0, 0.0, 1.0), cap=N.CAP_ROUND)
    c.push_line(40, 250, 40, 250, 9, tk.Brush.solid(0.5, 0.0, 0.5, 1.0), cap=N.CAP_SQUARE)
    c.push_rect_shadow(60, 40, 160, 110, tk.Brush.solid(0, 0, 0, 1), offset=(4, 6), expand=8, intensity=0.6,
                       radius=10)
    c.push_path(cubic_path(rng, W, H), tk.Brush.solid(0.8, 0.5, 0.1, 0.8), fill_rule=1)
    c.push_clip_layer(cubic_path(rng, W, H, 8))
    c.push_rect(100, 100, 300, 250, gradient(rng, W, H))
    c.push_circle_shadow(200, 150, 40, tk.Brush.solid(0.2, 0.0, 0.4, 1), expand=5, intensity=0.8)
    c.pop_layer()
    c.push_blur_group(3.0)
    c.push_line_shadow(20, 20, 200, 280, 4, tk.Brush.solid(0.1, 0.1, 0.1, 1), offset=(2, 2), expand=3)
    c.push_rect(250, 180, 330, 260, tk.Brush.solid(0.9, 0.9, 0.0, 1.0), radius=20)
    c.pop_layer()
    return c


def test_gpu_sdf_kinds_beside_paths_and_clips(renderer):
    c = kinds_scene(np.random.default_rng(7))
    compare_frame(renderer, c)
    # the batches' tile kinds (BATCH_BEGIN colour words)
    ptcl = renderer.debug(N.STAGE_PTCL, 0)
    kinds = ptcl["color"][ptcl["tag"] == N.PTCL_BATCH_BEGIN] & 7
    for k in (N.TILE_KIND_COLOR, N.TILE_KIND_SDF, N.TILE_KIND_INTERPRETER):
        assert (kinds == k).any(), k
    # MIXED tiles: colours and solid rect edges only (fine/specialized.hlsli:47-108 in the oracle)
    m = tk.Canvas(96, 80)
    m.push_rect(0, 0, 96, 80, tk.Brush.solid(0.9, 0.9, 0.9, 1.0))
    m.push_rect(5.5, 7.25, 60, 41.5, tk.Brush.solid(0.1, 0.2, 0.3, 0.7), radius=(3, 0, 9, 1.5))
    m.push_rect(40, 30, 90.75, 70, tk.Brush.solid(0.6, 0.1, 0.1, 1.0))
    compare_frame(renderer, m)
    ptcl = renderer.debug(N.STAGE_PTCL, 0)
    assert ((ptcl["color"][ptcl["tag"] == N.PTCL_BATCH_BEGIN] & 7) == N.TILE_KIND_MIXED).any()


@pytest.mark.parametrize("seed,scale", [(1, 1.0), (2, 1.5), (3, 0.75)])
def test_gpu_random_sdf_scenes(renderer, seed, scale):
    W, H = 480, 360
    rng = np.random.default_rng(seed)
    c = tk.Canvas(W, H, scale=scale)
    c.set_clear_color(0xFF202020)
    random_shapes(c, rng, 240, W, H)
    for _ in range(10):
        c.push_path(cubic_path(rng, W, H), tk.Brush.solid(*rng.uniform(0, 1, 3), 0.6))
    random_shapes(c, rng, 60, W, H)
    compare_frame(renderer, c)


@pytest.mark.parametrize("seed,scale", [(11, 1.0), (12, 1.25)])
def test_gpu_extended_sdf_kinds(renderer, seed, scale):
    W, H = 480, 360
    rng = np.random.default_rng(seed)
    c = tk.Canvas(W, H, scale=scale)
    c.set_clear_color(0xFF303030)
    extended_shapes(c, rng, 160, W, H)
    random_shapes(c, rng, 40, W, H)
    c.push_clip_layer(cubic_path(rng, W, H, 8))
    extended_shapes(c, rng, 40, W, H)
    c.pop_layer()
    compare_frame(renderer, c)


def sdf_scene(seed, w, h, n):
    rng = np.random.default_rng(seed)
    c = tk.Canvas(w, h)
    random_shapes(c, rng, n, w, h)
    return c


def test_gpu_sdf_batch_matches_serial(renderer):
    scenes = [sdf_scene(50 + i, 96 + 64 * i, 80 + 48 * i, 30 + 20 * i) for i in range(6)]
    ext = tk.Canvas(200, 150)
    extended_shapes(ext, np.random.default_rng(60), 40, 200, 150)
    scenes.append(ext)
    scenes += [tk.generate(4, 9)]
    serial = [serial_outputs(renderer, c) for c in scenes]
    r = tk.NativeRenderer(0)
    try:
        r.batch_upload(scenes)
        r.batch_render()
        check_batch_against_serial(r, scenes, serial)
    finally:
        r.close()


def small_shapes(c, rng, ox, oy):
    """One of each SDF kind, within about 40 pixels of (ox, oy)."""
    b = lambda: tk.Brush.solid(*rng.uniform(0, 1, 3), float(rng.uniform(0.4, 1)))
    r = lambda lo, hi: float(rng.uniform(lo, hi))
    c.push_rect(ox, oy, ox + r(5, 30), oy + r(5, 30), b(), radius=r(0, 6))
    c.push_rect_stroke(ox + 3, oy + 3, ox + r(10, 35), oy + r(10, 35), r(0.5, 4), b(), radius=(1, 2, 3, 4))
    c.push_circle(ox + r(5, 30), oy + r(5, 30), r(2, 10), b())
    c.push_circle_stroke(ox + 20, oy + 20, r(5, 15), r(0.5, 3), b())
    c.push_line(ox, oy + r(0, 30), ox + r(5, 35), oy + r(0, 30), r(0.5, 4), b(), cap=int(rng.integers(0, 3)))
    c.push_rect_shadow(ox + 5, oy + 5, ox + 25, oy + 20, b(), offset=(2, 3), expand=r(0, 3), intensity=0.6)
    c.push_circle_shadow(ox + 15, oy + 15, r(3, 8), b(), expand=r(0, 2), intensity=0.8)
    c.push_line_shadow(ox, oy, ox + 30, oy + 25, r(1, 3), b(), offset=(1, 1), expand=1.5, cap=N.CAP_ROUND)


def test_gpu_sdf_incremental_frames_equal_full_frames(renderer):
    W, H = 384, 256
    full = tk.NativeRenderer(0)
    try:
        rs = tk.RetainedScene(W, H)
        rs.set_clear_color(0xFFFFFFFF)
        nodes = []
        for k in range(8):
            node = tk.Canvas(W, H)
            node.keep_commands()
            small_shapes(node, np.random.default_rng(200 + k), 0.0, 0.0)
            nodes.append(node)
            rs.insert(k + 1, node, (1, 0, 0, 1, 40.0 * k + 10.5, 25.0 * (k % 4) + 8.25))
        renderer.render_retained(rs)
        for step, mutate in enumerate([lambda: rs.set_transform(2, (1, 0, 0, 1, 177.5, 131.25)),
                                       lambda: rs.remove(4),
                                       lambda: rs.move_before(6, 1),
                                       lambda: rs.replace(3, nodes[0]),
                                       lambda: None]):
            mutate()
            st = renderer.render_retained(rs)
            assert st["full_redraw"] == 0 and st["dirty_tiles"] < st["total_tiles"], (step, st)
            img = renderer.readback().view(np.uint8).reshape(H, W, 4)
            want = full.render_to_image(rs.materialize()[0])
            assert np.array_equal(img, want), step
    finally:
        full.close()


def test_gpu_rejects_unsupported_sdf_records(renderer):
    c = tk.Canvas(64, 64)
    c.push_rect(1, 1, 30, 30, tk.Brush.solid(1, 0, 0, 1))
    a = c.scene_arrays()
    bad_kind = dict(a)
    bad_kind["sdf"] = a["sdf"].copy()
    bad_kind["sdf"][0] = 20  # no such kind
    short = dict(a)
    short["sdf"] = a["sdf"][:10].copy()  # the record runs past the blob
    clip = dict(a)
    clip["draws"] = a["draws"].copy()
    clip["draws"]["tag"][0] = 2  # an SDF opacity group: outside this path
    for arrays in (bad_kind, short, clip):
        with pytest.raises(tk.TileinkError) as e:
            renderer.upload(N.ArrayScene(arrays))
        assert e.value.code == N.TK_E_INVALID
    renderer.render_to_image(c)


def test_gpu_rect_known_answers_match_fine_only_oracle(renderer):
    """The reference's coarse known-answer pixel tests for SDF rects
    (coarse_count/rect_pixels.rs:110-283, occlusion_pixels.rs:85-116): the
    sm_100a pipeline, with coarse's full-tile colour, hollow-stroke and
    occlusion proofs, gives exactly the pixels of fine interpreting every draw
    in every tile. Edge, huge (1e7, 1.7e38) and far-translated geometry, draw
    transforms, 0-257 stacked rects of alpha 0/127/255."""
    import oracle
    from sdf_cases import all_cases, desc_of
    for name, scene in all_cases():
        keep, d = desc_of(scene)
        want = oracle.interpret_sdf_draws(d)
        renderer.upload(keep)
        renderer.render()
        got = renderer.readback().view(np.uint8).reshape(want.shape)
        assert np.array_equal(got, want), (name, int((got != want).any(axis=2).sum()))


def test_gpu_partial_sdf_clip_matches_fine_only_oracle(renderer):
    """occlusion_pixels.rs:48-83 on the GPU: the pipeline with SDF clip
    wrappers gives exactly the fine-only oracle's pixels."""
    import oracle
    from sdf_cases import partial_clip_cases
    for name, canvas, stream in partial_clip_cases():
        want = oracle.interpret_particles(canvas.scene_desc(), stream)
        got = renderer.render_to_image(canvas)
        assert np.array_equal(got, want), name


@pytest.mark.parametrize("seed", [21, 22])
def test_gpu_sdf_clip_layers(renderer, seed):
    """Nested SDF clip layers (rect, circle, line, arc) around paths and
    shapes, next to path clips, against the oracle bit for bit."""
    W, H = 400, 300
    rng = np.random.default_rng(seed)
    c = tk.Canvas(W, H)
    c.set_clear_color(0xFFFFFFFF)
    random_shapes(c, rng, 30, W, H)
    for depth in range(3):
        k = int(rng.integers(0, 4))
        x0, y0 = rng.uniform(-20, W / 2), rng.uniform(-20, H / 2)
        if k == 0:
            c.push_clip_sdf_rect_layer(x0, y0, x0 + rng.uniform(40, 300), y0 + rng.uniform(40, 250),
                                       radius=float(rng.uniform(0, 40)))
        elif k == 1:
            c.push_clip_sdf_circle_layer(x0 + 60, y0 + 60, float(rng.uniform(20, 150)))
        elif k == 2:
            c.push_clip_sdf_line_layer(x0, y0, x0 + rng.uniform(50, 300), y0 + rng.uniform(50, 200),
                                       float(rng.uniform(4, 60)), cap=int(rng.integers(0, 3)))
        else:
            c.push_clip_sdf_arc_layer(x0 + 80, y0 + 80, float(rng.uniform(30, 120)), float(rng.uniform(-3, 3)),
                                      float(rng.uniform(-5, 5)), float(rng.uniform(6, 40)))
        random_shapes(c, rng, 20, W, H)
        c.push_path(cubic_path(rng, W, H), tk.Brush.solid(*rng.uniform(0, 1, 3), 0.7))
        if depth == 1:
            c.push_clip_layer(cubic_path(rng, W, H, 8))
            extended_shapes(c, rng, 12, W, H)
            c.pop_layer()
    for _ in range(3):
        c.pop_layer()
    img, ref = compare_frame(renderer, c)
    ptcl = renderer.debug(N.STAGE_PTCL, 0)
    assert (ptcl["tag"] == N.PTCL_BEGIN_SDF_CLIP).any()
