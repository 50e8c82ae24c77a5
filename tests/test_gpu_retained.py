"""Incremental rendering of retained scenes: after any sequence of mutations,
redrawing only the damaged tiles over the previous frame gives exactly the
image a full render of the same scene gives, and frames fall back to full
redraws where they must (FullRedrawReason, src/render/incremental/config.rs:52-63)."""
from __future__ import annotations

import numpy as np
import pytest

import tileink_b200 as tk
from tileink_b200 import _native as N

from test_retained import calls, node_canvas

pytestmark = pytest.mark.gpu

W, H = 512, 384


@pytest.fixture(scope="module")
def reference_renderer():
    r = tk.NativeRenderer(0)
    yield r
    r.close()


def full_image(r, canvas):
    return r.render_to_image(canvas)


def incremental_image(renderer, scene, ratio=0.7):
    stats = renderer.render_retained(scene, ratio)
    img = renderer.readback().view(np.uint8).reshape(H, W, 4)
    return img, stats


def big_node(seed, n):
    """n seeded fills and strokes spread over the canvas."""
    c = tk.Canvas(W, H)
    c.keep_commands()
    rng = np.random.default_rng(seed)
    for k in range(n):
        cx, cy = rng.uniform(20, W - 20), rng.uniform(20, H - 20)
        p = tk.BezPath()
        p.move_to(cx, cy)
        for _ in range(3):
            p.cubic_to(*(rng.uniform(-40, 40, 6) + np.tile([cx, cy], 3)))
        p.close()
        b = tk.Brush.solid(*rng.uniform(0, 1, 3), float(rng.uniform(0.4, 1.0)))
        if k % 3 == 2:
            c.push_stroke(p, b, float(rng.uniform(0.5, 5.0)))
        else:
            c.push_path(p, b, fill_rule=k % 2)
    return c


@pytest.mark.parametrize("device_flatten", [False, True])
def test_gpu_incremental_frames_equal_full_frames(renderer, reference_renderer, device_flatten):
    rs = tk.RetainedScene(W, H, device_flatten=device_flatten)
    rs.set_clear_color(0xFFFFFFFF)
    for k in range(12):
        rs.insert(k + 1, big_node(100 + k, 8), None if k % 2 else (1, 0, 0, 1, 2.0 * k, 0.0))
    img, st = incremental_image(renderer, rs)
    assert st["full_redraw"] == 1 and st["reason"] == N.FULL_REQUESTED  # the first materialization
    canvas = rs.materialize()[0]  # no change: the same canvas again
    assert np.array_equal(img, full_image(reference_renderer, canvas))

    small = [
        lambda: rs.set_transform(3, (1, 0, 0, 1, 6.5, -4.25)),
        lambda: rs.set_transform(3, (0.9, 0.2, -0.2, 0.9, 30.0, 10.0)),
        lambda: rs.remove(7),
        lambda: rs.replace(5, node_canvas(calls(77, n=3))),
        lambda: rs.move_before(12, 1),
        lambda: rs.insert(40, node_canvas(calls(41, n=2)), (1, 0, 0, 1, 100.0, 60.0), before=4),
        lambda: rs.invalidate_rect(0, 0, 40, 40),
        lambda: None,  # nothing changed
    ]
    for step, mutate in enumerate(small):
        mutate()
        img, st = incremental_image(renderer, rs)
        canvas = rs.materialize()[0]
        want = full_image(reference_renderer, canvas)
        assert np.array_equal(img, want), step
        assert st["full_redraw"] == 0, (step, st)
        assert st["dirty_tiles"] < st["total_tiles"], (step, st)

    # a node with clip layers: every tile
    rs.insert(50, node_canvas(calls(8, n=3, layered=True)))
    img, st = incremental_image(renderer, rs)
    assert st["full_redraw"] == 1 and st["reason"] == N.FULL_REQUESTED
    assert np.array_equal(img, full_image(reference_renderer, rs.materialize()[0]))
    # damage over the threshold: every tile
    rs.set_transform(1, (1, 0, 0, 1, 1.0, 1.0))
    rs.invalidate_rect(0, 0, W, H // 2 + 64)
    img, st = incremental_image(renderer, rs, ratio=0.5)
    assert st["full_redraw"] == 1 and st["reason"] == N.FULL_THRESHOLD
    assert np.array_equal(img, full_image(reference_renderer, rs.materialize()[0]))


def test_gpu_incremental_fallbacks(renderer):
    # blur layers reach across tiles: full redraws
    blur = tk.generate(5, 1, width=256, height=256, paths=12)
    renderer.upload(blur)
    st = renderer.render_incremental({"full": False, "rects": [[0, 0, 16, 16]]})
    assert st["full_redraw"] == 1
    st = renderer.render_incremental({"full": False, "rects": [[0, 0, 16, 16]]})
    assert st["full_redraw"] == 1 and st["reason"] == N.FULL_FILTERS
    # so do filter layers, and the full redraw is the frame
    from layer_cases import filter_chains, filter_scene
    fl = filter_scene(4, filter_chains()["chain"], (30.5, 28.0, 165.2, 117.9))
    want = renderer.render_to_image(fl).copy()
    renderer.upload(fl)
    st = renderer.render_incremental({"full": False, "rects": [[0, 0, 16, 16]]})
    assert st["full_redraw"] == 1 and st["reason"] == N.FULL_FILTERS
    assert np.array_equal(renderer.readback().view(np.uint8).reshape(want.shape), want)
    # a new size has no history
    c = tk.generate(1, 2, width=200, height=120, paths=20, device_segment_plan=True)
    renderer.upload(c)
    st = renderer.render_incremental({"full": False, "rects": [[0, 0, 16, 16]]})
    assert st["reason"] == N.FULL_NO_HISTORY
    first = renderer.readback().copy()
    # the same scene again with empty damage: nothing is redrawn, the frame stands
    renderer.upload(c)
    st = renderer.render_incremental({"full": False, "rects": np.zeros((0, 4), np.int32)})
    assert st["full_redraw"] == 0 and st["dirty_tiles"] == 0
    assert np.array_equal(renderer.readback(), first)
    # and with damage somewhere: those tiles are redrawn to the same pixels
    st = renderer.render_incremental({"full": False, "rects": [[10, 10, 90, 50]]})
    assert st["full_redraw"] == 0 and 0 < st["dirty_tiles"] < st["total_tiles"]
    assert np.array_equal(renderer.readback(), first)
    with pytest.raises(tk.TileinkError):
        renderer.render_incremental({"full": False, "rects": [[0, 0, 1, 1]]}, full_redraw_ratio=0.0)


def test_gpu_incremental_frames_reuse_the_unchanged_scan(renderer, reference_renderer):
    """Partial redraws of a scene that was not uploaded again reuse its scan
    (scene_scan.rs:116-125's unchanged-history reuse) and still equal full
    renders; an upload ends the reuse."""
    c = tk.generate(2, 11, width=W, height=H, paths=300)
    want = full_image(reference_renderer, c).copy()
    renderer.upload(c)
    st = renderer.render_incremental(None)
    assert st["full_redraw"] == 1 and st["scan_reused"] == 0
    for k, rect in enumerate([[0, 0, 100, 80], [200, 150, 330, 300], [400, 0, 512, 384]]):
        st = renderer.render_incremental({"full": False, "rects": [rect]})
        assert st["full_redraw"] == 0 and st["scan_reused"] == 1, st
        img = renderer.readback().view(np.uint8).reshape(H, W, 4)
        assert np.array_equal(img, want), k
    renderer.upload(c)
    renderer.render_incremental(None)
    st = renderer.render_incremental({"full": False, "rects": [[10, 10, 50, 50]]})
    assert st["scan_reused"] == 1
    renderer.upload(c)
    st = renderer.render_incremental({"full": False, "rects": [[10, 10, 50, 50]]})
    assert st["full_redraw"] == 0 and st["scan_reused"] == 0
    assert np.array_equal(renderer.readback().view(np.uint8).reshape(H, W, 4), want)


def jittered_paths(arrays, candidates, dx):
    """A copy of the scene arrays with the lines of some candidate paths moved
    by dx, keeping their records: only paths whose every line keeps its
    planned tile count (and so its segment slice) are moved."""
    b = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in arrays.items()}
    moved = []
    for p in candidates:
        rec = b["paths"][p]
        s, n = int(rec["line_start"]), int(rec["line_count"])
        bbox = (int(rec["tile_x0"]), int(rec["tile_y0"]), int(rec["tile_x1"]), int(rec["tile_y1"]))
        new = b["lines"][s:s + n].copy()
        new["p0"][:, 0] += dx
        new["p1"][:, 0] += dx
        if all(tk.plan_line_tile_count(new[i], bbox) == tk.plan_line_tile_count(b["lines"][s + i], bbox)
               for i in range(n)):
            b["lines"][s:s + n] = new
            moved.append(p)
    return b, moved


def array_scene(arrays, device_plan):
    scene = N.ArrayScene(arrays)
    if device_plan:
        scene.desc.flags |= N.SCENE_SEGMENTS_FROM_DEVICE
    return scene


def same_scan_and_frame(renderer, reference_renderer, scene):
    """The renderer's last frame equals a full upload and render of `scene`
    in another context: image, segments, PTCL and path records."""
    img = renderer.readback().copy()
    segs = renderer.debug(N.STAGE_SEGMENTS).copy()
    ptcl = renderer.debug(N.STAGE_PTCL).copy()
    paths = renderer.debug(N.STAGE_PATHS).copy()
    want = reference_renderer.render_to_image(scene)
    assert np.array_equal(img.view(np.uint8).reshape(want.shape), want)
    assert segs.tobytes() == reference_renderer.debug(N.STAGE_SEGMENTS).tobytes()
    assert np.array_equal(ptcl, reference_renderer.debug(N.STAGE_PTCL))
    assert paths.tobytes() == reference_renderer.debug(N.STAGE_PATHS).tobytes()


@pytest.mark.parametrize("device_plan", [False, True])
def test_gpu_delta_upload_rescans_only_changed_paths(renderer, reference_renderer, device_plan):
    """tk_scene_upload_delta: the paths whose lines changed are scanned again
    and the others keep their scan; the frame equals a full upload and
    render of the new scene, stage by stage, with host segment plans and with
    device plans (each path keeps the slice the last scan planned)."""
    c = tk.generate(2, 13, width=W, height=H, paths=200, device_segment_plan=device_plan)
    a = c.scene_arrays()
    renderer.upload(c)
    renderer.render()
    b, moved = jittered_paths(a, range(0, 200, 17), 0.03125)
    assert len(moved) >= 3
    assert renderer.upload_delta(array_scene(b, device_plan), moved) == len(moved)
    renderer.render()
    same_scan_and_frame(renderer, reference_renderer, array_scene(b, device_plan))
    # an incremental frame after a delta scans just the replaced paths
    b2, moved2 = jittered_paths(b, moved[:2], -0.0625)
    assert renderer.upload_delta(array_scene(b2, device_plan), moved2) == len(moved2)
    st = renderer.render_incremental({"full": False, "rects": [[0, 0, W, 64]]})
    assert st["full_redraw"] == 0 and st["scanned_paths"] == len(moved2) and st["scan_reused"] == 0
    st = renderer.render_incremental({"full": True})
    want2 = reference_renderer.render_to_image(array_scene(b2, device_plan))
    assert np.array_equal(renderer.readback().view(np.uint8).reshape(want2.shape), want2)


def test_gpu_device_plan_delta_with_a_changed_total_scans_everything(renderer, reference_renderer):
    """Device plans: a replaced path whose segment total changes would move
    every later slice, so the render finds that after counting it and scans
    the whole scene; the frame still equals a full upload and render."""
    c = tk.generate(2, 16, width=W, height=H, paths=150, device_segment_plan=True)
    a = c.scene_arrays()
    renderer.upload(c)
    renderer.render()
    b = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in a.items()}
    rec = b["paths"][40]
    s, n = int(rec["line_start"]), int(rec["line_count"])
    seg = b["lines"][s:s + n]
    cx, cy = float(seg["p0"][:, 0].mean()), float(seg["p0"][:, 1].mean())
    for end in ("p0", "p1"):  # shrunk about its centre: inside its bbox, fewer tile crossings
        seg[end][:, 0] = cx + 0.25 * (seg[end][:, 0] - cx)
        seg[end][:, 1] = cy + 0.25 * (seg[end][:, 1] - cy)
    b["lines"][s:s + n] = seg
    assert renderer.upload_delta(array_scene(b, True), [40]) == 1
    st = renderer.render_incremental({"full": True})
    assert st["scanned_paths"] == len(a["paths"])
    same_scan_and_frame(renderer, reference_renderer, array_scene(b, True))


def test_gpu_delta_upload_falls_back_when_the_layout_changes(renderer, reference_renderer):
    c = tk.generate(2, 14, width=W, height=H, paths=120)
    renderer.upload(c)
    renderer.render()
    other = tk.generate(2, 15, width=W, height=H, paths=121)  # other counts: a whole upload
    assert renderer.upload_delta(other, []) == other.scene_arrays()["paths"].shape[0]
    renderer.render()
    want = reference_renderer.render_to_image(other)
    assert np.array_equal(renderer.readback().view(np.uint8).reshape(want.shape), want)


def test_gpu_retained_recolor_keeps_the_whole_scan(renderer, reference_renderer):
    """A node replaced by the same geometry in another colour changes no
    line and no path record: the frame reuses the whole scan."""
    rs = tk.RetainedScene(W, H)
    rs.set_clear_color(0xFFFFFFFF)
    for k in range(6):
        rs.insert(k + 1, big_node(300 + k, 6))
    incremental_image(renderer, rs)
    recolored = tk.Canvas(W, H)
    recolored.keep_commands()
    src = big_node(302, 6)
    rng = np.random.default_rng(302)
    for k in range(6):
        cx, cy = rng.uniform(20, W - 20), rng.uniform(20, H - 20)
        p = tk.BezPath()
        p.move_to(cx, cy)
        for _ in range(3):
            p.cubic_to(*(rng.uniform(-40, 40, 6) + np.tile([cx, cy], 3)))
        p.close()
        rng.uniform(0, 1, 3), rng.uniform(0.4, 1.0)  # the original colour draws
        b = tk.Brush.solid(0.1 * k, 0.5, 0.9, 0.7)
        if k % 3 == 2:
            recolored.push_stroke(p, b, float(rng.uniform(0.5, 5.0)))
        else:
            recolored.push_path(p, b, fill_rule=k % 2)
    del src
    rs.replace(3, recolored)
    img, st = incremental_image(renderer, rs)
    assert st["full_redraw"] == 0
    assert st.get("rescan_paths") == 0 and st["scan_reused"] == 1 and st["scanned_paths"] == 0, st
    assert np.array_equal(img, full_image(reference_renderer, rs.materialize()[0]))
