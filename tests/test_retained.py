"""Retained scenes on the host: command replay reproduces a recording exactly,
and materialization reports the damage of every mutation (RetainedScene,
src/retained_scene/scene.rs:14-140, transaction.rs:74-255; damage planning,
src/render/incremental.rs:1-297). The GPU side (incremental frames equal full
frames) is in test_gpu_retained.py."""
from __future__ import annotations

import numpy as np
import pytest

import tileink_b200 as tk

W, H = 320, 240
SCENE_KEYS = ("lines", "paths", "draws", "brush", "layers", "draw_order", "draw_batch_ids", "ops")


def affine_after(o, i):
    """The composition the replay applies: `o` after `i`."""
    return (o[0] * i[0] + o[2] * i[1], o[1] * i[0] + o[3] * i[1], o[0] * i[2] + o[2] * i[3],
            o[1] * i[2] + o[3] * i[3], o[0] * i[4] + o[2] * i[5] + o[4], o[1] * i[4] + o[3] * i[5] + o[5])


def calls(seed: int, n: int = 6, layered: bool = False):
    """A seeded list of canvas calls: (kind, args) with kind fill / stroke /
    clip / pop, local transforms on some of them."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        pts = rng.uniform(-30, 140, 8)
        t = None if k % 3 else (1.0, 0.1 * k, -0.05 * k, 0.9, 5.0 * k, 3.0)
        if k % 4 == 3:
            brush = tk.Brush.linear((0, 0), (120, 40), [(0.0, (1, 0, 0, 1)), (1.0, (0, 0, 1, 0.5))])
        else:
            brush = tk.Brush.solid(*rng.uniform(0, 1, 3), 0.8)
        kind = "stroke" if k % 2 else "fill"
        out.append((kind, pts, brush, t, float(rng.uniform(0.5, 6.0))))
    if layered:
        out.insert(1, ("clip", rng.uniform(0, 150, 8), None, None, 0.0))
        out.append(("pop", None, None, None, 0.0))
    return out


def path_of(pts):
    p = tk.BezPath()
    p.move_to(pts[0], pts[1])
    p.cubic_to(*pts[2:8])
    p.quad_to(pts[0] + 20, pts[1] - 10, pts[6] - 5, pts[7] + 15)
    return p


def record(canvas, cs, outer=None):
    """Records `cs`, each call's transform preceded by `outer`."""
    for kind, pts, brush, t, width in cs:
        if outer is not None:
            t = affine_after(outer, t if t is not None else (1, 0, 0, 1, 0, 0))
        if kind == "fill":
            canvas.push_path(path_of(pts), brush, transform=t)
        elif kind == "stroke":
            canvas.push_stroke(path_of(pts), brush, width, transform=t)
        elif kind == "clip":
            canvas.push_clip_layer(path_of(pts), transform=t)
        else:
            canvas.pop_layer()


def node_canvas(cs):
    c = tk.Canvas(W, H)
    c.keep_commands()
    record(c, cs)
    return c


def fresh():
    c = tk.Canvas(W, H)
    c.set_host_segment_plan(False)
    return c


def assert_same_scene(a, b):
    sa, sb = a.scene_arrays(), b.scene_arrays()
    for k in SCENE_KEYS:
        assert sa[k].tobytes() == sb[k].tobytes(), k


def test_replay_reproduces_the_recording():
    cs = calls(1, layered=True)
    src = node_canvas(cs)
    direct = fresh()
    record(direct, cs)
    replayed = fresh()
    replayed.replay(src)
    assert_same_scene(direct, replayed)
    # under a transform: the same as recording with the transform composed in
    outer = (0.8, 0.3, -0.3, 0.8, 40.0, -10.0)
    direct_t = fresh()
    record(direct_t, cs, outer)
    replayed_t = fresh()
    replayed_t.replay(src, outer)
    assert_same_scene(direct_t, replayed_t)
    # a canvas without a command log, or with an open layer, cannot be replayed
    with pytest.raises(ValueError):
        fresh().replay(fresh())
    open_layer = tk.Canvas(W, H)
    open_layer.keep_commands()
    open_layer.push_clip_layer(path_of(np.arange(8.0)))
    with pytest.raises(ValueError):
        fresh().replay(open_layer)


def scene_of(nodes):
    """The canvas a retained scene with `nodes` [(id, calls, transform)] must
    materialize into."""
    c = fresh()
    for _, cs, t in nodes:
        c.replay(node_canvas(cs), t)
    return c


def draw_rects(canvas, first, count):
    d = canvas.scene_arrays()["draws"][first:first + count]["pixel_bounds"]
    return {tuple(int(v) for v in r) for r in d if r["x1"] > r["x0"] and r["y1"] > r["y0"]}


def draws_of(cs):
    return len(node_canvas(cs).scene_arrays()["draws"])


def test_retained_materialization_and_damage():
    rs = tk.RetainedScene(W, H)
    nodes = [(k + 1, calls(10 + k, n=3), None if k % 2 else (1, 0, 0, 1, 3.0 * k, 0.0)) for k in range(5)]
    for nid, cs, t in nodes:
        rs.insert(nid, node_canvas(cs), t)
    assert rs.version == 5
    canvas, damage = rs.materialize()
    assert damage["full"] and len(damage["rects"]) == 0
    assert_same_scene(canvas, scene_of(nodes))
    before = scene_of(nodes)

    # transform one node: its draw rectangles before and after
    rs.set_transform(3, (1, 0, 0, 1, 25.0, -12.0))
    nodes[2] = (3, nodes[2][1], (1, 0, 0, 1, 25.0, -12.0))
    canvas, damage = rs.materialize()
    assert not damage["full"]
    after = scene_of(nodes)
    assert_same_scene(canvas, after)
    first = sum(draws_of(cs) for _, cs, _ in nodes[:2])
    n3 = draws_of(nodes[2][1])
    want = draw_rects(before, first, n3) | draw_rects(after, first, n3)
    assert {tuple(r) for r in damage["rects"].tolist()} == want

    # nothing changed: no damage
    canvas, damage = rs.materialize()
    assert not damage["full"] and len(damage["rects"]) == 0

    # remove, reorder, replace, invalidate: the union of what each touched
    rs.remove(2)
    rs.move_before(5, 1)
    rs.replace(4, node_canvas(calls(99, n=2)))
    rs.invalidate_rect(1, 2, 30, 40)
    old = scene_of(nodes)
    old_rects = {nid: draw_rects(old, sum(draws_of(cs) for _, cs, _ in nodes[:k]), draws_of(nodes[k][1]))
                 for k, (nid, _, _) in enumerate(nodes)}
    nodes = [nodes[4], nodes[0], nodes[2], (4, calls(99, n=2), nodes[3][2])]
    canvas, damage = rs.materialize()
    new = scene_of(nodes)
    assert_same_scene(canvas, new)
    new_rects = {nid: draw_rects(new, sum(draws_of(cs) for _, cs, _ in nodes[:k]), draws_of(nodes[k][1]))
                 for k, (nid, _, _) in enumerate(nodes)}
    want = old_rects[2] | old_rects[5] | new_rects[5] | old_rects[4] | new_rects[4] | {(1, 2, 30, 40)}
    assert not damage["full"]
    assert {tuple(r) for r in damage["rects"].tolist()} == want

    # a node with layers regroups draw batches: everything is damaged
    rs.insert(9, node_canvas(calls(5, n=2, layered=True)), None, before=3)
    canvas, damage = rs.materialize()
    assert damage["full"]
    rs.set_clear_color(0xFF00FF00)
    assert rs.materialize()[1]["full"]
    rs.invalidate_all()
    assert rs.materialize()[1]["full"]


def test_retained_rejects_bad_mutations():
    rs = tk.RetainedScene(W, H)
    good = node_canvas(calls(3, n=2))
    rs.insert(1, good)
    with pytest.raises(ValueError):
        rs.insert(1, good)  # duplicate id
    with pytest.raises(ValueError):
        rs.insert(0, good)  # id 0 is "none"
    with pytest.raises(ValueError):
        rs.insert(2, fresh())  # no command log
    with pytest.raises(ValueError):
        rs.insert(2, good, before=7)  # unknown sibling
    for bad in (lambda: rs.remove(7), lambda: rs.set_transform(7, None), lambda: rs.replace(7, good),
                lambda: rs.move_before(1, 1), lambda: rs.move_before(1, 7)):
        with pytest.raises(ValueError):
            bad()
    v = rs.version
    rs.move_before(1, 0)
    assert rs.version == v + 1
