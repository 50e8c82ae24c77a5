"""Device flattening: fills flattened on the GPU give the host Canvas's lines
bit for bit, and therefore the same segments, PTCL and pixels."""
from __future__ import annotations

import numpy as np
import pytest

import tileink_b200 as tk
from tileink_b200 import _native as N

pytestmark = pytest.mark.gpu

WORKLOADS = [
    (1, 4, {}),
    (2, 6, {"width": 512, "height": 384, "paths": 400}),
    (3, 2, {"width": 480, "height": 270, "paths": 600}),
    (5, 1, {"width": 256, "height": 256, "paths": 24}),
]


def render_with(renderer, canvas):
    img = renderer.render_to_image(canvas)
    return {
        "img": img,
        "paths": renderer.debug(N.STAGE_PATHS),
        "lines": renderer.debug(N.STAGE_LINES),
        "segments": renderer.debug(N.STAGE_SEGMENTS),
        "ranges": renderer.debug(N.STAGE_RANGES),
        "ptcl": [renderer.debug(N.STAGE_PTCL, p) for p in range(renderer.stats()["passes"])],
    }


@pytest.mark.parametrize("config,seed,kw", WORKLOADS)
def test_gpu_device_flattening_matches_host_flattening(renderer, config, seed, kw):
    host = render_with(renderer, tk.generate(config, seed, device_segment_plan=True, **kw))
    dev_canvas = tk.generate(config, seed, device_flatten=True, **kw)
    assert dev_canvas.flatten_desc() is not None
    dev = render_with(renderer, dev_canvas)
    hp, dp = host["paths"], dev["paths"]
    assert np.array_equal(hp["line_count"], dp["line_count"])
    # every path's lines, wherever they sit in the line array
    for k in range(len(hp)):
        a = host["lines"][hp["line_start"][k]:hp["line_start"][k] + hp["line_count"][k]]
        b = dev["lines"][dp["line_start"][k]:dp["line_start"][k] + dp["line_count"][k]]
        assert a.tobytes() == b.tobytes(), k
    assert dev["segments"].tobytes() == host["segments"].tobytes()
    assert np.array_equal(dev["ranges"], host["ranges"])
    for a, b in zip(host["ptcl"], dev["ptcl"]):
        assert a.tobytes() == b.tobytes()
    assert np.array_equal(dev["img"], host["img"])


def test_gpu_device_flattening_rejects_inconsistent_elements(renderer):
    import ctypes
    canvas = tk.generate(1, 3, width=128, height=96, paths=5, device_flatten=True)
    d = canvas.scene_desc()
    f = canvas.flatten_desc()
    path_els = np.ctypeslib.as_array((ctypes.c_uint32 * (2 * d.path_count)).from_address(f.path_elements)).copy()
    path_els[1] = f.element_count + 5  # the first path claims elements past the end
    bad = N.FlattenDesc(f.elements, f.element_count, path_els.ctypes.data)
    with pytest.raises(tk.TileinkError):
        renderer._check(renderer._lib.tk_scene_upload_flatten(renderer._h, ctypes.byref(d), ctypes.byref(bad)))
    # elements the device refuses to flatten (their work would be unbounded):
    # reported, nothing flattened, the context stays usable
    arrays = canvas.scene_arrays()
    arrays.update(canvas.flatten_arrays())
    arrays["elements"] = arrays["elements"].copy()
    arrays["elements"]["tolerance"][0] = 1e-9
    with pytest.raises(tk.TileinkError, match="tolerance"):
        renderer.upload(N.ArrayScene(arrays))
    img = renderer.render_to_image(canvas)
    assert img.shape == (96, 128, 4)
    # a host-flattened scene without device planning cannot take elements either
    host = tk.generate(1, 3, width=128, height=96, paths=5)
    with pytest.raises(tk.TileinkError):
        renderer._check(renderer._lib.tk_scene_upload_flatten(renderer._h, ctypes.byref(host.scene_desc()),
                                                              ctypes.byref(f)))


def stroke_scene(device: bool):
    """Every stroke shape of the CPU stroke tests, at several widths and
    transforms (identity, rotation + scale, shear), plus seeded random curves:
    open, closed, dots, multiple subpaths, a close followed by more drawing."""
    from test_stroke import CASES
    c = tk.Canvas(320, 240)
    if device:
        c.set_device_flatten(True)
    else:
        c.set_host_segment_plan(False)
    transforms = [None, (0.9, 0.35, -0.35, 0.9, 40.0, -10.0), (1.0, 0.0, 0.4, 0.7, -20.0, 30.0)]
    k = 0
    for name in sorted(CASES):
        build, _, width = CASES[name]
        for t in transforms:
            for w in (width, 0.75, 2.5):
                p = tk.BezPath()
                build(p)
                c.push_stroke(p, tk.Brush.solid((k % 7) / 7, (k % 5) / 5, (k % 3) / 3, 0.6), w, transform=t,
                              tolerance=0.05 + 0.05 * (k % 3))
                k += 1
    # long polylines with repeated points inside and across groups of 32
    # points (the cleanup's sequential rule), open and closed back onto the start
    for closed in (False, True):
        pts = [(20.0 + 3.0 * i, 60.0 + (25.0 if i % 2 else 0.0) + 0.5 * i) for i in range(90)]
        for at in (88, 70, 34, 33, 32, 31, 5, 1):
            pts.insert(at, pts[at - 1])
        p = tk.BezPath()
        p.move_to(*pts[0])
        for q in pts[1:]:
            p.line_to(*q)
        if closed:
            p.line_to(*pts[0])
            p.close()
        c.push_stroke(p, tk.Brush.solid(0.2, 0.4, 0.6, 0.7), 3.0, tolerance=0.1)
    rng = np.random.default_rng(11)
    for _ in range(60):
        p = tk.BezPath()
        p.move_to(*rng.uniform(0, 320, 2))
        for _ in range(int(rng.integers(1, 9))):
            if rng.random() < 0.5:
                p.cubic_to(*rng.uniform(-20, 340, 6))
            else:
                p.quad_to(*rng.uniform(-20, 340, 4))
        if rng.random() < 0.4:
            p.close()
        c.push_stroke(p, tk.Brush.solid(*rng.uniform(0, 1, 3), 0.8), float(rng.uniform(0.3, 12.0)),
                      tolerance=float(rng.uniform(0.02, 0.3)))
    return c


def test_gpu_device_stroking_matches_host_stroking(renderer):
    host = render_with(renderer, stroke_scene(False))
    dev_canvas = stroke_scene(True)
    f = dev_canvas.flatten_desc()
    assert f is not None and f.stroke_count > 0 and dev_canvas.scene_desc().line_count == 0
    dev = render_with(renderer, dev_canvas)
    hp, dp = host["paths"], dev["paths"]
    assert np.array_equal(hp["line_count"], dp["line_count"])
    assert int(hp["line_count"].sum()) > 10000
    for k in range(len(hp)):
        a = host["lines"][hp["line_start"][k]:hp["line_start"][k] + hp["line_count"][k]]
        b = dev["lines"][dp["line_start"][k]:dp["line_start"][k] + dp["line_count"][k]]
        assert a.tobytes() == b.tobytes(), k
    assert dev["segments"].tobytes() == host["segments"].tobytes()
    for a, b in zip(host["ptcl"], dev["ptcl"]):
        assert a.tobytes() == b.tobytes()
    assert np.array_equal(dev["img"], host["img"])


def test_gpu_device_stroking_rejects_inconsistent_strokes(renderer):
    canvas = stroke_scene(True)
    base = canvas.scene_arrays()
    base.update(canvas.flatten_arrays())

    def upload(mutate):
        a = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in base.items()}
        mutate(a)
        renderer.upload(N.ArrayScene(a))

    def set_(key, field, index, value):
        def f(a):
            a[key][field][index] = value
        return f

    bad = [
        set_("strokes", "half_width", 0, 0.0),
        set_("strokes", "half_width", 1, np.nan),
        set_("strokes", "tolerance", 2, 1e-6),
        set_("strokes", "transform", 3, np.inf),
        set_("strokes", "path", 4, 10 ** 6),
        set_("strokes", "path", 5, 4),                 # two strokes on one path
        set_("strokes", "polyline_count", 6, 10 ** 6),
        set_("polylines", "stroke", 0, 1),              # owned by another stroke
        set_("polylines", "element_count", 1, 0),
        set_("polylines", "element0", 2, 10 ** 9),
    ]
    for mutate in bad:
        with pytest.raises(tk.TileinkError):
            upload(mutate)
    # element faults found on the device: reported, the context stays usable
    device_bad = [
        set_("stroke_elements", "verb", 0, N.EL_LINE),       # a polyline that does not start with a move
        set_("stroke_elements", "path", 1, 7),               # an element of another polyline
        set_("stroke_elements", "tolerance", 2, 1e-9),
        set_("stroke_elements", "verb", 3, 9),
    ]
    for mutate in device_bad:
        with pytest.raises(tk.TileinkError):
            upload(mutate)
    img = renderer.render_to_image(canvas)
    assert img.shape == (240, 320, 4)
