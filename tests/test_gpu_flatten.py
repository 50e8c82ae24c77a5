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
