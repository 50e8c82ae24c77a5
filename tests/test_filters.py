"""Filter layers on CPU: the oracle's colour filters and colour matrix
(filter/color.hlsli:7-76) against an independent float32 restatement in
numpy, their exact identities, the offset (filter/basic.hlsl:49-56), and the
Canvas's recording of filter layers (layers.rs:222-233, filter.rs:490-597)."""
from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
import tileink_b200 as tk
from tileink_b200 import _native as N

from layer_cases import SEPIA_MATRIX, filter_chains, filter_scene

F = np.float32


def premul_pixels(n, seed):
    """n premultiplied RGBA8 words with alpha 0, 255 and in between."""
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 256, n).astype(np.uint32)
    a[:8] = [0, 255, 255, 1, 128, 254, 0, 255]
    rgb = (rng.random((n, 3)) * (a[:, None] + 1)).astype(np.uint32)
    rgb = np.minimum(rgb, a[:, None])
    return rgb[:, 0] | (rgb[:, 1] << 8) | (rgb[:, 2] << 16) | (a << 24)


def oracle_chain(pixels, chain):
    """The oracle's filter chain over a one-row surface."""
    surf = np.ascontiguousarray(pixels, dtype=np.uint32).copy()
    filters = np.zeros(len(chain), dtype=N.FILTER_DTYPE)
    for k, (kind, value) in enumerate(chain):
        filters[k]["kind"] = kind
        if kind == N.FILTER_COLOR_MATRIX:
            filters[k]["matrix"] = np.asarray(value, dtype=np.float32)
        elif kind == N.FILTER_OFFSET:
            filters[k]["dx"], filters[k]["dy"] = value
        else:
            filters[k]["amount"] = value
    rect = np.array([0, 0, len(surf), 1], dtype=np.int32)
    oracle.lib().or_filter_chain(N.ptr(surf), len(surf), N.ptr(rect), N.ptr(filters), len(filters), None)
    return surf


def mad(a, b, c):
    """A fused multiply-add in float32: the float64 product of two float32
    values is exact, so one rounding of the sum and one to float32."""
    return F(np.float64(a) * np.float64(b) + np.float64(c))


def np_color_pixel(p, kind, amount):
    """filter_color_pixel restated with numpy float32 scalars."""
    amount = F(amount)
    ch = [F(int(p) >> s & 255) for s in (0, 8, 16)]
    alpha = int(p) >> 24
    if kind in (N.FILTER_INVERT, N.FILTER_SEPIA) and alpha:
        fa = F(alpha)
        m = [fa - c for c in ch]
        if kind == N.FILTER_SEPIA:
            r, g, b = ch
            m = [mad(F(0.393), r, mad(F(0.769), g, F(0.189) * b)), mad(F(0.349), r, mad(F(0.686), g, F(0.168) * b)),
                 mad(F(0.272), r, mad(F(0.534), g, F(0.131) * b))]
        t = F(min(max(amount, F(0)), F(1)))
        out = [int(F(min(max(mad(mm - c, t, c), F(0)), fa)) + F(0.5)) for mm, c in zip(m, ch)]
        return out + [alpha]
    scale = F(1.0) / F(255.0)
    c = [F(int(p) >> s & 255) * scale for s in (0, 8, 16, 24)]
    if kind == N.FILTER_OPACITY:
        a = F(min(max(amount, F(0)), F(1)))
        c = [x * a for x in c]
    elif c[3] > 0:
        st = [x / c[3] for x in c[:3]]
        lum = lambda v: (F(0.2126) * v[0] + F(0.7152) * v[1]) + F(0.0722) * v[2]  # noqa: E731
        if kind == N.FILTER_BRIGHTNESS:
            st = [x * amount for x in st]
        elif kind == N.FILTER_CONTRAST:
            st = [(x - F(0.5)) * amount + F(0.5) for x in st]
        elif kind == N.FILTER_GRAYSCALE:
            l, t = lum(st), F(min(max(amount, F(0)), F(1)))
            st = [mad(l - x, t, x) for x in st]
        elif kind == N.FILTER_HUE_ROTATE:
            ang = amount * F(0.017453292)
            co, si = F(math.cos(float(ang))), F(math.sin(float(ang)))
            r, g, b = st
            st = [((F(0.213) + co * F(0.787)) - si * F(0.213)) * r + ((F(0.715) - co * F(0.715)) - si * F(0.715)) * g
                  + ((F(0.072) - co * F(0.072)) + si * F(0.928)) * b,
                  ((F(0.213) - co * F(0.213)) + si * F(0.143)) * r + ((F(0.715) + co * F(0.285)) + si * F(0.140)) * g
                  + ((F(0.072) - co * F(0.072)) - si * F(0.283)) * b,
                  ((F(0.213) - co * F(0.213)) - si * F(0.787)) * r + ((F(0.715) - co * F(0.715)) + si * F(0.715)) * g
                  + ((F(0.072) + co * F(0.928)) + si * F(0.072)) * b]
        elif kind == N.FILTER_SATURATE:
            l = lum(st)
            st = [l + (x - l) * amount for x in st]
        c = [F(min(max(x, F(0)), F(1))) * c[3] for x in st] + [c[3]]
    return [int(F(min(max(x, F(0)), F(1))) * F(255) + F(0.5)) for x in c]


COLOR_CASES = [(N.FILTER_BRIGHTNESS, 1.6), (N.FILTER_BRIGHTNESS, 0.3), (N.FILTER_CONTRAST, 0.45),
               (N.FILTER_CONTRAST, 2.5), (N.FILTER_GRAYSCALE, 0.8), (N.FILTER_GRAYSCALE, 1.0),
               (N.FILTER_HUE_ROTATE, 137.0), (N.FILTER_HUE_ROTATE, -60.0), (N.FILTER_INVERT, 0.7),
               (N.FILTER_INVERT, 1.0), (N.FILTER_OPACITY, 0.55), (N.FILTER_SATURATE, 2.3),
               (N.FILTER_SATURATE, 0.0), (N.FILTER_SEPIA, 1.0), (N.FILTER_SEPIA, 0.4)]


@pytest.mark.parametrize("kind, amount", COLOR_CASES)
def test_color_filters_match_numpy_restatement(kind, amount):
    px = premul_pixels(3000, kind * 1000 + int(abs(amount) * 10))
    got = oracle_chain(px, [(kind, amount)])
    want = np.array([np_color_pixel(p, kind, amount) for p in px], dtype=np.int64)
    gotc = np.stack([(got >> s) & 255 for s in (0, 8, 16, 24)], axis=1).astype(np.int64)
    d = np.abs(gotc - want)
    assert d.max() <= 1, d.max()  # a double-rounded mad or a sin / cos last bit moves one level at most
    assert (d == 0).mean() >= 0.995


def test_color_filter_identities_are_exact():
    px = premul_pixels(4000, 5)
    for chain in ([(N.FILTER_INVERT, 0.0)], [(N.FILTER_SEPIA, 0.0)], [(N.FILTER_OPACITY, 1.0)],
                  [(N.FILTER_COLOR_MATRIX, [1, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 1, 0])], []):
        assert np.array_equal(oracle_chain(px, chain), px), chain
    # invert of an opaque pixel is 255 - c exactly; opacity 0 clears
    opaque = (px & 0x00FFFFFF) | 0xFF000000
    inv = oracle_chain(opaque, [(N.FILTER_INVERT, 1.0)])
    assert np.array_equal(inv, (0x00FFFFFF - (opaque & 0x00FFFFFF)) | 0xFF000000)
    assert not oracle_chain(px, [(N.FILTER_OPACITY, 0.0)]).any()


def test_color_matrix_keeps_bytes_and_saturates():
    px = premul_pixels(3000, 9)
    got = oracle_chain(px, [(N.FILTER_COLOR_MATRIX, SEPIA_MATRIX)])
    a = px >> 24
    assert np.array_equal(got >> 24, a)  # alpha row (0 0 0 1 0): alpha unchanged
    for s in (0, 8, 16):  # premultiplied channels stay within alpha
        assert np.all(((got >> s) & 255) <= a)
    # a bias of 1 on every channel saturates to the output alpha
    sat = oracle_chain(px, [(N.FILTER_COLOR_MATRIX, [0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 1, 0])])
    assert np.array_equal(sat, a * 0x01010101)


def test_offset_moves_pixels_inside_the_bounds():
    w, h = 23, 17
    surf = np.arange(1, w * h + 1, dtype=np.uint32)
    filters = np.zeros(1, dtype=N.FILTER_DTYPE)
    filters[0]["kind"], filters[0]["dx"], filters[0]["dy"] = N.FILTER_OFFSET, 4, -3
    rect = np.array([2, 1, 20, 15], dtype=np.int32)
    out = surf.copy()
    oracle.lib().or_filter_chain(N.ptr(out), w, N.ptr(rect), N.ptr(filters), 1, None)
    s2, o2 = surf.reshape(h, w), out.reshape(h, w)
    for y in range(h):
        for x in range(w):
            if not (2 <= x < 20 and 1 <= y < 15):
                assert o2[y, x] == s2[y, x]  # outside the bounds: untouched
                continue
            sx, sy = x - 4, y + 3
            want = s2[sy, sx] if (2 <= sx < 20 and 1 <= sy < 15) else 0
            assert o2[y, x] == want


def test_canvas_records_filter_layers():
    c = tk.Canvas(128, 96)
    c.push_filter_layer([(N.FILTER_GRAYSCALE, 0.5), (N.FILTER_OFFSET, (7.5, -4.2)), (N.FILTER_OFFSET, (-2.6, 0.4))],
                        (10.2, 20.7, 60.1, 50.0))
    c.push_path(tk.BezPath().move_to(20, 30).line_to(50, 35).line_to(40, 45).close(), tk.Brush.solid(1, 0, 0, 1))
    c.pop_layer()
    a = c.scene_arrays()
    ops = a["ops"]
    assert list(ops["kind"]) == [N.OP_FILTER_BEGIN, N.OP_DRAW_BATCH, N.OP_BLUR_END]
    L = a["filter_layers"][ops["batch_id"][0]]
    fl = a["filters"][L["first"]:L["first"] + L["count"]]
    assert list(fl["kind"]) == [N.FILTER_GRAYSCALE, N.FILTER_OFFSET, N.FILTER_OFFSET]
    # filter_offset_to_pixel_delta: ceil(d - 0.5)
    assert (fl["dx"][1], fl["dy"][1], fl["dx"][2], fl["dy"][2]) == (7, -4, -3, 0)
    # the region's pixel bounds (floor / ceil) grown by the chain's reach
    # (max(ceil|dx|, ceil|dy|) per offset: 8 + 3)
    assert list(L["surface"]) == [10 - 11, 20 - 11, 61 + 11, 50 + 11]
    assert list(ops["bounds"][0]) == [0, 9, 72, 61]  # clipped to the canvas
    # fixed_region: no reach; a canvas scale scales the region and the offsets
    c2 = tk.Canvas(128, 96, scale=2.0)
    c2.push_filter_layer([(N.FILTER_OFFSET, (1.3, 0.0))], (1.0, 2.0, 10.0, 12.0), fixed_region=True)
    c2.pop_layer()
    a2 = c2.scene_arrays()
    L2 = a2["filter_layers"][0]
    assert list(L2["surface"]) == [2, 4, 20, 24] and a2["filters"][0]["dx"] == 3  # ceil(2.6 - 0.5)
    c3 = tk.Canvas(128, 96)
    c3.push_filter_layer([(N.FILTER_DILATE, (3.0, 4.2)), (N.FILTER_ERODE, (6.0, 6.0))], (20.0, 20.0, 60.0, 50.0))
    c3.pop_layer()
    a3 = c3.scene_arrays()
    assert list(a3["filter_layers"][0]["surface"]) == [15, 15, 65, 55]  # a dilation reaches ceil(4.2); erosion 0
    assert [tuple(f) for f in a3["filters"][["dx", "dy"]]] == [(3, 5), (6, 6)]
    with pytest.raises(ValueError):
        c.push_filter_layer([(99, 1.0)], (0, 0, 10, 10))
    with pytest.raises(ValueError):
        c.push_filter_layer([(N.FILTER_BRIGHTNESS, float("nan"))], (0, 0, 10, 10))


def test_filter_layer_that_hides_its_children():
    # opacity 0 removes the group: the frame equals the one with an empty group
    rect = (20, 10, 180, 140)
    ca, cb = filter_scene(3, [(N.FILTER_OPACITY, 0.0)], rect), filter_scene(3, [], rect, children=False)
    a = oracle.OracleRun(ca.scene_desc(), threads=4)
    b = oracle.OracleRun(cb.scene_desc(), threads=4)
    assert np.array_equal(a.get(oracle.OR_IMAGE, np.uint32), b.get(oracle.OR_IMAGE, np.uint32))


@pytest.mark.parametrize("name", sorted(filter_chains()))
def test_filter_scenes_render_in_the_oracle(name):
    c = filter_scene(7, filter_chains()[name], (30.5, 28.0, 165.2, 117.9))
    img = oracle.OracleRun(c.scene_desc(), threads=4).get(oracle.OR_IMAGE, np.uint32)
    assert img.any()


def oracle_surface_chain(surf, w, rect, chain):
    """The oracle's chain over a w-wide surface (a copy), in place over rect."""
    out = np.ascontiguousarray(surf, dtype=np.uint32).copy()
    filters = np.zeros(len(chain), dtype=N.FILTER_DTYPE)
    for k, (kind, value) in enumerate(chain):
        filters[k]["kind"] = kind
        filters[k]["dx"], filters[k]["dy"] = value
    r = np.array(rect, dtype=np.int32)
    oracle.lib().or_filter_chain(N.ptr(out), w, N.ptr(r), N.ptr(filters), len(filters), None)
    return out


def np_morphology(img, rect, rx, ry, dilate):
    """filter_morphology_pixel along x then y, restated with numpy float32."""
    x0, y0, x1, y1 = rect
    sub = img[y0:y1, x0:x1]
    h, w = sub.shape

    def axis(src, radius, horizontal):
        out = np.zeros_like(src)
        n = w if horizontal else h
        for y in range(h):
            for x in range(w):
                pos = x if horizontal else y
                if not dilate and (pos < radius or pos + radius >= n):
                    continue
                acc = np.full(4, F(0.0) if dilate else F(1.0), dtype=np.float32)
                for sp in range(max(pos - radius, 0), min(n - 1, pos + radius) + 1):
                    p = int(src[y, sp] if horizontal else src[sp, x])
                    al = p >> 24
                    v = np.array([F(0) if al == 0 else F(p >> s & 255) / F(al) for s in (0, 8, 16)] + [F(al) / F(255)],
                                 dtype=np.float32)
                    acc = np.maximum(acc, v) if dilate else np.minimum(acc, v)
                ch = [acc[0] * acc[3], acc[1] * acc[3], acc[2] * acc[3], acc[3]]
                q = [int(F(min(max(c, F(0)), F(1))) * F(255) + F(0.5)) for c in ch]
                out[y, x] = q[0] | q[1] << 8 | q[2] << 16 | q[3] << 24
        return out

    res = img.copy()
    res[y0:y1, x0:x1] = axis(axis(sub, min(rx, w - 1), True), min(ry, h - 1), False)
    return res


@pytest.mark.parametrize("kind, rx, ry", [(N.FILTER_DILATE, 2, 1), (N.FILTER_ERODE, 1, 2), (N.FILTER_DILATE, 0, 3),
                                          (N.FILTER_ERODE, 3, 0)])
def test_morphology_matches_numpy_restatement(kind, rx, ry):
    w, h = 21, 15
    img = premul_pixels(w * h, 100 + kind + 10 * rx + ry).reshape(h, w)
    rect = (3, 2, 19, 14)
    got = oracle_surface_chain(img.reshape(-1), w, rect, [(kind, (rx, ry))]).reshape(h, w)
    assert np.array_equal(got, np_morphology(img, rect, rx, ry, kind == N.FILTER_DILATE))


def test_morphology_known_answers():
    w, h = 16, 12
    img = np.zeros((h, w), dtype=np.uint32)
    img[5, 7] = 0xFF204080
    d = oracle_surface_chain(img.reshape(-1), w, (0, 0, w, h), [(N.FILTER_DILATE, (2, 1))]).reshape(h, w)
    want = np.zeros_like(img)
    want[4:7, 5:10] = 0xFF204080  # the opaque pixel grows to a 5 x 3 block
    assert np.array_equal(d, want)
    e = oracle_surface_chain(want.reshape(-1), w, (0, 0, w, h), [(N.FILTER_ERODE, (2, 1))]).reshape(h, w)
    assert np.array_equal(e, img)  # and erodes back to the pixel
    # an erosion whose doubled radius reaches the surface clears it
    full = np.full((h, w), 0xFF00FF00, dtype=np.uint32)
    assert not oracle_surface_chain(full.reshape(-1), w, (0, 0, w, h), [(N.FILTER_ERODE, (8, 1))]).any()


def canvas_chain(chain):
    """A scene with one filter layer over an opaque 2 x 2 block and the
    frame's filter arrays."""
    c = tk.Canvas(64, 48)
    c.push_filter_layer(chain, (8.0, 8.0, 56.0, 40.0))
    c.push_path(tk.BezPath().move_to(20, 20).line_to(22, 20).line_to(22, 22).line_to(20, 22).close(),
                tk.Brush.solid(0.0, 1.0, 0.0, 1.0))
    c.pop_layer()
    return c


def test_flood_and_drop_shadow_known_answers():
    flood = canvas_chain([(N.FILTER_FLOOD, (1.0, 0.0, 0.0, 0.5))])
    img = oracle.OracleRun(flood.scene_desc(), threads=2).get(oracle.OR_IMAGE, np.uint32).reshape(48, 64)
    # the flood replaces the group over the bounds, composited over the
    # transparent clear: premultiplied (0.5, 0, 0, 0.5)
    assert np.all(img[8:40, 8:56] == 0x80000080) and not img[:8].any() and not img[:, :8].any()
    shadow = canvas_chain([(N.FILTER_DROP_SHADOW, (3.0, 2.0, 0.0, (0.0, 0.0, 1.0, 1.0)))])
    a = shadow.scene_arrays()
    L, f = a["filter_layers"][0], a["filters"][0]
    assert (f["dx"], f["dy"], f["color"]) == (3, 2, 0xFFFF0000)
    assert list(L["surface"]) == [5, 5, 59, 43]  # reach: ceil(3 * 0) + max(3, 2)
    img = oracle.OracleRun(shadow.scene_desc(), threads=2).get(oracle.OR_IMAGE, np.uint32).reshape(48, 64)
    assert np.all(img[20:22, 20:22] == 0xFF00FF00)  # the source over its shadow
    assert np.all(img[22:24, 23:25] == 0xFFFF0000)  # the shadow where the source is not
    assert not img[30:, 30:].any()
    # offsets round half away from zero; the reach adds ceil(3 std_dev)
    c = canvas_chain([(N.FILTER_DROP_SHADOW, (2.5, -2.5, 1.2, (0, 0, 0, 1)))])
    a = c.scene_arrays()
    assert (a["filters"][0]["dx"], a["filters"][0]["dy"]) == (3, -3)
    assert list(a["filter_layers"][0]["surface"]) == [8 - 7, 8 - 7, 56 + 7, 40 + 7]  # ceil(3.6) + 3


def test_component_transfer_matches_numpy_and_identity():
    rng = np.random.default_rng(21)
    table = rng.integers(0, 256, N.TRANSFER_TABLE_WORDS).astype(np.uint32)
    px = premul_pixels(4000, 13)
    filters = np.zeros(1, dtype=N.FILTER_DTYPE)
    filters[0]["kind"], filters[0]["color"] = N.FILTER_COMPONENT_TRANSFER, 0
    got = px.copy()
    rect = np.array([0, 0, len(px), 1], dtype=np.int32)
    oracle.lib().or_filter_chain(N.ptr(got), len(px), N.ptr(rect), N.ptr(filters), 1, N.ptr(table))
    # filter_transfer_pixel restated in numpy float32
    a = (px >> 24).astype(np.int64)
    idx = [np.where(a == 0, 0, np.minimum(((px >> s & 255).astype(np.int64) * 255 + a // 2) // np.maximum(a, 1), 255))
           for s in (0, 8, 16)]
    sc = F(1.0) / F(255.0)
    ch = [table[256 * k + idx[k]].astype(np.float32) * sc for k in range(3)]
    al = table[768 + a].astype(np.float32) * sc
    q = [(np.clip(c * al, 0, 1) * F(255) + F(0.5)).astype(np.uint32) for c in ch]
    qa = (np.clip(al, 0, 1) * F(255) + F(0.5)).astype(np.uint32)
    assert np.array_equal(got, q[0] | q[1] << 8 | q[2] << 16 | qa << 24)
    # the identity table keeps opaque pixels
    ident = np.tile(np.arange(256, dtype=np.uint32), 4)
    opaque = (px & 0x00FFFFFF) | 0xFF000000
    out = opaque.copy()
    oracle.lib().or_filter_chain(N.ptr(out), len(px), N.ptr(rect), N.ptr(filters), 1, N.ptr(ident))
    assert np.array_equal(out, opaque)
    # the Canvas copies tables and indexes them in order
    c = tk.Canvas(64, 48)
    c.push_filter_layer([(N.FILTER_COMPONENT_TRANSFER, table), (N.FILTER_COMPONENT_TRANSFER, ident)], (0, 0, 32, 32))
    c.pop_layer()
    arr = c.scene_arrays()
    assert list(arr["filters"]["color"]) == [0, 1024]
    assert np.array_equal(arr["filter_words"], np.concatenate([table, ident]))
    with pytest.raises(ValueError):
        c.push_filter_layer([(N.FILTER_COMPONENT_TRANSFER, np.full(1024, 300))], (0, 0, 8, 8))


def oracle_convolve(img, rect, kernel, target, divisor, bias, edge, preserve):
    """The oracle's convolution over rect of a 2-D surface (a copy)."""
    h, w = img.shape
    kern = np.ascontiguousarray(kernel, dtype=np.float32)
    words = kern.view(np.uint32).reshape(-1).copy()
    f = np.zeros(1, dtype=N.FILTER_DTYPE)
    f[0]["kind"], f[0]["color"] = N.FILTER_CONVOLVE, 0
    f[0]["rows"], f[0]["columns"] = kern.shape
    f[0]["target_x"], f[0]["target_y"] = target
    f[0]["divisor"], f[0]["bias"], f[0]["edge_mode"], f[0]["preserve_alpha"] = divisor, bias, edge, int(preserve)
    out = np.ascontiguousarray(img, dtype=np.uint32).reshape(-1).copy()
    r = np.array(rect, dtype=np.int32)
    oracle.lib().or_filter_chain(N.ptr(out), w, N.ptr(r), N.ptr(f), 1, N.ptr(words))
    return out.reshape(h, w)


def np_convolve(img, rect, kernel, target, divisor, bias, edge, preserve):
    """filter_convolve_pixel restated with numpy float32 (normal divisors)."""
    x0, y0, x1, y1 = rect
    kern = np.asarray(kernel, dtype=np.float32)
    rows, cols = kern.shape
    out = img.copy()
    sc = F(1.0) / F(255.0)
    for y in range(y0, y1):
        for x in range(x0, x1):
            acc = [F(0)] * 4
            for ky in range(rows):
                for kx in range(cols):
                    wt = kern[rows - 1 - ky, cols - 1 - kx]
                    px, py = x + kx - target[0], y + ky - target[1]
                    p = 0
                    if edge == N.CONVOLVE_EDGE_DUPLICATE:
                        p = int(img[min(max(py, y0), y1 - 1), min(max(px, x0), x1 - 1)])
                    elif edge == N.CONVOLVE_EDGE_WRAP:
                        p = int(img[y0 + (py - y0) % (y1 - y0), x0 + (px - x0) % (x1 - x0)])
                    elif x0 <= px < x1 and y0 <= py < y1:
                        p = int(img[py, px])
                    al = p >> 24
                    v = [F(p >> s & 255) * sc for s in (0, 8, 16, 24)]
                    if preserve:
                        v[:3] = [F(0) if al == 0 else c / v[3] for c in v[:3]]
                    v[3] = F(al)
                    acc = [mad(v[c], wt, acc[c]) for c in range(4)]
            rc = F(1.0) / F(divisor)
            q = [acc[c] * rc for c in range(3)]
            qa = (acc[3] * rc) * sc
            ua = F(int(img[y, x]) >> 24) * sc if preserve else qa + F(bias)
            a = F(min(max(ua, F(0)), F(1)))
            bb = F(bias) * ua
            col = [q[c] + bb for c in range(3)]
            col = [F(min(max(c, F(0)), F(1))) * a if preserve else F(min(max(c, F(0)), a)) for c in col]
            b = [int(F(min(max(c, F(0)), F(1))) * F(255) + F(0.5)) for c in col + [a]]
            out[y, x] = b[0] | b[1] << 8 | b[2] << 16 | b[3] << 24
    return out


CONVOLVE_CASES = [
    ([[1, 1, 1], [1, 1, 1], [1, 1, 1]], (1, 1), 9.0, 0.0, 1, False),
    ([[0, -1, 0], [-1, 4, -1], [0, -1, 0]], (1, 1), 1.0, 0.25, 2, False),
    ([[1, 2, 0.5, -1, 3], [0, 1, 0, 2, 1]], (3, 0), 6.5, -0.1, 0, True),
    ([[0.2, 0.7], [0.4, -0.3]], (0, 1), 0.8, 0.0, 0, False),
]


@pytest.mark.parametrize("case", range(len(CONVOLVE_CASES)))
def test_convolution_matches_numpy_restatement(case):
    kernel, target, divisor, bias, edge, preserve = CONVOLVE_CASES[case]
    w, h = 14, 11
    img = premul_pixels(w * h, 300 + case).reshape(h, w)
    rect = (2, 1, 13, 10)
    got = oracle_convolve(img, rect, kernel, target, divisor, bias, edge, preserve)
    want = np_convolve(img, rect, kernel, target, divisor, bias, edge, preserve)
    d = np.abs(np.stack([(got >> s) & 255 for s in (0, 8, 16, 24)]).astype(np.int64)
               - np.stack([(want >> s) & 255 for s in (0, 8, 16, 24)]).astype(np.int64))
    assert d.max() <= 1 and (d == 0).mean() >= 0.99, (d.max(), (d == 0).mean())


def test_convolution_identity_and_divisor_ranges():
    w, h = 12, 9
    img = premul_pixels(w * h, 77).reshape(h, w)
    ident = [[0, 0, 0], [0, 1, 0], [0, 0, 0]]
    for edge in (0, 1, 2):
        assert np.array_equal(oracle_convolve(img, (0, 0, w, h), ident, (1, 1), 1.0, 0.0, edge, False), img)
    # a zero divisor or an empty kernel keeps the centre
    assert np.array_equal(oracle_convolve(img, (0, 0, w, h), ident, (1, 1), 0.0, 0.0, 1, False), img)
    # kernel and divisor scaled together by 2^-140 (a subnormal divisor) or
    # 2^100 (a huge one) give the same image as unscaled
    base = oracle_convolve(img, (0, 0, w, h), [[1, 2, 1], [2, 4, 2], [1, 2, 1]], (1, 1), 16.0, 0.0, 1, False)
    tiny = np.float32(2.0 ** -140)
    sub = oracle_convolve(img, (0, 0, w, h), np.float32([[1, 2, 1], [2, 4, 2], [1, 2, 1]]) * tiny, (1, 1),
                          np.float32(16.0) * tiny, 0.0, 1, False)
    assert np.abs(sub.astype(np.int64) - base.astype(np.int64)).max() <= 0x01010101
    huge = np.float32(2.0 ** 100)
    big = oracle_convolve(img, (0, 0, w, h), np.float32([[1, 2, 1], [2, 4, 2], [1, 2, 1]]) * huge, (1, 1),
                          np.float32(16.0) * huge, 0.0, 1, False)
    assert np.array_equal(big, base)


def test_path_regions_and_transformed_replay():
    # a path region's bounds are its tight box under the transform and scale
    c = tk.Canvas(128, 96, scale=2.0)
    circle = tk.BezPath().move_to(30, 20)
    circle.cubic_to(30, 25.5, 25.5, 30, 20, 30).cubic_to(14.5, 30, 10, 25.5, 10, 20)
    circle.cubic_to(10, 14.5, 14.5, 10, 20, 10).cubic_to(25.5, 10, 30, 14.5, 30, 20).close()
    c.push_filter_layer([(N.FILTER_INVERT, 1.0)], circle, transform=(1, 0, 0, 1, 3.5, 0))
    c.pop_layer()
    L = c.scene_arrays()["filter_layers"][0]
    # the curve's extrema: x in [13.5, 33.5], y in [10, 30], times the scale 2
    assert list(L["surface"]) == [27, 20, 67, 60]
    # a retained node's rect region under a rotation becomes the rotated
    # rectangle's bounds; under a translation it moves
    node = tk.Canvas(128, 96)
    node.keep_commands()
    node.push_filter_layer([(N.FILTER_GRAYSCALE, 1.0)], (10.0, 10.0, 30.0, 20.0))
    node.push_path(tk.BezPath().move_to(12, 12).line_to(28, 12).line_to(28, 18).close(), tk.Brush.solid(1, 0, 0, 1))
    node.pop_layer()
    rs = tk.RetainedScene(128, 96)
    rs.insert(1, node, transform=(0.0, 1.0, -1.0, 0.0, 60.0, 0.0))  # x' = 60 - y, y' = x
    canvas, _ = rs.materialize()
    assert list(canvas.scene_arrays()["filter_layers"][0]["surface"]) == [40, 10, 50, 30]
    rs.set_transform(1, (1.0, 0.0, 0.0, 1.0, 5.0, 7.0))
    canvas, _ = rs.materialize()
    assert list(canvas.scene_arrays()["filter_layers"][0]["surface"]) == [15, 17, 35, 27]


def test_chain_blur_equals_a_blur_group_over_the_canvas():
    """Filter::Blur in a chain over a region covering the canvas blurs what a
    blur group of the same deviation blurs (both over the whole canvas)."""
    def scene(as_filter):
        from layer_cases import blob
        rng = np.random.default_rng(5)
        c = tk.Canvas(96, 72)
        c.set_clear_color(0xFFFFFFFF)
        if as_filter:
            c.push_filter_layer([(N.FILTER_BLUR, (3.0, 3.0))], (0.0, 0.0, 96.0, 72.0))
        else:
            c.push_blur_group(3.0)
        c.push_path(tk.BezPath().move_to(-5, -5).line_to(101, -5).line_to(101, 77).line_to(-5, 77).close(),
                    tk.Brush.solid(0.2, 0.5, 0.7, 0.6))
        for _ in range(5):
            c.push_path(blob(rng, rng.uniform(10, 86), rng.uniform(10, 62), 15), tk.Brush.solid(*rng.uniform(0, 1, 3), 1.0))
        c.pop_layer()
        return c
    a, b = scene(True), scene(False)
    ia = oracle.OracleRun(a.scene_desc(), threads=2).get(oracle.OR_IMAGE, np.uint32)
    ib = oracle.OracleRun(b.scene_desc(), threads=2).get(oracle.OR_IMAGE, np.uint32)
    assert np.array_equal(ia, ib)
    # one axis only blurs along it: a vertical stripe stays within its
    # columns, whole away from the top and bottom (transparent beyond them)
    c = tk.Canvas(40, 30)
    c.push_filter_layer([(N.FILTER_BLUR, (0.0, 2.0))], (0.0, 0.0, 40.0, 30.0))
    c.push_path(tk.BezPath().move_to(18, -2).line_to(22, -2).line_to(22, 32).line_to(18, 32).close(),
                tk.Brush.solid(0, 0, 0, 1))
    c.pop_layer()
    img = oracle.OracleRun(c.scene_desc(), threads=1).get(oracle.OR_IMAGE, np.uint32).reshape(30, 40)
    assert np.all(img[7:23, 18:22] == 0xFF000000) and not img[:, :18].any() and not img[:, 22:].any()
    assert np.all((img[0, 18:22] >> 24) < 255)

