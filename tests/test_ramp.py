"""Every word of the gradient ramps against an independent restatement of the
reference's build_ramp (src/shared/brush.rs:638-689).

The reference builds each ramp entry from peniko 0.6.1's premultiplied
interpolation, implemented by the `color` crate 0.3.3 (Cargo.lock:110-112;
neither is vendored): `left.interpolate(right, Srgb, Shorter)` premultiplies
both stops (rgb * alpha) and keeps their differences, `eval(t)` returns
premul = premul1 + delta_premul * t and alpha = alpha1 + t * delta_alpha and
un-premultiplies (scale by 1 / alpha, or by 1 when alpha is 0);
`to_alpha_color::<Srgb>()` is the identity in sRGB, and `premultiply()`
scales by alpha again. premul_f32_to_u32 (src/shared/pixel.rs:14-21) then
stores `(c * 255 + 0.5) as u8` (Rust's saturating cast). The restatement below
does those f32 operations in that order with numpy float32 scalars."""
from __future__ import annotations

import numpy as np
import pytest

import tileink_b200 as tk

F = np.float32


def u8(x) -> int:
    """Rust `f32 as u8`: truncation toward zero, saturating, NaN -> 0."""
    v = F(F(x) * F(255.0) + F(0.5))
    if np.isnan(v):
        return 0
    return int(min(max(np.trunc(v), 0.0), 255.0))


def interpolate_eval_premultiply(left, right, t):
    """color 0.3.3: DynamicColor::interpolate(...).eval(t), then
    to_alpha_color::<Srgb>().premultiply(), in f32."""
    (r1, g1, b1, a1), (r2, g2, b2, a2) = [[F(v) for v in c] for c in (left, right)]
    p1 = [F(r1 * a1), F(g1 * a1), F(b1 * a1)]
    p2 = [F(r2 * a2), F(g2 * a2), F(b2 * a2)]
    delta = [F(p2[k] - p1[k]) for k in range(3)]
    delta_alpha = F(a2 - a1)
    t = F(t)
    premul = [F(p1[k] + F(delta[k] * t)) for k in range(3)]
    alpha = F(a1 + F(t * delta_alpha))
    inv = F(1.0) if alpha == F(0.0) else F(F(1.0) / alpha)
    opaque = [F(c * inv) for c in premul]
    return [F(c * alpha) for c in opaque] + [alpha]


def reference_ramp(stops, size):
    """build_ramp (src/shared/brush.rs:638-689), one packed RGBA8 word per entry."""
    size = max(size, 2)
    if not stops:
        return [0] * size
    s = sorted(stops, key=lambda st: st[0])  # sort_by(total_cmp) is stable
    out = []
    for ix in range(size):
        t = F(F(ix) / F(size - 1))
        upper = sum(1 for st in s if F(st[0]) < t)  # partition_point(offset < t)
        if upper == 0:
            left = right = s[0]
        elif upper >= len(s):
            left = right = s[-1]
        else:
            left, right = s[upper - 1], s[upper]
        span = F(F(right[0]) - F(left[0]))
        if abs(span) <= F(np.finfo(np.float32).eps):
            lt = F(0.0)
        else:
            lt = F(min(max(F(F(t - F(left[0])) / span), F(0.0)), F(1.0)))
        c = interpolate_eval_premultiply(left[1], right[1], lt)
        r, g, b, a = (u8(v) for v in c)
        out.append(r | (g << 8) | (b << 16) | (a << 24))
    return out


def ramp_words(canvas):
    """The ramp payload of the canvas's first draw's brush (header word 2:
    payload offset from the brush start, word 3: its length)."""
    a = canvas.scene_arrays()
    off = int(a["draws"]["brush_offset"][0])
    blob = a["brush"]
    start, n = int(blob[off + 2]), int(blob[off + 3])
    return [int(w) for w in blob[off + start: off + start + n]]


def random_stops(rng, n):
    offsets = np.sort(rng.uniform(0, 1, n)).astype(np.float32)
    if rng.uniform() < 0.5:
        offsets[0], offsets[-1] = 0.0, 1.0
    if n > 2 and rng.uniform() < 0.3:
        offsets[1] = offsets[2]  # two stops at one offset: a hard edge
    cols = []
    for k in range(n):
        a = float(rng.choice([rng.uniform(0.02, 1.0), 1.0, 0.0, 0.5]))
        cols.append((*rng.uniform(0, 1, 3).astype(np.float32).tolist(), a))
    return [(float(o), c) for o, c in zip(offsets, cols)]


@pytest.mark.parametrize("seed", range(40))
def test_ramp_words_equal_the_reference_interpolation(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 7))
    stops = random_stops(rng, n)
    span = float(rng.choice([10.0, 300.0, 3000.0]))
    c = tk.Canvas(64, 64)
    path = tk.BezPath().move_to(0, 0).line_to(64, 0).line_to(64, 64).close()
    if seed % 2:
        c.push_path(path, tk.Brush.linear((0, 0), (span, 0), stops))
    else:
        c.push_path(path, tk.Brush.radial((0, 0), 0.0, (0, 0), span, stops))
    got = ramp_words(c)
    assert len(got) >= 64
    want = reference_ramp(stops, len(got))
    bad = [i for i in range(len(got)) if got[i] != want[i]]
    assert not bad, (len(bad), bad[:5], [hex(got[i]) for i in bad[:3]], [hex(want[i]) for i in bad[:3]])


def test_ramp_translucent_two_stop_interior():
    """Alpha below 1 on both ends: the interior entries go through the
    un-premultiply / premultiply round trip."""
    stops = [(0.0, (0.9, 0.2, 0.1, 0.35)), (1.0, (0.1, 0.7, 0.95, 0.8))]
    c = tk.Canvas(64, 64)
    c.push_path(tk.BezPath().move_to(0, 0).line_to(64, 0).line_to(64, 64).close(),
                tk.Brush.linear((0, 0), (2000, 0), stops))
    got = ramp_words(c)
    assert got == reference_ramp(stops, len(got))
    assert len(set(got)) > 100


@pytest.mark.parametrize("rgb0, alpha, want", [
    # (x * (1 / a)) * a lands one ulp across a byte boundary of x * 255 + 0.5
    (0.26179054379463196, 0.951216995716095, 63),   # direct premultiplied value: 64
    (0.689500629901886, 0.452160120010376, 80),      # direct: 79
    (0.0956406369805336, 0.9635743498802185, 23),    # direct: 24
])
def test_ramp_keeps_the_unpremultiply_round_trip(rgb0, alpha, want):
    """Entry 0 is the first stop evaluated at t = 0: premultiplied,
    un-premultiplied and premultiplied again, as the reference's
    interpolator does; a plain premultiply gives the neighbouring byte."""
    stops = [(0.0, (rgb0, 0.5, 0.5, alpha)), (1.0, (0.0, 0.0, 0.0, 1.0))]
    c = tk.Canvas(64, 64)
    c.push_path(tk.BezPath().move_to(0, 0).line_to(64, 0).line_to(64, 64).close(),
                tk.Brush.linear((0, 0), (100, 0), stops))
    got = ramp_words(c)
    assert got[0] & 0xFF == want
    assert got == reference_ramp(stops, len(got))
