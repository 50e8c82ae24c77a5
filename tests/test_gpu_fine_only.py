"""The GPU pipeline against the fine-only oracle for path fills
(src/native/runtime/tests/coarse_count/rect_pixels.rs:3-14, the method the
reference applies to SDF rects): every draw of every batch interpreted in
every tile with the tile's segment range and cumsum backdrop, and every clip
and opacity layer as an explicit BEGIN/END pair, with no tile bins, particle
or wrapper elision, colour promotion or occlusion skip. The device's coarse
decisions are thereby checked against something other than a restatement of
the same coarse algorithm. Pixels must be identical."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import tileink_b200 as tk

pytestmark = pytest.mark.gpu


def check(renderer, canvas):
    img = renderer.render_to_image(canvas)
    want = oracle.interpret_path_draws(canvas.scene_desc(), threads=8)
    assert np.array_equal(img, want), int((img != want).any(axis=2).sum())
    return img


def test_gpu_small_cubic_fills_equal_fine_only_oracle(renderer):
    """640x360, 240 closed cubic paths (seed 1)."""
    check(renderer, tk.generate(1, 1))


@pytest.mark.parametrize("seed", [2, 7])
def test_gpu_mixed_scene_equals_fine_only_oracle(renderer, seed):
    """768x512, 600 paths: fills and strokes, even-odd, gradients, clip
    layers nested to depth 4."""
    check(renderer, tk.generate(2, seed, width=768, height=512, paths=600))


def test_gpu_glyphs_equal_fine_only_oracle(renderer):
    check(renderer, tk.generate(3, 3, width=480, height=270, paths=1500))


def test_gpu_clip_stack_deeper_than_registers_equals_fine_only_oracle(renderer):
    cv = tk.Canvas(96, 96)
    cv.set_clear_color(0xFFFFFFFF)
    for k in range(6):
        s = 2 + k * 3
        cv.push_clip_layer(tk.BezPath().move_to(s, s + 1).line_to(96 - s, s).line_to(90 - s, 96 - s)
                           .line_to(s + 2, 94 - s).close())
    cv.push_path(tk.BezPath().move_to(0, 0).line_to(96, 10).line_to(80, 96).line_to(5, 90).close(),
                 tk.Brush.solid(1, 0, 0, 0.9))
    for _ in range(6):
        cv.pop_layer()
    cv.push_path(tk.BezPath().move_to(10, 10).line_to(60, 12).line_to(30, 70).close(),
                 tk.Brush.solid(0, 0.5, 1, 1))
    check(renderer, cv)
