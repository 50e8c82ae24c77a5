"""Clip, SDF-clip and opacity layers on the GPU: fused opacity layers against
the oracle (every stage) and the fine-only oracle, the reference's
nested-stack END order (src/native/runtime/tests/coarse_count/emit.rs:58-84)
and its draw-count cases across 256-draw pages (emit.rs:5-34)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import tileink_b200 as tk
from tileink_b200 import _native as N

from layer_cases import opacity_scene
from test_gpu_parity import compare_frame

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_gpu_opacity_layers_match_oracle_and_fine_only(renderer, seed):
    c = opacity_scene(seed)
    img, ref = compare_frame(renderer, c)
    tags = renderer.debug(N.STAGE_PTCL, 0)["tag"]
    assert (tags == N.PTCL_BEGIN_OPACITY).sum() > 10
    want = oracle.interpret_path_draws(c.scene_desc(), threads=8)
    assert np.array_equal(img, want), int((img != want).any(axis=2).sum())


def tile_stream(ptcl, tiles, t):
    return ptcl[int(tiles["ptcl_start"][t]):int(tiles["ptcl_end"][t])]


def test_gpu_nested_stack_end_order(renderer):
    """emit.rs:58-84 restated without the blend wrapper (blend layers are
    outside this path): an opacity layer, a clip that covers the tile (a
    no-op wrapper, dropped at both ends) and an SDF clip around a draw give
    BEGIN_OPACITY (payload in `color`), BEGIN_SDF_CLIP, the draw, then the
    ends in reverse: END_CLIP, END_OPACITY, END."""
    c = tk.Canvas(32, 32)
    c.set_clear_color(0xFFFFFFFF)
    c.push_opacity_layer(tk.BezPath().move_to(2, 3).line_to(14, 1).line_to(12, 15).line_to(1, 12).close(), 0.3)
    c.push_clip_layer(tk.BezPath().move_to(-40, -30).line_to(70, -35).line_to(75, 70).line_to(-35, 72).close())
    c.push_clip_sdf_circle_layer(8.0, 8.0, 6.5)
    c.push_path(tk.BezPath().move_to(3, 3).line_to(13, 4).line_to(9, 13).close(), tk.Brush.solid(0.2, 0.4, 0.8, 1))
    c.pop_layer()
    c.pop_layer()
    c.pop_layer()
    layers = c.scene_arrays()["layers"]
    assert list(layers["tag"]) == [N.LAYER_OPACITY, N.LAYER_CLIP, N.LAYER_CLIP]
    img = renderer.render_to_image(c)
    ptcl, tiles = renderer.debug(N.STAGE_PTCL, 0), renderer.debug(N.STAGE_TILES, 0)
    s = tile_stream(ptcl, tiles, 0)
    assert list(s["tag"]) == [N.PTCL_BATCH_BEGIN, N.PTCL_BEGIN_OPACITY, N.PTCL_BEGIN_SDF_CLIP, N.PTCL_FILL,
                              N.PTCL_END_CLIP, N.PTCL_END_OPACITY, N.PTCL_END]
    assert s[1]["color"] == 77  # opacity_f32_to_u8(0.3)
    assert s[2]["color"] == layers[2]["draw"]
    assert s[1]["segment_end"] > s[1]["segment_start"]
    ref = oracle.OracleRun(c.scene_desc(), threads=2)
    assert np.array_equal(ptcl, ref.get(oracle.OR_PASS_PTCL, N.PTCL_DTYPE, 0))
    assert np.array_equal(img, ref.get(oracle.OR_IMAGE, np.uint32).view(np.uint8).reshape(img.shape))
    assert np.array_equal(img, oracle.interpret_path_draws(c.scene_desc(), threads=2))


@pytest.mark.parametrize("draws", [0, 1, 255, 256, 257, 513])
@pytest.mark.parametrize("stack", [0, 1, 2, 3])
def test_gpu_draw_counts_across_pages(renderer, draws, stack):
    """emit.rs:5-34's draw counts around 256-draw pages under 0-3 clip
    wrappers: tile 0 of a 48x16 canvas holds every draw, in painter order,
    between its wrappers; the other tiles hold none."""
    rng = np.random.default_rng(draws * 7 + stack)
    c = tk.Canvas(48, 16)
    c.set_clear_color(0xFFFFFFFF)
    for k in range(stack):
        r = 7.5 - k
        c.push_clip_layer(tk.BezPath().move_to(8 - r, 8).line_to(8, 8 - r).line_to(8 + r, 8).line_to(8, 8 + r)
                          .close())
    for k in range(draws):
        x, y = rng.uniform(1, 12, 2)
        c.push_path(tk.BezPath().move_to(x, y).line_to(x + 3, y + 0.5).line_to(x + 1, y + 2.5).close(),
                    tk.Brush.solid(*rng.uniform(0, 1, 3), float(rng.uniform(0.2, 1))))
    for k in range(stack):
        c.pop_layer()
    c.push_path(tk.BezPath().move_to(20, 2).line_to(30, 3).line_to(25, 12).close(), tk.Brush.solid(0, 0, 0, 1))
    img = renderer.render_to_image(c)
    ptcl, tiles = renderer.debug(N.STAGE_PTCL, 0), renderer.debug(N.STAGE_TILES, 0)
    s = tile_stream(ptcl, tiles, 0)
    if draws:
        fills = s[s["tag"] == N.PTCL_FILL]
        assert len(fills) == draws
        assert list(fills["color"]) == list(range(stack, stack + draws))  # painter order: draw indices
        assert (s["tag"] == N.PTCL_BEGIN_CLIP).sum() == stack and (s["tag"] == N.PTCL_END_CLIP).sum() == stack
    ref = oracle.OracleRun(c.scene_desc(), threads=4)
    assert np.array_equal(tiles, ref.get(oracle.OR_PASS_TILES, N.TILE_DTYPE, 0))
    assert np.array_equal(ptcl, ref.get(oracle.OR_PASS_PTCL, N.PTCL_DTYPE, 0))
    assert np.array_equal(img, ref.get(oracle.OR_IMAGE, np.uint32).view(np.uint8).reshape(img.shape))
    assert np.array_equal(img, oracle.interpret_path_draws(c.scene_desc(), threads=4))


@pytest.mark.parametrize("factor, down, up", [(2, 1, 1), (3, 1, 1), (4, 0, 0), (4, 1, 0), (8, 0, 1), (5, 1, 1)])
def test_gpu_sampled_blur_matches_oracle(renderer, factor, down, up):
    """Blur groups through a copy reduced by `factor` (BlurSampling;
    filter/resample.hlsli): downsample, Gaussian at sigma / factor,
    upsample, composite — bit-exact against the oracle."""
    from layer_cases import sampled_blur_scene
    compare_frame(renderer, sampled_blur_scene(factor * 7 + down, factor, down, up, sigma=6.5))


@pytest.mark.parametrize("seed, sigma, quality, uniform", [(1, 6.0, 0, False), (2, 9.5, 1, False), (3, 4.0, 0, True),
                                                            (4, 0.9, 0, False), (5, 24.0, 1, False)])
def test_gpu_progressive_blur_matches_oracle(renderer, seed, sigma, quality, uniform):
    """Progressive blur groups (Filter::ProgressiveBlur; filter/progressive.hlsl):
    the pyramid reductions, the variance-bracketing resolve and the 7-tap
    shallow blur, bit-exact against the oracle."""
    from layer_cases import progressive_scene
    compare_frame(renderer, progressive_scene(seed, sigma=sigma, quality=quality, uniform=uniform))


@pytest.mark.parametrize("name", ["brightness", "contrast", "grayscale", "hue_rotate", "invert", "opacity",
                                  "saturate", "sepia", "matrix", "matrix_alpha", "offset", "chain", "erode",
                                  "dilate", "morphology_chain", "flood", "drop_shadow", "drop_shadow_sharp",
                                  "drop_shadow_wide", "component_transfer", "convolve_box", "convolve_edges",
                                  "convolve_preserve", "blur_xy", "blur_x_only"])
def test_gpu_filter_layers_match_oracle(renderer, name):
    """Filter layers (Canvas::push_filter_layer with a chain; filter/color.hlsli,
    filter/basic.hlsl): every colour filter, the colour matrix, offsets and a
    mixed chain, bit-exact against the oracle."""
    from layer_cases import filter_chains, filter_scene
    # the surface (the region grown by the chain's reach, up to 25 px here)
    # stays inside the 200 x 150 canvas, as spatial filters need
    compare_frame(renderer, filter_scene(11, filter_chains()[name], (30.5, 28.0, 165.2, 117.9)))


def test_gpu_filter_layer_regions(renderer):
    """Regions partly or wholly off the canvas (colour filters only), a fixed
    region with an offset, an empty region, and filter layers nested in blur
    groups and in each other."""
    from layer_cases import blob, filter_scene
    compare_frame(renderer, filter_scene(4, [(N.FILTER_SEPIA, 0.9), (N.FILTER_SATURATE, 1.7)], (-40.0, -20.5, 90.0, 80.0)))
    compare_frame(renderer, filter_scene(5, [(N.FILTER_INVERT, 1.0)], (150.0, 100.0, 400.0, 300.0)))
    compare_frame(renderer, filter_scene(6, [(N.FILTER_GRAYSCALE, 1.0)], (300.0, 300.0, 400.0, 400.0)))
    compare_frame(renderer, filter_scene(7, [(N.FILTER_OFFSET, (-9.0, 6.0))], (30.0, 30.0, 120.0, 110.0),
                                         fixed_region=True))
    compare_frame(renderer, filter_scene(8, [(N.FILTER_HUE_ROTATE, 90.0)], (50.0, 50.0, 50.0, 90.0)))
    compare_frame(renderer, filter_scene(12, [(N.FILTER_DILATE, (2.0, 2.0)), (N.FILTER_SEPIA, 1.0)],
                                         blob(np.random.default_rng(3), 100.0, 75.0, 40.0)))
    rng = np.random.default_rng(9)
    c = tk.Canvas(200, 150)
    c.set_clear_color(0xFF202020)
    c.push_blur_group(3.0)
    c.push_filter_layer([(N.FILTER_CONTRAST, 1.8), (N.FILTER_OFFSET, (4.0, 4.0))], (20.0, 20.0, 150.0, 120.0))
    for _ in range(6):
        c.push_path(blob(rng, rng.uniform(40, 130), rng.uniform(40, 100), 25), tk.Brush.solid(*rng.uniform(0, 1, 3), 0.9))
    c.push_filter_layer([(N.FILTER_INVERT, 0.6)], (60.0, 40.0, 140.0, 110.0))
    c.push_path(blob(rng, 100, 75, 30), tk.Brush.solid(0.9, 0.4, 0.1, 1.0))
    c.pop_layer()
    c.pop_layer()
    c.pop_layer()
    compare_frame(renderer, c)


def test_gpu_offset_filter_past_the_canvas_is_rejected(renderer):
    """An offset or morphology filter layer whose surface reaches past the
    canvas would read pixels this path's canvas-sized surfaces do not hold:
    refused at upload, and the context stays usable."""
    from layer_cases import filter_scene
    c = filter_scene(2, [(N.FILTER_OFFSET, (5.0, 5.0))], (-10.0, 0.0, 50.0, 50.0))
    with pytest.raises(tk.TileinkError, match="whose surface reaches past"):
        renderer.upload(c)
    c = filter_scene(2, [(N.FILTER_DILATE, (3.0, 3.0))], (10.0, 10.0, 198.0, 100.0))
    with pytest.raises(tk.TileinkError, match="whose surface reaches past"):
        renderer.upload(c)
    compare_frame(renderer, filter_scene(2, [(N.FILTER_OFFSET, (5.0, 5.0))], (10.0, 10.0, 50.0, 50.0)))
