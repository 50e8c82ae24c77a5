"""Differentiable rendering on the GPU against the FP64 restatement: the float
forward image, and dL/d(control points, colours, sigma) from the hand-written
adjoint against FP64 central finite differences of the same model (the
forward's flattening held fixed)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import tileink_b200 as tk
from tileink_b200 import diff
from tileink_b200.renderer import TileinkError

pytestmark = pytest.mark.gpu

GRAD_REL_TOLERANCE = 1e-3   # ||analytic - fd|| / ||fd|| over the checked parameters
IMAGE_TOLERANCE = 1e-5      # |f32 forward - f64 forward| per channel


def target_for(scene_target: diff.DiffScene) -> np.ndarray:
    lines, ep, w = diff.flatten(scene_target)
    zero = np.zeros((scene_target.height, scene_target.width, 4), np.float32)
    _, img = oracle.diff_loss(scene_target, lines, ep, w, scene_target.points, scene_target.colors,
                              scene_target.sigma, zero, return_image=True)
    return img.astype(np.float32)


def fd_check(renderer, sc, target, n_top=12, n_rand=6, n_col=8, h_pt=1e-3, h_col=1e-4, h_sigma=1e-3, seed=0):
    loss, img = renderer.diff_forward(sc, target, return_image=True)
    dp, dc, ds = renderer.diff_backward()
    lines, ep, w = diff.flatten(sc)

    def L(points=None, colors=None, sigma=None):
        return oracle.diff_loss(sc, lines, ep, w, sc.points if points is None else points,
                                sc.colors if colors is None else colors, sc.sigma if sigma is None else sigma,
                                target)

    rng = np.random.default_rng(seed)
    a, f = [], []
    flat = np.abs(dp).reshape(-1)
    for i in list(np.argsort(-flat)[:n_top]) + list(rng.choice(flat.size, n_rand, replace=False)):
        P = sc.points.astype(np.float64).reshape(-1).copy()
        P[i] += h_pt
        lp = L(points=P.reshape(sc.points.shape))
        P[i] -= 2 * h_pt
        lm = L(points=P.reshape(sc.points.shape))
        a.append(dp.reshape(-1)[i])
        f.append((lp - lm) / (2 * h_pt))
    flatc = np.abs(dc).reshape(-1)
    for i in list(np.argsort(-flatc)[:n_col // 2]) + list(rng.choice(flatc.size, n_col - n_col // 2, replace=False)):
        Cc = sc.colors.astype(np.float64).reshape(-1).copy()
        Cc[i] += h_col
        lp = L(colors=Cc.reshape(sc.colors.shape))
        Cc[i] -= 2 * h_col
        lm = L(colors=Cc.reshape(sc.colors.shape))
        a.append(dc.reshape(-1)[i])
        f.append((lp - lm) / (2 * h_col))
    if sc.sigma > 0:
        a.append(ds)
        f.append((L(sigma=sc.sigma + h_sigma) - L(sigma=sc.sigma - h_sigma)) / (2 * h_sigma))
    a, f = np.array(a, np.float64), np.array(f, np.float64)
    return loss, img, np.linalg.norm(a - f) / np.linalg.norm(f)


def test_gpu_diff_forward_matches_fp64_model(renderer):
    sc = diff.blur_group_scene(5, width=256, height=256, paths=16)
    target = target_for(diff.blur_group_scene(5, width=256, height=256, paths=16, jitter=3.0))
    loss, img = renderer.diff_forward(sc, target, return_image=True)
    lines, ep, w = diff.flatten(sc)
    ol, oimg = oracle.diff_loss(sc, lines, ep, w, sc.points, sc.colors, sc.sigma, target, return_image=True)
    assert np.abs(img - oimg).max() <= IMAGE_TOLERANCE
    assert abs(loss - ol) <= 1e-5 * ol


def test_gpu_diff_gradients_match_fp64_central_differences(renderer):
    sc = diff.blur_group_scene(7, width=256, height=256, paths=16)
    target = target_for(diff.blur_group_scene(7, width=256, height=256, paths=16, jitter=3.0))
    _, _, rel = fd_check(renderer, sc, target)
    assert rel <= GRAD_REL_TOLERANCE, rel


def test_gpu_diff_gradients_blur_group_workload(renderer):
    # 1024x1024, 256 closed paths x 12 cubics, sigma 4, target from parameters
    # jittered by N(0, 3^2) px
    sc = diff.blur_group_scene(5)
    target = target_for(diff.blur_group_scene(5, jitter=3.0))
    _, _, rel = fd_check(renderer, sc, target, n_top=8, n_rand=4, n_col=6)
    assert rel <= GRAD_REL_TOLERANCE, rel


def test_gpu_diff_gradients_without_blur(renderer):
    sc = diff.blur_group_scene(9, width=192, height=160, paths=10).with_params(sigma=0.0)
    tg = diff.blur_group_scene(9, width=192, height=160, paths=10, jitter=2.0).with_params(sigma=0.0)
    _, _, rel = fd_check(renderer, sc, target_for(tg))
    assert rel <= GRAD_REL_TOLERANCE, rel


def test_gpu_diff_zero_loss_has_zero_gradient(renderer):
    sc = diff.blur_group_scene(3, width=128, height=128, paths=6)
    _, img = renderer.diff_forward(sc, np.zeros((128, 128, 4), np.float32), return_image=True)
    loss = renderer.diff_forward(sc, img)
    dp, dc, ds = renderer.diff_backward()
    assert loss == 0.0
    assert not dp.any() and not dc.any() and ds == 0.0


def test_gpu_diff_backward_needs_a_forward():
    r = tk.NativeRenderer(0)
    try:
        with pytest.raises(TileinkError):
            r.diff_backward()
        # a plain scene upload invalidates the last differentiable forward
        sc = diff.blur_group_scene(3, width=64, height=64, paths=3)
        r.diff_forward(sc, np.zeros((64, 64, 4), np.float32))
        r.upload(tk.generate(1, 1, width=64, height=64, paths=3))
        with pytest.raises(TileinkError):
            r.diff_backward()
    finally:
        r.close()
