"""Differentiable rendering: the Python side of include/tileink_diff.h.

A `DiffScene` holds closed cubic paths (move_to, `cubics` cubic_to, close)
drawn with straight RGBA colours into one Gaussian blur group over an opaque
background. `NativeRenderer.diff_forward` renders it and returns the mean
squared error against a target; `NativeRenderer.diff_backward` returns
dL/d(points, colours, sigma) from the hand-written adjoint on the GPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .canvas import generate


@dataclass
class DiffScene:
    width: int
    height: int
    points: np.ndarray            # [paths, 1 + 3 * cubics, 2] float32
    colors: np.ndarray            # [paths, 4] float32, straight RGBA
    sigma: float = 4.0
    tolerance: float = 0.1
    background: tuple = (1.0, 1.0, 1.0, 1.0)
    # pixel rows [r0, r1) of the loss; None: every row (the rows of a
    # row-split objective, whose ranks sum their gradients)
    loss_rows: tuple | None = None
    _keep: list = field(default_factory=list, repr=False)

    @property
    def path_count(self) -> int:
        return int(self.points.shape[0])

    @property
    def cubics(self) -> int:
        return (int(self.points.shape[1]) - 1) // 3

    def desc(self) -> N.DiffScene:
        pts = np.ascontiguousarray(self.points, dtype=np.float32)
        cols = np.ascontiguousarray(self.colors, dtype=np.float32)
        if pts.ndim != 3 or pts.shape[2] != 2 or (pts.shape[1] - 1) % 3 or cols.shape != (pts.shape[0], 4):
            raise ValueError("points must be [paths, 1 + 3k, 2] and colors [paths, 4]")
        self._keep = [pts, cols]
        d = N.DiffScene()
        d.width, d.height = int(self.width), int(self.height)
        d.path_count, d.cubics_per_path = pts.shape[0], (pts.shape[1] - 1) // 3
        d.points, d.colors = pts.ctypes.data, cols.ctypes.data
        d.sigma, d.tolerance = float(self.sigma), float(self.tolerance)
        for i in range(4):
            d.background[i] = float(self.background[i])
        if self.loss_rows is not None:
            d.loss_row0, d.loss_row1 = int(self.loss_rows[0]), int(self.loss_rows[1])
        return d

    def with_params(self, points=None, colors=None, sigma=None) -> "DiffScene":
        return DiffScene(self.width, self.height,
                         self.points if points is None else np.asarray(points, dtype=np.float32),
                         self.colors if colors is None else np.asarray(colors, dtype=np.float32),
                         self.sigma if sigma is None else float(sigma), self.tolerance, self.background,
                         self.loss_rows)


def blur_group_scene(seed: int, *, width=1024, height=1024, paths=256, sigma=4.0, jitter=0.0) -> DiffScene:
    """The seeded blur-group workload (256 closed paths of 12 cubics with
    control points uniform over the canvas, straight RGBA uniform, sigma 4 over
    opaque white) as differentiable parameters; `jitter` adds N(0, jitter^2)
    px to every control point (the target scene)."""
    c = generate(5, seed, width=width, height=height, paths=paths, sigma=sigma, jitter=jitter)
    pts = c.param_points().astype(np.float32).reshape(paths, -1, 2)
    cols = c.param_colors().astype(np.float32).reshape(paths, 4)
    return DiffScene(width, height, pts, cols, sigma=sigma)


def flatten(scene: DiffScene):
    """(lines, endpoint_point [L, 2], endpoint_weights [L, 2, 4]) of the
    forward's frozen flattening."""
    lib = N.library()
    d = scene.desc()
    n = lib.tk_diff_flatten(C.byref(d), None, None, None, 0)
    lines = np.zeros(n, dtype=N.LINE_DTYPE)
    ep = np.zeros((n, 2), dtype=np.uint32)
    w = np.zeros((n, 2, 4), dtype=np.float32)
    lib.tk_diff_flatten(C.byref(d), N.ptr(lines), N.ptr(ep), N.ptr(w), n)
    return lines, ep, w
