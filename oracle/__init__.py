"""Oracle loader: CPU restatement of the reference's rasterization path.

TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg import this package, and only to check or time the CUDA
path; the product (tileink_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

OR_COUNTS, OR_BACKDROPS, OR_RANGES, OR_SEGMENTS = 0, 1, 2, 3
OR_BATCH_PTCL, OR_BATCH_TILES, OR_BATCH_KINDS, OR_IMAGE = 4, 5, 6, 7
OR_PASS_PTCL, OR_PASS_TILES, OR_PASS_KINDS, OR_PATHS, OR_BUMPS = 8, 9, 10, 11, 12
OR_PASS_GLYPHS = 13

_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        sources = [HERE / "oracle.cpp", HERE / "diff_oracle.cpp", HERE / "oracle.h"]
        if not LIB.exists() or any(LIB.stat().st_mtime < f.stat().st_mtime for f in sources):
            build()
        l = C.CDLL(str(LIB))
        P, U32, U64, I32, F32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_float
        l.or_run.restype = I32
        l.or_run.argtypes = [P, I32, U32, U32, C.POINTER(P)]
        l.or_prepare.restype = I32
        l.or_prepare.argtypes = [P, I32, C.POINTER(P)]
        l.or_raster.restype = I32
        l.or_raster.argtypes = [P, I32, U32, U32, U32]
        l.or_get_range.restype = U64
        l.or_get_range.argtypes = [P, U32, U64, U64, P]
        l.or_free.argtypes = [P]
        l.or_error.restype = C.c_char_p
        l.or_get.restype = C.c_size_t
        l.or_get.argtypes = [P, U32, U32, P, C.c_size_t]
        l.or_batch_count.restype = U32
        l.or_batch_count.argtypes = [P]
        l.or_pass_count.restype = U32
        l.or_pass_count.argtypes = [P]
        l.or_stage_times.argtypes = [P, P]
        l.or_line_scanned_tile_count.restype = U32
        l.or_line_scanned_tile_count.argtypes = [P, U32, U32, U32, U32]
        l.or_scan_count.argtypes = [P, U64, P, U32, P, P]
        l.or_scan_prefix.argtypes = [P, P, U32, P, P, P]
        l.or_blur_pass.argtypes = [P, P, U32, U32, P, P, F32, U32]
        l.or_fill_value.restype = F32
        l.or_fill_value.argtypes = [P, U32, I32, U32, U32]
        l.or_sdf_coverage.restype = F32
        l.or_sdf_coverage.argtypes = [P, F32, F32, P]
        l.or_exp_nonpos.restype = F32
        l.or_exp_nonpos.argtypes = [F32]
        l.or_sincos.argtypes = [F32, P, P]
        l.or_atan2.restype = F32
        l.or_atan2.argtypes = [F32, F32]
        l.or_progressive_blur.restype = I32
        l.or_progressive_blur.argtypes = [P, U32, U32, P, P]
        l.or_progressive_levels.restype = U32
        l.or_progressive_levels.argtypes = [U32, U32, F32, U32, P, U32]
        l.or_text_pow.restype = F32
        l.or_text_pow.argtypes = [F32, F32]
        l.or_filter_chain.restype = None
        l.or_filter_chain.argtypes = [P, U32, P, P, U32, P]
        l.or_glyph_over.restype = U32
        l.or_glyph_over.argtypes = [U32, U32, U32]
        l.or_interpret_particles.restype = I32
        l.or_interpret_particles.argtypes = [P, P, U32, P]
        l.or_interpret_path_draws.restype = I32
        l.or_interpret_path_draws.argtypes = [P, I32, P]
        l.or_interpret_sdf_draws.restype = I32
        l.or_interpret_sdf_draws.argtypes = [P, P]
        l.or_diff_loss.restype = C.c_double
        l.or_diff_loss.argtypes = [U32, U32, U32, U64, P, P, P, P, P, C.c_double, I32, P, P, P, I32]
        _lib = l
    return _lib


class OracleRun:
    """Result of the reference frame restated on the CPU.

    OracleRun(desc, threads, tile_rows=(y0, y1)) runs the whole frame, with
    coarse and fine restricted to tile rows [y0, y1) (y1 == 0: all rows).
    OracleRun.prepare(desc, threads) runs only the scan and the tile bins;
    raster(y0, y1, row_step) then draws tile rows y0, y0 + row_step, ... < y1
    and may be called again for other rows of the same frame."""

    def __init__(self, desc, threads: int = 1, tile_rows=(0, 0), _prepare_only=False):
        self._l = lib()
        self._desc = desc
        h = C.c_void_p()
        if _prepare_only:
            rc = self._l.or_prepare(C.byref(desc), int(threads), C.byref(h))
        else:
            rc = self._l.or_run(C.byref(desc), int(threads), int(tile_rows[0]), int(tile_rows[1]), C.byref(h))
        if rc != 0:
            raise RuntimeError("oracle: " + self._l.or_error().decode())
        self._h = h.value

    @classmethod
    def prepare(cls, desc, threads: int = 1) -> "OracleRun":
        return cls(desc, threads, _prepare_only=True)

    def raster(self, tile_y0: int = 0, tile_y1: int = 0, row_step: int = 1, threads: int = 1) -> None:
        if self._l.or_raster(self._h, int(threads), int(tile_y0), int(tile_y1), int(row_step)) != 0:
            raise RuntimeError("oracle: " + self._l.or_error().decode())

    def get_range(self, what: int, dtype, first: int, count: int) -> np.ndarray:
        """Elements [first, first + count) of a flat output (counts,
        backdrops, ranges, segments, image, bumps)."""
        n = self._l.or_get_range(self._h, what, 0, 0, None)
        k = max(0, min(count, n - first))
        out = np.zeros(k, dtype=dtype)
        if k:
            self._l.or_get_range(self._h, what, first, k, out.ctypes.data)
        return out

    def size(self, what: int) -> int:
        return self._l.or_get_range(self._h, what, 0, 0, None)

    def __del__(self):
        if getattr(self, "_h", None):
            self._l.or_free(self._h)
            self._h = None

    def get(self, what: int, dtype, index: int = 0) -> np.ndarray:
        n = self._l.or_get(self._h, what, index, None, 0)
        out = np.zeros(n // np.dtype(dtype).itemsize, dtype=dtype)
        if n:
            self._l.or_get(self._h, what, index, out.ctypes.data, n)
        return out

    @property
    def batch_count(self) -> int:
        return self._l.or_batch_count(self._h)

    @property
    def pass_count(self) -> int:
        return self._l.or_pass_count(self._h)

    def stage_times(self) -> list:
        t = (C.c_double * 7)()
        self._l.or_stage_times(self._h, t)
        return list(t)


def diff_loss(scene, lines, endpoint_point, endpoint_weights, points, colors, sigma, target, radius=None,
              return_image=False, threads=8):
    """FP64 loss of the differentiable model for parameters (points, colors,
    sigma) with the flattening (lines, endpoint weights) of a forward held
    fixed; radius defaults to ceil(3 sigma) of the scene."""
    import math
    h, w = scene.height, scene.width
    pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1)
    cols = np.ascontiguousarray(colors, dtype=np.float64).reshape(-1)
    tgt = np.ascontiguousarray(target, dtype=np.float32)
    bg = np.asarray(scene.background, dtype=np.float64)
    r = int(math.ceil(3.0 * float(np.float32(scene.sigma)))) if radius is None else int(radius)
    if scene.sigma <= 0:
        r = 0
    img = np.zeros((h, w, 4), dtype=np.float64) if return_image else None
    lines = np.ascontiguousarray(lines)
    ep = np.ascontiguousarray(endpoint_point, dtype=np.uint32)
    ew = np.ascontiguousarray(endpoint_weights, dtype=np.float32)
    loss = lib().or_diff_loss(w, h, scene.path_count, len(lines), lines.ctypes.data, ep.ctypes.data,
                              ew.ctypes.data, pts.ctypes.data, cols.ctypes.data, float(sigma), r, bg.ctypes.data,
                              tgt.ctypes.data, img.ctypes.data if img is not None else None, threads)
    return (loss, img) if return_image else loss


def interpret_particles(desc, particles: np.ndarray) -> np.ndarray:
    """Fine-only image with `particles` (PTCL records) as every tile's stream."""
    img = np.zeros((desc.height, desc.width, 4), np.uint8)
    p = np.ascontiguousarray(particles)
    if lib().or_interpret_particles(C.byref(desc), p.ctypes.data, len(p), img.ctypes.data) != 0:
        raise RuntimeError("oracle: " + lib().or_error().decode())
    return img


def interpret_path_draws(desc, threads: int = 8) -> np.ndarray:
    """Fine-only image (H, W, 4 RGBA8) of a scene of path and SDF draws in
    clip / opacity layers: every batch's stack and draws interpreted in every
    tile after the scan, with no coarse stage."""
    img = np.zeros((desc.height, desc.width, 4), np.uint8)
    if lib().or_interpret_path_draws(C.byref(desc), int(threads), img.ctypes.data) != 0:
        raise RuntimeError("oracle: " + lib().or_error().decode())
    return img


def interpret_sdf_draws(desc) -> np.ndarray:
    """Fine-only image (H, W, 4 RGBA8) of a scene of SDF draws: every draw
    interpreted as a PTCL_SDF particle in every tile, no coarse stage."""
    img = np.zeros((desc.height, desc.width, 4), np.uint8)
    if lib().or_interpret_sdf_draws(C.byref(desc), img.ctypes.data) != 0:
        raise RuntimeError("oracle: " + lib().or_error().decode())
    return img
