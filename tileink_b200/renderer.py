"""NativeRenderer: the reference's public render entry for the vector path
(src/native/renderer.rs:51-260, render_to_image at 177-190), backed by the
sm_100a C ABI (include/tileink.h).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


class TileinkError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"tileink error {code}: {message}")
        self.code = code


class NativeRenderer:
    """One CUDA context + stream on `device`; not thread-safe (like the reference's !Send runtime)."""

    def __init__(self, device: int = 0):
        self._lib = N.library()
        h = C.c_void_p()
        rc = self._lib.tk_ctx_create(int(device), C.byref(h))
        if rc != 0:
            raise TileinkError(rc, f"cannot create a context on CUDA device {device}")
        self._h = h.value
        self.width = self.height = 0

    def close(self):
        if getattr(self, "_h", None):
            self._lib.tk_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise TileinkError(rc, self._lib.tk_last_error(self._h).decode())

    @property
    def stream(self) -> int:
        return self._lib.tk_ctx_stream(self._h)

    def upload(self, scene) -> None:
        """Uploads a Canvas (its fills flattened on the GPU when it recorded
        them as elements) or a pre-flattened scene description."""
        d = scene.scene_desc() if hasattr(scene, "scene_desc") else scene.desc
        fl = scene.flatten_desc() if hasattr(scene, "flatten_desc") else getattr(scene, "flatten", None)
        if fl is not None:
            self._check(self._lib.tk_scene_upload_flatten(self._h, C.byref(d), C.byref(fl)))
        else:
            self._check(self._lib.tk_scene_upload(self._h, C.byref(d)))
        self.width, self.height = d.width, d.height

    def render(self) -> None:
        self._check(self._lib.tk_render(self._h))

    def render_incremental(self, damage=None, full_redraw_ratio: float = 0.7) -> dict:
        """Renders the uploaded scene, redrawing only the tiles under `damage`
        ({"full": bool, "rects": n x 4 int32 [x0, y0, x1, y1] pixels}; None =
        everything) over the previous frame, or everything when it must
        (tk_render_incremental). Returns the frame's statistics."""
        d = N.Damage()
        rects = None
        if damage is None or damage.get("full"):
            d.full = 1
        else:
            rects = np.ascontiguousarray(np.asarray(damage["rects"], dtype=np.int32).reshape(-1, 4))
            d.rect_count = len(rects)
            d.rects = rects.ctypes.data if len(rects) else None
        st = N.IncrementalStats()
        self._check(self._lib.tk_render_incremental(self._h, C.byref(d), float(full_redraw_ratio), C.byref(st)))
        return {k: int(getattr(st, k)) for k, _ in N.IncrementalStats._fields_}

    def render_retained(self, scene, full_redraw_ratio: float = 0.7) -> dict:
        """NativeRenderer::render_retained (src/native/renderer/retained.rs:17-23):
        materializes the retained scene, uploads it and redraws its damage.
        A materialization with the same path and line counts as the last one
        goes through tk_scene_upload_delta with the paths whose lines changed,
        so only they (and paths whose records changed) are scanned again."""
        canvas, damage = scene.materialize()
        prev = getattr(self, "_retained_lines", None)
        stats_extra = {}
        if canvas.flatten_desc() is None:
            a = canvas.scene_arrays()
            lines = a["lines"]
            if prev is not None and len(prev) == len(lines) and len(prev):
                differs = (prev.view(np.uint8).reshape(-1, N.LINE_DTYPE.itemsize) !=
                           lines.view(np.uint8).reshape(-1, N.LINE_DTYPE.itemsize)).any(axis=1)
                changed = np.unique(lines["path_id"][differs])
                stats_extra["rescan_paths"] = self.upload_delta(canvas, changed)
            else:
                self.upload(canvas)
            self._retained_lines = lines.copy()
        else:
            self._retained_lines = None
            self.upload(canvas)
        st = self.render_incremental(damage, full_redraw_ratio)
        st.update(stats_extra)
        return st

    def synchronize(self) -> None:
        self._check(self._lib.tk_synchronize(self._h))

    def readback(self, out: np.ndarray | None = None) -> np.ndarray:
        n = self.width * self.height
        if out is None:
            out = np.empty(n, dtype=np.uint32)
        self._check(self._lib.tk_readback(self._h, N.ptr(out), out.size))
        return out

    def render_to_image(self, scene) -> np.ndarray:
        """Premultiplied RGBA8 image, shape (H, W, 4), uint8."""
        self.upload(scene)
        self.render()
        return self.readback().view(np.uint8).reshape(self.height, self.width, 4)

    STAGE_NAMES = ("pool_clear", "scan_count", "pool_scan", "scan_emit", "bins", "coarse_count", "coarse_emit",
                   "fine", "blur")

    def set_timing(self, enabled: bool) -> None:
        self._check(self._lib.tk_set_timing(self._h, 1 if enabled else 0))

    def stage_times(self) -> dict:
        """Per-stage milliseconds of the last frame (CUDA events on the context stream)."""
        out = (C.c_float * len(self.STAGE_NAMES))()
        self._check(self._lib.tk_get_stage_times(self._h, out, len(self.STAGE_NAMES)))
        return dict(zip(self.STAGE_NAMES, list(out)))

    def stats(self) -> dict:
        s = N.Stats()
        self._check(self._lib.tk_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in N.Stats._fields_}

    def debug(self, stage: int, index: int = 0) -> np.ndarray:
        need = C.c_size_t(0)
        self._check(self._lib.tk_debug_readback(self._h, stage, index, None, 0, C.byref(need)))
        dt = self.DEBUG_DTYPES[stage]
        out = np.zeros(need.value // np.dtype(dt).itemsize, dtype=dt)
        self._check(self._lib.tk_debug_readback(self._h, stage, index, N.ptr(out), need.value, None))
        return out

    def upload_delta(self, scene, changed_paths=()) -> int:
        """tk_scene_upload_delta: replace the uploaded scene, keeping the scan
        of every path whose record and lines (`changed_paths` lists the
        paths whose lines changed) are unchanged. Returns how many paths the
        next render scans."""
        d = scene.scene_desc() if hasattr(scene, "scene_desc") else scene.desc
        ch = np.ascontiguousarray(np.asarray(list(changed_paths), dtype=np.uint32))
        n = C.c_uint32(0)
        self._check(self._lib.tk_scene_upload_delta(self._h, C.byref(d), N.ptr(ch) if len(ch) else None, len(ch),
                                                    C.byref(n)))
        self.width, self.height = d.width, d.height
        return n.value

    def set_band(self, tile_y0: int, tile_y1: int) -> None:
        """Render tile rows [tile_y0, tile_y1) from the next upload on
        (tk_set_band); (0, 0) returns to whole frames."""
        self._check(self._lib.tk_set_band(self._h, int(tile_y0), int(tile_y1)))

    def readback_rows(self, row0: int, row1: int, out=None) -> np.ndarray:
        """Pixel rows [row0, row1) as a (rows, width) uint32 array; `out` may
        be a host array or (int) a device address of that many words."""
        n = self.width * (row1 - row0)
        if isinstance(out, int):
            self._check(self._lib.tk_readback_rows(self._h, int(row0), int(row1), out, n))
            return None
        if out is None:
            out = np.zeros((row1 - row0, self.width), np.uint32)
        self._check(self._lib.tk_readback_rows(self._h, int(row0), int(row1), N.ptr(out), n))
        return out

    DEBUG_DTYPES = {N.STAGE_COUNTS: np.uint32, N.STAGE_BACKDROPS: np.int32, N.STAGE_RANGES: N.RANGE_DTYPE,
                    N.STAGE_SEGMENTS: N.SEGMENT_DTYPE, N.STAGE_PTCL: N.PTCL_DTYPE, N.STAGE_TILES: N.TILE_DTYPE,
                    N.STAGE_KINDS: np.uint32, N.STAGE_IMAGE: np.uint32, N.STAGE_PATHS: N.PATH_DTYPE,
                    N.STAGE_LINES: N.LINE_DTYPE, N.STAGE_GLYPHS: np.uint32}

    def debug_size(self, stage: int, index: int = 0) -> int:
        """Element count of a debug stage buffer."""
        total = C.c_uint64(0)
        self._check(self._lib.tk_debug_readback_range(self._h, stage, index, 0, 0, None, C.byref(total)))
        return total.value

    def debug_range(self, stage: int, first: int, count: int, index: int = 0) -> np.ndarray:
        """Elements [first, first + count) of a debug stage buffer (clipped)."""
        total = self.debug_size(stage, index)
        k = max(0, min(count, total - first))
        out = np.zeros(k, dtype=self.DEBUG_DTYPES[stage])
        if k:
            self._check(self._lib.tk_debug_readback_range(self._h, stage, index, first, k, N.ptr(out), None))
        return out

    # --- stage harnesses -------------------------------------------------------
    def stage_scan_prefix(self, counts, paths, ranges, cursors):
        counts = np.ascontiguousarray(counts, dtype=np.uint32)
        paths = np.ascontiguousarray(paths, dtype=N.PATH_DTYPE)
        ranges = np.ascontiguousarray(ranges, dtype=N.RANGE_DTYPE).copy()
        cursors = np.ascontiguousarray(cursors, dtype=np.uint32).copy()
        bumps = np.zeros(len(paths), dtype=np.uint32)
        self._check(self._lib.tk_stage_scan_prefix(self._h, N.ptr(counts), len(counts), N.ptr(paths), len(paths),
                                                   N.ptr(ranges), N.ptr(cursors), N.ptr(bumps)))
        return ranges, cursors, bumps

    def stage_tile_prefix(self, tiles, poll_limit: int = 0, withhold_first: bool = False):
        """Tile prefix (tk_stage_tile_prefix) on TILE_DTYPE records whose
        ptcl_count is set; returns (tiles, total). Raises TileinkError with
        code TK_E_TIMEOUT when the look-back wait gives up."""
        tiles = np.ascontiguousarray(tiles, dtype=N.TILE_DTYPE).copy()
        total = C.c_uint32(0)
        self._check(self._lib.tk_stage_tile_prefix(self._h, N.ptr(tiles), len(tiles), int(poll_limit),
                                                   1 if withhold_first else 0, C.byref(total)))
        return tiles, total.value

    def pool_scan_noalloc(self, paths, d_counts: int, d_backdrops: int, d_ranges: int, d_cursors: int,
                          pool_len: int, d_bumps: int) -> None:
        """Allocation-free pool scan on caller-owned device buffers (raw device
        addresses); `paths` is a host array. Waits for the context's stream."""
        paths = np.ascontiguousarray(paths, dtype=N.PATH_DTYPE)
        self._check(self._lib.tk_pool_scan_noalloc(self._h, N.ptr(paths), len(paths), d_counts, d_backdrops,
                                                   d_ranges, d_cursors, int(pool_len), d_bumps))

    # --- batched mode -----------------------------------------------------------
    def batch_upload(self, canvases) -> None:
        """Uploads independent one-pass scenes as one batch."""
        descs = [c.scene_desc() if hasattr(c, "scene_desc") else getattr(c, "desc", c) for c in canvases]
        arr = (N.SceneDesc * len(descs))(*descs)
        self._batch_keep = (canvases, descs, arr)
        self._check(self._lib.tk_batch_upload(self._h, C.cast(arr, C.c_void_p), len(descs)))
        self._batch_info = [self.batch_info(i) for i in range(len(descs))]

    def batch_render(self) -> None:
        self._check(self._lib.tk_batch_render(self._h))

    def batch_info(self, scene: int) -> N.BatchInfo:
        out = N.BatchInfo()
        self._check(self._lib.tk_batch_info_get(self._h, int(scene), C.byref(out)))
        return out

    def batch_readback(self, out: np.ndarray | None = None):
        """Every scene's premultiplied RGBA8 image, (H, W, 4) uint8 each,
        views into one buffer of all scenes' pixels (`out`: a caller's uint32
        buffer of exactly that many pixels, e.g. in pinned memory)."""
        infos = self._batch_info
        total = sum(i.width * i.height for i in infos)
        buf = np.empty(total, dtype=np.uint32) if out is None else out  # every pixel is written
        if buf.dtype != np.uint32 or buf.size != total or not buf.flags.c_contiguous:
            raise ValueError(f"batch readback needs a contiguous uint32 buffer of {total} pixels")
        self._check(self._lib.tk_batch_readback(self._h, N.ptr(buf), total))
        return [buf[i.image_offset:i.image_offset + i.width * i.height].view(np.uint8).reshape(i.height, i.width, 4)
                for i in infos]

    def autotune(self, iterations: int = 3) -> N.TuneResult:
        out = N.TuneResult()
        self._check(self._lib.tk_autotune(self._h, int(iterations), C.byref(out)))
        return out

    # --- differentiable rendering ---------------------------------------------
    def diff_forward(self, scene, target, return_image=False):
        """Loss (and optionally the [H, W, 4] f32 image) of a DiffScene against
        `target` ([H, W, 4] premultiplied f32)."""
        d = scene.desc()
        tgt = np.ascontiguousarray(target, dtype=np.float32)
        if tgt.shape != (scene.height, scene.width, 4):
            raise ValueError("target must be [height, width, 4]")
        loss = C.c_double(0.0)
        img = np.zeros_like(tgt) if return_image else None
        self._check(self._lib.tk_diff_forward(self._h, C.byref(d), N.ptr(tgt), C.byref(loss),
                                              N.ptr(img) if img is not None else None))
        self._diff_shape = (scene.points.shape, scene.colors.shape)
        return (loss.value, img) if return_image else loss.value

    def diff_backward(self):
        """(d_points, d_colors, d_sigma) of the last diff_forward."""
        pshape, cshape = getattr(self, "_diff_shape", ((0, 0, 2), (0, 4)))
        dp = np.zeros(pshape, dtype=np.float32)
        dc = np.zeros(cshape, dtype=np.float32)
        ds = C.c_float(0.0)
        self._check(self._lib.tk_diff_backward(self._h, N.ptr(dp), N.ptr(dc), C.byref(ds)))
        return dp, dc, ds.value

    def stage_scan_count(self, lines, paths, backdrops, counts):
        lines = np.ascontiguousarray(lines, dtype=N.LINE_DTYPE)
        paths = np.ascontiguousarray(paths, dtype=N.PATH_DTYPE)
        backdrops = np.ascontiguousarray(backdrops, dtype=np.int32).copy()
        counts = np.ascontiguousarray(counts, dtype=np.uint32).copy()
        self._check(self._lib.tk_stage_scan_count(self._h, N.ptr(lines), len(lines), N.ptr(paths), len(paths),
                                                  N.ptr(backdrops), N.ptr(counts), len(counts)))
        return backdrops, counts

    def stage_blur(self, src, dst, width, height, region, source, sigma, axis):
        src = np.ascontiguousarray(src, dtype=np.uint32)
        dst = np.ascontiguousarray(dst, dtype=np.uint32).copy()
        reg = np.asarray(region, dtype=np.uint32)
        srcb = np.asarray(source, dtype=np.uint32)
        self._check(self._lib.tk_stage_blur(self._h, N.ptr(src), N.ptr(dst), int(width), int(height), N.ptr(reg),
                                            N.ptr(srcb), float(sigma), int(axis)))
        return dst
