#!/usr/bin/env python
"""Benchmark: frames/s of the 4096x4096, 50,000-path mixed scene.

One step renders one full frame through the whole path (scan count, pool
prefix + backdrop cumsum, emit, tile binning, coarse count/prefix/emit, fine)
with the scene resident in HBM (`value`), and end to end through the C ABI
with the scene in pinned host memory, its host->device copy and the RGBA8
image readback inside every step (`e2e`).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tileink|reference]

Multi-GPU: one process per GPU (torchrun). The frame is split into tile-row
bands, one per rank (tk_set_band: each rank scans only the lines that reach
its band and draws only its rows), and every step ends with an NCCL
all-gather of the bands, so `value` is whole frames/s (strong scaling); the
time is the max over ranks. The batched leg splits the scenes over ranks and
the differentiable leg splits the loss rows and all-reduces the gradients.
`--impl reference` times the reference path's CPU restatement (the oracle
port; the reference itself is Rust + HLSL and cannot run here) on the host
cores: each step draws every 32nd tile row of the same frame, with the
whole-scene scan once per 32 steps.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "4K 50k-path frames/s"
UNIT = "frames/s"
WORKLOAD = "4096x4096 canvas, 50,000 paths (60% fills / 40% round-join strokes), cubic+quadratic, " \
           "200 Gaussian clusters sigma 300 px, nonzero/even-odd, solid/linear/radial paint, " \
           "10% in clip layers nested <=4"
SEED = 2


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="tileink", choices=["tileink", "reference"])
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--paths", type=int, default=0, help="override the path count (smaller trial runs)")
    p.add_argument("--size", type=int, default=0, help="override the canvas side (smaller trial runs)")
    p.add_argument("--diff-steps", type=int, default=10, help="timed fwd+bwd steps of the blur-group workload (0: skip)")
    p.add_argument("--batch-scenes", type=int, default=512, help="scenes of the batched-mode leg (0: skip)")
    p.add_argument("--incremental-steps", type=int, default=10, help="frames of the incremental leg (0: skip)")
    p.add_argument("--sdf-steps", type=int, default=10, help="frames of the SDF-shape leg (0: skip)")
    p.add_argument("--filter-steps", type=int, default=10, help="frames of the filter-layer leg (0: skip)")
    p.add_argument("--sdf-shapes", type=int, default=50000, help="shapes of the SDF-shape leg")
    p.add_argument("--sdf-kinds", default="base", choices=["base", "all"],
                   help="SDF-only runs: the base kinds, or all nineteen (the extended-kind kernel instance)")
    p.add_argument("--config-steps", type=int, default=10,
                   help="frames of the 640x360 and 1920x1080 glyph legs (0: skip)")
    p.add_argument("--cpu-profile", action="store_true",
                   help="time only the oracle on the benchmarked frame (full, every band, one thread) and print it")
    p.add_argument("--sdf-only", action="store_true",
                   help="run only the SDF-shape leg (rank 0, one GPU) and print its line (profiling runs)")
    return p.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.perf_counter(), [v.strip() for v in line.split(",")]))

    def window(self, t0, t1):
        """Keep the samples taken inside [t0, t1] (all samples if none fell inside)."""
        inside = [r for r in self.rows if t0 <= r[0] <= t1]
        self.rows = inside or self.rows

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=5)
        return False

    def summary(self, fallback_max=1965.0):
        rows = [r for _, r in self.rows]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": fallback_max, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else fallback_max,
                "reasons": sorted(reasons), "samples": len(rows)}


def max_over_ranks(value: float, world: int, device: str = "cuda") -> float:
    """The largest `value` over all ranks; every rank calls it at the same
    point (NCCL on the GPUs, gloo in the CPU tests)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def fp32_peak_tflops() -> float:
    """The FP32 FMA peak measured on a B200 by fp32_probe.cu, committed in
    profiles/fp32_peak_fma.txt."""
    for line in (ROOT / "profiles" / "fp32_peak_fma.txt").read_text().splitlines():
        if line.startswith("fp32_tflops "):
            return float(line.split()[1])
    raise RuntimeError("profiles/fp32_peak_fma.txt has no fp32_tflops line")


def measured_peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        return {}


def scene(size=0, paths=0, device_plan=True, seed=SEED):
    import tileink_b200 as tk
    return tk.generate(2, seed, width=size, height=size, paths=paths, device_segment_plan=device_plan)


def diff_timing(renderer, steps, warmup):
    """fwd+bwd latency of the differentiable blur-group workload (1024x1024,
    256 closed paths x 12 cubics, sigma 4, MSE against the image of the
    parameters jittered by N(0, 3^2) px) through the public API: host
    parameters in, loss and host gradients out, flattening and scene build
    included. The target is the GPU forward's own image of the jittered scene."""
    from tileink_b200 import diff
    sc = diff.blur_group_scene(5)
    tg = diff.blur_group_scene(5, jitter=3.0)
    _, target = renderer.diff_forward(tg, np.zeros((sc.height, sc.width, 4), np.float32), return_image=True)
    for _ in range(max(warmup, 3)):
        renderer.diff_forward(sc, target)
        renderer.diff_backward()
    fwd, bwd = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        loss = renderer.diff_forward(sc, target)
        t1 = time.perf_counter()
        dp, dc, ds = renderer.diff_backward()
        t2 = time.perf_counter()
        fwd.append((t1 - t0) * 1e3)
        bwd.append((t2 - t1) * 1e3)
    return {"workload": "1024x1024, 256 closed paths x 12 cubics, blur group sigma 4, MSE vs jittered target",
            "fwd_bwd_ms": float(np.median(np.add(fwd, bwd))), "fwd_ms": float(np.median(fwd)),
            "bwd_ms": float(np.median(bwd)), "steps": steps, "loss": loss,
            "timing": "host wall clock per call (median), host buffers in and out",
            "gradient_check": "tests/test_gpu_diff.py: FP64 central differences, relative error <= 1e-3"}


def diff_split_timing(device, steps, warmup, world, rank):
    """fwd+bwd of the blur-group workload over N GPUs: every rank renders the
    frame and takes the loss and the adjoint of its own pixel rows
    (tk_diff_scene.loss_row0/1); the partial gradients are all-reduced
    (NCCL sum). The time of a step is the max over ranks."""
    import torch
    import torch.distributed as dist
    import tileink_b200 as tk
    from tileink_b200 import diff
    r = tk.NativeRenderer(device)
    sc = diff.blur_group_scene(5)
    tg = diff.blur_group_scene(5, jitter=3.0)
    _, target = r.diff_forward(tg, np.zeros((sc.height, sc.width, 4), np.float32), return_image=True)
    h = sc.height
    sc.loss_rows = (h * rank // world, h * (rank + 1) // world)
    grads = torch.zeros(sc.points.size + sc.colors.size + 1, dtype=torch.float32, device="cuda")

    def step():
        loss = r.diff_forward(sc, target)
        dp, dc, ds = r.diff_backward()
        grads.copy_(torch.from_numpy(np.concatenate([dp.reshape(-1), dc.reshape(-1), [np.float32(ds)]])))
        dist.all_reduce(grads)
        lt = torch.tensor([loss], dtype=torch.float64, device="cuda")
        dist.all_reduce(lt)
        return float(lt.item())

    for _ in range(max(warmup, 3)):
        step()
    dist.barrier()
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        loss = step()
        torch.cuda.synchronize()
        times.append(max_over_ranks((time.perf_counter() - t0) * 1e3, world))
    r.close()
    return {"workload": "1024x1024, 256 closed paths x 12 cubics, blur group sigma 4, MSE vs jittered target; "
                        f"loss rows split over {world} ranks, gradients all-reduced",
            "fwd_bwd_ms": float(np.median(times)), "steps": steps, "loss": loss,
            "timing": "host wall clock per step (forward, backward, NCCL all-reduce), max over ranks, median"}


def batch_parallel_timing(device, n_scenes, steps, world, rank):
    """The uneven-batch workload over N GPUs: scenes partitioned by line
    count (shard.scene_partition), each rank batch-renders its own (one CUDA
    graph launch); scenes/s of the whole batch from the max over ranks."""
    import torch
    import tileink_b200 as tk
    from tileink_b200 import shard
    scenes = [tk.generate(4, 1000 + i) for i in range(n_scenes)]
    parts = shard.scene_partition([int(s.scene_desc().line_count) for s in scenes], world)
    mine = [scenes[i] for i in parts[rank]]
    b = tk.NativeRenderer(device)
    b.batch_upload(mine)  # warm-up: first allocations and graph capture
    b.batch_render()
    b.batch_readback()
    t0 = time.perf_counter()
    b.batch_upload(mine)
    b.batch_render()
    b.batch_readback()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    b.batch_render()
    b.batch_readback()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        b.batch_render()
    b.batch_readback()
    render_s = max_over_ranks((time.perf_counter() - t0) / steps, world)
    b.close()
    return {"workload": f"{n_scenes} scenes, W and H log-uniform in [64, 1024], 10-2000 closed cubic paths, solid; "
                        f"scenes split over {world} ranks by line count",
            "batched_scenes_per_s": n_scenes / render_s, "batched_e2e_scenes_per_s": n_scenes / e2e_s,
            "batched_ms": render_s * 1e3, "steps": steps, "scenes_per_rank": [len(p) for p in parts],
            "timing": "host wall clock, max over ranks; batched = graph replays + one readback"}


def batch_timing(n_scenes, steps):
    """Batched vs serial scenes/s on the uneven-batch workload: n_scenes
    independent scenes, width and height each log-uniform in [64, 1024],
    log-uniform 10..2000 closed cubic paths with solid fills (seeds 1000..).
    The scenes' records sit in pinned host memory and the images are read
    back into a pinned buffer, as in the end-to-end frame leg.
    serial: upload + render + readback per scene (tk_scene_upload,
    tk_render, tk_readback).
    batched: the whole batch in one CUDA graph launch (tk_batch_render) after
    the autotuner picked the pool-scan work item size; `value` with the
    scenes resident on the device, `e2e` with upload and readback."""
    import torch
    import tileink_b200 as tk
    canvases = [tk.generate(4, 1000 + i) for i in range(n_scenes)]
    scenes = [pinned_scene(c)[0] for c in canvases]
    pixels = [c.scene_desc().width * c.scene_desc().height for c in canvases]
    del canvases
    out = torch.empty(sum(pixels) * 4, dtype=torch.uint8, pin_memory=True).numpy().view(np.uint32)
    r = tk.NativeRenderer(0)
    for ps in scenes[:8]:
        r.upload(ps)
        r.render()
        r.readback(out)
    t0 = time.perf_counter()
    for ps in scenes:
        r.upload(ps)
        r.render()
        r.readback(out)
    serial_s = time.perf_counter() - t0
    r.close()
    b = tk.NativeRenderer(0)
    b.batch_upload(scenes)  # warm-up, as the serial path had: first allocations and graph capture
    b.batch_render()
    imgs = b.batch_readback(out)
    e2e = []
    for _ in range(steps):  # upload (host merge + copies), render, readback, each cycle
        t0 = time.perf_counter()
        b.batch_upload(scenes)
        b.batch_render()
        imgs = b.batch_readback(out)
        e2e.append(time.perf_counter() - t0)
    e2e_s = statistics.median(e2e)
    tune = b.autotune(3)
    b.batch_render()
    b.batch_readback()
    t0 = time.perf_counter()
    for _ in range(steps):
        b.batch_render()
    b.batch_readback()
    render_s = (time.perf_counter() - t0) / steps
    del imgs
    b.close()
    return {"workload": f"{n_scenes} scenes, W and H log-uniform in [64, 1024], 10-2000 closed cubic paths, solid",
            "serial_scenes_per_s": n_scenes / serial_s, "batched_scenes_per_s": n_scenes / render_s,
            "batched_e2e_scenes_per_s": n_scenes / e2e_s, "speedup": serial_s / render_s,
            "speedup_e2e": serial_s / e2e_s, "batched_ms": render_s * 1e3, "steps": steps,
            "scan_item_elems": tune.scan_item_elems, "tile": f"{tune.tile_width}x{tune.tile_height}",
            "tune_ms": {str(tune.candidate_elems[i]): tune.candidate_ms[i] for i in range(tune.candidates)},
            "timing": "host wall clock, warmed up; batched = graph replays + one readback, batched e2e = "
                      "median of upload + render + readback cycles, serial = per-scene upload, render and "
                      "readback; records in pinned host memory, images read into a pinned buffer"}


def incremental_timing(r, size, steps):
    """Incremental frames of the resident scene (tk_render_incremental, the
    retained path's damage-driven redraw): each frame a 256x256-pixel damage
    rectangle at a new place, the scene's scan reused (nothing was uploaded
    since) and coarse + fine run on the damaged tiles only over the previous
    frame; against full frames of the same scene (scan included). Host wall
    clock per frame, synchronized."""
    side = 256
    W = size or 4096
    r.render_incremental(None)  # the history frame
    r.synchronize()
    t0 = time.perf_counter()
    for _ in range(2):
        r.render_incremental(None)
    r.synchronize()
    full_ms = (time.perf_counter() - t0) * 1e3 / 2
    st = None
    t0 = time.perf_counter()
    for k in range(steps):
        x, y = (k * 331) % (W - side), (k * 197) % (W - side)
        st = r.render_incremental({"full": False, "rects": [[x, y, x + side, y + side]]})
    r.synchronize()
    inc_ms = (time.perf_counter() - t0) * 1e3 / steps
    return {"workload": f"the frame's scene, a {side}x{side}-pixel damage rectangle moved every frame",
            "incremental_ms": inc_ms, "full_ms": full_ms, "speedup": full_ms / inc_ms,
            "dirty_tiles": st["dirty_tiles"], "total_tiles": st["total_tiles"], "steps": steps,
            "timing": "host wall clock per frame, synchronized"}


def delta_timing(r, canvas, steps, k=8):
    """Delta frames (tk_scene_upload_delta + tk_render_incremental, the
    retained path after an edit): each frame the scene is uploaded again
    with k paths listed as changed (their lines re-uploaded), only
    those paths are scanned again (counted, prefixed, emitted into the slices
    the device plan gave them) and their tiles redrawn. Host wall clock per
    frame from the upload call to the synchronized render."""
    a = canvas.scene_arrays()
    paths = a["paths"]
    cut = np.percentile(paths["data_len"], 2)  # the smallest 2% of the paths' bboxes
    small = np.nonzero((paths["data_len"] > 0) & (paths["data_len"] <= cut))[0]
    k = min(k, len(small))
    rng = np.random.default_rng(5)
    r.upload(canvas)
    r.render_incremental(None)
    r.synchronize()
    times, st, n = [], None, 0
    for _ in range(steps):
        pick = np.sort(rng.choice(small, k, replace=False)).astype(np.uint32)
        rects = [[int(paths["tile_x0"][p]) * 16, int(paths["tile_y0"][p]) * 16, int(paths["tile_x1"][p]) * 16,
                  int(paths["tile_y1"][p]) * 16] for p in pick]
        t0 = time.perf_counter()
        n = r.upload_delta(canvas, pick)
        st = r.render_incremental({"full": False, "rects": rects})
        r.synchronize()
        times.append((time.perf_counter() - t0) * 1e3)
    return {"workload": f"the frame's scene uploaded again with {k} paths (among the 2% with the smallest bboxes, "
                        f"<= {int(cut)} tiles) listed as changed each frame; their bbox tiles redrawn",
            "delta_ms": float(np.median(times)), "rescan_paths": int(n), "scanned_paths": int(st["scanned_paths"]),
            "dirty_tiles": int(st["dirty_tiles"]), "scan_reused": int(st["scan_reused"]), "steps": steps,
            "timing": "host wall clock per frame (upload call to synchronized render), median"}


def sdf_scene(size, n, seed, kinds="base"):
    """n SDF shapes on a size^2 canvas, clustered like the path workload (200
    Gaussian centres, sigma 300 px): rects (half rounded), rect strokes,
    circles, circle strokes, lines with butt/square/round caps and rect,
    circle and line shadows, 4-160 px; paint 50% opaque solid, 25%
    translucent solid, 25% linear/radial gradients."""
    import tileink_b200 as tk
    from tileink_b200 import _native as N
    rng = np.random.default_rng(seed)
    c = tk.Canvas(size, size)
    c.set_clear_color(0xFFFFFFFF)
    centres = rng.uniform(0, size, (200, 2))
    for k in range(n):
        x, y = centres[rng.integers(200)] + rng.normal(0, 300, 2)
        w, h = rng.uniform(4, 160, 2)
        u = rng.uniform()
        if u < 0.5:
            b = tk.Brush.solid(*rng.uniform(0, 1, 3), 1.0)
        elif u < 0.75:
            b = tk.Brush.solid(*rng.uniform(0, 1, 3), float(rng.uniform(0.2, 0.9)))
        else:
            stops = [(0.0, (*rng.uniform(0, 1, 3), 1.0)), (1.0, (*rng.uniform(0, 1, 3), float(rng.uniform(0.3, 1))))]
            b = (tk.Brush.linear((x, y), (x + w, y + h), stops) if rng.uniform() < 0.5
                 else tk.Brush.radial((x, y), 0.0, (x, y), float(max(w, h)), stops))
        kind = k % 9 if kinds == "base" else k % 19
        if kind >= 9:  # the extended kinds
            r = float(max(w, h) / 2)
            if kind == 9:
                c.push_dash_line(x, y, x + w, y + h, float(rng.uniform(1, 6)), 8.0, 4.0, b, cap=int(rng.integers(0, 3)))
            elif kind == 10:
                c.push_triangle((x, y), (x + w, y + rng.uniform(0, h)), (x + rng.uniform(0, w), y + h), b,
                                corner_radius=float(rng.uniform(0, 4)))
            elif kind == 11:
                c.push_checkerboard(x, y, x + w, y + h, float(rng.uniform(4, 16)), b, tk.Brush.solid(1, 1, 1, 1))
            elif kind == 12:
                c.push_candlestick(x, y, y + h, y + h / 4, y + 3 * h / 4, int(rng.integers(3, 20)), 1, b)
            elif kind in (13, 14):
                c.push_sdf_arc(x, y, r, float(rng.uniform(0, 6.28)), float(rng.uniform(-6, 6)), float(rng.uniform(1, 8)),
                               b, cap=int(rng.integers(0, 3))) if kind == 13 else \
                    c.push_arc_shadow(x, y, r, 0.5, 4.0, 4.0, b, offset=(3, 3), expand=4.0, intensity=0.5)
            elif kind in (15, 16):
                if kind == 15:
                    c.push_star(x, y, r, r * 0.45, b, corner_radius=1.0, rotation=float(rng.uniform(-3, 3)))
                else:
                    c.push_star_stroke(x, y, r, r * 0.45, 2.0, b, rotation=float(rng.uniform(-3, 3)))
            else:
                tail = (int(rng.integers(0, 4)), w / 2, float(min(w, h) / 3), 12.0, 2.0)
                if kind == 17:
                    c.push_callout((x, y, x + w, y + h), 8.0, tail, b)
                else:
                    c.push_callout_stroke((x, y, x + w, y + h), 8.0, tail, 2.0, b)
        elif kind in (0, 1):
            c.push_rect(x, y, x + w, y + h, b, radius=float(rng.uniform(0, 20)) if kind else 0.0)
        elif kind == 2:
            c.push_rect_stroke(x, y, x + w, y + h, float(rng.uniform(1, 8)), b, radius=float(rng.uniform(0, 12)))
        elif kind == 3:
            c.push_circle(x, y, w / 2, b)
        elif kind == 4:
            c.push_circle_stroke(x, y, w / 2, float(rng.uniform(1, 6)), b)
        elif kind == 5:
            c.push_line(x, y, x + rng.uniform(-w, w), y + rng.uniform(-h, h), float(rng.uniform(1, 8)), b,
                        cap=int(rng.integers(0, 3)))
        elif kind == 6:
            c.push_rect_shadow(x, y, x + w, y + h, b, offset=(4, 4), expand=float(rng.uniform(0, 8)),
                               intensity=0.5, radius=8.0)
        elif kind == 7:
            c.push_circle_shadow(x, y, w / 2, b, offset=(3, 3), expand=float(rng.uniform(0, 6)), intensity=0.6)
        else:
            c.push_line_shadow(x, y, x + w, y + h, float(rng.uniform(1, 6)), b, offset=(2, 2), expand=3.0,
                               intensity=0.5, cap=N.CAP_ROUND)
    return c


def filter_timing(r, size, steps):
    """A filter layer over the whole canvas (Canvas::push_filter_layer with a
    chain of grayscale, contrast, a colour matrix and a component transfer)
    over 400 translucent fills: the group's filter-and-composite stage by
    CUDA events, against the HBM bytes it must move (8 per pixel for the
    fused per-pixel chain, 12 per pixel for the composite)."""
    import tileink_b200 as tk
    from tileink_b200 import _native as N
    size = size or 4096
    rng = np.random.default_rng(SEED + 11)
    c = tk.Canvas(size, size)
    c.set_clear_color(0xFFFFFFFF)
    table = np.concatenate([255 - np.arange(256), np.arange(256), (np.arange(256) ** 2) // 255, np.arange(256)])
    chain = [(N.FILTER_GRAYSCALE, 0.6), (N.FILTER_CONTRAST, 1.3),
             (N.FILTER_COLOR_MATRIX, [0.393, 0.769, 0.189, 0, 0, 0.349, 0.686, 0.168, 0, 0, 0.272, 0.534, 0.131, 0, 0,
                                      0, 0, 0, 1, 0]),
             (N.FILTER_COMPONENT_TRANSFER, table)]
    c.push_filter_layer(chain, (0.0, 0.0, float(size), float(size)))
    for _ in range(400):
        x0, y0 = rng.uniform(-200, size), rng.uniform(-200, size)
        w, h = rng.uniform(50, 1200, 2)
        c.push_path(tk.BezPath().move_to(x0, y0).line_to(x0 + w, y0).line_to(x0 + w, y0 + h).line_to(x0, y0 + h)
                    .close(), tk.Brush.solid(*rng.uniform(0, 1, 3), float(rng.uniform(0.3, 1.0))))
    c.pop_layer()
    r.upload(c)
    r.set_timing(True)
    for _ in range(3):
        r.render()
    r.synchronize()
    acc = {}
    for _ in range(steps):
        r.render()
        r.synchronize()
        for k, v in r.stage_times().items():
            acc[k] = acc.get(k, 0.0) + v / steps
    r.set_timing(False)
    filt_ms = acc["blur"]
    px = size * size
    algo = px * (8 + 12)  # the chain's per-pixel filters run fused: one read and one write per pixel
    hbm = measured_peaks().get("hbm_gbs", 6650.0)
    return {"workload": f"{size}x{size} canvas, 400 translucent rect fills inside one filter layer over the canvas: "
                        "grayscale, contrast, colour matrix, component transfer",
            "frame_ms": sum(acc.values()), "filter_stage_ms": filt_ms, "stage_ms": acc, "steps": steps,
            "roofline": {"bound": "hbm", "achieved": algo / (filt_ms * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                         "frac": algo / (filt_ms * 1e-3) / 1e9 / hbm, "algorithmic_bytes": algo,
                         "bytes_rule": "8 B/px for the fused run of per-pixel filters (read and write the "
                                       "surface once), 12 B/px for the composite (read the surface, read and "
                                       "write the target)"},
            "timing": "device, CUDA events per stage (the filter stage: the chain and the composite)"}


def sdf_timing(r, size, steps, cpu, n=50000, kinds="base"):
    """Frames of an SDF-shape scene (PTCL_SDF coverage in fine, full-tile
    colour and hollow-stroke proofs in coarse), device stage times by CUDA
    events; and the oracle on 1/4 of the shapes, scaled, as its CPU
    baseline."""
    from tileink_b200 import _native as N
    size = size or 4096
    c = sdf_scene(size, n, SEED + 7, kinds)
    r.upload(c)
    r.set_timing(True)
    for _ in range(3):
        r.render()
    r.synchronize()
    acc = {}
    for _ in range(steps):
        r.render()
        r.synchronize()
        for k, v in r.stage_times().items():
            acc[k] = acc.get(k, 0.0) + v / steps
    frame_ms = sum(acc.values())
    ptcl = r.debug(N.STAGE_PTCL, 0)
    tags = ptcl["tag"]
    tile_kind = ptcl["color"][tags == N.PTCL_BATCH_BEGIN] & 7
    what = ("rects, rounded rects, rect strokes, circles, circle strokes, lines, rect/circle/line shadows"
            if kinds == "base" else "all nineteen kinds: the base kinds plus dash lines, triangles, checkerboards, "
            "candlesticks, arcs, arc shadows, stars, star strokes, callouts and callout strokes")
    line = {"workload": f"{size}x{size} canvas, {n} SDF shapes ({what}), 200 Gaussian clusters "
                        "sigma 300 px, 50% opaque / 25% translucent solid / 25% gradient paint",
            "frames_per_s": 1e3 / frame_ms, "ms_per_frame": frame_ms, "stage_ms": acc, "steps": steps,
            "sdf_records": int((tags == N.PTCL_SDF).sum()), "color_records": int((tags == N.PTCL_COLOR).sum()),
            "tile_kinds": {name: int((tile_kind == k).sum()) for k, name in
                           ((0, "interpreter"), (1, "empty"), (2, "color"), (3, "sdf"), (4, "mixed"))},
            "timing": "device, CUDA events per stage, summed"}
    if cpu:
        import oracle
        div = 4  # the oracle renders SDF shapes faster than paths: a larger sample
        small = sdf_scene(size, n // div, SEED + 7)
        t0 = time.perf_counter()
        run = oracle.OracleRun(small.scene_desc(), threads=os.cpu_count() or 1)
        dt = time.perf_counter() - t0
        del run
        line["cpu_baseline"] = {"frames_per_s": 1.0 / (dt * div), "cores": os.cpu_count() or 1,
                                "kind": "port", "sample": f"{n // div} shapes (1/{div}), {dt:.2f} s, scaled x{div}"}
    return line


BANDS = 64  # the CPU arms' step: every BANDS-th tile row of the frame


def oracle_band_step(run, desc, k, threads):
    """Step k of the CPU rotation over the frame: at the start of every
    rotation the whole-scene scan (count, prefix + cumsum, emit) and the tile
    bins (OracleRun.prepare), then coarse and fine of the tile rows
    ty = k mod BANDS, k mod BANDS + BANDS, ... Returns (run, scan seconds or
    None, raster seconds)."""
    import oracle
    t_scan = None
    if k % BANDS == 0 or run is None:
        t0 = time.perf_counter()
        run = oracle.OracleRun.prepare(desc, threads=threads)
        t_scan = time.perf_counter() - t0
    t0 = time.perf_counter()
    run.raster(k % BANDS, 0, BANDS, threads=threads)
    return run, t_scan, time.perf_counter() - t0


def cpu_baseline(desc, threads=None):
    """The oracle (the CPU restatement of the reference path) on the host
    cores, on a bounded sample of the benchmarked frame itself: the
    whole-scene scan plus one interleaved band (every BANDS-th tile row);
    the frame time is the scan plus BANDS times the band."""
    threads = threads or os.cpu_count() or 1
    run, t_scan, t_band = oracle_band_step(None, desc, 0, threads)
    stages = run.stage_times()
    del run
    frame_s = t_scan + BANDS * t_band
    return {"value": 1.0 / frame_s, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"the benchmarked scene: the whole-scene scan ({t_scan:.2f} s) and tile rows 0, 16, 32, ... "
                      f"({t_band:.2f} s, 1/{BANDS} of the rows); frame = scan + {BANDS} x band",
            "scan_seconds": t_scan, "band_seconds": t_band, "stage_seconds": stages}


def run_reference(args):
    """The reference arm: the oracle port of the reference path on all host
    cores, on the same 4096^2, 50,000-path scene (seed 2) as the GPU arm.
    Step k draws tile rows k mod BANDS, k mod BANDS + BANDS, ... of the frame
    (coarse and fine); the whole-scene scan and tile bins run once per
    BANDS-step rotation, inside the step that starts it. frames/s =
    1 / (scan + the BANDS band times) when every band was timed, else
    1 / (scan + BANDS x the mean timed band): the bands interleave rows over
    the whole frame, so each is an even sample of it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    c = scene(args.size, args.paths, device_plan=False)
    d = c.scene_desc()
    threads = os.cpu_count() or 1
    warmup = max(args.warmup, 3)
    run = None
    for k in range(warmup):
        run, _, _ = oracle_band_step(run, d, k, threads)
    step_s, band_s, scan_s = [], {}, []
    for k in range(warmup, warmup + args.steps):
        run, t_scan, t_band = oracle_band_step(run, d, k, threads)
        step_s.append(t_band + (t_scan or 0.0))
        band_s.setdefault(k % BANDS, []).append(t_band)
        if t_scan is not None:
            scan_s.append(t_scan)
    if not scan_s:  # no rotation started inside the timed steps: time the scan once more
        run, t_scan, _ = oracle_band_step(None, d, 0, threads)
        scan_s.append(t_scan)
    del run
    measured = sorted(band_s)
    band_mean = {b: statistics.mean(v) for b, v in band_s.items()}
    if len(measured) == BANDS:
        frame_s = statistics.mean(scan_s) + sum(band_mean.values())
        how = f"scan + all {BANDS} bands, each measured in this run"
    else:
        frame_s = statistics.mean(scan_s) + BANDS * statistics.mean(band_mean.values())
        how = f"scan + {BANDS} x the mean of the {len(measured)} bands measured (fewer steps than bands)"
    value = 1.0 / frame_s
    sample = (f"oracle port of the reference path on the benchmarked scene; each step draws every {BANDS}th tile "
              f"row (1/{BANDS} of the frame), the whole-scene scan once per {BANDS}-step rotation; frame = {how}")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": warmup, "ms_per_step": statistics.mean(step_s) * 1e3,
            "frame_ms": frame_s * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded generator, seed 2)",
            "config": {"workload": WORKLOAD, "width": args.size or 4096, "height": args.size or 4096,
                       "paths": args.paths or 50000, "step": f"tile rows k mod {BANDS} (+ the scan at k mod "
                                                          f"{BANDS} == 0)", "segment_plan": "host"},
            "scan_ms": statistics.mean(scan_s) * 1e3,
            "band_ms": {str(b): band_mean[b] * 1e3 for b in measured},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_leg(r, config, seed, steps, cpu, name, what):
    """One of the other measured configurations at full size: device-resident
    frames (CUDA events on the context stream), the same frame end to end
    through tk_render_to_image (host records in, RGBA8 image out), and the
    oracle's full frame on all host threads and on one thread."""
    import torch
    import tileink_b200 as tk
    c = tk.generate(config, seed)
    d = c.scene_desc()
    img = r.render_to_image(c)  # uploads, warms up
    for _ in range(3):
        r.render()
    r.synchronize()
    stream = torch.cuda.ExternalStream(r.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        r.render()
    e1.record(stream)
    e1.synchronize()
    gpu_ms = e0.elapsed_time(e1) / steps
    r.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        img = r.render_to_image(c)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / steps
    line = {"workload": what, "gpu_frame_ms": gpu_ms, "frames_per_s": 1e3 / gpu_ms,
            "gpix_per_s": d.width * d.height / (gpu_ms * 1e-3) / 1e9, "e2e_ms": e2e_ms,
            "e2e_timing": "host wall clock per tk_render_to_image call (host records in, image out)",
            "steps": steps, "data": f"synthetic (seeded generator, seed {seed})"}
    if cpu:
        import oracle
        for threads in (os.cpu_count() or 1, 1):
            t0 = time.perf_counter()
            run = oracle.OracleRun(d, threads=threads)
            dt = time.perf_counter() - t0
            if threads > 1:
                ok = np.array_equal(img.reshape(-1).view(np.uint32), run.get(oracle.OR_IMAGE, np.uint32))
                line["cpu_matches_gpu"] = bool(ok)
            del run
            line[f"cpu_frame_ms_{threads}t" if threads == 1 else "cpu_frame_ms"] = dt * 1e3
        line["cpu_threads"] = os.cpu_count() or 1
        line["cpu_kind"] = "port"
    return line


def cpu_profile(args):
    """The oracle on the benchmarked frame, for profiles/: the unbanded frame
    on all threads, the band rotation on all threads (scan once plus every
    band), and one thread on the scan and on 1/256 of the tile rows."""
    import oracle
    c = scene(args.size, args.paths, device_plan=False)
    d = c.scene_desc()
    threads = os.cpu_count() or 1
    out = {"workload": WORKLOAD, "threads": threads}
    t0 = time.perf_counter()
    run = oracle.OracleRun(d, threads=threads)
    out["full_frame_s"] = time.perf_counter() - t0
    out["full_frame_stage_s"] = run.stage_times()
    del run
    run, bands = None, []
    scan = None
    for k in range(BANDS):
        run, t_scan, t_band = oracle_band_step(run, d, k, threads)
        scan = t_scan if t_scan is not None else scan
        bands.append(t_band)
    del run
    out["rotation_scan_s"] = scan
    out["rotation_band_s"] = bands
    out["rotation_frame_s"] = scan + sum(bands)
    out["rotation_over_full"] = out["rotation_frame_s"] / out["full_frame_s"]
    t0 = time.perf_counter()
    run = oracle.OracleRun.prepare(d, threads=1)
    out["one_thread_scan_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    run.raster(0, 0, 256, threads=1)
    out["one_thread_rows_1_in_256_s"] = time.perf_counter() - t0
    del run
    out["one_thread_frame_s"] = out["one_thread_scan_s"] + 256 * out["one_thread_rows_1_in_256_s"]
    print(json.dumps(out), flush=True)


def bin_ref_count(canvas):
    """(bin-list entries, bins, drawn draws) of the binning stage: every drawn
    draw lands in each 16x16-tile bin its tile box meets."""
    a = canvas.scene_arrays()
    d = canvas.scene_desc()
    tw, th = (d.width + 15) // 16, (d.height + 15) // 16
    nbx, nby = (tw + 15) // 16, (th + 15) // 16
    pb = a["draws"]["pixel_bounds"][a["draw_order"]]
    x0 = np.minimum(np.maximum(pb["x0"], 0) // 16, tw)
    y0 = np.minimum(np.maximum(pb["y0"], 0) // 16, th)
    x1 = np.minimum((np.maximum(pb["x1"], 0) + 15) // 16, tw)
    y1 = np.minimum((np.maximum(pb["y1"], 0) + 15) // 16, th)
    ok = (x0 < x1) & (y0 < y1)
    bx = (x1 - 1) // 16 - x0 // 16 + 1
    by = (y1 - 1) // 16 - y0 // 16 + 1
    return int((bx * by)[ok].sum()), nbx * nby, len(pb)


def pinned_scene(canvas):
    """Copy the recorded scene into pinned host buffers (page-locked, like a
    caller that keeps its records in pinned memory)."""
    import torch
    from tileink_b200 import _native as N
    arrays = canvas.scene_arrays()
    arrays.update(canvas.flatten_arrays())
    pinned = {}
    keep = []
    for k, v in arrays.items():
        if isinstance(v, np.ndarray) and v.nbytes:
            t = torch.empty(v.nbytes, dtype=torch.uint8, pin_memory=True)
            view = t.numpy().view(v.dtype)
            view[...] = v
            keep.append(t)
            pinned[k] = view
        else:
            pinned[k] = v
    s = N.ArrayScene(pinned)
    s._keep = keep
    bytes_in = sum(v.nbytes for v in pinned.values() if isinstance(v, np.ndarray))
    return s, bytes_in


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.cpu_profile:
        cpu_profile(args)
        return
    import torch
    import torch.distributed as dist

    import tileink_b200 as tk

    if args.sdf_only:
        r = tk.NativeRenderer(0)
        print(json.dumps({"sdf": sdf_timing(r, args.size, max(args.sdf_steps, 1), False, args.sdf_shapes,
                                            args.sdf_kinds)}), flush=True)
        r.close()
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)

    def barrier():
        if world > 1:
            dist.barrier()

    t_gen = time.perf_counter()
    canvas = scene(args.size, args.paths)
    gen_s = time.perf_counter() - t_gen
    r = tk.NativeRenderer(local)
    # N GPUs: one frame split into tile-row bands (tk_set_band), balanced by
    # backdrop tiles per row; each step renders every band and all-gathers
    # the bands' pixels into the whole frame on every rank (NCCL)
    from tileink_b200 import shard
    d0 = canvas.scene_desc()
    H, W = d0.height, d0.width
    bands = shard.band_partition(shard.row_weights(canvas.scene_arrays()["paths"], (H + 15) // 16), world)
    band = bands[rank]
    rows = shard.pixel_rows(band, H)
    if world > 1:
        r.set_band(*band)
        tallest = max(b - a for a, b in (shard.pixel_rows(x, H) for x in bands))
        band_buf = torch.zeros((tallest, W), dtype=torch.int32, device="cuda")
        frame_buf = torch.empty((world * tallest, W), dtype=torch.int32, device="cuda")
    r.upload(canvas)
    stream = torch.cuda.ExternalStream(r.stream)

    def frame():
        r.render()
        if world > 1:  # this band's rows into the gather buffer, then the all-gather
            r.readback_rows(rows[0], rows[1], out=band_buf.data_ptr())
            dist.all_gather_into_tensor(frame_buf, band_buf)

    clocks = ClockSampler(local).__enter__()
    for _ in range(max(args.warmup, 3)):
        frame()
    r.synchronize()
    torch.cuda.synchronize()
    stats = r.stats()
    r.set_timing(True)
    stage_sum = {k: 0.0 for k in r.STAGE_NAMES}
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_on = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        frame()
        for k, v in r.stage_times().items():
            stage_sum[k] += v
    if world > 1:
        e1.record(torch.cuda.current_stream())  # after the last all-gather
    else:
        e1.record(stream)
    e1.synchronize()
    t_off = time.perf_counter()
    time.sleep(0.25)
    clocks.__exit__(None, None, None)
    clocks.window(t_on - 0.1, t_off + 0.1)
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    r.set_timing(False)
    ms = max_over_ranks(ms, world)
    value = 1000.0 / ms  # whole frames: all ranks' bands make one frame

    # the oracle on a bounded sample of this frame (the scan and 1/BANDS of
    # the tile rows), with the device's segment plan (equal to the host
    # planner's: tests/test_gpu_fullsize.py)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from tileink_b200 import _native as N
        arrays = canvas.scene_arrays()
        arrays["paths"] = r.debug(N.STAGE_PATHS).copy()
        cpu_scene = N.ArrayScene(arrays)
        cpu = cpu_baseline(cpu_scene.desc)
        del cpu_scene, arrays
    # tile-draw refs per 16x16-tile bin, for the binning stage's bytes
    bin_refs, nbins, draw_n = bin_ref_count(canvas)

    # end to end: pinned host scene -> H2D -> frame -> D2H image, every step
    out = torch.empty(r.width * r.height * 4, dtype=torch.uint8, pin_memory=True).numpy().view(np.uint32)

    out_rows = out.reshape(r.height, r.width)[rows[0]:rows[1]]

    def read_frame():
        if world > 1:  # this rank's band rows (each rank reads its own)
            r.readback_rows(rows[0], rows[1], out=out_rows)
        else:
            r.readback(out)

    def e2e_ms_of(ps):
        r.upload(ps)
        r.render()
        read_frame()
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(args.e2e_steps):
            r.upload(ps)
            r.render()
            read_frame()
        s1.record(stream)
        s1.synchronize()
        dev_ms = s0.elapsed_time(s1) / args.e2e_steps
        wall_ms = (time.perf_counter() - t0) * 1000.0 / args.e2e_steps
        return max_over_ranks(max(dev_ms, wall_ms), world)

    ps, bytes_in = pinned_scene(canvas)
    e2e_ms = e2e_ms_of(ps)
    del ps
    # the same scene with its fills and stroke centerlines as Bezier
    # elements, flattened and stroked on the GPU at upload
    flat_canvas = tk.generate(2, SEED, width=args.size, height=args.size, paths=args.paths, device_flatten=True)
    ps_flat, bytes_in_flat = pinned_scene(flat_canvas)
    e2e_flat_ms = e2e_ms_of(ps_flat)
    inc_line = None
    if rank == 0 and world == 1 and args.incremental_steps > 0:
        inc_line = incremental_timing(r, args.size, args.incremental_steps)
        inc_line["delta"] = delta_timing(r, canvas, args.incremental_steps)
    sdf_line = None
    if rank == 0 and world == 1 and args.sdf_steps > 0:
        sdf_line = sdf_timing(r, args.size, args.sdf_steps, not args.no_cpu_baseline, args.sdf_shapes)
    filter_line = None
    if rank == 0 and world == 1 and args.filter_steps > 0:
        filter_line = filter_timing(r, args.size, args.filter_steps)
    del ps_flat, flat_canvas
    bytes_out = out.nbytes  # the whole frame per step (with N GPUs: every rank's band together)
    if world > 1:
        bytes_in, bytes_in_flat = world * bytes_in, world * bytes_in_flat  # every rank uploads the scene

    # roofline of the dominant kernel
    stage_ms = {k: v / args.steps for k, v in stage_sum.items()}
    peaks = measured_peaks()
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    fp32_peak = fp32_peak_tflops()
    T = stats["tiles"]
    L, B, S = stats["lines"], stats["backdrop_len"], stats["segments"]
    K, refs = stats["ptcl_records"], stats["tile_draw_refs"]
    fills, visits = stats["fill_particles"], stats["segment_visits"]
    algo = {
        # algorithmic bytes per launch (the bytes each stage must move)
        "scan_count": ("hbm", 24 * L + 4 * S),
        "pool_scan": ("hbm", (4 + 4 + 8 + 4 + 4) * B),
        "scan_emit": ("hbm", 24 * L + 20 * S),
        # each draw's order word and bounds read once, one word per (bin, draw) hit written
        "bins": ("hbm", 20 * draw_n + 4 * bin_refs + 4 * nbins),
        "coarse_count": ("hbm", 12 * refs + 24 * T),
        "coarse_emit": ("hbm", 12 * refs + 24 * K),
        "fine": ("fp32", 256 * (24 * visits + 10 * fills)),
    }
    rooflines = {}
    for name, (bound, amount) in algo.items():
        t = stage_ms.get(name, 0.0)
        if t <= 0:
            continue
        if bound == "hbm":
            ach = amount / (t * 1e-3) / 1e9
            rooflines[name] = {"bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
                               "frac": ach / hbm_peak, "ms": t, "algorithmic_bytes": amount}
        else:
            ach = amount / (t * 1e-3) / 1e12
            rooflines[name] = {"bound": "fp32", "achieved": ach, "peak": fp32_peak, "unit": "TFLOP/s",
                               "frac": ach / fp32_peak, "ms": t, "algorithmic_flops": amount}
    dominant = max(rooflines, key=lambda k: rooflines[k]["ms"])
    roof = dict(rooflines[dominant])
    roof["kernel"] = dominant
    roof["peak_source"] = ("measured FMA probe (fp32_probe.cu, profiles/fp32_peak_fma.txt)" if roof["bound"] == "fp32"
                           else "measured (MEASURED_PEAKS.json hbm_gbs)")
    # DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from
    # the committed ncu launch list of the default 4096^2 / 50k workload; other
    # sizes have no capture.
    roof["traffic"] = None
    traffic_file = ROOT / "profiles" / "dram_traffic_c2_4096x4096_50k.txt"
    if traffic_file.exists() and (args.size or 4096) == 4096 and (args.paths or 50000) == 50000:
        for line in traffic_file.read_text().splitlines():
            parts = line.split()
            if len(parts) == 2 and not line.startswith("#") and parts[0] == dominant:
                roof["traffic"] = int(parts[1])

    configs = None
    if rank == 0 and world == 1 and args.config_steps > 0:
        configs = {
            "c1_640x360_240_paths": config_leg(
                r, 1, 1, args.config_steps, not args.no_cpu_baseline, "c1",
                "640x360, 240 closed paths of 8-40 cubics, nonzero, alpha 0.3-1 over white"),
            "c3_1920x1080_20k_glyphs": config_leg(
                r, 3, 3, args.config_steps, not args.no_cpu_baseline, "c3",
                "1920x1080, 20,000 glyphs of 2-4 quadratic contours (6-24 segments), 8-64 px em, black on white"),
        }
    if world == 1:
        diff_line = diff_timing(r, args.diff_steps, args.warmup) if args.diff_steps > 0 else None
        batch_line = batch_timing(args.batch_scenes, 5) if args.batch_scenes > 0 else None
    else:  # every rank takes part: split objective and scene-parallel batches
        diff_line = diff_split_timing(local, args.diff_steps, args.warmup, world, rank) if args.diff_steps > 0 else None
        batch_line = (batch_parallel_timing(local, args.batch_scenes, 5, world, rank)
                      if args.batch_scenes > 0 else None)

    # per frame: pool clear (k_fill), scan count, item sums, item prefix,
    # pool scan, path totals, scan emit; per target pass: bins, coarse count,
    # tile prefix, coarse emit, fine
    launches_per_frame = 7 + 5 * stats["passes"]
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, seed 2)",
            "config": {"workload": WORKLOAD, "width": args.size or 4096, "height": args.size or 4096,
                       "paths": args.paths or 50000,
                       "parallelism": (f"band split x{world}: tile rows {bands} (one band per rank, paths clamped "
                                       "to the band at upload), NCCL all-gather of the bands every frame"
                                       if world > 1 else "one GPU"),
                       "l2": "inputs > L2 (lines %.1f GB), no flush" % (L * 24 / 1e9),
                       "segment_plan": "device",
                       "stage_times": "rank 0's band" if world > 1 else "the frame"},
            # the headline: the recorded Canvas (fills and stroke centerlines as
            # Bezier elements) uploaded, flattened, stroked, rendered and read
            # back every step
            "e2e": {"value": 1000.0 / e2e_flat_ms, "unit": UNIT, "h2d_bytes_per_step": int(bytes_in_flat),
                    "d2h_bytes_per_step": int(bytes_out), "ms_per_step": e2e_flat_ms,
                    "input": "fills and stroke centerlines as Bezier elements, flattened and stroked on the GPU "
                             "at upload"},
            "e2e_host_lines": {"value": 1000.0 / e2e_ms, "unit": UNIT, "h2d_bytes_per_step": int(bytes_in),
                               "d2h_bytes_per_step": int(bytes_out), "ms_per_step": e2e_ms,
                               "input": "host-flattened lines (the reference's Line records)"},
            "gpu_launches": launches_per_frame * args.steps,
            "roofline": roof,
            "stage_ms": stage_ms,
            "rooflines": rooflines,
            "counts": {"lines": L, "backdrop_tiles": B, "segments": S, "ptcl_records": K, "tile_draw_refs": refs,
                       "fill_particles": fills, "segment_visits": visits, "tiles": T, "passes": stats["passes"]},
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
            "fwd_bwd": diff_line,
            "batched": batch_line,
            "incremental": inc_line,
            "sdf": sdf_line,
            "filters": filter_line,
            "configs": configs,
            "scene_generation_s": gen_s,
        }
        print(json.dumps(line), flush=True)
    r.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
