#!/usr/bin/env python
"""Benchmark: frames/s of the 4096x4096, 50,000-path mixed scene.

One step renders one full frame through the whole path (scan count, pool
prefix + backdrop cumsum, emit, tile binning, coarse count/prefix/emit, fine)
with the scene resident in HBM (`value`), and end to end through the C ABI
with the scene in pinned host memory, its host->device copy and the RGBA8
image readback inside every step (`e2e`).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tileink|reference]

Multi-GPU: one process per GPU (torchrun); every rank renders its own frame
(replicas, weak scaling); the time is the max over ranks.
`--impl reference` times the reference path's CPU restatement (the oracle
port; the reference itself is Rust + HLSL and cannot run here) on the host
cores, on a bounded sample of the same workload.
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
CPU_SAMPLE_DIV = 16


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
    p.add_argument("--sdf-shapes", type=int, default=50000, help="shapes of the SDF-shape leg")
    p.add_argument("--sdf-kinds", default="base", choices=["base", "all"],
                   help="SDF-only runs: the base kinds, or all nineteen (the extended-kind kernel instance)")
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


def batch_timing(n_scenes, steps):
    """Batched vs serial scenes/s on the uneven-batch workload: n_scenes
    independent scenes, width and height each log-uniform in [64, 1024],
    log-uniform 10..2000 closed cubic paths with solid fills (seeds 1000..).
    serial: upload + render + readback per scene through tk_render_to_image.
    batched: the whole batch in one CUDA graph launch (tk_batch_render) after
    the autotuner picked the pool-scan work item size; `value` with the
    scenes resident on the device, `e2e` with upload and readback."""
    import tileink_b200 as tk
    scenes = [tk.generate(4, 1000 + i) for i in range(n_scenes)]
    r = tk.NativeRenderer(0)
    for c in scenes[:8]:
        r.render_to_image(c)
    t0 = time.perf_counter()
    for c in scenes:
        r.render_to_image(c)
    serial_s = time.perf_counter() - t0
    r.close()
    b = tk.NativeRenderer(0)
    t0 = time.perf_counter()
    b.batch_upload(scenes)
    b.batch_render()
    imgs = b.batch_readback()
    e2e_s = time.perf_counter() - t0
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
            "timing": "host wall clock; batched = graph replays + one readback, serial = per-scene upload, "
                      "render and readback"}


def incremental_timing(r, size, steps):
    """Incremental frames of the resident scene (tk_render_incremental, the
    retained path's damage-driven redraw): each frame a 256x256-pixel damage
    rectangle at a new place, the scene scanned in full and coarse + fine run
    on the damaged tiles only over the previous frame; against full frames of
    the same scene. Host wall clock per frame, synchronized."""
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


def cpu_baseline(size, paths):
    """The oracle (CPU restatement of the reference path) on all host cores,
    on 1/16 of the workload's paths over the same canvas; the frame time is
    scaled by 16 (scan, coarse and fine work grow linearly with paths)."""
    import oracle
    n = max(1, (paths or 50000) // CPU_SAMPLE_DIV)
    c = scene(size, n, device_plan=False, seed=SEED + 1)
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    run = oracle.OracleRun(c.scene_desc(), threads=threads)
    dt = time.perf_counter() - t0
    stages = run.stage_times()
    del run
    est = dt * CPU_SAMPLE_DIV
    return {"value": 1.0 / est, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"same generator, {n} paths (1/{CPU_SAMPLE_DIV}) on the {size or 4096}^2 canvas; "
                      f"one full oracle frame took {dt:.2f} s, scaled x{CPU_SAMPLE_DIV}",
            "sample_seconds": dt, "stage_seconds": stages}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle  # noqa: F401
    n = max(1, (args.paths or 50000) // CPU_SAMPLE_DIV)
    c = scene(args.size, n, device_plan=False, seed=SEED + 1)
    d = c.scene_desc()
    threads = os.cpu_count() or 1
    import oracle as O
    for _ in range(args.warmup):
        O.OracleRun(d, threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.OracleRun(d, threads=threads)
    dt = (time.perf_counter() - t0) / args.steps
    value = 1.0 / (dt * CPU_SAMPLE_DIV)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * CPU_SAMPLE_DIV * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded generator)",
            "config": {"workload": WORKLOAD, "width": args.size or 4096, "height": args.size or 4096,
                       "paths": args.paths or 50000, "sample_paths": n},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"oracle port of the reference path, {n} paths (1/{CPU_SAMPLE_DIV}) per step, "
                                       f"scaled x{CPU_SAMPLE_DIV}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


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
    r.upload(canvas)
    stream = torch.cuda.ExternalStream(r.stream)
    clocks = ClockSampler(local).__enter__()
    for _ in range(max(args.warmup, 3)):
        r.render()
    r.synchronize()
    stats = r.stats()
    r.set_timing(True)
    stage_sum = {k: 0.0 for k in r.STAGE_NAMES}
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_on = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        r.render()
        for k, v in r.stage_times().items():
            stage_sum[k] += v
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
    value = world * 1000.0 / ms

    # end to end: pinned host scene -> H2D -> frame -> D2H image, every step
    out = torch.empty(r.width * r.height * 4, dtype=torch.uint8, pin_memory=True).numpy().view(np.uint32)

    def e2e_ms_of(ps):
        r.upload(ps)
        r.render()
        r.readback(out)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for _ in range(args.e2e_steps):
            r.upload(ps)
            r.render()
            r.readback(out)
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
    if rank == 0 and args.incremental_steps > 0:
        inc_line = incremental_timing(r, args.size, args.incremental_steps)
    sdf_line = None
    if rank == 0 and args.sdf_steps > 0:
        sdf_line = sdf_timing(r, args.size, args.sdf_steps, not args.no_cpu_baseline, args.sdf_shapes)
    del ps_flat, flat_canvas
    bytes_out = out.nbytes

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
        "bins": ("hbm", 4 * refs),
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

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.size, args.paths)
    diff_line = diff_timing(r, args.diff_steps, args.warmup) if (rank == 0 and args.diff_steps > 0) else None
    batch_line = batch_timing(args.batch_scenes, 5) if (rank == 0 and args.batch_scenes > 0) else None

    launches_per_frame = 5 + 5 * stats["passes"]
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, seed 2)",
            "config": {"workload": WORKLOAD, "width": args.size or 4096, "height": args.size or 4096,
                       "paths": args.paths or 50000, "parallelism": f"replicas x{world}",
                       "l2": "inputs > L2 (lines %.1f GB), no flush" % (L * 24 / 1e9),
                       "segment_plan": "device"},
            # the headline: the recorded Canvas (fills and stroke centerlines as
            # Bezier elements) uploaded, flattened, stroked, rendered and read
            # back every step
            "e2e": {"value": world * 1000.0 / e2e_flat_ms, "unit": UNIT, "h2d_bytes_per_step": int(bytes_in_flat),
                    "d2h_bytes_per_step": int(bytes_out), "ms_per_step": e2e_flat_ms,
                    "input": "fills and stroke centerlines as Bezier elements, flattened and stroked on the GPU "
                             "at upload"},
            "e2e_host_lines": {"value": world * 1000.0 / e2e_ms, "unit": UNIT, "h2d_bytes_per_step": int(bytes_in),
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
            "scene_generation_s": gen_s,
        }
        print(json.dumps(line), flush=True)
    r.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
