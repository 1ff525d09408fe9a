"""Benchmark: pixel-hours/s of Tmrt + UTCI on a seeded 2000 x 2000 scene (1 m).

One step = one calendar day (24 hourly steps: shadow sweep, ground view
factors, anisotropic K/L fluxes, Tmrt, UTCI) over the whole raster, with the
static geometry (walls, 153-patch SVF) prepared once before timing.  The
timed number is the chosen form (``--form``); the plain form is timed beside
it.  ``e2e`` is the same metric through the public API from host rasters:
rasters uploaded, walls + SVF prepared, the day computed and every hour's
Tmrt and UTCI copied back to host memory.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl solweig|reference]

With N > 1 (torchrun, one rank per GPU) every rank runs its own day of the
same tile (days are independent: the thermal state resets daily), so the
work per GPU is fixed ("weak" scaling) and there is no data-path collective.
``--impl reference`` times the float64 CPU port of the reference path on the
host cores (one process per core, each stepping the 200 x 200 px, 24 h CPU
configuration of the reference's benchmark) and prints its own line.  The
headline line also carries the 720 h target (30 days in one CUDA graph vs the
plain form over the same days) and a per-stage roofline.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "pixel-hours/s Tmrt+UTCI at 2000² px: chosen vs plain form on 1 B200 at ≤0.1 K"
UNIT = "pixel-hours/s"


def _args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("solweig", "reference"), default="solweig")
    p.add_argument("--size", type=int, default=2000)
    p.add_argument("--form", choices=("plain", "batched", "chosen"), default="chosen")
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-month", action="store_true",
                   help="skip the 720 h (30 days in one graph) figure of the headline line")
    p.add_argument("--workload", choices=("day", "month", "tiles", "precision", "gradient", "float64",
                                          "geometry_walls"),
                   default="day",
                   help="day: the headline 2000^2 x 24 h line; month: 2000^2 x 720 h in one graph; "
                        "tiles: 64 uneven tiles in one graph; precision: 4000^2 patch-sum error report; "
                        "float64: the float64 radiation switch, hour by hour; geometry_walls: footprint walls")
    p.add_argument("--no-tune", dest="tune", action="store_false",
                   help="skip the launch-shape autotuner (cached per shape) of the batched form")
    return p.parse_args()


# ----------------------------------------------------------------------------
# CPU reference arm: the float64 port of the reference path on host cores
# ----------------------------------------------------------------------------

# The CPU configuration of the reference's headline (C1): the 200 x 200 px
# synthetic scene (seed 0, 53 N, DOY 172, 24 hourly steps) through the
# float64 numpy port of the reference path (walls, 153-patch SVF, hourly
# Solweig_2022a_calc restatement, UTCI).  Static preparation is done once per
# process, untimed (as the GPU arm prepares walls and SVF before timing);
# timed samples are consecutive hours of the day with the thermal state
# carried, a new day starting after hour 23.
C1 = 200
C1_LOC = dict(latitude=53.0, longitude=0.0, altitude=3.0)
_C1 = {}


def _c1_init():
    from oracle import step as ST
    from solweig_cuda_b200 import synthetic
    sc = synthetic.make_scene(C1, seed=0)
    _C1["met"] = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    _C1["s"] = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    _C1["gen"] = None


def _c1_step(hours):
    """The next ``hours`` hours of the C1 day in this process: (pixel-hours, seconds)."""
    from oracle import step as ST
    if not _C1:
        _c1_init()
    t0 = time.perf_counter()
    done = 0
    while done < hours:
        if _C1["gen"] is None:
            _C1["gen"] = ST.day_hours(_C1["s"], _C1["met"], C1_LOC, 0.0)
        try:
            next(_C1["gen"])
            done += 1
        except StopIteration:
            _C1["gen"] = None
    return C1 * C1 * hours, time.perf_counter() - t0


def run_reference(a, rank, world):
    """pixel-hours/s of the port on every host core: one process per core, each
    stepping its own C1 day 4 hours per timed step."""
    if rank != 0:
        return
    import multiprocessing as mp
    workers = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    hours = 4
    ctx = mp.get_context("spawn")
    vals = []
    with ctx.Pool(workers, initializer=_c1_init) as pool:
        pool.map(_c1_step, [0] * workers, chunksize=1)  # every process prepared
        for i in range(a.warmup + a.steps):
            t0 = time.perf_counter()
            res = pool.map(_c1_step, [hours] * workers, chunksize=1)
            wall = time.perf_counter() - t0
            if i >= a.warmup:
                vals.append((sum(r[0] for r in res) / wall, wall))
    value = sum(v for v, _ in vals) / len(vals)
    ms = 1000.0 * sum(w for _, w in vals) / len(vals)
    sample = (f"{workers} processes x {hours} consecutive hours of the {C1}x{C1} px day (state carried) "
              f"per step; walls + 153-patch SVF prepared per process before timing")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"float64 CPU port of the reference path on the {C1}x{C1} px, 24 h CPU "
                               f"configuration (seed 0, 53N, DOY 172): hourly Tmrt+UTCI",
                   "size": C1, "hours": 24, "cores": workers},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_single():
    """The port on one host core: 12 consecutive hours (0-11) of the C1 day."""
    _c1_init()
    work, sec = _c1_step(12)
    return {"value": work / sec, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{C1}x{C1} px (seed 0, 53N, DOY 172), hours 0-11 with the thermal state carried, "
                      f"walls + 153-patch SVF prepared before timing; float64 numpy port of the reference "
                      f"path, {sec:.1f} s"}


# ----------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi samples (SM clock, throttle reasons) while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self):
        import statistics
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def _peaks():
    """(HBM GB/s, sustained BF16 TFLOP/s, source): the measured copy bandwidth and
    cuBLAS BF16 throughput of this pool's B200s, else the recorded fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        tf = d.get("bf16_tflops_sustained", d.get("bf16_tflops"))
        return float(d["hbm_gbs"]), float(tf), "measured (MEASURED_PEAKS.json hbm_gbs, bf16_tflops_sustained)"
    except (OSError, KeyError, ValueError, TypeError):
        return 6650.0, 1400.0, "fallback (6.65 TB/s, 1.4 PFLOP/s sustained BF16)"


# What bounds each stage of the batched day (from the ncu summaries in
# profiles/): the HBM fraction of the gather-bound stages is small by nature.
STAGE_LIMITER = {
    "day_shadow_kernel": "latency of the ray-step gathers through L1/L2 and lane divergence of the walk lengths",
    "day_gvf_kernel": "instruction issue of the 18 x 22 walks and the block barriers of the 4-hour passes "
                      "(shared-memory wavefronts about half of their peak)",
    "day_tables_kernel": "negligible (one block per hour)",
    "patch_gemm_kernel": "expansion of the mask bits into the BF16 operand stages (the MMAs overlap it)",
    "day_radiation_kernel": "latency of the per-pixel hour loop",
}


def _stage_kernels(cfg):
    """The kernel that does the work of each timed stage for a launch config."""
    return {
        "day_shadow_kernel": "day_sweep_tma_kernel" if cfg.sweep_window else "day_shadow_kernel",
        "day_gvf_kernel": "day_gvf_hv_kernel" if cfg.gvf_hours == 1 else "day_gvf_kernel",
        "day_tables_kernel": "day_tables_kernel",
        "patch_gemm_kernel": "patch_gemm_pipe_kernel",  # the combined sums of <= 24 hours
        "day_radiation_kernel": "day_radiation_kernel",
    }


def _traffic(kernel):
    """Per-launch DRAM bytes of ``kernel`` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith(kernel + "="):
                    return float(line.split("=", 1)[1].split()[0])
    except OSError:
        pass
    return None


def _events_ms(fn, steps, warmup, flush):
    """Mean device ms of fn() over `steps` runs after `warmup`, L2 flushed before each."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        torch.cuda.synchronize()
        times.append(s.elapsed_time(e))
    return sum(times) / len(times)


def run_month(a):
    """2000^2 px x 720 h (30 days, state reset daily) as one CUDA-graph replay."""
    import numpy as np
    import torch
    from solweig_cuda_b200 import batched, engine, synthetic, tune
    dev = torch.device("cuda", 0)
    n = a.size
    sc = synthetic.make_scene(n, seed=0)
    scene = engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover, device=dev)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0, days=30)
    day = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0)
    cfg = tune.apply(day, met[:24]) if a.tune else day.config
    del day
    md = batched.MultiDay(scene, 53.0, 0.0, 3.0, 0.0, days=30, config=cfg)
    t0 = time.perf_counter()
    md.plan(met)
    plan_s = time.perf_counter() - t0
    md.capture()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    with ClockSampler(0) as clocks:
        ms = _events_ms(md.replay, a.steps, a.warmup, flush)
    work = n * n * 720
    print(json.dumps({
        "metric": "pixel-hours/s Tmrt+UTCI, 2000^2 px x 720 h (30 days) in one CUDA graph",
        "value": work / (ms / 1000.0), "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms, "higher_is_better": True, "dtype": "f32+f64+bf16", "data": "synthetic",
        "config": {"workload": f"{n}x{n} px, DOY 172-201, 53N, thermal state reset daily, batched form",
                   "launch_config": list(cfg.astuple()), "kernel_launches": md.launches,
                   "host_plan_s_30_days": plan_s, "l2": "flushed before every replay"},
        "clocks": clocks.summary()}), flush=True)


def run_float64(a):
    """The float64 switch (dtype=float64): 2000^2 px x 24 h through the float64
    step, hour by hour, beside the float32 per-hour form on the same day."""
    import torch
    from solweig_cuda_b200 import engine, synthetic
    dev = torch.device("cuda", 0)
    n = a.size
    sc = synthetic.make_scene(n, seed=0)
    scene = engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover, device=dev)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    r64 = engine.DayRunner64(scene, 53.0, 0.0, 3.0, 0.0)
    r32 = engine.DayRunner(scene, 53.0, 0.0, 3.0, 0.0)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    with ClockSampler(0) as clocks:
        ms64 = _events_ms(lambda: r64.run_day(met), a.steps, a.warmup, flush)
    ms32 = _events_ms(lambda: r32.run_day(met), a.steps, a.warmup, flush)
    t64 = r64.run_day(met, outputs=("tmrt",))["tmrt"]
    t32 = r32.run_day(met, outputs=("tmrt",))["tmrt"]
    diff = float((t64 - t32.double()).abs().max())
    work = n * n * 24
    print(json.dumps({
        "metric": f"pixel-hours/s Tmrt+UTCI, {n}^2 px x 24 h, float64 radiation (dtype=float64)",
        "value": work / (ms64 / 1000.0), "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms64, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{n}x{n} px at 1 m, 24 hourly steps (DOY 172, 53N), solweig_step64 per hour",
                   "float32_per_hour_ms": ms32, "max_abs_tmrt_f64_minus_f32_K": diff,
                   "kernel_launches_per_day": 3 * 24, "l2": "flushed before every day"},
        "clocks": clocks.summary()}), flush=True)


def run_geometry_walls(a):
    """The geometry wall method on a 2000^2 px, 1 m raster: 20 000 seeded
    footprints (rectangles and pentagons, 4-40 m) burned into the wall rasters."""
    import numpy as np
    import torch
    from solweig_cuda_b200 import _lib, walls
    from solweig_cuda_b200.engine import device_ptr
    n = a.size
    rng = np.random.default_rng(7)
    buildings = []
    for k in range(20000):
        x, y = rng.uniform(0, n - 40, 2)
        w, h = rng.uniform(4, 40, 2)
        ring = [[x, y], [x + w, y], [x + w, y + h], [x + w / 2, y + 1.3 * h], [x, y + h], [x, y]]
        if k % 2:
            ring = [ring[0], ring[1], ring[2], ring[4], ring[5]]
        buildings.append(({"type": "Polygon", "coordinates": [ring]}, float(rng.uniform(3, 30))))
    ghsl = np.where(rng.random((n, n)) < 0.3, rng.uniform(0, 30, (n, n)), 0).astype(np.float32)
    transform = (1.0, 0.0, 0.0, 0.0, -1.0, float(n))
    t0 = time.perf_counter()
    w_host, _ = walls.calculate_geometry_walls(buildings, ghsl, (n, n), transform, 2.0)
    call_s = time.perf_counter() - t0
    # the two device kernels alone, on the segments of that call
    seg = []
    for g, h in buildings:
        hh, aa = walls.wall_segments(g, h)
        seg += [list(s[0]) + list(s[1]) for s, _ in hh]
    seg = np.asarray(seg, dtype=np.float64)
    pix = np.column_stack([seg[:, 0], n - seg[:, 1], seg[:, 2], n - seg[:, 3]])
    dev = torch.device("cuda", 0)
    t_seg = torch.from_numpy(np.ascontiguousarray(pix)).to(dev)
    t_h = torch.ones(len(pix), dtype=torch.float64, device=dev)
    t_g = torch.from_numpy(ghsl).to(dev)
    owner = torch.empty((n, n), dtype=torch.int32, device=dev)
    out_w = torch.empty((n, n), dtype=torch.float32, device=dev)
    out_a = torch.empty((n, n), dtype=torch.float32, device=dev)
    L = _lib.lib()

    def kernels():
        _lib.check(L.solweig_wall_segments_burn(device_ptr(t_seg), len(pix), n, n, device_ptr(owner), None), "burn")
        _lib.check(L.solweig_geometry_walls(device_ptr(owner), device_ptr(t_h), device_ptr(t_h), device_ptr(t_g),
                                            n * n, 2.0, device_ptr(out_w), device_ptr(out_a), None), "merge")

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    ms = _events_ms(kernels, a.steps, a.warmup, flush)
    print(json.dumps({
        "metric": f"raster pixels/s, geometry wall method (footprint edges burned, GHSL merge), {n}^2 px",
        "value": n * n / (ms / 1000.0), "unit": "pixels/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms, "higher_is_better": True, "dtype": "f64+f32", "data": "synthetic",
        "config": {"workload": f"{n}x{n} px at 1 m, 20000 footprints (seed 7), {len(pix)} edges",
                   "kernels": ["segment_burn_kernel", "geometry_walls_kernel"], "gpu_launches_per_step": 2,
                   "calculate_geometry_walls_s": call_s, "wall_pixels": int((w_host > 0).sum()),
                   "l2": "flushed before every step"}}), flush=True)


def _tile_specs(count=64):
    import numpy as np
    rng = np.random.default_rng(2024)
    sides = rng.integers(256, 1537, size=count)
    lats = rng.uniform(35.0, 60.0, size=count)
    return [(int(sides[i]), int(i + 1), float(lats[i])) for i in range(count)]


def run_tiles(a):
    """64 tiles, sides U{256..1536}, seeds 1-64, latitudes U[35, 60] N, one day each, one graph."""
    import numpy as np
    import torch
    from solweig_cuda_b200 import batched, engine, synthetic, tune
    dev = torch.device("cuda", 0)
    specs = _tile_specs()
    scenes, mets, lats = [], [], []
    for side, seed, lat in specs:
        sc = synthetic.make_scene(side, seed=seed)
        scenes.append(engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover, device=dev))
        mets.append(synthetic.make_met(doy=172, latitude=lat, longitude=0.0, seed=seed))
        lats.append(lat)
    configs = []
    tuned = {}
    for s, met, lat in zip(scenes, mets, lats):
        day = batched.ChosenDay(s, lat, 0.0, 3.0, 0.0)
        key = tune.tune_key(day)
        if a.tune and key not in tuned:
            tuned[key] = tune.apply(day, met)
        configs.append(tuned.get(key, day.config))
        del day
    tb = batched.TileBatch(scenes, lats, [0.0] * len(scenes), configs=configs)
    tb.plan(mets)
    tb.capture()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    with ClockSampler(0) as clocks:
        ms = _events_ms(tb.replay, a.steps, a.warmup, flush)
    work = tb.pixels * 24
    print(json.dumps({
        "metric": "pixel-hours/s Tmrt+UTCI, 64 uneven tiles x 24 h in one CUDA graph",
        "value": work / (ms / 1000.0), "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms, "higher_is_better": True, "dtype": "f32+f64+bf16", "data": "synthetic",
        "config": {"workload": "64 tiles, sides U{256..1536} (seed 2024), generator seeds 1-64, "
                               "latitudes U[35,60] N, DOY 172, batched form",
                   "pixels": tb.pixels, "tuned_shapes": {k: list(v.astuple()) for k, v in tuned.items()},
                   "kernel_launches": tb.launches, "l2": "flushed before every replay"},
        "clocks": clocks.summary()}), flush=True)


def run_precision(a):
    """4000^2 px: the BF16 patch contraction's error against FP64 sums on a pixel
    sample, and the batched form's Kdown/Ldown/Tmrt against the per-hour FP32 form."""
    import numpy as np
    import torch
    from solweig_cuda_b200 import batched, engine, synthetic
    dev = torch.device("cuda", 0)
    n = 4000 if a.size == 2000 else a.size
    sc = synthetic.make_scene(n, seed=0)
    scene = engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover, device=dev)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    outs = ("tmrt", "kdown", "ldown")
    day = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0, outputs=outs)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    ms = _events_ms(lambda: day.run_day(met), a.steps, a.warmup, flush)
    stage = day.profile_day(met)
    got = {k: v.clone() for k, v in day.run_day(met).items()}
    torch.cuda.synchronize()
    sums = day.patch_sums()
    # FP64 reference of the contraction on a pixel sample, all hours
    rng = np.random.default_rng(7)
    idx = torch.from_numpy(rng.choice(scene.pixels, size=65536, replace=False)).to(dev)
    L = scene.layout.host
    P = L.count
    words = scene.masks.view(torch.int32).view(10, -1)[:, idx].to(torch.int64) & 0xFFFFFFFF
    bit = torch.arange(P, device=dev)
    Sb = (words[bit // 32] >> (bit % 32)[:, None]) & 1
    Vb = (words[5 + bit // 32] >> (bit % 32)[:, None]) & 1
    sky = (Sb * (1 - Vb)).to(torch.float64).T
    veg = (Sb * Vb).to(torch.float64).T
    W = np.zeros((2 * 24, P))
    for h, s_ in enumerate(day.last_scalars):
        if s_.lv is not None:
            lum = s_.lv[:, 2]
            W[2 * h] = lum
            W[2 * h + 1] = lum * L.cos_alt * L.steradian
    Wt = torch.from_numpy(W).to(dev)
    ref_sky, ref_veg = sky @ Wt.T, veg @ Wt.T
    gsum = sums[:, idx].T.to(torch.float64)
    rsum = ref_sky + 0.03 * ref_veg
    scale = Wt.abs().sum(dim=1).clamp_min(1e-30)
    err_sum = ((gsum - rsum).abs() / scale).max().item()
    abs_sum = (gsum - rsum).abs().max().item()
    # the per-hour FP32 form (per-patch loop, no tensor cores) beside it
    plain = engine.DayRunner(scene, 53.0, 0.0, 3.0, 0.0)
    ref = plain.run_day(met, outputs=outs)
    torch.cuda.synchronize()
    diffs = {k: float(torch.nan_to_num((got[k] - ref[k]).abs(), nan=0.0).max()) for k in outs}
    gemm_flops = batched.ChosenDay.gemm_flops(scene.pixels, 24, P)
    print(json.dumps({
        "metric": "patch-sum contraction error vs FP64 and batched-vs-FP32 differences, 4000^2 px x 24 h",
        "value": n * n * 24 / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms,
        "steps": a.steps, "warmup": a.warmup, "higher_is_better": True,
        "config": {"workload": f"{n}x{n} px at 1 m, DOY 172, 53N, BF16 hi/lo weights, FP32 accumulation",
                   "sample_pixels": 65536},
        "patch_sums_max_rel_error_vs_fp64": err_sum,
        "patch_sums_max_abs_error_vs_fp64": abs_sum,
        "patch_sums": "sky + 0.03 x vegetation sums of luminance and luminance*cos*omega, per hour",
        "max_abs_diff_vs_fp32_form": diffs,
        "stages_ms": stage,
        "patch_gemm_tflops": gemm_flops / (stage["patch_gemm_kernel"] / 1000.0) / 1e12}), flush=True)


def run_gradient(a):
    """1000^2 px x 24 h: adjoint of the daily-mean UTCI (masks fixed) w.r.t. albedo
    U[0.1,0.4], emissivity U[0.9,0.98], vegetation transmissivity U[0.02,0.2] and
    Ta/RH/wind; timed, and checked against central differences along random
    directions."""
    import numpy as np
    import torch
    from solweig_cuda_b200 import engine, grad, synthetic
    dev = torch.device("cuda", 0)
    n = 1000 if a.size == 2000 else a.size
    sc = synthetic.make_scene(n, seed=0)
    scene = engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover, device=dev)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    rng = np.random.default_rng(0)
    prm = {"albedo": rng.uniform(0.1, 0.4, scene.shape).astype(np.float32),
           "emissivity": rng.uniform(0.9, 0.98, scene.shape).astype(np.float32),
           "transmissivity": rng.uniform(0.02, 0.2, scene.shape).astype(np.float32)}
    w = np.ones(scene.shape, np.float32) / scene.pixels
    dg = grad.DayGradient(scene, 53.0, 0.0, 3.0, 0.0)
    P = {k: torch.from_numpy(v).to(dev) for k, v in prm.items()}
    Wt = torch.from_numpy(w).to(dev)

    def fwd():
        return dg.forward(P["albedo"], P["emissivity"], P["transmissivity"], met)

    def bwd():
        return dg.backward(P["albedo"], P["emissivity"], P["transmissivity"], met, Wt)

    for _ in range(a.warmup):
        fwd()
        bwd()
    t_f, t_b = [], []
    for _ in range(a.steps):
        t0 = time.perf_counter()
        fwd()
        t_f.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        out = bwd()
        t_b.append(time.perf_counter() - t0)
    t0 = time.perf_counter()
    jac = dg.forcing_jacobian(met)
    t_jac = time.perf_counter() - t0
    fg = dg.forcing_grad(met, out[3], out[4], jac)
    g = {"albedo": out[0].cpu().numpy().astype(np.float64), "emissivity": out[1].cpu().numpy().astype(np.float64),
         "transmissivity": out[2].cpu().numpy().astype(np.float64), **fg}

    def J(p, m):
        d = dg.forward(p["albedo"], p["emissivity"], p["transmissivity"], m).cpu().numpy()
        return float(np.nansum(d * w))

    steps = {"albedo": 1e-2, "emissivity": 1e-2, "transmissivity": 1e-2, "ta": 1e-2, "rh": 1e-1, "ws": 1e-2}
    rng = np.random.default_rng(1)
    checks = {}
    for name, h in steps.items():
        v = rng.uniform(-1, 1, scene.shape if name in prm else 24)
        pp = {k: x.copy() for k, x in prm.items()}
        pm = {k: x.copy() for k, x in prm.items()}
        mp, mm = met.copy(), met.copy()
        if name in prm:
            pp[name] = (prm[name] + h * v).astype(np.float32)
            pm[name] = (prm[name] - h * v).astype(np.float32)
        else:
            col = grad.FORCING_COLUMNS[name]
            mp[:, col] += h * v
            mm[:, col] -= h * v
        fd = (J(pp, mp) - J(pm, mm)) / (2 * h)
        ad = float(np.sum(g[name] * v))
        checks[name] = {"adjoint": ad, "central_difference": fd, "rel_error": abs(ad - fd) / max(abs(fd), 1e-30)}
    print(json.dumps({
        "metric": "daily-mean UTCI adjoint, 1000^2 px x 24 h (masks fixed)",
        "value": float(np.mean(t_b)), "unit": "s per backward (forward recomputed inside)",
        "higher_is_better": False, "steps": a.steps, "warmup": a.warmup,
        "forward_s": float(np.mean(t_f)), "forcing_jacobian_s": t_jac,
        "config": {"workload": f"{n}x{n} px at 1 m, DOY 172, 53N; albedo U[0.1,0.4], emissivity U[0.9,0.98], "
                               "transmissivity U[0.02,0.2]; J = mean over pixels of daily-mean UTCI",
                   "timing": "host wall clock around each synchronous call"},
        "directional_checks": checks,
        "gradient_norms": {k: float(np.linalg.norm(v)) for k, v in g.items()}}), flush=True)


def main():
    a = _args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if a.impl == "reference":
        run_reference(a, rank, world)
        return 0
    if a.workload != "day":
        if rank == 0:
            import torch
            torch.cuda.set_device(0)
            {"month": run_month, "tiles": run_tiles, "precision": run_precision,
             "gradient": run_gradient, "float64": run_float64,
             "geometry_walls": run_geometry_walls}[a.workload](a)
        return 0
    import numpy as np
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from solweig_cuda_b200 import batched, engine, synthetic
    dev = torch.device("cuda", local)
    n = a.size
    sc = synthetic.make_scene(n, seed=0)
    doy = 172 + rank
    met = synthetic.make_met(doy=doy, latitude=53.0, longitude=0.0)
    scene = engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover, device=dev)
    torch.cuda.synchronize()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2

    plain = engine.DayRunner(scene, 53.0, 0.0, 3.0, 0.0)
    if a.form == "chosen":
        chosen = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0)
        if a.tune:
            from solweig_cuda_b200 import tune
            tune.apply(chosen, met)
    elif a.form == "batched":
        chosen = batched.BatchedDay(scene, 53.0, 0.0, 3.0, 0.0)
    else:
        chosen = plain

    def day(runner):
        return runner.run_day(met, outputs=("tmrt", "utci"))

    def timed(runner, steps, warmup):
        for _ in range(warmup):
            day(runner)
        torch.cuda.synchronize()
        times = []
        for _ in range(steps):
            flush.zero_()
            if dist is not None:
                dist.barrier()
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            day(runner)
            e.record()
            torch.cuda.synchronize()
            times.append(s.elapsed_time(e))
        return times

    sun_alt = __import__("solweig_cuda_b200.sun", fromlist=["metdata"]).metdata(met, 53.0, 0.0, 3.0, 0.0).altitude
    # our kernels per timed day: 7 for the batched form, shadow/GVF/radiation per hour otherwise
    launches_per_day = chosen.launches_per_day if a.form == "chosen" else 3 * len(met)
    plain_times = timed(plain, max(1, min(a.steps, 3)), 1)
    with ClockSampler(local) as clocks:
        chosen_times = timed(chosen, a.steps, a.warmup)
    ms = float(np.mean(chosen_times))
    ms_plain = float(np.mean(plain_times))
    if dist is not None:
        t = torch.tensor([ms, ms_plain], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_plain = float(t[0]), float(t[1])
    work = n * n * 24
    value = world * work / (ms / 1000.0)
    value_plain = world * work / (ms_plain / 1000.0)

    # Per-kernel timing of one instrumented day (events on the launching stream).
    peak, peak_tf, peak_src = _peaks()
    roof = None
    if a.form == "chosen":
        stage_ms = chosen.profile_day(met)
        day_hours = int(sum(1 for x in sun_alt if x > 0))
        px = n * n
        bytes_per = batched.ChosenDay.stage_bytes(px, 24, day_hours)
        gemm_flops = batched.ChosenDay.gemm_flops(px, 24, scene.layout.host.count)
        kernels = _stage_kernels(chosen.config)
        total = sum(stage_ms.values())
        stages = {}
        for k, v in stage_ms.items():
            if k == "patch_gemm_kernel":
                ach = gemm_flops / (v / 1000.0) / 1e12
                e = {"bound": "tensor", "achieved": ach, "peak": peak_tf, "unit": "TFLOP/s",
                     "frac": ach / peak_tf, "algorithmic": gemm_flops}
            else:
                ach = bytes_per[k] / (v / 1000.0) / 1e9
                e = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                     "algorithmic": bytes_per[k]}
            e.update({"kernel": kernels[k], "ms": round(v, 4), "share": round(v / total, 4),
                      "limiter": STAGE_LIMITER[k], "traffic": _traffic(kernels[k])})
            stages[k] = e
        dom = max(stages, key=lambda k: stages[k]["ms"])
        d = stages[dom]
        roof = {"bound": d["bound"], "kernel": d["kernel"], "achieved": d["achieved"], "peak": d["peak"],
                "unit": d["unit"], "frac": d["frac"], "peak_source": peak_src, "traffic": d["traffic"],
                "launch_ms": d["ms"], "limiter": d["limiter"], "stages": stages,
                "patch_gemm_tflops": stages["patch_gemm_kernel"]["achieved"]}
    else:
        kern = plain.profile_day(met)
        dom = max(kern, key=lambda k: kern[k]["ms"])
        info = kern[dom]
        achieved = info["bytes_per_launch"] / (info["ms"] / info["launches"] / 1000.0) / 1e9
        roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_src,
                "traffic": _traffic(dom), "launch_ms": info["ms"] / info["launches"],
                "share": {k: round(v["ms"] / sum(x["ms"] for x in kern.values()), 4) for k, v in kern.items()}}

    # The 720 h target of the metric: 30 days (state reset daily) in ONE graph
    # replay against the plain per-hour form over the same 30 days.
    month = None
    if a.form == "chosen" and world == 1 and not a.no_month:
        met30 = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0, days=30)
        md = batched.MultiDay(scene, 53.0, 0.0, 3.0, 0.0, days=30, config=chosen.config)
        t0 = time.perf_counter()
        md.plan(met30)
        plan_s = time.perf_counter() - t0
        md.capture()
        month_ms = _events_ms(md.replay, 2, 1, flush)
        launches_month = md.launches
        del md
        torch.cuda.empty_cache()
        torch.cuda.synchronize()
        flush.zero_()
        torch.cuda.synchronize()
        s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s_ev.record()
        for d in range(30):
            plain.run_day(met30[24 * d:24 * (d + 1)], outputs=("tmrt", "utci"))
        e_ev.record()
        torch.cuda.synchronize()
        plain_month_ms = s_ev.elapsed_time(e_ev)
        work30 = n * n * 720
        month = {"value": work30 / (month_ms / 1000.0), "ms_per_step": month_ms,
                 "value_with_host_plan": work30 / (month_ms / 1000.0 + plan_s),
                 "plain_value": work30 / (plain_month_ms / 1000.0), "plain_ms": plain_month_ms,
                 "ratio_vs_plain": plain_month_ms / month_ms,
                 "ratio_vs_plain_with_host_plan": plain_month_ms / (month_ms + 1000.0 * plan_s),
                 "kernel_launches": launches_month, "host_plan_s": plan_s,
                 "workload": f"{n}x{n} px x 720 h (DOY 172-201, thermal state reset daily): the batched "
                             "form in one CUDA-graph replay (host plan of the 30 days outside it; also "
                             "reported with it) vs the plain per-hour form over the same days (its host "
                             "plan interleaved); L2 flushed before each"}

    # End to end through the public API with host buffers: the input rasters
    # sit in page-locked host memory (as a caller streaming tiles keeps them),
    # the results come back into the API's page-locked buffers.
    from solweig_cuda_b200 import api

    def _pinned_host(x):
        t = torch.empty(x.shape, dtype=torch.from_numpy(np.ascontiguousarray(x)).dtype, pin_memory=True)
        t.copy_(torch.from_numpy(np.ascontiguousarray(x)))
        return t

    host_in = {k: _pinned_host(getattr(sc, k)) for k in ("dsm", "trees", "dem", "landcover")}
    e2e_times, h2d, d2h = [], 0, 0
    for i in range(a.e2e_steps + 1 if a.e2e_steps > 0 else 0):
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = api.simulate_day(host_in["dsm"].numpy(), host_in["trees"].numpy(), host_in["dem"].numpy(), met,
                               latitude=53.0, longitude=0.0, landcover=host_in["landcover"].numpy(),
                               pixel_size=1.0, device=dev, form=a.form)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if i > 0:
            e2e_times.append(dt)
        h2d, d2h = res["h2d_bytes"], res["d2h_bytes"]
    # median over the steps (a step that meets a cold allocator or a busy host
    # would otherwise dominate a short run); every step is listed in the line
    e2e_s = float(np.median(e2e_times)) if e2e_times else float("nan")
    if dist is not None:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t[0])
    e2e_value = world * work / e2e_s if e2e_times else None
    if not e2e_times:
        e2e_s = None

    # the reference's driver call (series.run_timeseries, no files written):
    # rasters from host arrays, walls + SVF, 3 calendar days in the batched form
    series_e2e = None
    if rank == 0 and world == 1 and a.e2e_steps > 0:
        import tempfile
        from solweig_cuda_b200 import series
        met3 = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0, days=3)
        with tempfile.TemporaryDirectory() as tmp:
            def run_series(m):
                series.run_timeseries(sc.dsm, sc.trees, sc.dem, m, tmp, 0.0, 53.0, landcover_path=sc.landcover,
                                      utc_offset_hours=0.0, no_write=True, device=dev)
            run_series(met3[:24])  # warm-up: kernel attributes, allocator
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            run_series(met3)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
        series_e2e = {"value": n * n * 72 / dt, "unit": UNIT, "seconds": dt,
                      "includes": "series.run_timeseries(no_write=True): H2D rasters, walls, 153-patch SVF, "
                                  "3 days x 24 h in the batched form"}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline_single()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64+bf16" if a.form == "chosen" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": f"{n}x{n} px at 1 m, 24 hourly steps (one day, DOY 172, 53N), "
                                   f"static walls + 153-patch SVF prepared before timing",
                       "form": a.form, "size": n, "hours": 24, "l2": "flushed (256 MB write) before every timed step",
                       "parallelism": f"days over {world} GPU(s)"},
            "plain": {"value": value_plain, "ms_per_step": ms_plain, "ratio": value / value_plain},
            "month_720h": month,
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "seconds_per_step": e2e_s,
                    "seconds_each_step": [round(t, 4) for t in e2e_times],
                    "includes": "H2D rasters (page-locked), walls, 153-patch SVF, 24 h, D2H Tmrt+UTCI",
                    "run_timeseries_no_write": series_e2e},
            "gpu_launches": launches_per_day * a.steps,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
