"""Autotuner for the launch shapes of the batched day.

The search space is :class:`_lib.SolweigDayConfig`:

* sweep: the shared-memory window sweep (TMA-staged 48 x 48 or 40 x 40
  windows, fixed 16 x 16 tiles), or the raster sweep with a shadow block
  (columns x rows) of 32x8, 64x4, 16x16, 32x4, 128x2
* GVF: tile rows per block of the per-hour kernel: 4, 8, 16 (32 columns,
  halo of ``second`` - 1), or the hour-vectorized kernel on 32 x 32 tiles
* radiation block: 128 or 256 pixels
* patch-contraction CTAs per SM: 1 or 2

``solweig_day_batched_timed`` times every stage with CUDA events on the
launching stream, and each stage's time depends only on its own parameter,
so the search is one pass per parameter with the others held (7 + 4 + 2 + 2
timed days, each repeated and the minimum taken).  Results are cached per
(device, tile-size bucket, hours, patches) in a JSON file
(``$SOLWEIG_TUNE_CACHE`` or ``~/.cache/solweig_cuda_b200/autotune.json``),
shared by threads of one process through a lock and replaced atomically.
"""
from __future__ import annotations

import json
import os
import threading
from pathlib import Path

import torch

from . import _lib

__all__ = ["SHADOW_BLOCKS", "GVF_ROWS", "GVF_HOURS", "RAD_THREADS", "GEMM_CTAS", "cache_path", "tune_key",
           "tune", "lookup", "apply"]

SHADOW_BLOCKS = ((32, 8), (64, 4), (16, 16), (32, 4), (128, 2))
GVF_ROWS = (4, 8, 16)
GVF_HOURS = (0, 1)
RAD_THREADS = (128, 256)
GEMM_CTAS = (1, 2)

_lock = threading.Lock()


def cache_path():
    env = os.environ.get("SOLWEIG_TUNE_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "solweig_cuda_b200" / "autotune.json"


def _bucket(n):
    """Tile sides are grouped to the nearest multiple of 256 (at least 256)."""
    return max(256, int(round(n / 256.0)) * 256)


def tune_key(runner):
    sc = runner.scene
    name = torch.cuda.get_device_name(sc.device)
    return f"v5|{name}|{_bucket(sc.rows)}x{_bucket(sc.cols)}|h{runner.hours}|p{sc.struct.patches}"


def _load():
    p = cache_path()
    try:
        with open(p) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(key, config, stages):
    p = cache_path()
    with _lock:
        data = _load()
        data[key] = {"config": list(config.astuple()), "stage_ms": stages}
        p.parent.mkdir(parents=True, exist_ok=True)
        tmp = p.with_suffix(f".{os.getpid()}.{threading.get_ident()}.tmp")
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, p)


def lookup(runner):
    """Cached config for this runner's shape, or None."""
    with _lock:
        entry = _load().get(tune_key(runner))
    if entry is None:
        return None
    return _lib.SolweigDayConfig(*entry["config"])


def _timed(runner, met, config, repeats):
    runner.set_config(config)
    best = None
    for _ in range(repeats):
        ms = runner.profile_day(met)
        best = ms if best is None else {k: min(best[k], ms[k]) for k in ms}
    return best


def tune(runner, met, repeats=2, use_cache=True):
    """Pick the launch shapes for ``runner`` (a :class:`batched.ChosenDay`) on
    the forcing ``met``; returns (config, per-stage ms of the chosen config)."""
    key = tune_key(runner)
    if use_cache:
        cached = lookup(runner)
        if cached is not None:
            runner.set_config(cached)
            return cached, None
    cfg = list(_lib.SolweigDayConfig.default().astuple())
    runner.profile_day(met)  # warm-up: kernel attributes, caches
    stages = {}

    def pick(stage, candidates, assign):
        nonlocal cfg
        best_t, best_c = None, None
        for cand in candidates:
            trial = list(cfg)
            assign(trial, cand)
            t = _timed(runner, met, _lib.SolweigDayConfig(*trial), repeats)[stage]
            if best_t is None or t < best_t:
                best_t, best_c = t, trial
        cfg = best_c
        stages[stage] = best_t

    def set_shadow(c, v):
        c[0], c[1], c[7] = v

    def set_gvf(c, v):
        c[2], c[5] = v

    def set_rad(c, v):
        c[3] = v

    def set_gemm(c, v):
        c[4] = v

    pick("day_shadow_kernel", [(cfg[0], cfg[1], w) for w in (1, 2)] + [(bx, by, 0) for bx, by in SHADOW_BLOCKS],
         set_shadow)
    pick("day_gvf_kernel", [(cfg[2], h) for h in GVF_HOURS if h] + [(r, 0) for r in GVF_ROWS], set_gvf)
    pick("day_radiation_kernel", RAD_THREADS, set_rad)
    pick("patch_gemm_kernel", GEMM_CTAS, set_gemm)
    config = _lib.SolweigDayConfig(*cfg)
    runner.set_config(config)
    if use_cache:
        _store(key, config, stages)
    return config, stages


def apply(runner, met, repeats=2):
    """Tuned config from the cache, or tune now; sets it on the runner."""
    return tune(runner, met, repeats=repeats, use_cache=True)[0]
