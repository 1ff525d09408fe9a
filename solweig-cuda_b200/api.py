"""Public end-to-end call: host rasters and forcing in, host Tmrt and UTCI out.

``simulate_day`` is the whole per-tile workflow of ``run_timeseries`` for one
calendar day without file I/O: rasters uploaded, walls and the 153-patch SVF
prepared on the device, the 24 hourly steps run, and every hour's Tmrt and
UTCI copied back into pinned host memory.
"""
from __future__ import annotations

import threading

import numpy as np
import torch

from . import engine, tune
from .batched import BatchedDay, ChosenDay

__all__ = ["simulate_day"]

# Page-locked host buffers for the results, reused across calls: page-locking
# hundreds of megabytes on every call costs several times the day itself.
_PINNED = {}
_PINNED_LOCK = threading.Lock()


def _pinned(name, shape):
    key = (name, tuple(shape))
    with _PINNED_LOCK:
        buf = _PINNED.get(key)
        if buf is None:
            buf = torch.empty(shape, dtype=torch.float32, pin_memory=True)
            _PINNED[key] = buf
    return buf


def simulate_day(dsm, trees, dem, met, latitude, longitude, landcover=None, pixel_size=1.0,
                 site_altitude=3.0, utc=0.0, device="cuda", form="chosen", reuse_output=True):
    """Returns {"tmrt": [H, rows, cols] float32, "utci": ..., "h2d_bytes", "d2h_bytes"}.

    form: "chosen" (batched day, tensor-core patch sums), "batched" (per-hour
    kernels in one launch sequence) or "plain" (per-hour loop).
    reuse_output: the returned arrays live in page-locked buffers that the
    next call with the same shape overwrites (copy them to keep them); False
    page-locks fresh buffers for every call."""
    # rasters are uploaded in their own dtype and widened on the device
    arrays = [np.ascontiguousarray(a) for a in (dsm, trees, dem)]
    lc = None if landcover is None else np.ascontiguousarray(landcover)
    h2d = sum(a.nbytes for a in arrays) + (lc.nbytes if lc is not None else 0)
    scene = engine.Scene(arrays[0], arrays[1], arrays[2], pixel_size, landcover=lc, device=device)
    met = np.asarray(met, dtype=np.float64)
    if form == "chosen":
        runner = ChosenDay(scene, latitude, longitude, site_altitude, utc, hours=len(met),
                           use_graph=False)
        # launch shapes tuned earlier for this device and tile size, if any
        # (the call itself never tunes)
        cached = tune.lookup(runner)
        if cached is not None:
            runner.set_config(cached)
    elif form == "batched":
        runner = BatchedDay(scene, latitude, longitude, site_altitude, utc, hours=len(met),
                            use_graph=False)
    else:
        runner = engine.DayRunner(scene, latitude, longitude, site_altitude, utc)
    res = runner.run_day(met, outputs=("tmrt", "utci"))
    out = {}
    d2h = 0
    for k in ("tmrt", "utci"):
        host = (_pinned(k, res[k].shape) if reuse_output
                else torch.empty(res[k].shape, dtype=torch.float32, pin_memory=True))
        host.copy_(res[k], non_blocking=True)
        out[k] = host
        d2h += host.numel() * 4
    torch.cuda.current_stream().synchronize()
    if hasattr(runner, "check_errors"):
        runner.check_errors()
    out = {k: v.numpy() for k, v in out.items()}
    out["h2d_bytes"] = h2d
    out["d2h_bytes"] = d2h
    return out
