"""Batched form: a whole day (or many days) per CUDA-graph replay.

All hours of a day are planned on the host first (FP64 solar geometry,
Perez luminance, patch weights, sun rays), written into pinned memory and
replayed as one captured graph: the hour-record and ray uploads, the state
reset and the 2 kernels of every hour (``solweig_day``).  The graph is
captured once per scene and replays for any forcing of the same length,
because every kernel reads its hour record from device memory.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .engine import HourBuffers, device_ptr, outputs_struct, plan_day, stream_handle

__all__ = ["BatchedDay", "ChosenDay"]


class BatchedDay:
    """Run days of ``hours`` rows each through one captured graph."""

    def __init__(self, scene, latitude, longitude, site_altitude=3.0, utc=0.0, hours=24,
                 outputs=("tmrt", "utci"), use_graph=True):
        self.scene = scene
        self.latitude, self.longitude, self.site_altitude, self.utc = latitude, longitude, site_altitude, utc
        self.hours = hours
        dev = scene.device
        self.state = {k: torch.zeros(scene.shape, dtype=torch.float32, device=dev)
                      for k in _lib.STATE_FIELDS}
        self.scratch = torch.empty((_lib.SCRATCH_PLANES, scene.rows, scene.cols), dtype=torch.float32,
                                   device=dev)
        self.buffers = HourBuffers(scene, hours)
        self.layout_dev = scene.layout.device(dev)
        self.out_names = tuple(outputs)
        self.out = {k: torch.empty((hours,) + scene.shape, dtype=torch.float32, device=dev)
                    for k in self.out_names}
        self.use_graph = use_graph
        self.graph = None
        self.launches_per_day = 2 * hours

    def _state_struct(self):
        s = _lib.SolweigState()
        for k in _lib.STATE_FIELDS:
            setattr(s, k, self.state[k].data_ptr())
        return s

    def _sequence(self):
        """Uploads, state reset and the day's kernels, on the current stream."""
        self.buffers.upload(0, self.hours, self.buffers.kmax)
        for t in self.state.values():
            t.zero_()
        sc = self.scene
        base = outputs_struct(self.out, 0)
        stride = sc.pixels
        _lib.check(_lib.lib().solweig_day(
            ctypes.byref(sc.struct), device_ptr(self.layout_dev), self.buffers.ptr(), self.hours,
            ctypes.byref(self._state_struct()), ctypes.byref(base), stride, sc.gvf_host_ptr,
            sc.first_steps, sc.second_steps, device_ptr(self.scratch), stream_handle()),
            "solweig_day")

    def plan(self, met):
        met = np.asarray(met, dtype=np.float64)
        if len(met) != self.hours:
            raise ValueError(f"expected {self.hours} forcing rows, got {len(met)}")
        plan = plan_day(self.scene, met, self.latitude, self.longitude, self.site_altitude, self.utc)
        self.buffers.wait_free()
        for i, (h, ray, _) in enumerate(plan):
            self.buffers.put(i, h, ray)
        self.last_scalars = [p[2] for p in plan]
        return plan

    def run_day(self, met, outputs=None):
        """Plan the day on the host and replay; returns {name: [H, rows, cols]} views
        that stay valid until the next call."""
        self.plan(met)
        if not self.use_graph:
            self._sequence()
        else:
            if self.graph is None:
                self._sequence()          # eager pass: kernel attributes, allocator warm-up
                torch.cuda.synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    self._sequence()
                self.graph = g
            self.graph.replay()
        self.buffers.mark()
        names = self.out_names if outputs is None else outputs
        return {k: self.out[k] for k in names}


class ChosenDay(BatchedDay):
    """The batched form: every hour of a day in seven launches
    (``solweig_day_batched``: per-launch shadow and GVF over all hours, the
    BF16 tensor-core patch contraction, hour-looping radiation), replayed as
    one CUDA graph together with the hour-record uploads.

    Produces the all-direction planes (Tmrt, UTCI, Kdown, Kup, Ldown, Lup,
    Kside, Lside, shadow, Tg ...); the cardinal E/S/W/N planes are only made
    by the per-hour form."""

    CARDINAL = ("keast", "ksouth", "kwest", "knorth", "least", "lsouth", "lwest", "lnorth")

    def __init__(self, scene, latitude, longitude, site_altitude=3.0, utc=0.0, hours=24,
                 outputs=("tmrt", "utci"), use_graph=True):
        bad = [o for o in outputs if o in self.CARDINAL]
        if bad:
            raise ValueError(f"the batched form does not produce {bad}")
        super().__init__(scene, latitude, longitude, site_altitude, utc, hours, outputs, use_graph)
        self.scratch = None
        L = _lib.lib()
        self.work_bytes = int(L.solweig_day_batched_work_bytes(scene.rows, scene.cols, hours,
                                                               int(scene.struct.has_water)))
        if self.work_bytes <= 0:
            raise ValueError("bad batched-day shape")
        self.work = torch.empty(self.work_bytes, dtype=torch.uint8, device=scene.device)
        self.launches_per_day = 7

    def _sequence(self):
        self.buffers.upload(0, self.hours, self.buffers.kmax)
        for t in self.state.values():
            t.zero_()
        sc = self.scene
        base = outputs_struct(self.out, 0)
        _lib.check(_lib.lib().solweig_day_batched(
            ctypes.byref(sc.struct), device_ptr(self.layout_dev), self.buffers.ptr(), self.hours,
            ctypes.byref(self._state_struct()), ctypes.byref(base), sc.pixels, sc.gvf_host_ptr,
            sc.first_steps, sc.second_steps, device_ptr(self.work), self.work_bytes, stream_handle()),
            "solweig_day_batched")

    def error_flag(self):
        """Device error flag of the last day (0 = ok, 1 = a tensor-core wait timed out)."""
        flag = torch.zeros(1, dtype=torch.int32, device=self.scene.device)
        sc = self.scene
        _lib.check(_lib.lib().solweig_day_batched_error(
            device_ptr(self.work), sc.rows, sc.cols, self.hours, int(sc.struct.has_water),
            device_ptr(flag), stream_handle()), "solweig_day_batched_error")
        return int(flag.item())
