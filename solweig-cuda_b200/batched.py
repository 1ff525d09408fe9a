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
from .engine import HourBuffers, device_ptr, outputs_struct, plan_day, plan_hours, stream_handle

__all__ = ["BatchedDay", "ChosenDay", "MultiDay", "TileBatch", "DayError"]

# Bits of the sticky error word (word 1 of the flag pair at the start of the
# work buffer): bit v is set when a day raised flag v.  Flags 1 (a tensor-core
# wait of the contraction timed out) and 3 (a sun ray stayed inside the raster
# for more than max(rows, cols) + 2 steps) leave invalid results; flag 2 (a
# window sweep's TMA wait timed out) does not (that tile walked from the raster).
_INVALID_BITS = (1 << 1) | (1 << 3)
_FLAG_TEXT = {1: "a tensor-core wait of the patch contraction timed out",
              2: "a sweep window's TMA wait timed out (results exact)",
              3: "a sun ray table stayed inside the raster longer than max(rows, cols) + 2 steps"}


class DayError(RuntimeError):
    """A batched day raised a device error flag that invalidates its results."""


def _error_words(work):
    """The flag pair at the start of a batched-day work buffer (int32 view)."""
    return work[:8].view(torch.int32)


def clear_day_errors(work):
    """Zero both words of the flag pair (the days never clear the sticky word)."""
    _error_words(work).zero_()


def check_day_errors(work, what="batched day"):
    """Raise DayError when a day run in `work` since the last clear raised a
    flag that invalidates results; returns the sticky bit set (synchronises)."""
    bits = int(_error_words(work)[1].item())
    if bits & _INVALID_BITS:
        raised = [v for v in _FLAG_TEXT if bits & (1 << v)]
        raise DayError(f"{what}: " + "; ".join(_FLAG_TEXT[v] for v in raised) + " - results invalid")
    return bits


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

    @property
    def launches_per_day(self):
        """Shadow, GVF and radiation kernel of every hour."""
        return 3 * self.hours

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


def day_launches(scene, config, sweep_parts=1):
    """Kernel launches of one batched day for this scene and launch shapes,
    with the sweep stage issued in ``sweep_parts`` hour ranges: per range the
    ray exits, the ceilings and the sweep; once the height dilation (and the
    tile maxima of the window sweep); then the GVF (the hour-vectorized
    kernel or the per-hour one), weights, two splits (sky and vegetation
    weights), tables, contraction and radiation."""
    c = int(not config.no_ceiling)
    win = int(config.sweep_window != 0 and scene.geo32 is not None and not scene.struct.has_water)
    return sweep_parts * (2 + c) + c + win + 7


class ChosenDay(BatchedDay):
    """The batched form: every hour of a day in a few launches
    (``solweig_day_batched``: ray ceilings and shadow sweep over ranges of
    hours, GVF over all hours, the BF16 tensor-core patch contraction,
    hour-looping radiation).  Each sweep range is a CUDA graph (with the
    upload of its hour records) replayed as soon as its hours are planned, so
    the host plans the next range while the GPU sweeps; the rest of the day is
    one more graph.

    Produces the all-direction planes (Tmrt, UTCI, Kdown, Kup, Ldown, Lup,
    Kside, Lside, shadow, Tg ...); the cardinal E/S/W/N planes are only made
    by the per-hour form."""

    CARDINAL = ("keast", "ksouth", "kwest", "knorth", "least", "lsouth", "lwest", "lnorth")

    def __init__(self, scene, latitude, longitude, site_altitude=3.0, utc=0.0, hours=24,
                 outputs=("tmrt", "utci"), use_graph=True, pipeline_hours=(2, 2, 2, 2, 4, 4, 8)):
        bad = [o for o in outputs if o in self.CARDINAL]
        if bad:
            raise ValueError(f"the batched form does not produce {bad}")
        super().__init__(scene, latitude, longitude, site_altitude, utc, hours, outputs, use_graph)
        self.scratch = None
        # pipeline_hours: the sweep stage runs in ranges of hours, each launched
        # as soon as its hours are planned (the host plans the next range while
        # the GPU sweeps this one): an int gives ranges of that many hours, a
        # sequence the successive range lengths (the last one repeats), 0 plans
        # the whole day first.  The default starts with short ranges, so the
        # GPU starts early, and grows them, so fewer launches are paid for.
        self.ranges = self._ranges(hours, pipeline_hours)
        self.part_graphs = None
        L = _lib.lib()
        self.work_bytes = int(L.solweig_day_batched_work_bytes(scene.rows, scene.cols, hours,
                                                               int(scene.struct.has_water)))
        if self.work_bytes <= 0:
            raise ValueError("bad batched-day shape")
        self.work = torch.empty(self.work_bytes, dtype=torch.uint8, device=scene.device)
        clear_day_errors(self.work)
        self.config = _lib.SolweigDayConfig.default()

    @staticmethod
    def _ranges(hours, pipeline_hours):
        if isinstance(pipeline_hours, int):
            if pipeline_hours <= 0:
                return None
            lengths = [pipeline_hours]
        else:
            lengths = [int(x) for x in pipeline_hours]
            if not lengths or min(lengths) <= 0:
                raise ValueError("pipeline_hours: range lengths must be positive")
        out, h, i = [], 0, 0
        while h < hours:
            n = lengths[min(i, len(lengths) - 1)]
            out.append((h, min(h + n, hours)))
            h, i = h + n, i + 1
        return out

    @property
    def launches_per_day(self):
        """Kernels of one day (``day_launches``)."""
        return day_launches(self.scene, self.config, len(self.ranges) if self.ranges else 1)

    def set_config(self, config):
        """Launch shapes (``SolweigDayConfig`` or a tuple of its fields); drops captured graphs."""
        if not isinstance(config, _lib.SolweigDayConfig):
            config = _lib.SolweigDayConfig(*config)
        self.config = config
        self.graph = None
        self.part_graphs = None

    def _part(self, part, h0=0, h1=0):
        """One part of the day on the current stream (``solweig_day_batched_part``):
        part 0 uploads the records and rays of hours [h0, h1) and sweeps them,
        part 1 runs the rest of the day."""
        if part == 0:
            self.buffers.upload(h0, h1 - h0, self.buffers.kmax)
        sc = self.scene
        base = outputs_struct(self.out, 0)
        _lib.check(_lib.lib().solweig_day_batched_part(
            ctypes.byref(sc.struct), device_ptr(self.layout_dev), self.buffers.ptr(), self.hours,
            ctypes.byref(_lib.SolweigState()), ctypes.byref(base), sc.pixels, sc.gvf_host_ptr,
            sc.first_steps, sc.second_steps, device_ptr(self.work), self.work_bytes,
            ctypes.byref(self.config), part, h0, h1, stream_handle()), "solweig_day_batched_part")

    def run_day(self, met, outputs=None):
        """Plan the day on the host and run it; with pipelined ranges each sweep
        range starts as soon as its hours are planned.  Returns {name: [H, rows,
        cols]} views that stay valid until the next call."""
        if self.ranges is None:
            return super().run_day(met, outputs)
        met = np.asarray(met, dtype=np.float64)
        if len(met) != self.hours:
            raise ValueError(f"expected {self.hours} forcing rows, got {len(met)}")
        self.buffers.wait_free()
        rows = plan_hours(self.scene, met, self.latitude, self.longitude, self.site_altitude, self.utc)
        scalars = []
        capture = self.use_graph and self.part_graphs is None
        for c, (h0, h1) in enumerate(self.ranges):
            for i in range(h0, h1):
                h, ray, scal = next(rows)
                self.buffers.put(i, h, ray)
                scalars.append(scal)
            if self.use_graph and not capture:
                self.part_graphs[c].replay()
            else:
                self._part(0, h0, h1)
        if self.use_graph and not capture:
            self.part_graphs[-1].replay()
        else:
            self._part(1)
        if capture:
            # the eager pass above produced this day; capture the parts for the next ones
            torch.cuda.synchronize()
            graphs = []
            for h0, h1 in self.ranges:
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    self._part(0, h0, h1)
                graphs.append(g)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._part(1)
            graphs.append(g)
            self.part_graphs = graphs
        self.last_scalars = scalars
        self.buffers.mark()
        names = self.out_names if outputs is None else outputs
        return {k: self.out[k] for k in names}

    def _sequence(self):
        # Each day starts from the reset state (src/series.py:425-436): the
        # batched kernel starts from zero state when no state planes are given,
        # and nothing needs the day's final state.
        self.buffers.upload(0, self.hours, self.buffers.kmax)
        sc = self.scene
        base = outputs_struct(self.out, 0)
        _lib.check(_lib.lib().solweig_day_batched_ex(
            ctypes.byref(sc.struct), device_ptr(self.layout_dev), self.buffers.ptr(), self.hours,
            ctypes.byref(_lib.SolweigState()), ctypes.byref(base), sc.pixels, sc.gvf_host_ptr,
            sc.first_steps, sc.second_steps, device_ptr(self.work), self.work_bytes,
            ctypes.byref(self.config), stream_handle()), "solweig_day_batched_ex")

    @staticmethod
    def stage_bytes(pixels, hours, day_hours):
        """Algorithmic HBM bytes of each stage of one day.

        shadow (with the ray ceilings): per daytime pixel-hour 16 B packed
        geometry read and a 4 B ceiling written and read back, 40 B float64
        geometry + 1 B flags + 20 B float32 fields read, 16 B quad written
        (101 B); GVF: 16 B quad + 4 B face
        bits + 4 B emissivity read, 3 planes + the albedo-without-shadow plane
        written (40 B); tables: per-hour tables (negligible); contraction: 40 B
        of mask words per pixel read, 2 sums per pixel-hour written (8 B: sky
        plus transmitted vegetation, luminance and luminance*cos*omega);
        radiation: 109 B of per-pixel statics and 16 B of state per day, 20 B
        per daytime pixel-hour (3 GVF planes, 2 sums) and 8 B per pixel-hour
        written (Tmrt, UTCI)."""
        return {
            "day_shadow_kernel": pixels * day_hours * 101,
            "day_gvf_kernel": pixels * day_hours * 40,
            "day_tables_kernel": hours * 9680,
            "patch_gemm_kernel": pixels * (40 + 8 * hours),
            "day_radiation_kernel": pixels * (125 + 20 * day_hours + 8 * hours),
        }

    @staticmethod
    def gemm_flops(pixels, hours, patches):
        """Algorithmic FLOPs of the contraction: 2 x pixels x patches x 2 hour
        columns (luminance, luminance x cos x omega) x 2 masks (sky,
        vegetation); the BF16 hi/lo duplication is not counted."""
        return 2 * pixels * patches * (2 * hours) * 2

    STAGES = ("day_shadow_kernel", "day_gvf_kernel", "day_tables_kernel", "patch_gemm_kernel",
              "day_radiation_kernel")

    def profile_day(self, met):
        """Device time of each stage of one day, {stage: ms}, from CUDA events
        recorded on the launching stream between the stages."""
        self.plan(met)
        self.buffers.upload(0, self.hours, self.buffers.kmax)
        sc = self.scene
        base = outputs_struct(self.out, 0)
        ms = (ctypes.c_float * len(self.STAGES))()
        _lib.check(_lib.lib().solweig_day_batched_timed(
            ctypes.byref(sc.struct), device_ptr(self.layout_dev), self.buffers.ptr(), self.hours,
            ctypes.byref(_lib.SolweigState()), ctypes.byref(base), sc.pixels, sc.gvf_host_ptr,
            sc.first_steps, sc.second_steps, device_ptr(self.work), self.work_bytes,
            ctypes.byref(self.config), stream_handle(), ms), "solweig_day_batched_timed")
        self.buffers.mark()
        return dict(zip(self.STAGES, (float(x) for x in ms)))

    WORK_FIELDS = ("quads", "lup_first", "gvf", "nosh", "sums", "wf32", "bw", "tables", "error", "tilemax",
                   "total")

    def work_offsets(self):
        """{field: byte offset} of the work buffer (``solweig_day_batched_layout``)."""
        sc = self.scene
        off = (ctypes.c_int64 * 11)()
        _lib.check(_lib.lib().solweig_day_batched_layout(sc.rows, sc.cols, self.hours,
                                                         int(sc.struct.has_water), off),
                   "solweig_day_batched_layout")
        return dict(zip(self.WORK_FIELDS, (int(x) for x in off)))

    def quads(self):
        """The sweep's per-pixel GVF inputs of the last day as a [H, rows, cols, 4]
        float32 view: shadow, Lup excess, albedo and the ground (1) / sunlit-wall
        (2) bits as an int32 bit pattern (daytime hours only; night hours hold
        stale values)."""
        o = self.work_offsets()
        n = 16 * self.hours * self.scene.pixels
        return self.work[o["quads"]:o["quads"] + n].view(torch.float32).view(self.hours, self.scene.rows,
                                                                                 self.scene.cols, 4)

    def patch_sums(self):
        """The contraction's output of the last day as a [2H, pixels] view: row
        2h + 0 the luminance and 2h + 1 the luminance*cos*omega summed over the
        sky patches plus 0.03 x the same over the vegetation patches."""
        o = self.work_offsets()
        n = 2 * self.hours * self.scene.pixels
        return self.work[o["sums"]:o["sums"] + 4 * n].view(torch.float32).view(2 * self.hours, self.scene.pixels)

    def check_errors(self):
        """Raise DayError if any day run by this object left invalid results."""
        return check_day_errors(self.work, "batched day")

    def error_flag(self):
        """Device error flag of the last day (0 = ok, 1 = a tensor-core wait timed
        out, 2 = a sweep window's TMA wait timed out: that tile walked from the raster,
        3 = a sun ray stayed inside the raster for more than max(rows, cols) + 2 steps)."""
        flag = torch.zeros(1, dtype=torch.int32, device=self.scene.device)
        sc = self.scene
        _lib.check(_lib.lib().solweig_day_batched_error(
            device_ptr(self.work), sc.rows, sc.cols, self.hours, int(sc.struct.has_water),
            device_ptr(flag), stream_handle()), "solweig_day_batched_error")
        return int(flag.item())


class MultiDay:
    """``days`` consecutive days of ``hours`` rows each through ONE captured
    graph: every hour record and sun ray uploaded once, then per day the state
    reset (``src/series.py:425-436``) and the batched day
    (``solweig_day_batched_ex``).  Outputs [days * hours, rows, cols]."""

    def __init__(self, scene, latitude, longitude, site_altitude=3.0, utc=0.0, days=30, hours=24,
                 outputs=("tmrt", "utci"), config=None):
        self.scene = scene
        self.latitude, self.longitude, self.site_altitude, self.utc = latitude, longitude, site_altitude, utc
        self.days, self.hours = days, hours
        dev = scene.device
        self.state = {k: torch.zeros(scene.shape, dtype=torch.float32, device=dev)
                      for k in _lib.STATE_FIELDS}
        self.buffers = HourBuffers(scene, days * hours)
        self.layout_dev = scene.layout.device(dev)
        self.out_names = tuple(outputs)
        self.out = {k: torch.empty((days * hours,) + scene.shape, dtype=torch.float32, device=dev)
                    for k in self.out_names}
        self.work_bytes = int(_lib.lib().solweig_day_batched_work_bytes(scene.rows, scene.cols, hours,
                                                                        int(scene.struct.has_water)))
        self.work = torch.empty(self.work_bytes, dtype=torch.uint8, device=dev)
        clear_day_errors(self.work)
        self.config = config if config is not None else _lib.SolweigDayConfig.default()
        self.graph = None
        self.launches = day_launches(scene, self.config) * days

    def plan(self, met):
        met = np.asarray(met, dtype=np.float64)
        if len(met) != self.days * self.hours:
            raise ValueError(f"expected {self.days * self.hours} forcing rows, got {len(met)}")
        self.buffers.wait_free()
        H = self.hours
        for d in range(self.days):
            plan = plan_day(self.scene, met[d * H:(d + 1) * H], self.latitude, self.longitude,
                            self.site_altitude, self.utc)
            for i, (h, ray, _) in enumerate(plan):
                self.buffers.put(d * H + i, h, ray)

    def _sequence(self):
        sc = self.scene
        L = _lib.lib()
        self.buffers.upload(0, self.days * self.hours, self.buffers.kmax)
        st = _lib.SolweigState()  # zero state at the start of every day
        hsize = self.buffers.hsize
        for d in range(self.days):
            base = outputs_struct(self.out, d * self.hours)
            hours_ptr = ctypes.c_void_p(self.buffers.h_dev.data_ptr() + d * self.hours * hsize)
            _lib.check(L.solweig_day_batched_ex(
                ctypes.byref(sc.struct), device_ptr(self.layout_dev), hours_ptr, self.hours,
                ctypes.byref(st), ctypes.byref(base), sc.pixels, sc.gvf_host_ptr, sc.first_steps,
                sc.second_steps, device_ptr(self.work), self.work_bytes, ctypes.byref(self.config),
                stream_handle()), "solweig_day_batched_ex")

    def capture(self):
        self._sequence()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._sequence()
        self.graph = g

    def replay(self):
        self.graph.replay()
        self.buffers.mark()
        return self.out

    def run(self, met):
        self.plan(met)
        if self.graph is None:
            self.capture()
        return self.replay()

    def check_errors(self):
        """Raise DayError if any day of any replay so far left invalid results."""
        return check_day_errors(self.work, "multi-day batch")


class TileBatch:
    """Independent tiles (own scene, latitude and forcing) for one day each,
    captured as ONE graph; a single work buffer sized for the largest tile is
    reused tile after tile on the stream.  Each tile may carry its own launch
    shapes (from :mod:`tune`)."""

    def __init__(self, scenes, latitudes, longitudes, site_altitude=3.0, utc=0.0, hours=24,
                 outputs=("tmrt", "utci"), configs=None):
        self.scenes = list(scenes)
        n = len(self.scenes)
        self.latitudes = list(latitudes)
        self.longitudes = list(longitudes)
        self.site_altitude, self.utc, self.hours = site_altitude, utc, hours
        dev = self.scenes[0].device
        L = _lib.lib()
        self.work_bytes = max(int(L.solweig_day_batched_work_bytes(s.rows, s.cols, hours,
                                                                   int(s.struct.has_water)))
                              for s in self.scenes)
        self.work = torch.empty(self.work_bytes, dtype=torch.uint8, device=dev)
        clear_day_errors(self.work)
        self.buffers = [HourBuffers(s, hours) for s in self.scenes]
        self.layouts = [s.layout.device(dev) for s in self.scenes]
        self.state = [{k: torch.zeros(s.shape, dtype=torch.float32, device=dev) for k in ("tgmap1", "tgout1")}
                      for s in self.scenes]
        self.out_names = tuple(outputs)
        self.out = [{k: torch.empty((hours,) + s.shape, dtype=torch.float32, device=dev) for k in outputs}
                    for s in self.scenes]
        self.configs = list(configs) if configs is not None else [_lib.SolweigDayConfig.default()] * n
        self.graph = None
        self.launches = sum(day_launches(s_, c) for s_, c in zip(self.scenes, self.configs))

    @property
    def pixels(self):
        return sum(s.pixels for s in self.scenes)

    def plan(self, mets):
        for s, b, met, lat, lon in zip(self.scenes, self.buffers, mets, self.latitudes, self.longitudes):
            met = np.asarray(met, dtype=np.float64)
            if len(met) != self.hours:
                raise ValueError(f"expected {self.hours} forcing rows, got {len(met)}")
            b.wait_free()
            for i, (h, ray, _) in enumerate(plan_day(s, met, lat, lon, self.site_altitude, self.utc)):
                b.put(i, h, ray)

    def _sequence(self):
        L = _lib.lib()
        for s, b, lay, state, out, cfg in zip(self.scenes, self.buffers, self.layouts, self.state, self.out,
                                              self.configs):
            b.upload(0, self.hours, b.kmax)
            st = _lib.SolweigState()  # zero state at the start of the day
            base = outputs_struct(out, 0)
            _lib.check(L.solweig_day_batched_ex(
                ctypes.byref(s.struct), device_ptr(lay), b.ptr(), self.hours, ctypes.byref(st),
                ctypes.byref(base), s.pixels, s.gvf_host_ptr, s.first_steps, s.second_steps,
                device_ptr(self.work), self.work_bytes, ctypes.byref(cfg), stream_handle()),
                "solweig_day_batched_ex")

    def capture(self):
        self._sequence()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._sequence()
        self.graph = g

    def replay(self):
        self.graph.replay()
        for b in self.buffers:
            b.mark()
        return self.out

    def run(self, mets):
        self.plan(mets)
        if self.graph is None:
            self.capture()
        return self.replay()

    def check_errors(self):
        """Raise DayError if any tile-day of any replay so far left invalid results."""
        return check_day_errors(self.work, "tile batch")
