"""Drop-in for the reference's ``src/series.py``: forcing loader and time-series driver.

``load_meteorology`` and ``run_timeseries`` keep the reference's names,
arguments and day grouping (``src/series.py:91-194``).  Differences, by design:

* rasters are read from ``.npy`` files (or passed as arrays); GeoTIFF input
  works only where ``rasterio`` or GDAL is importable;
* outputs are written as ``.npy`` stacks [steps, rows, cols] float32 with a
  JSON sidecar of timestamps instead of DEFLATE GeoTIFFs;
* each day runs as one captured CUDA graph (:class:`batched.BatchedDay`) and
  its outputs are copied to pinned host memory on a separate stream while the
  next day computes; a bounded writer thread stores them
  (``src/output.py:11-102``, ``src/runtime.py:79-163``).
"""
from __future__ import annotations

import json
import os
import queue
import threading
from dataclasses import dataclass
from datetime import datetime, timedelta
from pathlib import Path

import numpy as np
import torch

from . import engine
from .batched import BatchedDay

__all__ = ["DayForcing", "Meteorology", "load_meteorology", "run_timeseries", "load_raster",
           "OutputWriter"]


@dataclass(frozen=True)
class DayForcing:
    date: str
    values: np.ndarray
    timestamps: tuple


@dataclass(frozen=True)
class Meteorology:
    values: np.ndarray
    timestamps: tuple
    days: tuple
    timestep_minutes: float


def _read_values(source):
    if isinstance(source, np.ndarray):
        values = np.array(source, dtype=np.float64, order="C", copy=True)
        return values.reshape(1, -1) if values.ndim == 1 else values
    paths = [Path(source)] if isinstance(source, (str, os.PathLike)) else [Path(p) for p in source]
    arrays = [np.loadtxt(p.expanduser().resolve(), skiprows=1, ndmin=2, dtype=np.float64,
                         encoding="utf-8-sig") for p in paths]
    return np.ascontiguousarray(arrays[0] if len(arrays) == 1 else np.concatenate(arrays), dtype=np.float64)


def load_meteorology(source) -> Meteorology:
    """UMEP forcing table(s) grouped into calendar days (``src/series.py:175-194``)."""
    if isinstance(source, Meteorology):
        return source
    values = _read_values(source)
    stamps = []
    for year, doy, hour, minute in values[:, :4].astype(np.int64):
        stamps.append(datetime(int(year), 1, 1) + timedelta(days=int(doy) - 1, hours=int(hour),
                                                            minutes=int(minute)))
    timestamps = tuple(stamps)
    timestep = (stamps[1] - stamps[0]).total_seconds() / 60 if len(stamps) > 1 else 0.0
    values.setflags(write=False)
    groups = []
    start = 0
    for stop in range(1, len(stamps) + 1):
        if stop == len(stamps) or stamps[stop].date() != stamps[start].date():
            groups.append(DayForcing(stamps[start].date().isoformat(), values[start:stop],
                                     timestamps[start:stop]))
            start = stop
    return Meteorology(values, timestamps, tuple(groups), timestep)


def load_raster(path):
    """A 2-D float64 raster from ``.npy`` (or GeoTIFF with rasterio / GDAL installed)."""
    if isinstance(path, np.ndarray):
        return np.asarray(path, dtype=np.float64)
    p = Path(path)
    if p.suffix.lower() == ".npy":
        return np.load(p).astype(np.float64)
    try:
        import rasterio
        with rasterio.open(p) as src:
            return src.read(1).astype(np.float64)
    except ImportError:
        pass
    try:
        from osgeo import gdal
        ds = gdal.Open(os.fspath(p))
        return ds.GetRasterBand(1).ReadAsArray().astype(np.float64)
    except ImportError as exc:
        raise RuntimeError(f"cannot read {p}: only .npy rasters are supported without "
                           "rasterio/GDAL") from exc


class OutputWriter:
    """Bounded background writer: at most ``max_inflight`` chunks queued; a
    worker failure is re-raised by the next ``check``/``submit``/``finish``."""

    def __init__(self, enabled=True, max_inflight=2):
        self.enabled = enabled
        self._q = queue.Queue(maxsize=max(1, int(max_inflight)))
        self._error = None
        self._thread = None
        if enabled:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()

    def _run(self):
        while True:
            job = self._q.get()
            if job is None:
                return
            if self._error is not None:
                continue
            try:
                job()
            except BaseException as exc:  # noqa: BLE001 - surfaced through check()
                self._error = exc

    def check(self):
        if self._error is not None:
            err, self._error = self._error, None
            raise RuntimeError("output writer failed") from err

    def submit(self, job):
        self.check()
        if self.enabled:
            self._q.put(job)
        else:
            job()

    def finish(self):
        if self._thread is not None:
            self._q.put(None)
            self._thread.join()
            self._thread = None
        self.check()

    def abort(self):
        if self._thread is not None:
            while True:
                try:
                    self._q.get_nowait()
                except queue.Empty:
                    break
            self._q.put(None)
            self._thread.join(timeout=30)
            self._thread = None


def _write_chunk(folder, names, host, steps, copy_done, crop, meta):
    copy_done.synchronize()
    folder.mkdir(parents=True, exist_ok=True)
    r, c = crop
    for name in names:
        arr = host[name][:steps][:, r, c]
        np.save(folder / f"{name}.npy", np.ascontiguousarray(arr))
    (folder / "timestamps.json").write_text(json.dumps(meta))


def run_timeseries(building_dsm_path, tree_path, dem_path, met_file, output_path,
                   longitude, latitude, *, landcover_path=None, utc_offset_hours=None,
                   site_altitude_m=3., wall_method='dsm', building_geometry_path=None,
                   building_height_path=None, minimum_wall_height_m=2., dsm_wall_threshold_m=3.,
                   default_building_height_m=6., level_height_m=3., minimum_building_height_m=2.,
                   save_tmrt=True, save_svf=False, save_kup=False, save_kdown=False,
                   save_lup=False, save_ldown=False, save_shadow=False, dtype=np.float32,
                   no_write=False, output_core=None, output_chunk_steps=24,
                   async_output=True, output_queue_size=2, output_valid_mask=None, progress=False,
                   pixel_size=1.0, device="cuda"):
    """Simulate every day of the forcing on one tile (``src/series.py:91-156``).

    Returns ``{"static": {...}, "days": {date: {variable: [paths]}}}``.
    """
    if str(wall_method).strip().lower() != "dsm":
        raise NotImplementedError("only wall_method='dsm' is supported")
    forcing = load_meteorology(met_file)
    output = Path(output_path).resolve()
    dsm = load_raster(building_dsm_path)
    trees = load_raster(tree_path)
    dem = load_raster(dem_path)
    lc = load_raster(landcover_path) if landcover_path is not None else None
    utc = float(longitude) / 15.0 if utc_offset_hours is None else float(utc_offset_hours)
    stamp = lambda msg: print(f"[{datetime.now():%H:%M:%S}] {msg}", flush=True) if progress else None  # noqa: E731
    stamp("Spatial preparation started")
    scene = engine.Scene(dsm, trees, dem, pixel_size, landcover=lc, wall_threshold=dsm_wall_threshold_m,
                         device=device, keep_planes=save_svf)
    files = {"static": {}, "days": {}}
    writer = OutputWriter(enabled=bool(async_output and not no_write), max_inflight=output_queue_size)
    if output_core is None:
        crop = (slice(None), slice(None))
    else:
        row, col, nr, nc = output_core
        crop = (slice(row, row + nr), slice(col, col + nc))
    if not no_write:
        static = output / "static"
        static.mkdir(parents=True, exist_ok=True)
        np.save(static / "walls.npy", scene.walls_host.astype(np.float32))
        np.save(static / "aspect.npy", scene.aspect_host.astype(np.float32))
        files["static"] = {"walls": str(static / "walls.npy"), "aspect": str(static / "aspect.npy")}
        if save_svf:
            total = scene.svf32[0] - (1.0 - scene.svf32[5]) * (1.0 - 0.03)
            np.save(static / "SVF.npy", total.cpu().numpy().astype(np.float32))
            files["static"]["SVF"] = str(static / "SVF.npy")
    variables = ["UTCI"] + [n for n, on in (("TMRT", save_tmrt), ("Kup", save_kup), ("Kdown", save_kdown),
                                            ("Lup", save_lup), ("Ldown", save_ldown),
                                            ("Shadow", save_shadow)) if on]
    abi = {"UTCI": "utci", "TMRT": "tmrt", "Kup": "kup", "Kdown": "kdown", "Lup": "lup",
           "Ldown": "ldown", "Shadow": "shadow"}
    runners = {}
    copy_stream = torch.cuda.Stream(device=scene.device)
    stamp("Time-series simulation started")
    pending = []
    try:
        for day in forcing.days:
            writer.check()
            nh = len(day.values)
            if nh not in runners:
                runners[nh] = BatchedDay(scene, float(latitude), float(longitude), float(site_altitude_m),
                                         utc, hours=nh, outputs=tuple(abi[v] for v in variables))
            res = runners[nh].run_day(day.values)
            if no_write:
                continue
            done = torch.cuda.Event()
            host = {}
            copy_stream.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(copy_stream):
                for v in variables:
                    h = torch.empty(res[abi[v]].shape, dtype=torch.float32, pin_memory=True)
                    h.copy_(res[abi[v]], non_blocking=True)
                    host[v] = h.numpy()
                done.record(copy_stream)
            # the next day's graph writes the same device buffers: wait for the copy
            torch.cuda.current_stream().wait_event(done)
            if output_valid_mask is not None:
                mask = np.asarray(output_valid_mask, dtype=bool)
            else:
                mask = None
            folder = output / day.date
            chunks = []
            step = max(1, int(output_chunk_steps))
            for k, start in enumerate(range(0, nh, step)):
                stop = min(nh, start + step)
                sub = folder if nh <= step else folder / f"chunk_{k + 1:04d}"
                meta = {"timestamps": [t.isoformat() for t in day.timestamps[start:stop]],
                        "utc_offset_hours": utc}
                view = {v: host[v][start:stop] for v in variables}
                if mask is not None:
                    for v in variables:
                        view[v] = np.where(mask[None], view[v], np.nan)
                writer.submit(lambda sub=sub, view=view, n=stop - start, meta=meta:
                              _write_chunk(sub, variables, view, n, done, crop, meta))
                chunks.append(str(sub))
            files["days"][day.date] = {v: [str(Path(c) / f"{v}.npy") for c in chunks] for v in variables}
            pending.append(done)
            stamp(f"Daily calculation completed: {day.date}")
        writer.finish()
        torch.cuda.synchronize()
        return files
    except BaseException:
        writer.abort()
        raise
