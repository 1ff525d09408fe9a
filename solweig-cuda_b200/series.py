"""Drop-in for the reference's ``src/series.py``: forcing loader and time-series driver.

``load_meteorology`` and ``run_timeseries`` keep the reference's names,
arguments and day grouping (``src/series.py:91-194``).  Differences, by design:

* rasters are read from ``.npy`` files (or passed as arrays); GeoTIFF input
  works only where ``rasterio`` or GDAL is importable;
* outputs are written as ``.npy`` stacks [steps, rows, cols] float32 with a
  JSON sidecar of timestamps instead of DEFLATE GeoTIFFs;
* each day runs in the batched form (:class:`batched.ChosenDay`: all hours
  of the day in a few launches, replayed from captured CUDA graphs) and its
  outputs are copied to pinned host memory on a separate stream while the
  next day computes; a bounded writer thread stores them
  (``src/output.py:11-102``, ``src/runtime.py:79-163``);
* calendar days can be split over ranks (one process per GPU, no exchange);
* ``dtype=float64`` (the reference's radiation precision switch) runs every
  hour through the float64 step (:class:`engine.DayRunner64`) instead.
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

from . import engine, shard
from .batched import BatchedDay, ChosenDay

__all__ = ["DayForcing", "Meteorology", "load_meteorology", "run_timeseries", "load_raster",
           "OutputWriter", "rank_and_world", "Float64Day"]


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


def _write_chunk(folder, names, host, steps, copy_done, crop, meta, valid=None):
    """Writer job of one output chunk: waits for its device-to-host copy, crops
    to the output core and, with an output mask, sets the pixels outside it
    to NaN on the cropped array (``src/output.py:205-216``)."""
    copy_done.synchronize()
    folder.mkdir(parents=True, exist_ok=True)
    r, c = crop
    for name in names:
        arr = np.array(host[name][:steps][:, r, c], dtype=np.float32)
        if valid is not None:
            arr[:, ~valid] = np.nan
        np.save(folder / f"{name}.npy", arr)
    (folder / "timestamps.json").write_text(json.dumps(meta))


class _HostCopy:
    """Device-to-host copy of one day's output planes into page-locked memory
    on a side stream; ``synchronize`` waits for it (a no-op on CPU tensors)."""

    def __init__(self, planes, copy_stream):
        self.host = {}
        self.event = None
        if copy_stream is None:
            for k, v in planes.items():
                self.host[k] = v.detach().cpu().numpy().copy()
            return
        copy_stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(copy_stream):
            for k, v in planes.items():
                h = torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
                h.copy_(v, non_blocking=True)
                self.host[k] = h.numpy()
            self.event = torch.cuda.Event()
            self.event.record(copy_stream)
        # the next day writes the same device buffers: the compute stream waits for the copy
        torch.cuda.current_stream().wait_event(self.event)

    def synchronize(self):
        if self.event is not None:
            self.event.synchronize()


def rank_and_world(rank=None, world_size=None):
    """This process's rank and the number of ranks: the arguments, else an
    initialised ``torch.distributed`` group, else RANK / WORLD_SIZE from the
    environment (as ``torchrun`` sets them), else (0, 1)."""
    if rank is not None or world_size is not None:
        r, w = int(rank or 0), int(world_size or 1)
    else:
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            r, w = dist.get_rank(), dist.get_world_size()
        else:
            r, w = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))
    if w < 1 or not 0 <= r < w:
        raise ValueError(f"rank {r} outside a world of {w}")
    return r, w


def _default_device(rank, world):
    if world > 1:
        return f"cuda:{int(os.environ.get('LOCAL_RANK', rank)) % max(1, torch.cuda.device_count())}"
    return "cuda"


def _make_runner(scene, latitude, longitude, site_altitude, utc, hours, outputs, form):
    """Runner of one day length: the batched form (``ChosenDay``: every hour
    of the day in a few launches, tensor-core patch sums) for days of up to
    64 rows, the per-hour kernels in one captured graph (``BatchedDay``) for
    longer days or ``form="batched"``."""
    if form == "chosen" and hours <= 64:
        return ChosenDay(scene, latitude, longitude, site_altitude, utc, hours=hours, outputs=outputs)
    return BatchedDay(scene, latitude, longitude, site_altitude, utc, hours=hours, outputs=outputs)


class Float64Day:
    """Day runner of the float64 switch (``dtype=float64``, ``run.py:27``):
    every hour through the float64 step (:class:`engine.DayRunner64`), for
    any day length; the requested planes come back as float64 (UTCI float32)."""

    def __init__(self, scene, latitude, longitude, site_altitude, utc, hours, outputs):
        self.runner = engine.DayRunner64(scene, latitude, longitude, site_altitude, utc, hours=hours)
        self.outputs = tuple(outputs)

    def run_day(self, met):
        return self.runner.run_day(met, self.outputs)


def _make_runner64(scene, latitude, longitude, site_altitude, utc, hours, outputs, form):
    return Float64Day(scene, latitude, longitude, site_altitude, utc, hours, outputs)


def _check_dtype(dtype):
    dt = np.dtype(dtype)
    if dt not in (np.float32, np.float64):
        raise NotImplementedError(f"dtype must be float32 or float64 (the reference's choices), not {dt}")
    return dt == np.float64


def run_timeseries(building_dsm_path, tree_path, dem_path, met_file, output_path,
                   longitude, latitude, *, landcover_path=None, utc_offset_hours=None,
                   site_altitude_m=3., wall_method='dsm', building_geometry_path=None,
                   building_height_path=None, minimum_wall_height_m=2., dsm_wall_threshold_m=3.,
                   default_building_height_m=6., level_height_m=3., minimum_building_height_m=2.,
                   save_tmrt=True, save_svf=False, save_kup=False, save_kdown=False,
                   save_lup=False, save_ldown=False, save_shadow=False, dtype=np.float32,
                   no_write=False, output_core=None, output_chunk_steps=24,
                   async_output=True, output_queue_size=2, output_valid_mask=None, progress=False,
                   pixel_size=1.0, device=None, form="chosen", rank=None, world_size=None,
                   scene_factory=None, runner_factory=None, crs=None, geotransform=None):
    """Simulate every day of the forcing on one tile (``src/series.py:91-156``).

    Days run in the batched form (``form="chosen"``, :class:`batched.ChosenDay`)
    unless ``form="batched"``.  With several ranks (``rank``/``world_size``, an
    initialised process group, or RANK/WORLD_SIZE from ``torchrun``) each rank
    runs a contiguous share of the calendar days on its own GPU
    (``LOCAL_RANK``) and writes those days' folders; rank 0 also writes the
    static rasters.  Days are independent (the thermal state resets every
    day), so ranks exchange nothing.  ``dtype=float64`` runs every hour
    through the float64 step (:class:`Float64Day`; ``form`` is then not
    used: the batched forms compute in float32 and BF16).  ``scene_factory`` and
    ``runner_factory`` replace :class:`engine.Scene` and the day runner (for
    tests of the host logic).

    ``wall_method="geometry"`` takes the walls from building footprints
    (``building_geometry_path``: GeoJSON in EPSG:4326; ``building_height_path``:
    the GHSL height raster) as ``src/series.py:218-233`` does; the ``.npy``
    rasters carry no georeferencing, so ``crs`` (the rasters' coordinate
    system) and ``geotransform`` (GDAL order) must then be given.

    Returns ``{"static": {...}, "days": {date: {variable: [paths]}}}`` with the
    days this rank ran.
    """
    method = str(wall_method).strip().lower()
    if method not in ("dsm", "geometry"):
        raise ValueError(f"wall_method must be 'dsm' or 'geometry', not {wall_method!r}")
    if method == "geometry" and not (building_geometry_path and building_height_path):
        raise ValueError("wall_method='geometry' requires building_geometry_path and building_height_path")
    if method == "geometry" and (crs is None or geotransform is None):
        raise ValueError("wall_method='geometry' needs the rasters' crs and geotransform (GDAL order)")
    f64 = _check_dtype(dtype)
    if form not in ("chosen", "batched"):
        raise ValueError(f"form must be 'chosen' or 'batched', not {form!r}")
    rank, world = rank_and_world(rank, world_size)
    forcing = load_meteorology(met_file)
    days = shard.split(forcing.days, rank, world)
    output = Path(output_path).resolve()
    dsm = load_raster(building_dsm_path)
    trees = load_raster(tree_path)
    dem = load_raster(dem_path)
    lc = load_raster(landcover_path) if landcover_path is not None else None
    utc = float(longitude) / 15.0 if utc_offset_hours is None else float(utc_offset_hours)
    stamp = lambda msg: print(f"[{datetime.now():%H:%M:%S}] {msg}", flush=True) if progress else None  # noqa: E731
    if output_core is None:
        crop = (slice(None), slice(None))
        cropped = dsm.shape
    else:
        row, col, nr, nc = (int(x) for x in output_core)
        crop = (slice(row, row + nr), slice(col, col + nc))
        cropped = (nr, nc)
    valid = None
    if output_valid_mask is not None:
        valid = np.array(output_valid_mask, dtype=bool, copy=True)
        if valid.shape != tuple(cropped):
            raise ValueError(f"output_valid_mask has shape {valid.shape}; the cropped output is {tuple(cropped)}")
        valid.setflags(write=False)
    stamp("Spatial preparation started")
    if device is None:
        device = _default_device(rank, world)
    make_scene = scene_factory or engine.Scene
    wall_args = {}
    if method == "geometry":
        from . import walls as _walls
        buildings = _walls.load_buildings(building_geometry_path, crs, default_height_m=default_building_height_m,
                                          level_height_m=level_height_m,
                                          minimum_height_m=minimum_building_height_m)
        ghsl = load_raster(building_height_path).astype(np.float32)
        w, a = _walls.calculate_geometry_walls(buildings, ghsl, dsm.shape, _walls.affine_from_gdal(geotransform),
                                               minimum_wall_height_m, device=device)
        wall_args = dict(walls=w.astype(np.float64), aspect=a.astype(np.float64))
    scene = make_scene(dsm, trees, dem, pixel_size, landcover=lc, wall_threshold=dsm_wall_threshold_m,
                       device=device, keep_planes=save_svf, **wall_args)
    files = {"static": {}, "days": {}}
    writer = OutputWriter(enabled=bool(async_output and not no_write), max_inflight=output_queue_size)
    if not no_write and rank == 0:
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
    make = runner_factory or (_make_runner64 if f64 else _make_runner)
    runners = {}
    on_gpu = torch.device(scene.device).type == "cuda"
    copy_stream = torch.cuda.Stream(device=scene.device) if on_gpu and not no_write else None
    stamp("Time-series simulation started")
    try:
        for day in days:
            writer.check()
            nh = len(day.values)
            if nh not in runners:
                runners[nh] = make(scene, float(latitude), float(longitude), float(site_altitude_m), utc, nh,
                                   tuple(abi[v] for v in variables), form)
            res = runners[nh].run_day(day.values)
            if no_write:
                continue
            copy = _HostCopy({v: res[abi[v]] for v in variables}, copy_stream)
            folder = output / day.date
            chunks = []
            step = max(1, int(output_chunk_steps))
            for k, start in enumerate(range(0, nh, step)):
                stop = min(nh, start + step)
                sub = folder if nh <= step else folder / f"chunk_{k + 1:04d}"
                meta = {"timestamps": [t.isoformat() for t in day.timestamps[start:stop]],
                        "utc_offset_hours": utc}
                view = {v: copy.host[v][start:stop] for v in variables}
                writer.submit(lambda sub=sub, view=view, n=stop - start, meta=meta:
                              _write_chunk(sub, variables, view, n, copy, crop, meta, valid))
                chunks.append(str(sub))
            files["days"][day.date] = {v: [str(Path(c) / f"{v}.npy") for c in chunks] for v in variables}
            stamp(f"Daily calculation completed: {day.date}")
        writer.finish()
        if on_gpu:
            torch.cuda.synchronize(scene.device)
        for runner in runners.values():  # device error flags of every day run
            if hasattr(runner, "check_errors"):
                runner.check_errors()
        return files
    except BaseException:
        writer.abort()
        raise


def run_tiles(tiles, met_file, output_path, longitude, latitude, *, utc_offset_hours=None,
              site_altitude_m=3., dsm_wall_threshold_m=3., save_tmrt=True, save_kup=False,
              save_kdown=False, save_lup=False, save_ldown=False, save_shadow=False, dtype=np.float32,
              no_write=False, output_chunk_steps=24, async_output=True, output_queue_size=2,
              progress=False, pixel_size=1.0, device=None, rank=None, world_size=None,
              group_pixels=48_000_000):
    """Every tile of a tiled case, day by day, with all tiles of a group in ONE
    captured graph per day (:class:`batched.TileBatch`); the reference runs
    ``run_timeseries`` once per tile (``run.py:62-68``, ``:113-129``).

    ``tiles``: sequence of dicts with ``tile_id``, ``dsm``, ``trees``, ``dem``,
    optional ``landcover`` (2-D arrays of the tile's input window) and
    ``output_core`` (row, col, rows, cols of the core inside the window).
    Tiles are grouped so that a group holds at most ``group_pixels`` pixels;
    each group's scenes stay on the device while its days run.  With several
    ranks each takes a contiguous share of the tiles.  Outputs go to
    ``output_path/<tile_id>/<date>/<VAR>.npy`` (cropped to the core) and
    ``output_path/<tile_id>/static``.  Days longer than 64 rows run tile by
    tile in the per-hour graph form.  ``dtype=float64`` runs every tile-day
    through the float64 step (:class:`Float64Day`), tile by tile.

    Returns ``{tile_id: {"static": {...}, "days": {date: {variable: [paths]}}}}``.
    """
    from .batched import TileBatch
    f64 = _check_dtype(dtype)
    rank, world = rank_and_world(rank, world_size)
    forcing = load_meteorology(met_file)
    mine = shard.split(list(tiles), rank, world)
    output = Path(output_path).resolve()
    utc = float(longitude) / 15.0 if utc_offset_hours is None else float(utc_offset_hours)
    stamp = lambda msg: print(f"[{datetime.now():%H:%M:%S}] {msg}", flush=True) if progress else None  # noqa: E731
    if device is None:
        device = _default_device(rank, world)
    variables = ["UTCI"] + [n for n, on in (("TMRT", save_tmrt), ("Kup", save_kup), ("Kdown", save_kdown),
                                            ("Lup", save_lup), ("Ldown", save_ldown),
                                            ("Shadow", save_shadow)) if on]
    abi = {"UTCI": "utci", "TMRT": "tmrt", "Kup": "kup", "Kdown": "kdown", "Lup": "lup",
           "Ldown": "ldown", "Shadow": "shadow"}
    outs = tuple(abi[v] for v in variables)
    groups, cur, size = [], [], 0
    for t in mine:
        px = int(np.prod(np.shape(t["dsm"])))
        if cur and size + px > group_pixels:
            groups.append(cur)
            cur, size = [], 0
        cur.append(t)
        size += px
    if cur:
        groups.append(cur)
    files = {}
    writer = OutputWriter(enabled=bool(async_output and not no_write), max_inflight=output_queue_size)
    copy_stream = None if no_write else torch.cuda.Stream(device=torch.device(device))
    try:
        for group in groups:
            scenes = []
            for t in group:
                stamp(f"Tile {t['tile_id']}: spatial preparation")
                sc = engine.Scene(t["dsm"], t["trees"], t["dem"], pixel_size, landcover=t.get("landcover"),
                                  wall_threshold=dsm_wall_threshold_m, device=device)
                scenes.append(sc)
                rec = files.setdefault(t["tile_id"], {"static": {}, "days": {}})
                if not no_write:
                    static = output / t["tile_id"] / "static"
                    static.mkdir(parents=True, exist_ok=True)
                    np.save(static / "walls.npy", sc.walls_host.astype(np.float32))
                    np.save(static / "aspect.npy", sc.aspect_host.astype(np.float32))
                    rec["static"] = {"walls": str(static / "walls.npy"), "aspect": str(static / "aspect.npy")}
            batches, runners64 = {}, {}
            for day in forcing.days:
                writer.check()
                nh = len(day.values)
                if f64:
                    results = []
                    for i, sc in enumerate(scenes):
                        if (i, nh) not in runners64:
                            runners64[(i, nh)] = Float64Day(sc, float(latitude), float(longitude),
                                                            float(site_altitude_m), utc, nh, outs)
                        results.append(runners64[(i, nh)].run_day(day.values))
                elif nh <= 64:
                    if nh not in batches:
                        batches[nh] = TileBatch(scenes, [float(latitude)] * len(scenes),
                                                [float(longitude)] * len(scenes), float(site_altitude_m), utc,
                                                hours=nh, outputs=outs)
                    results = batches[nh].run([day.values] * len(scenes))
                else:
                    results = [BatchedDay(sc, float(latitude), float(longitude), float(site_altitude_m), utc,
                                          hours=nh, outputs=outs).run_day(day.values) for sc in scenes]
                if no_write:
                    continue
                for t, res in zip(group, results):
                    copy = _HostCopy({v: res[abi[v]] for v in variables}, copy_stream)
                    row, col, nr, nc = (int(x) for x in t["output_core"])
                    crop = (slice(row, row + nr), slice(col, col + nc))
                    folder = output / t["tile_id"] / day.date
                    chunks = []
                    step = max(1, int(output_chunk_steps))
                    for k, start in enumerate(range(0, nh, step)):
                        stop = min(nh, start + step)
                        sub = folder if nh <= step else folder / f"chunk_{k + 1:04d}"
                        meta = {"timestamps": [s.isoformat() for s in day.timestamps[start:stop]],
                                "utc_offset_hours": utc}
                        view = {v: copy.host[v][start:stop] for v in variables}
                        writer.submit(lambda sub=sub, view=view, n=stop - start, meta=meta, crop=crop, copy=copy:
                                      _write_chunk(sub, variables, view, n, copy, crop, meta))
                        chunks.append(str(sub))
                    files[t["tile_id"]]["days"][day.date] = {v: [str(Path(c) / f"{v}.npy") for c in chunks]
                                                             for v in variables}
                stamp(f"Daily calculation completed: {day.date} ({len(group)} tiles)")
            torch.cuda.synchronize(torch.device(device))
            for batch in batches.values():  # device error flags of every tile-day
                batch.check_errors()
            del batches, runners64, scenes
        writer.finish()
        return files
    except BaseException:
        writer.abort()
        raise
