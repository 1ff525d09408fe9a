"""Validation of the forcing table and of case options before a run.

Restates the rules of the reference's ``scripts/input_check.py``:
``check_weather`` (``:28-76``), ``validate_preparation_options`` (``:79-129``),
``check_options`` / ``check_output_window`` (``:132-196``) and the option part of
``check_case`` (``:199-226``).  Raster checks that need GDAL (projection,
geotransform) are not restated; :func:`check_arrays` checks in-memory rasters
(shape, finiteness) instead.
"""
from __future__ import annotations

import calendar
import json
import math
import operator
import os
from datetime import date
from pathlib import Path

import numpy as np

from .series import Meteorology, _read_values, load_meteorology

__all__ = ["PATH_KEYS", "PREPARATION_KEYS", "check_weather", "validate_preparation_options",
           "check_options", "check_output_window", "check_case", "check_arrays"]

PATH_KEYS = frozenset({"building_dsm_path", "tree_path", "dem_path", "met_file", "building_geometry_path",
                       "building_height_path", "landcover_path", "output_path"})
PREPARATION_KEYS = frozenset({"case_name", "case_type", "case_size_m", "core_area_m", "buffer_area_m",
                              "resolution_m", "start_date", "end_date"})
_REQUIRED = frozenset({"building_dsm_path", "tree_path", "dem_path", "met_file", "longitude", "latitude"})
_OPTIONAL = frozenset({"minimum_wall_height_m", "dsm_wall_threshold_m", "default_building_height_m",
                       "level_height_m", "minimum_building_height_m", "save_tmrt", "save_svf", "save_kup",
                       "save_kdown", "save_lup", "save_ldown", "save_shadow", "wall_method",
                       "utc_offset_hours", "site_altitude_m", "output_core", "output_chunk_steps",
                       "async_output", "output_queue_size",
                       # georeferencing of .npy rasters for wall_method=geometry (a GeoTIFF
                       # carries them; these keys have no counterpart in the reference)
                       "crs", "geotransform"})
_SAVE_FLAGS = ("save_tmrt", "save_svf", "save_kup", "save_kdown", "save_lup", "save_ldown", "save_shadow")
_POSITIVE_LENGTHS = ("minimum_wall_height_m", "dsm_wall_threshold_m", "default_building_height_m",
                     "level_height_m", "minimum_building_height_m")
# forcing column, lower bound, upper bound, name (UMEP 24-column table)
_FORCING_RANGES = ((9, 0.0, math.inf, "wind"), (10, 0.0, 100.0, "relative humidity"),
                   (11, -100.0, 100.0, "air temperature"), (12, 0.001, math.inf, "pressure"),
                   (14, 0.0, math.inf, "global shortwave"))


def _is_bool(x):
    return isinstance(x, (bool, np.bool_))


def _is_real(x):
    return not _is_bool(x) and isinstance(x, (int, float, np.number))


def _forcing_paths(source):
    if isinstance(source, (str, os.PathLike)):
        paths = [source]
    elif isinstance(source, (list, tuple)) and source:
        if not all(isinstance(p, (str, os.PathLike)) for p in source):
            raise TypeError("forcing file lists must contain only paths; use an ndarray for numeric data")
        paths = list(source)
    else:
        raise TypeError("forcing must be a path, ndarray, nonempty ordered path list, or Meteorology")
    resolved = [Path(p).expanduser().resolve() for p in paths]
    if len(set(resolved)) != len(resolved):
        raise ValueError("forcing file list contains a duplicate path")
    return resolved


def check_weather(source):
    """Validate a UMEP forcing table (path, ordered path list, array or
    :class:`series.Meteorology`); returns the grouped :class:`Meteorology`."""
    if isinstance(source, Meteorology):
        source = source.values
    if not isinstance(source, np.ndarray):
        source = _forcing_paths(source)
    values = _read_values(source)
    if values.ndim != 2 or values.shape[0] == 0 or values.shape[1] < 23:
        raise ValueError("forcing requires at least one row and 23 SOLWEIG columns in a two-dimensional array")
    if not np.isfinite(values).all():
        raise ValueError("forcing contains non-finite values")
    stamp = values[:, :4]
    if not np.array_equal(stamp, np.floor(stamp)):
        raise ValueError("forcing year, day-of-year, hour and minute must be integers")
    limits = ((0, 1, 9999, "forcing year must be between 1 and 9999"),
              (1, 1, 366, "forcing day-of-year must be valid for its calendar year"),
              (2, 0, 23, "forcing hour must be between 0 and 23"),
              (3, 0, 59, "forcing minute must be between 0 and 59"))
    for col, lo, hi, message in limits:
        if np.any((stamp[:, col] < lo) | (stamp[:, col] > hi)):
            raise ValueError(message)
    for year, doy in stamp[:, :2].astype(np.int64):
        if doy > 365 + int(calendar.isleap(int(year))):
            raise ValueError(f"forcing day-of-year {doy} is invalid for calendar year {year}")
    for col, lo, hi, name in _FORCING_RANGES:
        if np.any((values[:, col] < lo) | (values[:, col] > hi)):
            raise ValueError(f"forcing contains missing or invalid {name} values")
    forcing = load_meteorology(values)
    steps = [(b - a).total_seconds() / 60 for a, b in zip(forcing.timestamps, forcing.timestamps[1:])]
    if any(s <= 0 for s in steps):
        raise ValueError("forcing timestamps must be strictly increasing with no duplicates")
    if steps and any(s != steps[0] for s in steps[1:]):
        raise ValueError("forcing timestamps must have one constant timestep; missing samples or days are "
                         "not supported")
    return forcing


def _finite_measure(value):
    try:
        return _is_real(value) and math.isfinite(value)
    except OverflowError:
        return False


def validate_preparation_options(raw):
    """The case-preparation keys of ``case.json``; returns them with defaults."""
    if not isinstance(raw, dict):
        raise ValueError("case.json must contain a JSON object")
    opts = {k: raw[k] for k in PREPARATION_KEYS & raw.keys()}
    kind = opts.setdefault("case_type", "local")
    if kind not in ("local", "open_data"):
        raise ValueError("case_type must be local or open_data")
    if "case_name" in opts and (not isinstance(opts["case_name"], str) or not opts["case_name"].strip()):
        raise ValueError("case_name must be a nonempty string")
    if kind == "open_data" and "case_size_m" not in opts:
        raise ValueError("case_type=open_data requires case_size_m")
    opts.setdefault("resolution_m", 1)
    for key in ("case_size_m", "core_area_m", "buffer_area_m", "resolution_m"):
        if key not in opts:
            continue
        value = opts[key]
        negative_ok = key == "buffer_area_m"
        if not _finite_measure(value) or (value < 0 if negative_ok else value <= 0):
            raise ValueError(f"{key} must be a {'nonnegative' if negative_ok else 'positive'} finite number")
    if ("core_area_m" in opts) != ("buffer_area_m" in opts):
        raise ValueError("core_area_m and buffer_area_m must be supplied together")
    for key in ("core_area_m", "buffer_area_m"):
        if key in opts:
            px = opts[key] / opts["resolution_m"]
            if not math.isfinite(px) or abs(px - round(px)) > 1e-9:
                raise ValueError(f"{key} must be a whole number of resolution_m pixels")
    if ("start_date" in opts) != ("end_date" in opts):
        raise ValueError("start_date and end_date must be supplied together")
    if "start_date" in opts:
        days = []
        for key in ("start_date", "end_date"):
            value = opts[key]
            try:
                parsed = date.fromisoformat(value) if isinstance(value, str) else None
            except ValueError:
                parsed = None
            if parsed is None or parsed.isoformat() != value:
                raise ValueError(f"{key} must be a calendar date in YYYY-MM-DD format")
            days.append(parsed)
        if days[1] < days[0]:
            raise ValueError("end_date must not precede start_date")
        utc = raw.get("utc_offset_hours")
        if kind == "open_data" and (_is_bool(utc) or utc != 0):
            raise ValueError("Open-data meteorology requires utc_offset_hours=0")
    return opts


def check_output_window(core, shape, mask=None):
    """``output_core`` = [row, col, rows, cols] inside ``shape`` (if given) and an
    optional boolean mask of the cropped shape."""
    if core is not None:
        ok = (isinstance(core, (list, tuple)) and len(core) == 4
              and all(not _is_bool(x) and isinstance(x, (int, np.integer)) for x in core)
              and min(core[:2]) >= 0 and min(core[2:]) >= 1)
        if not ok:
            raise ValueError("output_core must be [row, col, rows, cols] with nonnegative offsets and "
                             "positive dimensions")
        row, col, rows, cols = core
        if shape is not None and (row + rows > shape[0] or col + cols > shape[1]):
            raise ValueError("output_core must lie inside the computational raster")
        shape = (rows, cols)
    if mask is not None:
        m = np.asarray(mask)
        if m.dtype != np.dtype(bool):
            raise TypeError("output_valid_mask must have boolean dtype")
        if m.ndim != 2 or m.shape != tuple(shape):
            raise ValueError("output_valid_mask must be two-dimensional and match the cropped output shape")


def check_options(case, *, dtype=np.float32, output_path=None, no_write=False):
    """Run options of a case (dtype, output chunking, location, wall method ...)."""
    if np.dtype(dtype) not in (np.dtype(np.float32), np.dtype(np.float64)):
        raise ValueError("dtype must be float32 or float64")
    for name, default in (("output_chunk_steps", 24), ("output_queue_size", 2)):
        value = case.get(name, default)
        if _is_bool(value):
            raise ValueError(f"{name} must be a positive integer")
        try:
            value = operator.index(value)
        except TypeError:
            raise ValueError(f"{name} must be a positive integer") from None
        if value < 1:
            raise ValueError(f"{name} must be a positive integer")
    if not _is_bool(case.get("async_output", True)):
        raise ValueError("async_output must be boolean")
    for name, lo, hi in (("longitude", -180, 180), ("latitude", -90, 90), ("utc_offset_hours", -24, 24)):
        value = case.get(name)
        if name in case and value is None and name != "utc_offset_hours":
            raise ValueError(f"{name} must be a finite number between {lo} and {hi}")
        if value is not None and (not _is_real(value) or not math.isfinite(value) or not lo <= value <= hi):
            raise ValueError(f"{name} must be a finite number between {lo} and {hi}")
    alt = case.get("site_altitude_m", 3.0)
    if not _is_real(alt) or not math.isfinite(alt):
        raise ValueError("site_altitude_m must be finite")
    for name in _POSITIVE_LENGTHS:
        value = case.get(name, 1.0)
        if not _is_real(value) or not math.isfinite(value) or value <= 0:
            raise ValueError(f"{name} must be a positive finite number")
    for name in _SAVE_FLAGS:
        if name in case and not _is_bool(case[name]):
            raise ValueError(f"{name} must be true or false")
    method = case.get("wall_method", "dsm")
    if method not in ("dsm", "geometry"):
        raise ValueError("wall_method must be dsm or geometry")
    if method == "geometry" and not all(case.get(k) for k in ("building_geometry_path", "building_height_path")):
        raise ValueError("wall_method=geometry requires building_geometry_path and building_height_path")
    # georeferencing of .npy rasters (no counterpart in the reference: a GeoTIFF carries it)
    gt = case.get("geotransform")
    if gt is not None:
        if (not isinstance(gt, (list, tuple)) or len(gt) != 6
                or not all(_is_real(v) and math.isfinite(v) for v in gt)):
            raise ValueError("geotransform must be six finite numbers (GDAL order)")
        if gt[1] * gt[5] - gt[2] * gt[4] == 0:
            raise ValueError("geotransform must be invertible")
    if case.get("crs") is not None:
        from . import crs as _crs
        try:
            _crs.project_lonlat([0.0], [0.0], case["crs"])
        except NotImplementedError as exc:
            raise ValueError(f"crs: {exc}") from None
    check_output_window(case.get("output_core"), None)
    if output_path is not None and not no_write:
        out = Path(output_path).resolve()
        if out.exists() and (not out.is_dir() or any(out.iterdir())):
            raise FileExistsError(f"Output must be a new or empty directory: {out}")


def check_case(path):
    """Read and check ``case.json``; returns (case options with resolved paths,
    preparation settings)."""
    path = Path(path).resolve()
    raw = json.loads(path.read_text(encoding="utf-8-sig"))
    settings = validate_preparation_options(raw)
    case = {k: v for k, v in raw.items() if k not in PREPARATION_KEYS}
    missing = _REQUIRED - case.keys()
    if missing:
        raise ValueError("Missing case options: " + ", ".join(sorted(missing)))
    unknown = case.keys() - (PATH_KEYS | _REQUIRED | _OPTIONAL)
    if unknown:
        raise ValueError("Unknown case options: " + ", ".join(sorted(unknown)))
    for key in PATH_KEYS & case.keys():
        value = case[key]
        if value is None and key not in _REQUIRED and key != "output_path":
            continue
        entries = value if key == "met_file" and isinstance(value, list) else [value]
        if not entries or any(not isinstance(e, str) or not e.strip() for e in entries):
            raise ValueError(f"{key} must be a nonempty path" + (" or ordered path list" if key == "met_file" else ""))
        resolved = [str((path.parent / Path(e).expanduser()).resolve()) for e in entries]
        case[key] = resolved if isinstance(value, list) else resolved[0]
    case.setdefault("async_output", True)
    case.setdefault("output_queue_size", 2)
    case.setdefault("output_chunk_steps", 24)
    check_options(case)
    return case, settings


def check_arrays(dsm, trees, dem, landcover=None):
    """In-memory rasters: two-dimensional, one shape, finite."""
    arrays = {"building DSM": dsm, "trees": trees, "DEM": dem}
    if landcover is not None:
        arrays["land cover"] = landcover
    shape = None
    for name, a in arrays.items():
        a = np.asarray(a)
        if a.ndim != 2:
            raise ValueError(f"{name} must be two-dimensional")
        if shape is not None and a.shape != shape:
            raise ValueError(f"{name} is not aligned with the building DSM")
        if not np.isfinite(a).all():
            raise ValueError(f"{name} contains non-finite values")
        shape = a.shape
    return shape
