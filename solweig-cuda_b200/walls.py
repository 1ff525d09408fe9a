"""Drop-in for the DSM wall method of the reference's ``src/walls.py``.

``calculate_dsm_walls`` keeps the reference's signature and returns host
float64 arrays ``(walls, aspect)`` like ``src/walls.py:132-142``: wall height
from the 4-neighbour maximum and the wall aspect from 180 rotated line
templates, both scored on the device; the gradient fallback for walls no
template resolves runs on the host for the few pixels concerned.

The geometry wall method (``src/walls.py:145-332``) keeps its names too:
``building_height`` (the reference's height/level rules for GeoJSON
properties), ``load_buildings`` (GeoJSON footprints projected from EPSG:4326
into the raster's system, :mod:`crs` standing in for PROJ), ``wall_segments``
(every polygon edge, rings oriented as shapely's ``orient(sign=1)``, with its
outward aspect) and ``calculate_geometry_walls`` (the edges burned into the
raster on the device, ``csrc/geowalls.cu``).  Geometries are GeoJSON-like
mappings (``{"type": "Polygon" | "MultiPolygon", "coordinates": ...}``) or
objects with ``__geo_interface__`` (shapely geometries among them).
"""
from __future__ import annotations

import ctypes
import json
import math
import re
from pathlib import Path
from typing import Any, Mapping

import numpy as np
import torch

from . import _lib, crs as _crs
from .engine import _upload, device_ptr, stream_handle, wall_aspect, wall_heights_device

__all__ = ["calculate_dsm_walls", "calculate_geometry_walls", "building_height", "load_buildings",
           "wall_segments", "affine_from_gdal"]


def calculate_dsm_walls(dsm, pixel_size_m, minimum_wall_height_m=3.0, device="cuda"):
    surface = np.asarray(dsm, dtype=np.float64)
    dsm_dev = _upload(surface, np.float64, torch.device(device))
    walls_dev = wall_heights_device(dsm_dev, float(minimum_wall_height_m))
    aspect, walls = wall_aspect(surface, dsm_dev, walls_dev, float(pixel_size_m))
    return walls, aspect


# Building heights from GeoJSON properties (src/walls.py:145-205): the same
# keys, number syntax, ranges, lists and feet conversion.
_NUMBER = re.compile(r"\d+(?:[\.,]\d+)?")
_HEIGHT_KEYS = ("height", "building:height", "est_height", "building:part:height")
_LEVEL_KEYS = ("building:levels", "levels", "building_levels")
_NOT_A_NUMBER = frozenset({"yes", "no", "none", "null", "nan"})


def _positive(value: Any):
    try:
        x = float(value)
    except (TypeError, ValueError):
        return None
    return x if math.isfinite(x) and x > 0 else None


def _numbers(value: Any):
    text = str(value).strip().lower()
    if not text or text in _NOT_A_NUMBER:
        return []
    out = []
    for token in _NUMBER.findall(text):
        x = _positive(token.replace(",", "."))
        if x is not None:
            out.append(x)
    return out


def _length_metres(value: Any):
    x = _positive(value)
    if x is not None:
        return x
    text = str(value).strip().lower()
    if ";" in text:
        parts = [v for v in (_length_metres(part) for part in text.split(";")) if v is not None]
        return max(parts) if parts else None
    values = _numbers(text)
    if not values:
        return None
    x = max(values) if ("-" in text or " to " in text) else values[0]
    if "ft" in text or "feet" in text or "'" in text:
        x *= 0.3048
    return x


def building_height(properties: Mapping[str, Any] | None, *, default_height_m=6.0, level_height_m=3.0,
                    minimum_height_m=2.0) -> float:
    """Height of one building from its properties: an explicit height key,
    else levels x level height, else the default; never below the minimum."""
    minimum = float(minimum_height_m)
    props = properties or {}
    for key in _HEIGHT_KEYS:
        if key in props:
            h = _length_metres(props.get(key))
            if h is not None:
                return max(minimum, h)
    for key in _LEVEL_KEYS:
        if key in props:
            levels = max(_numbers(props.get(key)) or [0])
            if levels > 0:
                return max(minimum, levels * float(level_height_m))
    return max(minimum, float(default_height_m))


def _geometry_mapping(geometry):
    g = getattr(geometry, "__geo_interface__", geometry)
    if not isinstance(g, Mapping):
        raise TypeError("a geometry must be a GeoJSON-like mapping or provide __geo_interface__")
    return g


def _polygons(geometry):
    """Polygons of a Polygon / MultiPolygon as lists of (n, 2) float64 rings."""
    g = _geometry_mapping(geometry)
    kind = g.get("type")
    if kind == "Polygon":
        polys = [g.get("coordinates") or []]
    elif kind == "MultiPolygon":
        polys = g.get("coordinates") or []
    else:
        return []
    out = []
    for poly in polys:
        rings = []
        for ring in poly:
            r = np.asarray(ring, dtype=np.float64)
            r = r[:, :2] if r.ndim == 2 else np.zeros((0, 2))  # drop any z coordinate
            if len(r) and not np.array_equal(r[0], r[-1]):
                r = np.vstack([r, r[:1]])  # close the ring as shapely does
            rings.append(r)
        if rings and len(rings[0]) >= 4:
            out.append(rings)
    return out


def _signed_area(ring):
    x, y = ring[:, 0], ring[:, 1]
    return 0.5 * float(np.sum(x[:-1] * y[1:] - x[1:] * y[:-1]))


def _project_geometry(geometry, target_crs):
    g = _geometry_mapping(geometry)
    polys = []
    for rings in _polygons(g):
        out = []
        for r in rings:
            x, y = _crs.project_lonlat(r[:, 0], r[:, 1], target_crs)
            out.append(np.column_stack([x, y]).tolist())
        polys.append(out)
    return {"type": "MultiPolygon", "coordinates": polys}


def load_buildings(geojson_path, target_crs, *, default_height_m=6.0, level_height_m=3.0,
                   minimum_height_m=2.0):
    """(projected geometry, height) of every Polygon / MultiPolygon feature of a
    GeoJSON file (coordinates in EPSG:4326) in ``target_crs``."""
    data = json.loads(Path(geojson_path).read_text(encoding="utf-8"))
    buildings = []
    for feature in data.get("features") or []:
        geometry = feature.get("geometry")
        if not geometry or geometry.get("type") not in ("Polygon", "MultiPolygon"):
            continue
        projected = _project_geometry(geometry, target_crs)
        if not projected["coordinates"]:
            continue
        height = building_height(feature.get("properties") or {}, default_height_m=default_height_m,
                                 level_height_m=level_height_m, minimum_height_m=minimum_height_m)
        buildings.append((projected, height))
    return buildings


def wall_segments(geometry, height):
    """Wall segments of a footprint (``src/walls.py:241-267``): every edge of
    every ring, rings oriented as ``orient(polygon, sign=1.0)`` (exterior
    counter-clockwise, holes clockwise), zero-length edges dropped.  Returns
    ``(heights, aspects)``: lists of ``(((x0, y0), (x1, y1)), value)`` with the
    building height and the edge's aspect ``atan2(dy, -dx)`` in degrees [0, 360)."""
    heights, aspects = [], []
    for rings in _polygons(geometry):
        for k, ring in enumerate(rings):
            area = _signed_area(ring)
            if (k == 0 and area < 0.0) or (k > 0 and area > 0.0):
                ring = ring[::-1]
            for (x0, y0), (x1, y1) in zip(ring[:-1].tolist(), ring[1:].tolist()):
                dx, dy = float(x1 - x0), float(y1 - y0)
                if dx == 0 and dy == 0:
                    continue
                seg = ((x0, y0), (x1, y1))
                heights.append((seg, float(height)))
                aspects.append((seg, (math.degrees(math.atan2(dy, -dx)) + 360.0) % 360.0))
    return heights, aspects


def affine_from_gdal(geotransform):
    """rasterio's ``Affine.from_gdal``: (a, b, c, d, e, f) of a GDAL geotransform."""
    c, a, b, f, d, e = (float(v) for v in geotransform[:6])
    return (a, b, c, d, e, f)


def _to_pixels(xy, transform):
    """Pixel coordinates (column u, row v) of world points under the affine
    (a, b, c, d, e, f): x = a u + b v + c, y = d u + e v + f."""
    a, b, c, d, e, f = (float(v) for v in tuple(transform)[:6])
    x, y = xy[:, 0] - c, xy[:, 1] - f
    if b == 0.0 and d == 0.0:
        return x / a, y / e
    det = a * e - b * d
    return (e * x - b * y) / det, (a * y - d * x) / det


def calculate_geometry_walls(buildings, ghsl_height, out_shape, transform, minimum_wall_height_m,
                             device="cuda", stream=None):
    """Wall height and aspect rasters (host float32) from building footprints
    (``src/walls.py:270-332``).  ``buildings``: iterable of (geometry, height);
    ``ghsl_height``: the building-height raster (masked values read as 0,
    compared in float32 as the reference reads it); ``transform``: the raster's
    affine (a, b, c, d, e, f) (``affine_from_gdal`` of a GDAL geotransform).
    Every footprint edge becomes a wall of max(minimum, height) burned into the
    cells it touches on the device (the last edge touching a cell gives its
    values); where the GHSL height reaches the minimum it replaces the
    footprint height."""
    rows, cols = (int(v) for v in tuple(out_shape)[:2])
    minimum = float(minimum_wall_height_m)
    ghsl = np.ascontiguousarray(np.ma.filled(np.ma.asarray(ghsl_height), 0), dtype=np.float32)
    if ghsl.shape != (rows, cols):
        raise ValueError(f"ghsl_height has shape {ghsl.shape}; the raster is {(rows, cols)}")
    ends, seg_h, seg_a = [], [], []
    for geometry, fallback in buildings:
        heights, aspects = wall_segments(geometry, max(minimum, float(fallback)))
        for (seg, h), (_, asp) in zip(heights, aspects):
            ends.append(seg[0] + seg[1])
            seg_h.append(h)
            seg_a.append(asp)
    seg = np.asarray(ends, dtype=np.float64).reshape(-1, 4)
    u0, v0 = _to_pixels(seg[:, 0:2], transform)
    u1, v1 = _to_pixels(seg[:, 2:4], transform)
    pix = np.ascontiguousarray(np.column_stack([u0, v0, u1, v1]), dtype=np.float64)
    dev = torch.device(device)
    L = _lib.lib()
    st = stream_handle(stream)
    t_seg = _upload(pix if len(pix) else np.zeros((1, 4)), np.float64, dev)
    t_h = _upload(np.asarray(seg_h + [0.0]), np.float64, dev)
    t_a = _upload(np.asarray(seg_a + [0.0]), np.float64, dev)
    t_g = _upload(ghsl, np.float32, dev)
    owner = torch.empty((rows, cols), dtype=torch.int32, device=dev)
    walls = torch.empty((rows, cols), dtype=torch.float32, device=dev)
    aspect = torch.empty((rows, cols), dtype=torch.float32, device=dev)
    _lib.check(L.solweig_wall_segments_burn(device_ptr(t_seg), len(pix), rows, cols, device_ptr(owner), st),
               "solweig_wall_segments_burn")
    _lib.check(L.solweig_geometry_walls(device_ptr(owner), device_ptr(t_h), device_ptr(t_a), device_ptr(t_g),
                                        rows * cols, minimum, device_ptr(walls), device_ptr(aspect), st),
               "solweig_geometry_walls")
    return walls.cpu().numpy(), aspect.cpu().numpy()
