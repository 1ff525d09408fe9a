"""Oracle of the geometry wall method's raster stage (test infrastructure).

``src/walls.py:270-332`` (``calculate_geometry_walls``) burns every footprint
edge into the raster with ``rasterio.features.rasterize(..., all_touched=True)``
-- later shapes replacing earlier ones -- for the wall mask, the fallback
heights and the aspects, then merges them with the GHSL heights.  rasterio
(GDAL) is absent here, so its burn is restated with an explicit rule, exactly,
in rational arithmetic: a segment touches the cell (col, row) when one of its
points lies in the half-open square [col, col + 1) x [row, row + 1) of pixel
coordinates.  Every cell of the segment's bounding box is tested by
intersecting the parameter intervals of the two axes -- a different method
from the device's grid walk.  The merge restates ``src/walls.py:318-332``
with numpy.  Parity with GDAL's own burn is unpinned: neither it nor
rasterio can run in this image.
"""
from __future__ import annotations

import math
from fractions import Fraction

import numpy as np


def _axis_interval(p0, d, k):
    """{t : k <= p0 + t d < k + 1} as (lo, lo_closed, hi, hi_closed), or None."""
    if d == 0:
        return (Fraction(-10), True, Fraction(10), True) if k <= p0 < k + 1 else None
    a = (k - p0) / d        # p = k
    b = (k + 1 - p0) / d    # p = k + 1 (excluded)
    if d > 0:
        return (a, True, b, False)
    return (b, False, a, True)


def _meet(x, y):
    lo, lo_c = max((x[0], x[1]), (y[0], y[1]), key=lambda v: (v[0], not v[1]))
    hi, hi_c = min((x[2], x[3]), (y[2], y[3]), key=lambda v: (v[0], v[1]))
    return lo, lo_c, hi, hi_c


def _nonempty(iv):
    lo, lo_c, hi, hi_c = iv
    return lo < hi or (lo == hi and lo_c and hi_c)


def cells_touched(u0, v0, u1, v1):
    """Cells (col, row) holding a point of the segment, exactly."""
    u0, v0, u1, v1 = (Fraction(float(x)) for x in (u0, v0, u1, v1))
    du, dv = u1 - u0, v1 - v0
    unit = (Fraction(0), True, Fraction(1), True)
    out = []
    for i in range(math.floor(min(u0, u1)), math.floor(max(u0, u1)) + 1):
        xi = _axis_interval(u0, du, i)
        if xi is None:
            continue
        xi = _meet(xi, unit)
        if not _nonempty(xi):
            continue
        for j in range(math.floor(min(v0, v1)), math.floor(max(v0, v1)) + 1):
            yj = _axis_interval(v0, dv, j)
            if yj is not None and _nonempty(_meet(xi, yj)):
                out.append((i, j))
    return out


def burn(segments, rows, cols):
    """owner[row, col] = index of the last segment touching the cell, -1 if none."""
    owner = np.full((rows, cols), -1, dtype=np.int32)
    for s, (u0, v0, u1, v1) in enumerate(np.asarray(segments, dtype=np.float64).reshape(-1, 4)):
        for i, j in cells_touched(u0, v0, u1, v1):
            if 0 <= i < cols and 0 <= j < rows:
                owner[j, i] = s
    return owner


def merge(owner, heights, aspects, ghsl, minimum):
    """``src/walls.py:318-332``: the mask, fallback-height and aspect rasters
    (float32, the rasterize dtype) merged with the float32 GHSL heights."""
    mask = owner >= 0
    idx = np.where(mask, owner, 0)
    fallback = np.where(mask, np.asarray(heights, dtype=np.float64)[idx].astype(np.float32), np.float32(0))
    aspect = np.where(mask, np.asarray(aspects, dtype=np.float64)[idx].astype(np.float32), np.float32(0))
    ghsl = np.nan_to_num(np.asarray(ghsl, dtype=np.float32), nan=0.0, posinf=0.0, neginf=0.0)
    support = mask & (ghsl >= np.float32(minimum))
    walls = np.where(mask, np.where(support, ghsl, fallback), 0).astype(np.float32)
    aspect = np.where(mask, aspect, 0).astype(np.float32)
    np.remainder(aspect, np.float32(360.0), out=aspect)
    return walls, aspect
