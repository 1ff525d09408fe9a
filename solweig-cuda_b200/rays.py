"""Host-side ray tables (FP64, numpy): the digital rays that the kernels walk.

All three walks of the reference step along a digital line from each pixel:
the sun-shadow sweep (``src/umep_solweig.py:2289-2318``), the sky-patch
visibility rays of the SVF (``src/svf.py:47-75``) and the 18 ground-view
search directions (``src/umep_solweig.py:1459-1495``).  The offsets use
numpy's round-half-even and the step heights ``dz = (ds * index) * tan(alt) /
scale`` are computed here exactly as the reference computes them, so the
device compares the very same float64 values.
"""
from __future__ import annotations

import math

import numpy as np

__all__ = ["ShadowRay", "shadow_ray", "svf_rays", "gvf_offsets", "gvf_face_windows",
           "sun_window", "svf_patch_directions"]

_PI4 = np.pi / 4


def _ymajor(az):
    return (_PI4 <= az < 3 * _PI4) or (5 * _PI4 <= az < 7 * _PI4)


def _steps(az, index):
    """dx (rows), dy (cols) of a ray at ``az`` radians for integer ``index`` (array)."""
    s, c, t = np.sin(az), np.cos(az), np.tan(az)
    if _ymajor(az):
        dy = np.sign(s) * index
        dx = -np.sign(c) * np.abs(np.round(index / t))
        ds = np.abs(1 / s)
    else:
        dy = np.sign(s) * np.abs(np.round(index * t))
        dx = -np.sign(c) * index
        ds = np.abs(1 / c)
    return dx, dy, ds


class ShadowRay:
    """Offsets/heights of one sun ray plus the self-shadow azimuth window."""

    __slots__ = ("dxdy", "dz", "low", "high", "middle")

    def __init__(self, dxdy, dz, low, high, middle):
        self.dxdy, self.dz, self.low, self.high, self.middle = dxdy, dz, low, high, middle

    @property
    def steps(self):
        return self.dz.size


def sun_window(az):
    """(low, high, middle) of the wall self-shadow test for sun azimuth ``az`` radians."""
    low, high = az - np.pi / 2, az + np.pi / 2
    middle = low >= 0 and high < 2 * np.pi
    if not middle:
        if low < 0 and high <= 2 * np.pi:
            low += 2 * np.pi
        else:
            high -= 2 * np.pi
    return float(low), float(high), int(middle)


def shadow_ray(azimuth, altitude, scale, maximum, shape, vegetation=True):
    """Sun ray of ``shadowingfunction_wallheight_23`` (``vegetation``, index from 0,
    loop bound ``maximum = amaxvalue``) or ``_13`` (index from 1, ``maximum`` =
    the DSM maximum).  Steps run up to and including the first one whose dz
    exceeds ``maximum`` or whose offset leaves the raster.
    """
    rows, cols = shape
    if vegetation:
        az = azimuth * (np.pi / 180.)
        alt = altitude * (np.pi / 180.)
        first = 0
    else:
        az = math.radians(azimuth)
        alt = math.radians(altitude)
        first = 1
    index = np.arange(first, max(shape) + 2, dtype=np.float64)
    dx, dy, ds = _steps(az, index)
    tanab = np.tan(alt) / scale
    dz = (ds * index) * tanab
    bad = (~(maximum >= dz)) | (np.abs(dx) >= rows) | (np.abs(dy) >= cols)
    count = int(np.flatnonzero(bad)[0]) + 1 if bad.any() else index.size
    if maximum < 0:
        count = 0
    dxdy = np.ascontiguousarray(np.column_stack((dx[:count], dy[:count])).astype(np.int32))
    low, high, middle = sun_window(az)
    return ShadowRay(dxdy, np.ascontiguousarray(dz[:count]), low, high, middle)


def svf_patch_directions(patch_option):
    """Patch azimuth/altitude (degrees) as ordered by the SVF ray setup (``src/svf.py:31-35``)."""
    counts = {1: (30, 30, 24, 24, 18, 12, 6, 1), 2: (31, 30, 28, 24, 19, 13, 7, 1),
              3: (62, 60, 56, 48, 38, 26, 14, 1)}[int(patch_option)]
    starts = (0, 4, 2, 5, 8, 0, 10, 0)
    alts = (6, 18, 30, 42, 54, 66, 78, 90)
    azimuth = np.concatenate([np.arange(n) * (360. / n) + s for n, s in zip(counts, starts)])
    azimuth[azimuth > 360.] -= 360.
    altitude = np.asarray(alts, dtype=np.float64)[np.repeat(np.arange(len(counts)), counts)]
    return azimuth, altitude, counts


def svf_rays(patch_option, shape, amaxvalue, scale):
    """Per-patch visibility rays: ``(dxdy [P, cap, 2] int32, dz [P, cap], lengths [P], cap)``.

    ``lengths[p]`` is the index of the first step with dz > amaxvalue or an
    offset leaving the raster, plus one (``src/svf.py:53-72``).  The heights
    grow linearly with the index, so only a prefix of the steps (up to two
    past amaxvalue / slope) can hold that first step: each patch evaluates
    ``_steps`` on that prefix alone, with the same float64 operations.
    """
    rows, cols = shape
    azimuth, altitude, _ = svf_patch_directions(patch_option)
    P = azimuth.size
    capacity = max(rows, cols) + 1
    index_all = np.arange(capacity, dtype=np.float64)
    lengths = np.zeros(P, dtype=np.int32)
    if amaxvalue < 0:
        return np.zeros((P, 1, 2), dtype=np.int32), np.zeros((P, 1)), lengths, 1
    tables = []
    for p in range(P):
        az, el = azimuth[p] * (np.pi / 180.), altitude[p] * (np.pi / 180.)
        tz = np.tan(el) / scale
        s_, c_ = abs(np.sin(az)), abs(np.cos(az))
        slope = (1 / s_ if _ymajor(az) else 1 / c_) * tz
        m = capacity if not slope > 0 else int(min(capacity, np.ceil(amaxvalue / slope) + 2))
        index = index_all[:max(m, 1)]
        dx, dy, ds = _steps(az, index)
        z = (ds * index) * tz
        bad = np.flatnonzero((z > amaxvalue) | (np.abs(dx) >= rows) | (np.abs(dy) >= cols))
        if len(bad):
            n = int(bad[0]) + 1
        elif m >= capacity:
            n = capacity
        else:  # cannot happen (z exceeds amaxvalue within the prefix); the full table
            dx, dy, ds = _steps(az, index_all)
            z = (ds * index_all) * tz
            bad = np.flatnonzero((z > amaxvalue) | (np.abs(dx) >= rows) | (np.abs(dy) >= cols))
            n = int(bad[0]) + 1 if len(bad) else capacity
        lengths[p] = n
        tables.append((dx[:n], dy[:n], z[:n]))
    cap = max(1, int(lengths.max()))
    dxdy = np.zeros((P, cap, 2), dtype=np.int32)
    dz = np.zeros((P, cap), dtype=np.float64)
    for p, (dx, dy, z) in enumerate(tables):
        n = len(z)
        dxdy[p, :n, 0], dxdy[p, :n, 1] = dx, dy
        dz[p, :n] = z
    return dxdy, dz, lengths, cap


def _svf_rays_per_patch(patch_option, shape, amaxvalue, scale):
    """The per-patch loop form of ``svf_rays`` (kept for the equality test)."""
    rows, cols = shape
    azimuth, altitude, _ = svf_patch_directions(patch_option)
    P = azimuth.size
    capacity = max(rows, cols) + 1
    index = np.arange(capacity, dtype=np.float64)
    dxdy = np.zeros((P, capacity, 2), dtype=np.int32)
    dz = np.zeros((P, capacity), dtype=np.float64)
    lengths = np.zeros(P, dtype=np.int32)
    for p in range(P):
        if amaxvalue < 0:
            continue
        az, el = azimuth[p] * (np.pi / 180.), altitude[p] * (np.pi / 180.)
        dx, dy, ds = _steps(az, index)
        z = (ds * index) * (np.tan(el) / scale)
        bad = np.flatnonzero((z > amaxvalue) | (np.abs(dx) >= rows) | (np.abs(dy) >= cols))
        n = int(bad[0]) + 1 if len(bad) else capacity
        lengths[p] = n
        dxdy[p, :n, 0], dxdy[p, :n, 1] = dx[:n], dy[:n]
        dz[p, :n] = z[:n]
    cap = max(1, int(lengths.max()))
    return (np.ascontiguousarray(dxdy[:, :cap]), np.ascontiguousarray(dz[:, :cap]), lengths, cap)


def gvf_offsets(scale, first=1.0, second=22.0):
    """Offsets [18, second_steps, 2] of the ground-view search and the step counts.

    ``first``/``second`` are the reference's ``round(1.1)`` and ``round(1.1*20)``
    scaled by pixel density (``src/umep_solweig.py:1443-1447``).
    """
    first_steps = np.round(first * scale)
    if first_steps < 1:
        first_steps = 1
    second_steps = int(np.round(second * scale))
    first_steps = int(first_steps)
    out = np.zeros((18, max(second_steps, 1), 2), dtype=np.int32)
    for j, deg in enumerate(np.arange(5, 359, 20)):
        az = deg * (np.pi / 180)
        s, c, t = np.sin(az), np.cos(az), np.tan(az)
        for n in range(second_steps):
            if _ymajor(az):
                dy = np.sign(s) * n
                dx = -np.sign(c) * np.abs(np.round(n / t))
            else:
                dy = np.sign(s) * abs(round(n * t))
                dx = -np.sign(c) * n
            out[j, n] = int(dx), int(dy)
    return np.ascontiguousarray(out), first_steps, second_steps


def gvf_face_windows():
    """(low[18], high[18], middle[18]) self-shadow windows of the 18 GVF directions."""
    lows, highs, mids = [], [], []
    for deg in np.arange(5, 359, 20):
        low, high, mid = sun_window(deg * (np.pi / 180))
        lows.append(low)
        highs.append(high)
        mids.append(mid)
    return (np.asarray(lows, dtype=np.float64), np.asarray(highs, dtype=np.float64),
            np.asarray(mids, dtype=np.int32))
