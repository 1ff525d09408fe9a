"""Oracle restatement of the static and per-hour geometry (test infrastructure).

float64 numpy, written for clarity rather than speed.  Each function names the
reference code it restates.
"""
from __future__ import annotations

import math

import numpy as np

_PI4 = np.pi / 4


def _ray_step(azimuth_rad, index):
    """(dx, dy, ds) of step ``index`` along a digital ray at ``azimuth_rad``.

    dx moves along axis 0 (rows), dy along axis 1 (cols); numpy's
    round-half-even is part of the contract (``src/umep_solweig.py:2296-2303``).
    """
    s, c, t = np.sin(azimuth_rad), np.cos(azimuth_rad), np.tan(azimuth_rad)
    if (_PI4 <= azimuth_rad < 3 * _PI4) or (5 * _PI4 <= azimuth_rad < 7 * _PI4):
        return -np.sign(c) * np.abs(np.round(index / t)), np.sign(s) * index, np.abs(1 / s)
    return -np.sign(c) * index, np.sign(s) * np.abs(np.round(index * t)), np.abs(1 / c)


def _shift(field, dx, dy):
    """Return (values, inside): field sampled at (r + dx, c + dy); 0 where outside."""
    rows, cols = field.shape
    dx, dy = int(dx), int(dy)
    out = np.zeros_like(field)
    inside = np.zeros(field.shape, dtype=bool)
    r0, r1 = max(0, -dx), min(rows, rows - dx)
    c0, c1 = max(0, -dy), min(cols, cols - dy)
    if r1 > r0 and c1 > c0:
        out[r0:r1, c0:c1] = field[r0 + dx:r1 + dx, c0 + dy:c1 + dy]
        inside[r0:r1, c0:c1] = True
    return out, inside


def _self_shadow_faces(aspect, azimuth_rad, wallbol):
    """Wall faces turned away from the sun (facesh), ``src/umep_solweig.py:2372-2380``."""
    low, high = azimuth_rad - np.pi / 2, azimuth_rad + np.pi / 2
    if low >= 0 and high < 2 * np.pi:
        return np.logical_or(aspect < low, aspect >= high).astype(float) - wallbol + 1
    if low < 0 and high <= 2 * np.pi:
        low = low + 2 * np.pi
    else:
        high = high - 2 * np.pi
    return 1.0 - np.logical_or(aspect > low, aspect <= high).astype(float)


def shadow_sweep(dsm, vegdem, vegdem2, azimuth, altitude, scale, amaxvalue, bush, walls, aspect):
    """Building + vegetation shadows and wall shading for one sun position.

    Restates ``shadowingfunction_wallheight_23`` (``src/umep_solweig.py:2201-2406``).
    ``azimuth``/``altitude`` in degrees, ``aspect`` in radians.  Returns
    ``(vegsh, sh, vbshvegsh, wallsh, wallsun, wallshve, facesh, facesun)``.
    """
    dsm = np.asarray(dsm, dtype=np.float64)
    vegdem = np.asarray(vegdem, dtype=np.float64)
    vegdem2 = np.asarray(vegdem2, dtype=np.float64)
    walls = np.asarray(walls, dtype=np.float64)
    rows, cols = dsm.shape
    azi = azimuth * (np.pi / 180.)
    alt = altitude * (np.pi / 180.)
    tan_by_scale = np.tan(alt) / scale
    building_top = dsm.copy()          # running max of shifted (dsm - dz): "f"
    canopy_top = vegdem.copy()         # running max of shifted (vegdem - dz): "shvoveg"
    veg = (bush > 1).astype(float)     # vegetation shadow flag
    seen = np.zeros((rows, cols))      # accumulated veg flags before a building hit
    shaded = np.zeros((rows, cols))
    index, dx, dy, dz, dz_prev = 0, 0, 0, 0.0, 0.0
    while amaxvalue >= dz and abs(dx) < rows and abs(dy) < cols:
        dx, dy, ds = _ray_step(azi, index)
        dz = (ds * index) * tan_by_scale
        a_s, inside = _shift(dsm, dx, dy)
        top_s, _ = _shift(vegdem, dx, dy)
        bot_s, _ = _shift(vegdem2, dx, dy)
        temp = np.where(inside, a_s - dz, 0.0)
        top_now = np.where(inside, top_s - dz, 0.0)
        bot_now = np.where(inside, bot_s - dz, 0.0)
        top_prev = np.where(inside, top_s - dz_prev, 0.0)
        bot_prev = np.where(inside, bot_s - dz_prev, 0.0)
        building_top = np.fmax(building_top, temp)
        canopy_top = np.fmax(canopy_top, top_now)
        shaded = (building_top > dsm).astype(float)
        count = ((top_now > dsm).astype(float) + (bot_now > dsm) + (top_prev > dsm) + (bot_prev > dsm))
        step_veg = ((count > 0) & (count < 4)).astype(float)
        veg = np.fmax(veg, step_veg)
        veg[veg * shaded > 0] = 0
        seen = seen + veg
        dz_prev = dz
        index += 1

    wallbol = (walls > 0).astype(float)
    facesh = _self_shadow_faces(aspect, azi, wallbol)
    sh = 1 - shaded
    seen = (seen > 0).astype(float) - veg
    veg = (veg > 0).astype(float)
    canopy_volume = (canopy_top - dsm) * veg
    vegsh = 1 - veg
    vbshvegsh = 1 - seen
    volume = building_top - dsm
    facesun = np.logical_and(facesh + wallbol == 1, walls > 0).astype(float)
    wallsun = np.maximum(walls - volume, 0.0)
    wallsun[facesh == 1] = 0
    wallsh = walls - wallsun
    wallshve = np.maximum(canopy_volume * wallbol - wallsh, 0.0)
    over = wallshve > walls
    wallshve[over] = walls[over]
    wallsun = wallsun - wallshve
    neg = wallsun < 0
    wallshve[neg] = 0
    wallsun[neg] = 0
    return vegsh, sh, vbshvegsh, wallsh, wallsun, wallshve, facesh, facesun


def shadow_sweep_buildings(dsm, azimuth, altitude, scale, walls, aspect):
    """Building-only shadows, ``shadowingfunction_wallheight_13``
    (``src/umep_solweig.py:2063-2197``).  Returns ``(sh, wallsh, wallsun, facesh, facesun)``.
    """
    dsm = np.asarray(dsm, dtype=np.float64)
    walls = np.asarray(walls, dtype=np.float64)
    rows, cols = dsm.shape
    azi = math.radians(azimuth)
    alt = math.radians(altitude)
    tan_by_scale = np.tan(alt) / scale
    amax = np.max(dsm)
    top = dsm.copy()
    index, dx, dy, dz = 1, 0, 0, 0.0
    while amax >= dz and abs(dx) < rows and abs(dy) < cols:
        dx, dy, ds = _ray_step(azi, index)
        dz = ds * index * tan_by_scale
        a_s, inside = _shift(dsm, dx, dy)
        top = np.fmax(top, np.where(inside, a_s - dz, 0.0))
        index += 1
    wallbol = (walls > 0).astype(float)
    facesh = _self_shadow_faces(aspect, azi, wallbol)
    volume = top - dsm
    facesun = np.logical_and(facesh + wallbol == 1, walls > 0).astype(float)
    wallsun = np.maximum(walls - volume, 0.0)
    wallsun[facesh == 1] = 0
    wallsh = walls - wallsun
    sh = 1 - (volume != 0).astype(float)
    return sh, wallsh, wallsun, facesh, facesun


# ----------------------------------------------------------------------------
# Walls from the DSM
# ----------------------------------------------------------------------------

def wall_heights(dsm, threshold):
    """Wall height from the 4-neighbour maximum, ``src/kernels/geometry.cu:15-34``.

    Interior cells: max(N, S, W, E) - dsm where that is >= threshold.  Border
    cells are zero except row 0 at columns ``rows <= col < cols - 1`` which
    keep ``-dsm`` when that is >= threshold (the column bound uses the row
    count, a quirk inherited from UMEP's ``findwalls``).
    """
    dsm = np.asarray(dsm, dtype=np.float64)
    rows, cols = dsm.shape
    out = np.zeros_like(dsm)
    if rows >= 3 and cols >= 3:
        nb = np.fmax(np.fmax(dsm[:-2, 1:-1], dsm[2:, 1:-1]), np.fmax(dsm[1:-1, :-2], dsm[1:-1, 2:]))
        diff = nb - dsm[1:-1, 1:-1]
        out[1:-1, 1:-1] = np.where(diff >= threshold, diff, 0.0)
    if rows > 1:
        c0, c1 = rows, cols - 1
        if c1 > c0:
            edge = -dsm[0, c0:c1]
            out[0, c0:c1] = np.where(edge >= threshold, edge, 0.0)
    return out


def filter_size(pixel_size_m):
    """Template size for the wall aspect search, ``src/walls.py:24-30``."""
    size = int(np.floor((1.0 / pixel_size_m + 1e-10) * 9))
    if size <= 2:
        size = 3
    elif size != 9 and size % 2 == 0:
        size += 1
    return size


def aspect_templates(size):
    """180 rotated line/side templates, ``src/walls.py:33-56`` (scipy ``rotate``)."""
    from scipy.ndimage import rotate
    radius = size // 2
    line = np.zeros((size, size))
    line[:, radius] = 1
    sides = np.zeros((size, size))
    sides[radius, :radius] = 1
    sides[radius, radius + 1:] = 2
    out = []
    for angle in range(180):
        rl = np.round(rotate(line, angle, order=1, reshape=False, mode="nearest"))
        rs = np.round(rotate(sides, angle, order=0, reshape=False, mode="nearest"))
        if angle in (150, 30):
            rs[:, size - 1] = 0
        if 270 - angle == 225:
            rl[0, 0] = rl[size - 1, size - 1] = 1
        if 270 - angle == 135:
            rl[0, size - 1] = rl[size - 1, 0] = 1
        out.append(tuple(np.argwhere(m).astype(np.int64) - radius
                         for m in (rl != 0, rs == 1, rs == 2)))
    return out


def wall_aspect(walls, dsm, pixel_size):
    """Wall aspect in degrees, ``src/walls.py:83-129`` with ``geometry.cu:36-63``."""
    dsm = np.asarray(dsm, dtype=np.float64)
    mask = walls > 0
    aspect = np.zeros(dsm.shape)
    if not mask.any():
        return aspect
    rows, cols = dsm.shape
    size = filter_size(pixel_size)
    radius = size // 2
    if rows > 2 * radius + 2 and cols > 2 * radius + 2:
        templates = aspect_templates(size)
        occupied = mask.astype(np.int64)
        rr, cc = np.nonzero(mask)
        valid = (rr >= radius) & (rr < rows - radius - 2) & (cc >= radius) & (cc < cols - radius - 2)
        best = np.full(rr.size, -1)
        score_best = np.zeros(rr.size, dtype=np.int64)
        for angle, (line, _, _) in enumerate(templates):
            score = np.zeros(rr.size, dtype=np.int64)
            for dr, dc in line:
                score += occupied[np.clip(rr + dr, 0, rows - 1), np.clip(cc + dc, 0, cols - 1)]
            better = valid & (score > score_best)
            score_best[better] = score[better]
            best[better] = angle
        for angle in np.unique(best):
            if angle < 0:
                continue
            sel = best == angle
            _, s1, s2 = templates[int(angle)]
            r, c = rr[sel], cc[sel]
            first = sum(dsm[r + dr, c + dc] for dr, dc in s1) if len(s1) else np.zeros(r.size)
            second = sum(dsm[r + dr, c + dc] for dr, dc in s2) if len(s2) else np.zeros(r.size)
            direction = np.full(r.size, 270.0 - int(angle))
            direction[first > second] -= 180.0
            direction[direction < 0] += 360.0
            aspect[r, c] = direction
    step = 1.0 / (1.0 / pixel_size)
    fy, fx = np.gradient(dsm, step, step)
    grad = -np.arctan2(fx, fy)
    grad[grad < 0] += 2 * np.pi
    unresolved = mask & (aspect == 0)
    aspect += unresolved * (grad / (math.pi / 180.0))
    return aspect


# ----------------------------------------------------------------------------
# Sky view factor (153 patches)
# ----------------------------------------------------------------------------

def patch_directions(patch_option):
    """Patch azimuth/altitude/band layout and annulus weights, ``src/svf.py:19-46``."""
    counts = {1: (30, 30, 24, 24, 18, 12, 6, 1), 2: (31, 30, 28, 24, 19, 13, 7, 1),
              3: (62, 60, 56, 48, 38, 26, 14, 1)}[int(patch_option)]
    edges = (0, 12, 24, 36, 48, 60, 72, 84, 90)
    alts = (6, 18, 30, 42, 54, 66, 78, 90)
    starts = (0, 4, 2, 5, 8, 0, 10, 0)
    azimuth = np.concatenate([np.arange(n) * (360. / n) + s for n, s in zip(counts, starts)])
    azimuth[azimuth > 360.] -= 360.
    band = np.repeat(np.arange(len(counts)), counts)
    altitude = np.asarray(alts, dtype=np.float64)[band]
    weights = np.zeros((len(counts), 2))
    for b, n in enumerate(counts):
        for k in np.arange(edges[b] + 1, edges[b + 1] + 1):
            ring = 91. - k
            w = (1. / (2. * np.pi)) * np.sin(np.pi / 180.) * np.sin((np.pi * (2. * ring - 1.)) / 180.)
            weights[b, 0] += ((360. / n) * (np.pi / 180.)) * w
            weights[b, 1] += ((360. / np.ceil(n / 2.)) * (np.pi / 180.)) * w
    sectors = np.stack([(azimuth >= 0) & (azimuth < 180), (azimuth >= 90) & (azimuth < 270),
                        (azimuth >= 180) & (azimuth < 360), (azimuth >= 270) | (azimuth < 90)])
    return azimuth, altitude, band, weights, sectors


def svf_patch_masks(dsm, vegdem, vegdem2, bush, scale, amaxvalue, patch_option=2):
    """Per-patch visibility masks ``(shmat, vegmat, vbmat)`` as float arrays
    ``[rows, cols, P]`` (1 = patch visible through that class).

    Restates ``svf_visibility`` (``src/kernels/geometry.cu:66-119``): a shadow
    sweep toward every patch centre that stops at the first building hit.
    """
    azimuth, altitude, *_ = patch_directions(patch_option)
    rows, cols = dsm.shape
    P = azimuth.size
    shm = np.empty((rows, cols, P))
    vegm = np.empty((rows, cols, P))
    vbm = np.empty((rows, cols, P))
    zeros = np.zeros((rows, cols))
    for p in range(P):
        vegsh, sh, vbsh, *_ = shadow_sweep(dsm, vegdem, vegdem2, azimuth[p], altitude[p], scale,
                                           amaxvalue, bush, zeros, zeros)
        shm[:, :, p], vegm[:, :, p], vbm[:, :, p] = sh, vegsh, vbsh
    return shm, vegm, vbm


def svf_reduce(shm, vegm, vbm, vegdem2, patch_option=2, transmissivity=0.03):
    """Annulus-weighted sums of the patch masks, ``src/kernels/geometry.cu:121-159``.

    Returns the 16 planes (all, E, S, W, N) x (sh, veg, vb) + svftotal.
    """
    _, _, band, weights, sectors = patch_directions(patch_option)
    out = []
    for m in (shm, vegm, vbm):
        wf = weights[band, 0]
        wa = weights[band, 1]
        planes = [np.tensordot(m, wf, axes=([2], [0]))]
        for d in range(4):
            planes.append(np.tensordot(m, wa * sectors[d], axes=([2], [0])))
        out.extend(planes)
    eps = 3.0459e-4
    out[2] = out[2] + eps
    out[3] = out[3] + eps
    last = np.where(vegdem2 == 0, eps, 0.0)
    for i in (7, 8, 12, 13):
        out[i] = out[i] + last
    out = [np.minimum(v, 1.0) for v in out]
    total = out[0] - (1.0 - out[5]) * (1.0 - transmissivity)
    return out + [total]


def svf_calculator(patch_option, amaxvalue, dsm, vegdem, vegdem2, bush, scale, transmissivity=0.03):
    """19-tuple of ``src/svf.py:81-114``: 15 SVF planes, vegmat, vbmat, shmat, svftotal."""
    shm, vegm, vbm = svf_patch_masks(dsm, vegdem, vegdem2, bush, scale, amaxvalue, patch_option)
    r = svf_reduce(shm, vegm, vbm, vegdem2, patch_option, transmissivity)
    order = (0, 10, 1, 11, 6, 4, 14, 9, 2, 12, 7, 5, 3, 13, 8)
    return tuple(r[i] for i in order) + (vegm, vbm, shm, r[15])


def compute_diffsh(shmat, vegshmat, transmissivity):
    """``diffsh = sh - (1 - veg)(1 - tau)``, ``src/svf.py:117-131``."""
    return shmat - (1.0 - vegshmat) * (1.0 - transmissivity)
