"""Oracle restatement of the ground view factors (test infrastructure).

``gvf`` restates ``gvf_2018a`` (``src/umep_solweig.py:583-663``) and its inner
``sunonsurface_2018a`` (``src/umep_solweig.py:1400-1600``) in float64 numpy.
"""
from __future__ import annotations

import numpy as np

from .geometry import _ray_step


def _walk_direction(azimuth_deg, scale, buildings, shadow, sunwall, first, second, aspect,
                    walls, Lup, albshadow, alb, Lwall, albedo_b):
    """One search direction of ``sunonsurface_2018a``.

    Returns ``(gvf2, lup_dir, alb_dir, albnosh_dir)`` before the per-pixel
    corrections.  The shifted fields are NOT cleared between steps: a pixel
    whose sample has left the raster keeps the last sample it saw, as the
    reference's in-place slice assignment does.
    """
    rows, cols = buildings.shape
    azi = azimuth_deg * (np.pi / 180)
    first = np.round(first * scale)
    if first < 1:
        first = 1
    second = np.round(second * scale)
    f = buildings.copy()
    t_bu = np.zeros((rows, cols))
    t_sh = np.zeros((rows, cols))
    t_lup = np.zeros((rows, cols))
    t_albsh = np.zeros((rows, cols))
    t_alb = np.zeros((rows, cols))
    t_sunwall = np.zeros((rows, cols))
    sum_sh = np.zeros((rows, cols))
    sum_lup = np.zeros((rows, cols))
    sum_albsh = np.zeros((rows, cols))
    sum_alb = np.zeros((rows, cols))
    sum_wall = np.zeros((rows, cols))
    sum_lwall = np.zeros((rows, cols))
    sum_albwall = np.zeros((rows, cols))
    sum_albwall_nosh = np.zeros((rows, cols))
    seen_sunwall = np.zeros((rows, cols))
    seen_wall = np.zeros((rows, cols))
    near = None
    for n in range(int(second)):
        dx, dy, _ = _ray_step(azi, n)
        dx, dy = int(dx), int(dy)
        r0, r1 = max(0, -dx), min(rows, rows - dx)
        c0, c1 = max(0, -dy), min(cols, cols - dy)
        if r1 > r0 and c1 > c0:
            src = (slice(r0 + dx, r1 + dx), slice(c0 + dy, c1 + dy))
            dst = (slice(r0, r1), slice(c0, c1))
            t_bu[dst] = buildings[src]
            t_sh[dst] = shadow[src]
            t_lup[dst] = Lup[src]
            t_albsh[dst] = albshadow[src]
            t_alb[dst] = alb[src]
            t_sunwall[dst] = sunwall[src]
        f = np.minimum(f, t_bu)
        sum_sh += t_sh * f
        sum_lup += t_lup * f
        sum_albsh += t_albsh * f
        sum_alb += t_alb * f
        seen_sunwall = ((t_sunwall * f + seen_sunwall) > 0).astype(float)
        seen_wall = (((1 - f) + seen_wall) > 0).astype(float)
        sum_lwall += seen_sunwall * Lwall
        sum_albwall += seen_sunwall * albedo_b
        sum_wall += seen_sunwall
        sum_albwall_nosh += seen_wall * albedo_b
        if n + 1 <= first:
            near = (sum_wall.copy(), sum_sh.copy(), sum_lwall.copy(), sum_lup.copy(),
                    sum_albwall.copy(), sum_albsh.copy(), sum_albwall_nosh.copy(), sum_alb.copy())
    n_wall, n_sh, n_lwall, n_lup, n_albwall, n_albsh, n_albwall_nosh, n_alb = near
    sun_near = n_wall > 0
    wall_near = n_albwall_nosh > 0
    sun_far = sum_wall > 0
    wall_far = sum_albwall_nosh > 0

    wallbol = (walls > 0).astype(float)
    low, high = azi - np.pi / 2, azi + np.pi / 2
    if low >= 0 and high < 2 * np.pi:
        facesh = np.logical_or(aspect < low, aspect >= high).astype(float) - wallbol + 1
    elif low < 0 and high <= 2 * np.pi:
        facesh = 1 - np.logical_or(aspect > low + 2 * np.pi, aspect <= high).astype(float)
    else:
        facesh = 1 - np.logical_or(aspect > low, aspect <= high - 2 * np.pi).astype(float)
    keep = (sum_wall == second) - facesh
    keep[keep == -1] = 0
    drop = keep == 1

    def mix(wall_sum, ground_sum, wall_div, ground_div, influence):
        return (wall_sum + ground_sum) / wall_div * influence + ground_sum / ground_div * (1 - influence)

    sum_wall = np.where(drop, 0, sum_wall)
    gvf2 = np.minimum(mix(sum_wall, sum_sh, second + 1, second, sun_far), 1.)
    sum_lwall = np.where(drop, 0, sum_lwall)
    sum_albwall = np.where(drop, 0, sum_albwall)
    lup1 = mix(n_lwall, n_lup, first + 1, first, sun_near)
    lup2 = mix(sum_lwall, sum_lup, second + 1, second, sun_far)
    alb1 = mix(n_albwall, n_albsh, first + 1, first, sun_near)
    alb2 = mix(sum_albwall, sum_albsh, second + 1, second, sun_far)
    nosh1 = mix(n_albwall_nosh, n_alb, first + 1, first, wall_near)
    nosh2 = mix(sum_albwall_nosh, sum_alb, second, second, wall_far)
    return (gvf2, (lup1 * 0.5 + lup2 * 0.4) / 0.9, (alb1 * 0.5 + alb2 * 0.4) / 0.9,
            (nosh1 * 0.5 + nosh2 * 0.4) / 0.9)


def gvf(wallsun, walls, buildings, scale, shadow, first, second, dirwalls, Tg, Tgwall, Ta,
        emis_grid, ewall, alb_grid, SBC, albedo_b, Twater=None, lc_grid=None, landcover=0):
    """17 ground-view-factor planes of ``gvf_2018a``; also returns the surface
    temperature after the water override (the reference mutates ``Tg`` in place).

    Returns ``(planes, Tg_after)`` with ``planes`` in the reference order
    (gvfLup, gvfalb, gvfalbnosh, then E, S, W, N triples, gvfSum, gvfNorm).
    """
    Tg = np.array(Tg, dtype=np.float64, copy=True)
    shadow = np.asarray(shadow, dtype=np.float64)
    with np.errstate(divide='ignore', invalid='ignore'):
        sunwall = ((wallsun / walls * buildings) == 1).astype(float)
    aspect = dirwalls * np.pi / 180
    ambient = SBC * emis_grid * (Ta + 273.15) ** 4
    Lup_first = SBC * emis_grid * (Tg * shadow + Ta + 273.15) ** 4 - ambient
    if landcover == 1:
        Tg[lc_grid == 3] = Twater - Ta
    Lup_rest = SBC * emis_grid * (Tg * shadow + Ta + 273.15) ** 4 - ambient
    Lwall = SBC * ewall * (Tgwall + Ta + 273.15) ** 4 - SBC * ewall * (Ta + 273.15) ** 4
    albshadow = alb_grid * shadow
    ground = 1 - buildings
    acc = {k: np.zeros(buildings.shape) for k in
           ("lup", "alb", "nosh", "lupE", "albE", "noshE", "lupS", "albS", "noshS",
            "lupW", "albW", "noshW", "lupN", "albN", "noshN", "sum")}
    directions = np.arange(5, 359, 20)
    for j, az in enumerate(directions):
        Lup = Lup_first if j == 0 else Lup_rest
        gvf2, lup_d, alb_d, nosh_d = _walk_direction(
            az, scale, buildings, shadow, sunwall, first, second, aspect, walls, Lup, albshadow,
            alb_grid, Lwall, albedo_b)
        lup_d = lup_d + (SBC * emis_grid * (Tg * shadow + Ta + 273.15) ** 4 - ambient) * ground
        alb_d = alb_d + alb_grid * ground * shadow
        nosh_d = nosh_d * buildings + alb_grid * ground
        acc["lup"] += lup_d
        acc["alb"] += alb_d
        acc["nosh"] += nosh_d
        acc["sum"] += gvf2
        for key, hit in (("E", 0 <= az < 180), ("S", 90 <= az < 270), ("W", 180 <= az < 360),
                         ("N", az >= 270 or az < 90)):
            if hit:
                acc["lup" + key] += lup_d
                acc["alb" + key] += alb_d
                acc["nosh" + key] += nosh_d
    n = directions.size
    planes = [acc["lup"] / n + ambient, acc["alb"] / n, acc["nosh"] / n]
    for key in "ESWN":
        planes += [acc["lup" + key] / (n / 2) + ambient, acc["alb" + key] / (n / 2),
                   acc["nosh" + key] / (n / 2)]
    norm = acc["sum"] / n
    norm[buildings == 0] = 1
    planes += [acc["sum"], norm]
    return planes, Tg
