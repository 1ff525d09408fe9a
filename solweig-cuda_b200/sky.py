"""Host-side FP64 sky-vault geometry and per-hour patch weights.

The anisotropic sky of SOLWEIG 2022a divides the vault into patches
(153 for ``patch_option=2``) and, every hour, weights each patch by the Perez
luminance (shortwave) and a band emissivity (longwave).  This module builds:

* the patch layout            ``create_patches``, ``src/umep_solweig.py:1737-1786``;
* patch solid angles          as in ``Kside_veg_v2022a`` / ``Lcyl_v2022a``
                              (``src/umep_solweig.py:737-751``, ``:973-983``);
* Perez relative luminance    ``Perez_v3``, ``src/model.py:808-958``;
* band emissivities           Martin & Berdahl ``model2``, ``src/umep_solweig.py:509-541``;
* the exact sunlit/shaded
  wall-patch thresholds       ``shaded_or_sunlit``, ``src/umep_solweig.py:1362-1397``.

The shaded/sunlit test of the reference is ``atan(tan(asvf) + yi) * 180/pi``
compared with the patch altitude.  ``arctan_thresholds`` turns it into two
float64 thresholds on ``x = tan(asvf) + yi`` found by bisection over the
doubles with numpy's own ``arctan``, so the device decides every pixel with
two comparisons and no transcendental call, and still agrees with numpy.
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np

__all__ = [
    "PatchLayout", "create_patches", "patch_layout", "perez", "band_emissivity",
    "arctan_thresholds",
]

_D2R = np.pi / 180
_R2D = 180 / np.pi

# (band edges, band altitudes, azimuth start, patches per band), per option.
_LAYOUTS = {
    1: ((0, 12, 24, 36, 48, 60, 72, 84, 90), (6, 18, 30, 42, 54, 66, 78, 90),
        (0, 4, 2, 5, 8, 0, 10, 0), (30, 30, 24, 24, 18, 12, 6, 1)),
    2: ((0, 12, 24, 36, 48, 60, 72, 84, 90), (6, 18, 30, 42, 54, 66, 78, 90),
        (0, 4, 2, 5, 8, 0, 10, 0), (31, 30, 28, 24, 19, 13, 7, 1)),
    3: ((0, 12, 24, 36, 48, 60, 72, 84, 90), (6, 18, 30, 42, 54, 66, 78, 90),
        (0, 4, 2, 5, 8, 0, 10, 0), (62, 60, 56, 48, 38, 26, 14, 1)),
    4: ((0, 4.5, 9, 15, 21, 27, 33, 39, 45, 51, 57, 63, 69, 75, 81, 90),
        (3, 9, 15, 21, 27, 33, 39, 45, 51, 57, 63, 69, 75, 81, 90),
        (0, 0, 4, 4, 2, 2, 5, 5, 8, 8, 0, 0, 10, 10, 0),
        (62, 62, 60, 60, 56, 56, 48, 48, 38, 38, 26, 26, 14, 14, 1)),
}


def create_patches(patch_option):
    """Patch altitudes and azimuths in degrees (band-major order)."""
    edges, alts, starts, counts = _LAYOUTS[int(patch_option)]
    alt, azi = [], []
    for band_alt, start, count in zip(alts, starts, counts):
        step = 360 / count
        for k in range(count):
            alt.append(band_alt)
            azi.append(k * step + start)
    return (np.asarray(alt, dtype=np.float64), np.asarray(azi, dtype=np.float64),
            np.asarray(edges, dtype=np.float64), np.asarray(alts), np.asarray(counts))


class PatchLayout:
    """Static per-patch quantities of one sky-vault layout (all float64)."""

    def __init__(self, patch_option):
        alt, azi, edges, band_alt, counts = create_patches(patch_option)
        self.patch_option = int(patch_option)
        self.altitude = alt
        self.azimuth = azi
        self.count = alt.size
        self.band_edges = edges
        self.band_altitude = band_alt
        self.band_counts = counts
        self.band_of_patch = np.repeat(np.arange(counts.size), counts)
        self.band_offsets = np.r_[0, np.cumsum(counts)]
        # Solid angle of each patch (Kside_veg_v2022a / Lcyl_v2022a loop).
        uniq, uniq_counts = np.unique(alt, return_counts=True)
        omega = np.zeros(alt.size)
        for i in range(alt.size):
            n = int(uniq_counts[uniq == alt[i]][0])
            if n > 1:
                omega[i] = ((360 / n) * _D2R) * (np.sin((alt[i] + alt[0]) * _D2R)
                                                  - np.sin((alt[i] - alt[0]) * _D2R))
            else:
                omega[i] = ((360 / n) * _D2R) * (np.sin(alt[i] * _D2R)
                                                  - np.sin((alt[i - 1] + alt[0]) * _D2R))
        self.steradian = omega
        self.cos_alt = np.cos(alt * _D2R)
        self.sin_alt = np.sin(alt * _D2R)
        # Cardinal direction cosines used by the longwave per-direction sums
        # (define_patch_characteristics, src/umep_solweig.py:1262-1273).
        self.cardinal = np.column_stack([
            np.where((azi > 360) | (azi < 180), np.cos((90 - azi) * _D2R), 0.0),
            np.where((azi > 90) & (azi < 270), np.cos((180 - azi) * _D2R), 0.0),
            np.where((azi > 180) & (azi < 360), np.cos((270 - azi) * _D2R), 0.0),
            np.where((azi > 270) | (azi < 90), np.cos((0 - azi) * _D2R), 0.0),
        ])  # columns: east, south, west, north
        # Exact thresholds for shaded_or_sunlit against every patch altitude.
        self.sunlit_below, self.shaded_above = arctan_thresholds(alt)


@lru_cache(maxsize=8)
def patch_layout(patch_option):
    return PatchLayout(patch_option)


def _degrees(x):
    return np.arctan(np.float64(x)) * _R2D


def _first_at_least(target, strict):
    """Smallest positive double x with deg(x) >= target (> target if ``strict``).

    Positive doubles are ordered like their int64 bit patterns, so this is a
    bisection over integers; returns +inf when no finite x qualifies.
    """
    def ok(bits):
        v = _degrees(np.int64(bits).view(np.float64))
        return v > target if strict else v >= target

    lo = int(np.float64(0.0).view(np.int64))
    hi = int(np.float64(np.finfo(np.float64).max).view(np.int64))
    if not ok(hi):
        return np.inf
    if ok(lo):
        return 0.0
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if ok(mid):
            hi = mid
        else:
            lo = mid
    return float(np.int64(hi).view(np.float64))


def arctan_thresholds(altitudes):
    """Per-altitude thresholds (sunlit_below, shaded_above) on x = tan(asvf) + yi.

    ``x < sunlit_below``  <=>  arctan(x)*180/pi <  altitude (patch sunlit);
    ``x > shaded_above``  <=>  arctan(x)*180/pi >  altitude (patch shaded);
    values in between compare equal and are neither, as in the reference.
    Altitudes must be positive (sky patches are above the horizon).
    """
    altitudes = np.asarray(altitudes, dtype=np.float64)
    lo = np.empty(altitudes.size)
    hi = np.empty(altitudes.size)
    cache = {}
    for i, a in enumerate(altitudes):
        if a <= 0:
            raise ValueError("patch altitudes must be positive")
        if a not in cache:
            first_ge = _first_at_least(a, strict=False)
            first_gt = _first_at_least(a, strict=True)
            cache[a] = (first_ge, np.nextafter(first_gt, -np.inf))
        lo[i], hi[i] = cache[a]
    return lo, hi


def band_emissivity(esky, layout):
    """Martin & Berdahl per-patch sky emissivity (model2, unnormalised)."""
    cached = getattr(layout, "_band_index", None)
    if cached is None:
        uniq, index = np.unique(layout.altitude, return_inverse=True)
        cached = (uniq, 1 / np.cos((90 - uniq) * _D2R), index)
        layout._band_index = cached
    uniq, inv_cos, index = cached
    band = 1 - (1 - esky) * np.exp(0.308 * (1.7 - inv_cos))
    return band[index]


_PEREZ = np.array([
    # a1..a4
    [1.3525, -1.2219, -1.1000, -0.5484, -0.6000, -1.0156, -1.0000, -1.0500],
    [-0.2576, -0.7730, -0.2515, -0.6654, -0.3566, -0.3670, 0.0211, 0.0289],
    [-0.2690, 1.4148, 0.8952, -0.2672, -2.5000, 1.0078, 0.5025, 0.4260],
    [-1.4366, 1.1016, 0.0156, 0.7117, 2.3250, 1.4051, -0.5119, 0.3590],
    # b1..b4
    [-0.7670, -0.2054, 0.2782, 0.7234, 0.2937, 0.2875, -0.3000, -0.3250],
    [0.0007, 0.0367, -0.1812, -0.6219, 0.0496, -0.5328, 0.1922, 0.1156],
    [1.2734, -3.9128, -4.5000, -5.6812, -5.6812, -3.8500, 0.7023, 0.7781],
    [-0.1233, 0.9156, 1.1766, 2.6297, 1.8415, 3.3750, -1.6317, 0.0025],
    # c1..c4
    [2.8000, 6.9750, 24.7219, 33.3389, 21.0000, 14.0000, 19.0000, 31.0625],
    [0.6004, 0.1774, -13.0812, -18.3000, -4.7656, -0.9999, -5.0000, -14.5000],
    [1.2375, 6.4477, -37.7000, -62.2500, -21.5906, -7.1406, 1.2438, -46.1148],
    [1.0000, -0.1239, 34.8438, 52.0781, 7.2492, 7.5469, -1.9094, 55.3750],
    # d1..d4
    [1.8734, -1.5798, -5.0000, -3.5000, -3.5000, -3.4000, -4.0000, -7.2312],
    [0.6297, -0.5081, 1.5218, 0.0016, -0.1554, -0.1078, 0.0250, 0.4050],
    [0.9738, -1.7812, 3.9229, 1.1477, 1.4062, -1.0750, 0.3844, 13.3500],
    [0.2809, 0.1080, -2.6204, 0.1062, 0.3988, 1.5702, 0.2656, 0.6234],
    # e1..e4
    [0.0356, 0.2624, -0.0156, 0.4659, 0.0032, -0.0672, 1.0468, 1.5000],
    [-0.1246, 0.0672, 0.1597, -0.3296, 0.0766, 0.4016, -0.3788, -0.6426],
    [-0.5718, -0.2190, 0.4199, -0.0876, -0.0656, 0.3017, -2.4517, 1.8564],
    [0.9938, -0.4285, -0.5562, -0.0329, -0.1294, -0.4844, 1.4656, 0.5636],
])  # rows: coefficient (a1..e4), columns: clearness bin


def _clearness_bin(eps):
    # Strict inequalities on both sides, exactly as the reference: a value
    # equal to a bin edge keeps the previous assignment (bin 0 initially).
    edges = (1.065, 1.230, 1.500, 1.950, 2.800, 4.500, 6.200)
    b = 0
    if eps < edges[0]:
        b = 0
    for i in range(6):
        if edges[i] < eps < edges[i + 1]:
            b = i + 1
    if eps > edges[6]:
        b = 7
    return b


def perez(zen_deg, azimuth, rad_d, rad_i, jday, layout):
    """Perez (1993) relative luminance of every patch, normalised to sum 1.

    Returns an array ``(P, 3)`` of (altitude deg, azimuth deg, luminance), the
    ``lv`` of ``Perez_v3(..., patchchoice=1, patch_option)``.
    """
    altitude = (90 - zen_deg) * _D2R
    zen = zen_deg * _D2R
    az = azimuth * _D2R
    eps = ((rad_d + rad_i) / (rad_d + 1.041 * np.power(zen, 3))) / (1 + 1.041 * np.power(zen, 3))
    day_angle = jday * 2 * np.pi / 365
    i0 = 1367 * (1.00011 + 0.034221 * np.cos(day_angle) + 0.00128 * np.sin(day_angle)
                 + 0.000719 * np.cos(2 * day_angle) + 0.000077 * np.sin(2 * day_angle))
    if altitude >= 10 * _D2R:
        airmass = 1 / np.sin(altitude)
    elif altitude < 0:
        airmass = 1 / np.sin(altitude) + 0.50572 * np.power(180 * complex(altitude) / np.pi + 6.07995, -1.6364)
    else:
        airmass = 1 / np.sin(altitude) + 0.50572 * np.power(180 * altitude / np.pi + 6.07995, -1.6364)
    delta = (airmass * rad_d) / i0
    if rad_d <= 10:
        delta = 0
    b = _clearness_bin(eps)
    c = _PEREZ[:, b]

    def coef(j):
        return c[4 * j] + c[4 * j + 1] * zen + delta * (c[4 * j + 2] + c[4 * j + 3] * zen)

    m_a, m_b, m_e = coef(0), coef(1), coef(4)
    if b > 0:
        m_c, m_d = coef(2), coef(3)
    else:
        m_c = np.exp(np.power(delta * (c[8] + c[9] * zen), c[10])) - 1
        m_d = -np.exp(delta * (c[12] + c[13] * zen)) + c[14] + delta * c[15] * delta
    p_alt, p_azi = layout.altitude, layout.azimuth
    sv_zen = (90 - p_alt) * _D2R
    sv_alt = p_alt * _D2R
    sv_azi = p_azi * _D2R
    cos_ss = np.sin(sv_alt) * np.sin(altitude) + np.cos(altitude) * np.cos(sv_alt) * np.cos(np.abs(sv_azi - az))
    cos_ss = np.clip(cos_ss, -1.0, 1.0)
    lv = (1 + m_a * np.exp(m_b / np.cos(sv_zen))) * ((1 + m_c * np.exp(m_d * np.arccos(cos_ss))
                                                      + m_e * cos_ss * cos_ss))
    lv = lv / np.sum(lv)
    lv = np.real(lv).astype(np.float64) if np.iscomplexobj(lv) else lv
    return np.column_stack((sv_alt * _R2D, sv_azi * _R2D, lv))
