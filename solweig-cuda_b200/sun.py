"""Host-side FP64 solar geometry for the per-hour SOLWEIG step.

This module restates, in float64 numpy, the sun-position chain that the
reference runs on the host before every hour:

* ``sun_position``          NREL SPA (Reda & Andreas, NREL/TP-560-34302) as
                            retained by UMEP, ``src/umep_solweig.py:2529-3518``
                            (fixed refraction at 1010 mbar / 283 K, delta_t = 0);
* ``metdata``               ``Solweig_2015a_metdata_noload``,
                            ``src/umep_solweig.py:2412-2503`` (sun sampled at the
                            forcing time minus half a step, zenith clamp at 89
                            degrees, 15-minute daily altmax search from 10:00);
* ``daylen``                ``src/umep_solweig.py:430-448``;
* ``clearness_index``       ``clearnessindex_2013b``, ``src/umep_solweig.py:1654-1734``;
* ``diffuse_fraction``      ``diffusefraction``, ``src/umep_solweig.py:1789-1832``;
* ``sun_distance``          ``src/umep_solweig.py:2513-2523``.

Everything here is scalar FP64 work of well under a millisecond per hour; the
per-pixel work happens in the CUDA library.  The periodic-term tables are the
published SPA tables (they must be identical for the ephemeris to agree), laid
out as ``(amplitude, phase, frequency)`` rows in the published order so that
``np.sum`` reduces them in the same order as the reference.  Where the
reference's copy of a table differs from the publication, the reference's
value is kept (the goal is agreement with the reference's sun vectors): L0
row 26 phase 2.4458, L0 row 41 amplitude 71, L1 row 28 frequency 3286.6, R0
row 21 amplitude 85 and R2 row 6 frequency 18849.
"""
from __future__ import annotations

import calendar
import datetime as _dt
import math

import numpy as np

__all__ = [
    "sun_position", "metdata", "daylen", "clearness_index", "diffuse_fraction",
    "sun_distance", "SolarHours",
]

_D2R = np.pi / 180.0

# ----------------------------------------------------------------------------
# SPA periodic terms (A, B, C): term = A * cos(B + C * JME)
# ----------------------------------------------------------------------------
_L0 = np.array([
    [175347046.0, 0.0, 0.0], [3341656.0, 4.6692568, 6283.07585], [34894.0, 4.6261, 12566.1517],
    [3497.0, 2.7441, 5753.3849], [3418.0, 2.8289, 3.5231], [3136.0, 3.6277, 77713.7715],
    [2676.0, 4.4181, 7860.4194], [2343.0, 6.1352, 3930.2097], [1324.0, 0.7425, 11506.7698],
    [1273.0, 2.0371, 529.691], [1199.0, 1.1096, 1577.3435], [990.0, 5.233, 5884.927],
    [902.0, 2.045, 26.298], [857.0, 3.508, 398.149], [780.0, 1.179, 5223.694],
    [753.0, 2.533, 5507.553], [505.0, 4.583, 18849.228], [492.0, 4.205, 775.523],
    [357.0, 2.92, 0.067], [317.0, 5.849, 11790.629], [284.0, 1.899, 796.298],
    [271.0, 0.315, 10977.079], [243.0, 0.345, 5486.778], [206.0, 4.806, 2544.314],
    [205.0, 1.869, 5573.143], [202.0, 2.4458, 6069.777], [156.0, 0.833, 213.299],
    [132.0, 3.411, 2942.463], [126.0, 1.083, 20.775], [115.0, 0.645, 0.98],
    [103.0, 0.636, 4694.003], [102.0, 0.976, 15720.839], [102.0, 4.267, 7.114],
    [99.0, 6.21, 2146.17], [98.0, 0.68, 155.42], [86.0, 5.98, 161000.69],
    [85.0, 1.3, 6275.96], [85.0, 3.67, 71430.7], [80.0, 1.81, 17260.15],
    [79.0, 3.04, 12036.46], [71.0, 1.76, 5088.63], [74.0, 3.5, 3154.69],
    [74.0, 4.68, 801.82], [70.0, 0.83, 9437.76], [62.0, 3.98, 8827.39],
    [61.0, 1.82, 7084.9], [57.0, 2.78, 6286.6], [56.0, 4.39, 14143.5],
    [56.0, 3.47, 6279.55], [52.0, 0.19, 12139.55], [52.0, 1.33, 1748.02],
    [51.0, 0.28, 5856.48], [49.0, 0.49, 1194.45], [41.0, 5.37, 8429.24],
    [41.0, 2.4, 19651.05], [39.0, 6.17, 10447.39], [37.0, 6.04, 10213.29],
    [37.0, 2.57, 1059.38], [36.0, 1.71, 2352.87], [36.0, 1.78, 6812.77],
    [33.0, 0.59, 17789.85], [30.0, 0.44, 83996.85], [30.0, 2.74, 1349.87],
    [25.0, 3.16, 4690.48]])
_L1 = np.array([
    [628331966747.0, 0.0, 0.0], [206059.0, 2.678235, 6283.07585], [4303.0, 2.6351, 12566.1517],
    [425.0, 1.59, 3.523], [119.0, 5.796, 26.298], [109.0, 2.966, 1577.344],
    [93.0, 2.59, 18849.23], [72.0, 1.14, 529.69], [68.0, 1.87, 398.15],
    [67.0, 4.41, 5507.55], [59.0, 2.89, 5223.69], [56.0, 2.17, 155.42],
    [45.0, 0.4, 796.3], [36.0, 0.47, 775.52], [29.0, 2.65, 7.11],
    [21.0, 5.34, 0.98], [19.0, 1.85, 5486.78], [19.0, 4.97, 213.3],
    [17.0, 2.99, 6275.96], [16.0, 0.03, 2544.31], [16.0, 1.43, 2146.17],
    [15.0, 1.21, 10977.08], [12.0, 2.83, 1748.02], [12.0, 3.26, 5088.63],
    [12.0, 5.27, 1194.45], [12.0, 2.08, 4694.0], [11.0, 0.77, 553.57],
    [10.0, 1.3, 3286.6], [10.0, 4.24, 1349.87], [9.0, 2.7, 242.73],
    [9.0, 5.64, 951.72], [8.0, 5.3, 2352.87], [6.0, 2.65, 9437.76],
    [6.0, 4.67, 4690.48]])
_L2 = np.array([
    [52919.0, 0.0, 0.0], [8720.0, 1.0721, 6283.0758], [309.0, 0.867, 12566.152],
    [27.0, 0.05, 3.52], [16.0, 5.19, 26.3], [16.0, 3.68, 155.42],
    [10.0, 0.76, 18849.23], [9.0, 2.06, 77713.77], [7.0, 0.83, 775.52],
    [5.0, 4.66, 1577.34], [4.0, 1.03, 7.11], [4.0, 3.44, 5573.14],
    [3.0, 5.14, 796.3], [3.0, 6.05, 5507.55], [3.0, 1.19, 242.73],
    [3.0, 6.12, 529.69], [3.0, 0.31, 398.15], [3.0, 2.28, 553.57],
    [2.0, 4.38, 5223.69], [2.0, 3.75, 0.98]])
_L3 = np.array([
    [289.0, 5.844, 6283.076], [35.0, 0.0, 0.0], [17.0, 5.49, 12566.15],
    [3.0, 5.2, 155.42], [1.0, 4.72, 3.52], [1.0, 5.3, 18849.23],
    [1.0, 5.97, 242.73]])
_L4 = np.array([[114.0, 3.142, 0.0], [8.0, 4.13, 6283.08], [1.0, 3.84, 12566.15]])
_L5 = np.array([[1.0, 3.14, 0.0]])
_B0 = np.array([
    [280.0, 3.199, 84334.662], [102.0, 5.422, 5507.553], [80.0, 3.88, 5223.69],
    [44.0, 3.7, 2352.87], [32.0, 4.0, 1577.34]])
_B1 = np.array([[9.0, 3.9, 5507.55], [6.0, 1.73, 5223.69]])
_R0 = np.array([
    [100013989.0, 0.0, 0.0], [1670700.0, 3.0984635, 6283.07585], [13956.0, 3.05525, 12566.1517],
    [3084.0, 5.1985, 77713.7715], [1628.0, 1.1739, 5753.3849], [1576.0, 2.8469, 7860.4194],
    [925.0, 5.453, 11506.77], [542.0, 4.564, 3930.21], [472.0, 3.661, 5884.927],
    [346.0, 0.964, 5507.553], [329.0, 5.9, 5223.694], [307.0, 0.299, 5573.143],
    [243.0, 4.273, 11790.629], [212.0, 5.847, 1577.344], [186.0, 5.022, 10977.079],
    [175.0, 3.012, 18849.228], [110.0, 5.055, 5486.778], [98.0, 0.89, 6069.78],
    [86.0, 5.69, 15720.84], [86.0, 1.27, 161000.69], [85.0, 0.27, 17260.15],
    [63.0, 0.92, 529.69], [57.0, 2.01, 83996.85], [56.0, 5.24, 71430.7],
    [49.0, 3.25, 2544.31], [47.0, 2.58, 775.52], [45.0, 5.54, 9437.76],
    [43.0, 6.01, 6275.96], [39.0, 5.36, 4694.0], [38.0, 2.39, 8827.39],
    [37.0, 0.83, 19651.05], [37.0, 4.9, 12139.55], [36.0, 1.67, 12036.46],
    [35.0, 1.84, 2942.46], [33.0, 0.24, 7084.9], [32.0, 0.18, 5088.63],
    [32.0, 1.78, 398.15], [28.0, 1.21, 6286.6], [28.0, 1.9, 6279.55],
    [26.0, 4.59, 10447.39]])
_R1 = np.array([
    [103019.0, 1.10749, 6283.07585], [1721.0, 1.0644, 12566.1517], [702.0, 3.142, 0.0],
    [32.0, 1.02, 18849.23], [31.0, 2.84, 5507.55], [25.0, 1.32, 5223.69],
    [18.0, 1.42, 1577.34], [10.0, 5.91, 10977.08], [9.0, 1.42, 6275.96],
    [9.0, 0.27, 5486.78]])
_R2 = np.array([
    [4359.0, 5.7846, 6283.0758], [124.0, 5.579, 12566.152], [12.0, 3.14, 0.0],
    [9.0, 3.63, 77713.77], [6.0, 1.87, 5573.14], [3.0, 5.47, 18849.0]])
_R3 = np.array([[145.0, 4.273, 6283.076], [7.0, 3.92, 12566.15]])
_R4 = np.array([[4.0, 2.56, 6283.08]])

# Nutation: argument multipliers of (X0..X4) and (a, b, c, d) coefficients.
_NUT_Y = np.array([
    [0, 0, 0, 0, 1], [-2, 0, 0, 2, 2], [0, 0, 0, 2, 2], [0, 0, 0, 0, 2], [0, 1, 0, 0, 0],
    [0, 0, 1, 0, 0], [-2, 1, 0, 2, 2], [0, 0, 0, 2, 1], [0, 0, 1, 2, 2], [-2, -1, 0, 2, 2],
    [-2, 0, 1, 0, 0], [-2, 0, 0, 2, 1], [0, 0, -1, 2, 2], [2, 0, 0, 0, 0], [0, 0, 1, 0, 1],
    [2, 0, -1, 2, 2], [0, 0, -1, 0, 1], [0, 0, 1, 2, 1], [-2, 0, 2, 0, 0], [0, 0, -2, 2, 1],
    [2, 0, 0, 2, 2], [0, 0, 2, 2, 2], [0, 0, 2, 0, 0], [-2, 0, 1, 2, 2], [0, 0, 0, 2, 0],
    [-2, 0, 0, 2, 0], [0, 0, -1, 2, 1], [0, 2, 0, 0, 0], [2, 0, -1, 0, 1], [-2, 2, 0, 2, 2],
    [0, 1, 0, 0, 1], [-2, 0, 1, 0, 1], [0, -1, 0, 0, 1], [0, 0, 2, -2, 0], [2, 0, -1, 2, 1],
    [2, 0, 1, 2, 2], [0, 1, 0, 2, 2], [-2, 1, 1, 0, 0], [0, -1, 0, 2, 2], [2, 0, 0, 2, 1],
    [2, 0, 1, 0, 0], [-2, 0, 2, 2, 2], [-2, 0, 1, 2, 1], [2, 0, -2, 0, 1], [2, 0, 0, 0, 1],
    [0, -1, 1, 0, 0], [-2, -1, 0, 2, 1], [-2, 0, 0, 0, 1], [0, 0, 2, 2, 1], [-2, 0, 2, 0, 1],
    [-2, 1, 0, 2, 1], [0, 0, 1, -2, 0], [-1, 0, 1, 0, 0], [-2, 1, 0, 0, 0], [1, 0, 0, 0, 0],
    [0, 0, 1, 2, 0], [0, 0, -2, 2, 2], [-1, -1, 1, 0, 0], [0, 1, 1, 0, 0], [0, -1, 1, 2, 2],
    [2, -1, -1, 2, 2], [0, 0, 3, 2, 2], [2, -1, 0, 2, 2]], dtype=np.float64)
_NUT_PE = np.array([
    [-171996, -174.2, 92025, 8.9], [-13187, -1.6, 5736, -3.1], [-2274, -0.2, 977, -0.5],
    [2062, 0.2, -895, 0.5], [1426, -3.4, 54, -0.1], [712, 0.1, -7, 0],
    [-517, 1.2, 224, -0.6], [-386, -0.4, 200, 0], [-301, 0, 129, -0.1],
    [217, -0.5, -95, 0.3], [-158, 0, 0, 0], [129, 0.1, -70, 0], [123, 0, -53, 0],
    [63, 0, 0, 0], [63, 0.1, -33, 0], [-59, 0, 26, 0], [-58, -0.1, 32, 0],
    [-51, 0, 27, 0], [48, 0, 0, 0], [46, 0, -24, 0], [-38, 0, 16, 0], [-31, 0, 13, 0],
    [29, 0, 0, 0], [29, 0, -12, 0], [26, 0, 0, 0], [-22, 0, 0, 0], [21, 0, -10, 0],
    [17, -0.1, 0, 0], [16, 0, -8, 0], [-16, 0.1, 7, 0], [-15, 0, 9, 0], [-13, 0, 7, 0],
    [-12, 0, 6, 0], [11, 0, 0, 0], [-10, 0, 5, 0], [-8, 0, 3, 0], [7, 0, -3, 0],
    [-7, 0, 0, 0], [-7, 0, 3, 0], [-7, 0, 3, 0], [6, 0, 0, 0], [6, 0, -3, 0],
    [6, 0, -3, 0], [-6, 0, 3, 0], [-6, 0, 3, 0], [5, 0, 0, 0], [-5, 0, 3, 0],
    [-5, 0, 3, 0], [-5, 0, 3, 0], [4, 0, 0, 0], [4, 0, 0, 0], [4, 0, 0, 0],
    [-4, 0, 0, 0], [-4, 0, 0, 0], [-4, 0, 0, 0], [3, 0, 0, 0], [-3, 0, 0, 0],
    [-3, 0, 0, 0], [-3, 0, 0, 0], [-3, 0, 0, 0], [-3, 0, 0, 0], [-3, 0, 0, 0],
    [-3, 0, 0, 0]], dtype=np.float64)

# (cubic, quadratic, linear, constant) coefficients of the five nutation arguments.
_NUT_X = (
    ((1 / 189474), -0.0019142, 445267.11148, 297.85036),
    (-(1 / 300000), -0.0001603, 35999.05034, 357.52772),
    ((1 / 56250), 0.0086972, 477198.867398, 134.96298),
    ((1 / 327270), -0.0036825, 483202.017538, 93.27191),
    ((1 / 450000), 0.0020708, -1934.136261, 125.04452),
)
_OBLIQUITY = (2.45, 5.79, 27.87, 7.12, -39.05, -249.67, -51.38, 1999.25, -1.55, -4680.93, 84381.448)


def _wrap(value, period):
    """Reduce into [0, period) the way the SPA port does (floor-based)."""
    value = value - period * np.floor(value / period)
    if value < 0:
        value = value + period
    return value


def _series(table, jme):
    return np.sum(table[:, 0] * np.cos(table[:, 1] + (table[:, 2] * jme)))


def _julian(year, month, day, hour, minute, second, utc):
    """Julian day and centuries (delta_t = 0), Gregorian calendar after 1582."""
    if month in (1, 2):
        y, m = year - 1, month + 12
    else:
        y, m = year, month
    ut = ((hour - utc) / 24) + (minute / (60 * 24)) + (second / (60 * 60 * 24))
    d = day + ut
    if year < 1582 or (year == 1582 and (month < 10 or (month == 10 and day <= 4))):
        b = 0
    else:
        a = np.floor(y / 100)
        b = 2 - a + np.floor(a / 4)
    jd = d + b + np.floor(365.25 * (y + 4716)) + np.floor(30.6001 * (m + 1)) - 1524.5
    jc = (jd - 2451545) / 36525
    jce = jc
    jme = jce / 10
    return jd, jc, jce, jme


def sun_position(year, month, day, hour, minute, second, utc, latitude, longitude, altitude):
    """Topocentric sun zenith and azimuth in degrees (NREL SPA, UMEP variant).

    Follows ``sun_position`` at ``src/umep_solweig.py:2529-2677``: delta_t = 0,
    atmospheric refraction for 1010 mbar and 283 K applied unconditionally.
    Returns ``(zenith_deg, azimuth_deg)``.
    """
    jd, jc, jce, jme = _julian(year, month, day, hour, minute, second, utc)
    # Earth heliocentric longitude / latitude / radius.
    l_terms = [_series(t, jme) for t in (_L0, _L1, _L2, _L3, _L4)]
    l5 = _L5[:, 0] * np.cos(_L5[:, 1] + (_L5[:, 2] * jme))
    helio_lon = (l_terms[0] + (l_terms[1] * jme) + (l_terms[2] * np.power(jme, 2))
                 + (l_terms[3] * np.power(jme, 3)) + (l_terms[4] * np.power(jme, 4))
                 + (l5 * np.power(jme, 5))) / 1e8
    helio_lon = _wrap(float(np.asarray(helio_lon).item()) * 180 / np.pi, 360)
    b0, b1 = _series(_B0, jme), _series(_B1, jme)
    helio_lat = _wrap(((b0 + (b1 * jme)) / 1e8) * 180 / np.pi, 360)
    r_terms = [_series(t, jme) for t in (_R0, _R1, _R2, _R3)]
    r4 = _R4[:, 0] * np.cos(_R4[:, 1] + (_R4[:, 2] * jme))
    radius = float(np.asarray((r_terms[0] + (r_terms[1] * jme) + (r_terms[2] * np.power(jme, 2))
                               + (r_terms[3] * np.power(jme, 3)) + (r4 * np.power(jme, 4))) / 1e8).item())
    # Geocentric position.
    geo_lon = _wrap(helio_lon + 180, 360)
    geo_lat = _wrap(-helio_lat, 360)
    # Nutation.
    x = np.array([c3 * np.power(jce, 3) + c2 * np.power(jce, 2) + c1 * jce + c0
                  for (c3, c2, c1, c0) in _NUT_X])
    arg = _NUT_Y.dot(np.transpose(x)) * (np.pi / 180)
    d_psi = np.sum((_NUT_PE[:, 0] + (_NUT_PE[:, 1] * jce)) * np.sin(arg)) / 36000000
    d_eps = np.sum((_NUT_PE[:, 2] + (_NUT_PE[:, 3] * jce)) * np.cos(arg)) / 36000000
    # True obliquity.
    u = jme / 10
    p = _OBLIQUITY
    eps0 = (p[0] * np.power(u, 10) + p[1] * np.power(u, 9) + p[2] * np.power(u, 8)
            + p[3] * np.power(u, 7) + p[4] * np.power(u, 6) + p[5] * np.power(u, 5)
            + p[6] * np.power(u, 4) + p[7] * np.power(u, 3) + p[8] * np.power(u, 2)
            + p[9] * u + p[10])
    eps = (eps0 / 3600) + d_eps
    aberration = -20.4898 / (3600 * radius)
    lam = geo_lon + d_psi + aberration
    nu0 = (280.46061837 + (360.98564736629 * (jd - 2451545)) + (0.000387933 * np.power(jc, 2))
           - (np.power(jc, 3) / 38710000))
    nu0 = _wrap(nu0, 360)
    nu = nu0 + (d_psi * np.cos(eps * np.pi / 180))
    num = (np.sin(lam * np.pi / 180) * np.cos(eps * np.pi / 180)) - \
          (np.tan(geo_lat * np.pi / 180) * np.sin(eps * np.pi / 180))
    alpha = _wrap(np.arctan2(num, np.cos(lam * np.pi / 180)) * 180 / np.pi, 360)
    delta = np.arcsin((np.sin(geo_lat * np.pi / 180) * np.cos(eps * np.pi / 180))
                      + (np.cos(geo_lat * np.pi / 180) * np.sin(eps * np.pi / 180)
                         * np.sin(lam * np.pi / 180))) * 180 / np.pi
    hour_angle = _wrap(nu + longitude - alpha, 360)
    # Topocentric correction.
    xi = 8.794 / (3600 * radius)
    uu = np.arctan(0.99664719 * np.tan(latitude * np.pi / 180))
    xx = np.cos(uu) + ((altitude / 6378140) * np.cos(latitude * np.pi / 180))
    yy = (0.99664719 * np.sin(uu)) + ((altitude / 6378140) * np.sin(latitude * np.pi / 180))
    d_alpha = np.arctan2(-xx * np.sin(xi * np.pi / 180) * np.sin(hour_angle * np.pi / 180),
                         np.cos(delta * np.pi / 180)
                         - (xx * np.sin(xi * np.pi / 180) * np.cos(hour_angle * np.pi / 180)))
    delta_t = np.arctan2((np.sin(delta * np.pi / 180) - (yy * np.sin(xi * np.pi / 180))) * np.cos(d_alpha),
                         np.cos(delta * np.pi / 180)
                         - (yy * np.sin(xi * np.pi / 180)) * np.cos(hour_angle * np.pi / 180)) * 180 / np.pi
    h_t = hour_angle - d_alpha * 180 / np.pi
    e0 = np.arcsin((np.sin(latitude * np.pi / 180) * np.sin(delta_t * np.pi / 180))
                   + (np.cos(latitude * np.pi / 180) * np.cos(delta_t * np.pi / 180)
                      * np.cos(h_t * np.pi / 180))) * 180 / np.pi
    refraction = 1.02 / (60 * np.tan((e0 + (10.3 / (e0 + 5.11))) * np.pi / 180))
    zenith = 90 - (e0 + refraction)
    azimuth = (np.arctan2(np.sin(h_t * np.pi / 180),
                          (np.cos(h_t * np.pi / 180) * np.sin(latitude * np.pi / 180))
                          - (np.tan(delta_t * np.pi / 180) * np.cos(latitude * np.pi / 180)))
               * 180 / np.pi) + 180
    azimuth = _wrap(azimuth, 360)
    return float(np.asarray(zenith).item()), float(np.asarray(azimuth).item())


def sun_distance(jday):
    """Relative Earth-Sun distance (Partridge & Platt), ``src/umep_solweig.py:2513-2523``."""
    b = 2. * np.pi * jday / 365.
    return np.sqrt((1.00011 + np.dot(0.034221, np.cos(b)) + np.dot(0.001280, np.sin(b))
                    + np.dot(0.000719, np.cos((2. * b))) + np.dot(0.000077, np.sin((2. * b)))))


def daylen(doy, latitude):
    """(daylength, declination, sunset, sunrise) hours, ``src/umep_solweig.py:430-448``."""
    dec = -23.45 * np.cos(2.0 * np.pi * (doy + 10.0) / 365.0)
    soc = np.tan(_D2R * dec) * np.tan(_D2R * latitude)
    soc = min(max(soc, -1.0), 1.0)
    dayl = 12.0 + 24.0 * np.arcsin(soc) / np.pi
    return dayl, dec, 12.0 + dayl / 2.0, 12.0 - dayl / 2.0


_G_BY_LATITUDE = (
    (10., (3.37, 2.85, 2.80, 2.64)), (20., (2.99, 3.02, 2.70, 2.93)),
    (30., (3.60, 3.00, 2.98, 2.93)), (40., (3.04, 3.11, 2.92, 2.94)),
    (50., (2.70, 2.95, 2.77, 2.71)), (60., (2.52, 3.07, 2.67, 2.93)),
    (70., (1.76, 2.69, 2.61, 2.61)), (80., (1.60, 1.67, 2.24, 2.63)),
    (90., (1.11, 1.44, 1.94, 2.02)),
)


def clearness_index(zen, jday, ta, rh_fraction, rad_g, latitude, p_kpa):
    """Crawford & Duchon clearness index, ``src/umep_solweig.py:1654-1734``.

    ``zen`` in radians, ``rh_fraction`` in [0, 1], ``p_kpa`` the forcing pressure
    (kPa, -999 for missing).  Returns ``(I0, CI, Kt, I0et, CIuncorr)``.
    """
    p = 1013. if p_kpa == -999.0 else p_kpa * 10.
    itoa = 1370.0
    d = sun_distance(jday)
    m = 35. * np.cos(zen) * ((1224. * (np.cos(zen) ** 2) + 1) ** (-1 / 2.))
    trpg = 1.021 - 0.084 * (m * (0.000949 * p + 0.051)) ** 0.5
    g4 = None
    for bound, values in _G_BY_LATITUDE:
        if latitude < bound:
            g4 = values
            break
    if jday > 335 or jday <= 60:
        g = g4[0]
    elif jday <= 152:
        g = g4[1]
    elif jday <= 244:
        g = g4[2]
    else:
        g = g4[3]
    a2, b2 = 17.27, 237.7
    td = (b2 * (((a2 * ta) / (b2 + ta)) + np.log(rh_fraction))) / (a2 - (((a2 * ta) / (b2 + ta)) + np.log(rh_fraction)))
    td = (td * 1.8) + 32
    u = np.exp(0.1133 - np.log(g + 1) + 0.0393 * td)
    tw = 1 - 0.077 * ((u * m) ** 0.3)
    tar = 0.935 ** m
    i0 = itoa * np.cos(zen) * trpg * tw * d * tar
    if abs(zen) > np.pi / 2:
        i0 = 0
    if not np.isreal(i0):
        i0 = 0
    corr = 0.1473 * np.log(90 - (zen / np.pi * 180)) + 0.3454
    with np.errstate(divide='ignore', invalid='ignore'):
        ci_uncorr = np.float64(rad_g) / np.float64(i0)
    ci = ci_uncorr + (1 - corr)
    i0et = itoa * np.cos(zen) * d
    kt = rad_g / i0et
    if math.isnan(ci):
        ci = float('inf')
    return i0, ci, kt, i0et, ci_uncorr


def diffuse_fraction(rad_g, altitude, kt, ta, rh):
    """Reindl et al. (1990) direct/diffuse split, ``src/umep_solweig.py:1789-1832``.

    Returns ``(radI, radD)``; ``rh`` in percent.
    """
    alfa = altitude * (np.pi / 180)
    if ta <= -999.00 or rh <= -999.00 or np.isnan(ta) or np.isnan(rh):
        if kt <= 0.3:
            rad_d = rad_g * (1.020 - 0.248 * kt)
        elif kt < 0.78:
            rad_d = rad_g * (1.45 - 1.67 * kt)
        else:
            rad_d = rad_g * 0.147
    else:
        rhf = rh / 100
        if kt <= 0.3:
            rad_d = rad_g * (1 - 0.232 * kt + 0.0239 * np.sin(alfa) - 0.000682 * ta + 0.0195 * rhf)
        elif kt < 0.78:
            rad_d = rad_g * (1.329 - 1.716 * kt + 0.267 * np.sin(alfa) - 0.00357 * ta + 0.106 * rhf)
        else:
            rad_d = rad_g * (0.426 * kt - 0.256 * np.sin(alfa) + 0.00349 * ta + 0.0734 * rhf)
    rad_i = (rad_g - rad_d) / (np.sin(alfa))
    if rad_i < 0:
        rad_i = 0
    if altitude < 1 and rad_i > rad_g:
        rad_i = rad_g
    if rad_d > rad_g:
        rad_d = rad_g
    return rad_i, rad_d


class SolarHours:
    """Per-hour sun geometry for a block of forcing rows (all FP64, host side).

    Attributes mirror the tuple of ``Solweig_2015a_metdata_noload``:
    ``altitude``, ``azimuth`` (degrees), ``zen`` (radians), ``jday``,
    ``dectime`` and ``altmax`` are 1-D float64 arrays, one entry per row.
    """

    __slots__ = ("year", "altitude", "azimuth", "zen", "jday", "leafon", "dectime", "altmax")

    def __init__(self, **fields):
        for name in self.__slots__:
            setattr(self, name, fields[name])


def _datetime_fields(stamp):
    return stamp.year, stamp.month, stamp.day, stamp.hour, stamp.minute


def metdata(met, latitude, longitude, site_altitude, utc):
    """Sun position for every forcing row, ``src/umep_solweig.py:2412-2503``.

    ``met`` is the (rows, 24) UMEP forcing table.  The sun is evaluated at the
    forcing time minus half the forcing step; ``altmax`` is the maximum solar
    altitude of the calendar day found by a 15-minute search starting at
    10:15 local time; zenith angles in (89, 90] degrees are clamped to 89.
    All sun positions of the table (rows and altmax candidates) go through one
    vectorised SPA evaluation.
    """
    met = np.asarray(met, dtype=np.float64)
    n = met.shape[0]
    dectime = met[:, 1] + met[:, 2] / 24 + met[:, 3] / (60 * 24.)
    half = 0 if n == 1 else (dectime[1] - dectime[0]) / 2.
    out = {k: np.empty(n) for k in ("year", "altitude", "azimuth", "zen", "jday", "leafon", "altmax")}
    day0s = [_dt.datetime(int(met[i, 0]), 1, 1) + _dt.timedelta(int(met[i, 1]) - 1) for i in range(n)]
    starts = [i for i in range(n) if i == 0 or np.mod(dectime[i], np.floor(dectime[i])) == 0]
    K = 24  # 15-minute candidates after 10:00 evaluated up front (6 h); more on demand

    def candidates(i, k0, k1):
        out, fifteen = [], 0.
        for k in range(k1):
            fifteen = fifteen + 15. / 1440.
            if k >= k0:
                out.append(_datetime_fields(day0s[i] + _dt.timedelta(days=(60 * 10) / 1440.0 + fifteen)))
        return out

    fields = []
    for i in starts:
        fields += candidates(i, 0, K)
    for i in range(n):
        stamp = (day0s[i] + _dt.timedelta(hours=met[i, 2]) + _dt.timedelta(minutes=met[i, 3])
                 - _dt.timedelta(days=half))
        fields.append(_datetime_fields(stamp))
    f = np.asarray(fields, dtype=np.int64)
    zen_all, azi_all = sun_positions(f[:, 0], f[:, 1], f[:, 2], f[:, 3], f[:, 4], utc, latitude,
                                     longitude, site_altitude)
    altmax_of = {}
    for s_i, i in enumerate(starts):
        zc = list(zen_all[s_i * K:(s_i + 1) * K])
        sunmaximum, zenith_max = -90., 90.
        k = 0
        while sunmaximum <= 90. - zenith_max:
            sunmaximum = 90. - zenith_max
            if k == len(zc):  # the next block of 15-minute candidates
                g = np.asarray(candidates(i, len(zc), len(zc) + K), dtype=np.int64)
                zc += list(sun_positions(g[:, 0], g[:, 1], g[:, 2], g[:, 3], g[:, 4], utc, latitude,
                                         longitude, site_altitude)[0])
            zenith_max = float(zc[k])
            k += 1
        altmax_of[i] = sunmaximum
    base = len(starts) * K
    current = None
    for i in range(n):
        if i in altmax_of:
            current = altmax_of[i]
        out["altmax"][i] = current
        zenith = float(zen_all[base + i])
        azimuth = float(azi_all[base + i])
        if 89.0 < zenith <= 90.0:
            zenith = 89.0
        out["altitude"][i] = 90. - zenith
        out["azimuth"][i] = azimuth
        out["zen"][i] = zenith * (np.pi / 180.)
        out["year"][i] = met[i, 0]
        doy = day0s[i].timetuple().tm_yday
        out["jday"][i] = doy
        out["leafon"][i] = 1 if (doy > 97) | (doy < 300) else 0
    return SolarHours(dectime=dectime, **out)


def _series_rows(table, jme):
    """Row-wise periodic-term sums for a vector of JME (one row per time)."""
    return np.sum(table[None, :, 0] * np.cos(table[None, :, 1] + (table[None, :, 2] * jme[:, None])), axis=1)


def _wrap_vec(value, period):
    value = value - period * np.floor(value / period)
    return np.where(value < 0, value + period, value)


def _julian_vec(year, month, day, hour, minute, utc):
    year = np.asarray(year, dtype=np.int64)
    month = np.asarray(month, dtype=np.int64)
    early = (month == 1) | (month == 2)
    y = np.where(early, year - 1, year).astype(np.float64)
    m = np.where(early, month + 12, month).astype(np.float64)
    ut = ((np.asarray(hour, dtype=np.float64) - utc) / 24) + (np.asarray(minute, dtype=np.float64) / (60 * 24)) + (0 / (60 * 60 * 24))
    d = np.asarray(day, dtype=np.float64) + ut
    a = np.floor(y / 100)
    b = 2 - a + np.floor(a / 4)
    julian_cal = (year < 1582) | ((year == 1582) & ((month < 10) | ((month == 10) & (np.asarray(day) <= 4))))
    b = np.where(julian_cal, 0.0, b)
    jd = d + b + np.floor(365.25 * (y + 4716)) + np.floor(30.6001 * (m + 1)) - 1524.5
    jc = (jd - 2451545) / 36525
    return jd, jc, jc, jc / 10


def sun_positions(year, month, day, hour, minute, utc, latitude, longitude, altitude):
    """Vectorised :func:`sun_position` over arrays of calendar fields.

    Same operations as the scalar version, row by row; the periodic-term sums
    reduce along the contiguous axis, so they use the same summation order.
    """
    jd, jc, jce, jme = _julian_vec(year, month, day, hour, minute, utc)
    l_terms = [_series_rows(t, jme) for t in (_L0, _L1, _L2, _L3, _L4)]
    l5 = _L5[0, 0] * np.cos(_L5[0, 1] + (_L5[0, 2] * jme))
    helio_lon = (l_terms[0] + (l_terms[1] * jme) + (l_terms[2] * np.power(jme, 2))
                 + (l_terms[3] * np.power(jme, 3)) + (l_terms[4] * np.power(jme, 4))
                 + (l5 * np.power(jme, 5))) / 1e8
    helio_lon = _wrap_vec(helio_lon * 180 / np.pi, 360)
    b0, b1 = _series_rows(_B0, jme), _series_rows(_B1, jme)
    helio_lat = _wrap_vec(((b0 + (b1 * jme)) / 1e8) * 180 / np.pi, 360)
    r_terms = [_series_rows(t, jme) for t in (_R0, _R1, _R2, _R3)]
    r4 = _R4[0, 0] * np.cos(_R4[0, 1] + (_R4[0, 2] * jme))
    radius = (r_terms[0] + (r_terms[1] * jme) + (r_terms[2] * np.power(jme, 2))
              + (r_terms[3] * np.power(jme, 3)) + (r4 * np.power(jme, 4))) / 1e8
    geo_lon = _wrap_vec(helio_lon + 180, 360)
    geo_lat = _wrap_vec(-helio_lat, 360)
    x = np.stack([c3 * np.power(jce, 3) + c2 * np.power(jce, 2) + c1 * jce + c0
                  for (c3, c2, c1, c0) in _NUT_X], axis=1)          # (T, 5)
    arg = x.dot(np.transpose(_NUT_Y)) * (np.pi / 180)               # (T, 63)
    d_psi = np.sum((_NUT_PE[None, :, 0] + (_NUT_PE[None, :, 1] * jce[:, None])) * np.sin(arg), axis=1) / 36000000
    d_eps = np.sum((_NUT_PE[None, :, 2] + (_NUT_PE[None, :, 3] * jce[:, None])) * np.cos(arg), axis=1) / 36000000
    u = jme / 10
    p = _OBLIQUITY
    eps0 = (p[0] * np.power(u, 10) + p[1] * np.power(u, 9) + p[2] * np.power(u, 8)
            + p[3] * np.power(u, 7) + p[4] * np.power(u, 6) + p[5] * np.power(u, 5)
            + p[6] * np.power(u, 4) + p[7] * np.power(u, 3) + p[8] * np.power(u, 2)
            + p[9] * u + p[10])
    eps = (eps0 / 3600) + d_eps
    aberration = -20.4898 / (3600 * radius)
    lam = geo_lon + d_psi + aberration
    nu0 = (280.46061837 + (360.98564736629 * (jd - 2451545)) + (0.000387933 * np.power(jc, 2))
           - (np.power(jc, 3) / 38710000))
    nu0 = _wrap_vec(nu0, 360)
    nu = nu0 + (d_psi * np.cos(eps * np.pi / 180))
    num = (np.sin(lam * np.pi / 180) * np.cos(eps * np.pi / 180)) - \
          (np.tan(geo_lat * np.pi / 180) * np.sin(eps * np.pi / 180))
    alpha = _wrap_vec(np.arctan2(num, np.cos(lam * np.pi / 180)) * 180 / np.pi, 360)
    delta = np.arcsin((np.sin(geo_lat * np.pi / 180) * np.cos(eps * np.pi / 180))
                      + (np.cos(geo_lat * np.pi / 180) * np.sin(eps * np.pi / 180)
                         * np.sin(lam * np.pi / 180))) * 180 / np.pi
    hour_angle = _wrap_vec(nu + longitude - alpha, 360)
    xi = 8.794 / (3600 * radius)
    uu = np.arctan(0.99664719 * np.tan(latitude * np.pi / 180))
    xx = np.cos(uu) + ((altitude / 6378140) * np.cos(latitude * np.pi / 180))
    yy = (0.99664719 * np.sin(uu)) + ((altitude / 6378140) * np.sin(latitude * np.pi / 180))
    d_alpha = np.arctan2(-xx * np.sin(xi * np.pi / 180) * np.sin(hour_angle * np.pi / 180),
                         np.cos(delta * np.pi / 180)
                         - (xx * np.sin(xi * np.pi / 180) * np.cos(hour_angle * np.pi / 180)))
    delta_t = np.arctan2((np.sin(delta * np.pi / 180) - (yy * np.sin(xi * np.pi / 180))) * np.cos(d_alpha),
                         np.cos(delta * np.pi / 180)
                         - (yy * np.sin(xi * np.pi / 180)) * np.cos(hour_angle * np.pi / 180)) * 180 / np.pi
    h_t = hour_angle - d_alpha * 180 / np.pi
    e0 = np.arcsin((np.sin(latitude * np.pi / 180) * np.sin(delta_t * np.pi / 180))
                   + (np.cos(latitude * np.pi / 180) * np.cos(delta_t * np.pi / 180)
                      * np.cos(h_t * np.pi / 180))) * 180 / np.pi
    refraction = 1.02 / (60 * np.tan((e0 + (10.3 / (e0 + 5.11))) * np.pi / 180))
    zenith = 90 - (e0 + refraction)
    azimuth = (np.arctan2(np.sin(h_t * np.pi / 180),
                          (np.cos(h_t * np.pi / 180) * np.sin(latitude * np.pi / 180))
                          - (np.tan(delta_t * np.pi / 180) * np.cos(latitude * np.pi / 180)))
               * 180 / np.pi) + 180
    return zenith, _wrap_vec(azimuth, 360)
