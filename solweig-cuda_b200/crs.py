"""Projection of longitude/latitude (EPSG:4326, the GeoJSON coordinate system)
into the raster's coordinate system, for the geometry wall method.

The reference reprojects building footprints with ``rasterio.warp.
transform_geom("EPSG:4326", target_crs, geometry)`` (``src/walls.py:220``),
i.e. PROJ, which this image lacks.  The projections a city raster is
normally in are written out here:

* ``EPSG:4326`` -- longitude/latitude itself (identity);
* ``EPSG:3857`` -- spherical ("web") Mercator on the WGS84 semi-major axis;
* ``EPSG:32601``-``32660`` / ``32701``-``32760`` -- WGS84 / UTM zones north /
  south: the transverse Mercator projection by Krueger's series in the third
  flattening n (the form of Karney, J. Geodesy 85, 2011, eqs. 7-11 and 35),
  to sixth order in n, scale 0.9996 on the central meridian, false easting
  500 km, false northing 0 (north) or 10 000 km (south).

``target_crs`` may be an ``"EPSG:<code>"`` string, an integer code, or a WKT
string (as GDAL's ``GetProjection()`` returns) whose last EPSG authority names
the projected system.  Other systems raise ``NotImplementedError``.
"""
from __future__ import annotations

import math
import re

import numpy as np

__all__ = ["epsg_code", "project_lonlat", "utm_forward", "WGS84_A", "WGS84_F"]

WGS84_A = 6378137.0
WGS84_F = 1.0 / 298.257223563
UTM_K0 = 0.9996

_AUTHORITY = re.compile(r'(?:AUTHORITY\[\s*"EPSG"\s*,\s*"?|ID\[\s*"EPSG"\s*,\s*)(\d+)')


def epsg_code(crs) -> int:
    """The EPSG code of ``crs`` (``"EPSG:32633"``, ``32633`` or WKT)."""
    if isinstance(crs, (int, np.integer)):
        return int(crs)
    text = str(crs).strip()
    m = re.fullmatch(r"(?i)epsg:(\d+)", text)
    if m:
        return int(m.group(1))
    codes = _AUTHORITY.findall(text)
    if codes:
        return int(codes[-1])  # the outermost system's authority comes last in WKT
    raise NotImplementedError(f"cannot read an EPSG code from the coordinate system {text[:80]!r}")


def _krueger_alpha(n):
    """alpha_1..alpha_6 of the forward series (Karney 2011, eq. 35)."""
    n2, n3, n4, n5, n6 = n * n, n ** 3, n ** 4, n ** 5, n ** 6
    return (
        n / 2 - 2 * n2 / 3 + 5 * n3 / 16 + 41 * n4 / 180 - 127 * n5 / 288 + 7891 * n6 / 37800,
        13 * n2 / 48 - 3 * n3 / 5 + 557 * n4 / 1440 + 281 * n5 / 630 - 1983433 * n6 / 1935360,
        61 * n3 / 240 - 103 * n4 / 140 + 15061 * n5 / 26880 + 167603 * n6 / 181440,
        49561 * n4 / 161280 - 179 * n5 / 168 + 6601661 * n6 / 7257600,
        34729 * n5 / 80640 - 3418889 * n6 / 1995840,
        212378941 * n6 / 319334400,
    )


def utm_forward(lon, lat, zone, south=False, a=WGS84_A, f=WGS84_F):
    """Easting and northing (m) of WGS84 longitude/latitude (degrees) in a UTM zone."""
    lon = np.asarray(lon, dtype=np.float64)
    lat = np.asarray(lat, dtype=np.float64)
    n = f / (2 - f)
    e = 2 * math.sqrt(n) / (1 + n)
    big_a = a / (1 + n) * (1 + n * n / 4 + n ** 4 / 64 + n ** 6 / 256)
    lon0 = (int(zone) - 1) * 6 - 180 + 3
    lam = np.radians(lon - lon0)
    phi = np.radians(lat)
    s = np.sin(phi)
    t = np.sinh(np.arctanh(s) - e * np.arctanh(e * s))  # tangent of the conformal latitude
    xi_p = np.arctan2(t, np.cos(lam))
    eta_p = np.arctanh(np.sin(lam) / np.sqrt(1 + t * t))
    xi, eta = xi_p.copy(), eta_p.copy()
    for j, al in enumerate(_krueger_alpha(n), start=1):
        xi += al * np.sin(2 * j * xi_p) * np.cosh(2 * j * eta_p)
        eta += al * np.cos(2 * j * xi_p) * np.sinh(2 * j * eta_p)
    easting = 500000.0 + UTM_K0 * big_a * eta
    northing = UTM_K0 * big_a * xi + (10000000.0 if south else 0.0)
    return easting, northing


def project_lonlat(lon, lat, target_crs):
    """Coordinates of longitude/latitude (degrees) in ``target_crs``."""
    code = epsg_code(target_crs)
    lon = np.asarray(lon, dtype=np.float64)
    lat = np.asarray(lat, dtype=np.float64)
    if code == 4326:
        return lon.copy(), lat.copy()
    if code == 3857:
        return (WGS84_A * np.radians(lon),
                WGS84_A * np.log(np.tan(np.pi / 4 + np.radians(lat) / 2)))
    if 32601 <= code <= 32660:
        return utm_forward(lon, lat, code - 32600, south=False)
    if 32701 <= code <= 32760:
        return utm_forward(lon, lat, code - 32700, south=True)
    raise NotImplementedError(f"EPSG:{code} is not one of the projections provided "
                              "(EPSG:4326, EPSG:3857, WGS84 / UTM 326xx and 327xx)")
