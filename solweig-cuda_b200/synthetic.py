"""Seeded synthetic urban scenes and forcing (host side, numpy).

The reference ships no rasters for its published runs, so seeded synthetic
inputs with the stated shapes stand in for them:

* flat ground at 0 m (DEM = 0);
* axis-aligned rectangular buildings, footprints U[8, 30] m per side, heights
  U[5, 40] m, placed until ~30 % of the area is roof;
* Gaussian tree crowns, height U[3, 15] m, radius U[2, 6] m, ~10 % cover,
  never on roofs (the trunk zone, 25 % of the height, is applied by the
  static preparation as in the reference);
* land cover: building = 2, paved = 1, grass = 5 under trees;
* a 24-hour UMEP forcing table for one day: Ta = 16 + 6 sin(2 pi (h - 9)/24),
  RH = 72.5 - 12.5 sin(...), wind U[1, 5] m/s, global radiation = s_h * I0
  with s_h ~ U[0.6, 1.0] and I0 from the clearness-index model, 0 at night,
  pressure 101.3 kPa, every other column -999.
"""
from __future__ import annotations

import datetime as _dt

import numpy as np

from . import sun as _sun

__all__ = ["Scene", "make_scene", "make_met"]


class Scene:
    """Rasters of one synthetic tile (float32, metres)."""

    def __init__(self, dsm, trees, dem, landcover, pixel_size, latitude, longitude, seed):
        self.dsm = dsm
        self.trees = trees
        self.dem = dem
        self.landcover = landcover
        self.pixel_size = pixel_size
        self.latitude = latitude
        self.longitude = longitude
        self.seed = seed

    @property
    def shape(self):
        return self.dsm.shape


def make_scene(rows, cols=None, seed=0, pixel_size=1.0, building_cover=0.30, tree_cover=0.10,
               latitude=53.0, longitude=0.0):
    """Generate a seeded scene of ``rows x cols`` pixels (``numpy.random.default_rng(seed)``)."""
    cols = rows if cols is None else cols
    rng = np.random.default_rng(seed)
    dsm = np.zeros((rows, cols), dtype=np.float32)
    area = rows * cols
    roof = np.zeros((rows, cols), dtype=bool)
    m_to_px = 1.0 / pixel_size
    attempts = 0
    covered = 0  # roof.sum(), kept incrementally
    while covered < building_cover * area and attempts < 100000:
        attempts += 1
        h = max(1, int(round(rng.uniform(8, 30) * m_to_px)))
        w = max(1, int(round(rng.uniform(8, 30) * m_to_px)))
        if h >= rows or w >= cols:
            continue
        r0 = int(rng.integers(0, rows - h + 1))
        c0 = int(rng.integers(0, cols - w + 1))
        height = np.float32(rng.uniform(5, 40))
        block = dsm[r0:r0 + h, c0:c0 + w]
        np.maximum(block, height, out=block)
        footprint = roof[r0:r0 + h, c0:c0 + w]
        covered += int(footprint.size - np.count_nonzero(footprint))
        footprint[...] = True
    trees = np.zeros((rows, cols), dtype=np.float32)
    crown = np.zeros((rows, cols), dtype=bool)
    attempts = 0
    crowned = 0  # crown.sum(), kept incrementally
    while crowned < tree_cover * area and attempts < 200000:
        attempts += 1
        rc = int(rng.integers(0, rows))
        cc = int(rng.integers(0, cols))
        radius = rng.uniform(2, 6) * m_to_px
        height = rng.uniform(3, 15)
        if roof[rc, cc]:
            continue
        R = int(np.ceil(radius))
        r0, r1 = max(0, rc - R), min(rows, rc + R + 1)
        c0, c1 = max(0, cc - R), min(cols, cc + R + 1)
        yy, xx = np.mgrid[r0:r1, c0:c1]
        d2 = (yy - rc) ** 2 + (xx - cc) ** 2
        inside = (d2 <= radius * radius) & ~roof[r0:r1, c0:c1]
        sigma = radius / 2.0
        value = (height * np.exp(-d2 / (2 * sigma * sigma))).astype(np.float32)
        patch = trees[r0:r1, c0:c1]
        np.copyto(patch, np.maximum(patch, value), where=inside)
        cells = crown[r0:r1, c0:c1]
        grown = inside & (value > 0) & ~cells
        crowned += int(np.count_nonzero(grown))
        cells |= grown
    dem = np.zeros((rows, cols), dtype=np.float32)
    landcover = np.ones((rows, cols), dtype=np.float32)
    landcover[trees > 0] = 5
    landcover[roof] = 2
    return Scene(dsm, trees, dem, landcover, pixel_size, latitude, longitude, seed)


def make_met(year=2025, doy=172, latitude=53.0, longitude=0.0, site_altitude=3.0, utc=0.0,
             seed=0, days=1):
    """UMEP 24-column forcing table, hourly, for ``days`` consecutive days."""
    rng = np.random.default_rng(seed + 1000)
    rows = []
    start = _dt.datetime(year, 1, 1) + _dt.timedelta(days=doy - 1)
    for d in range(days):
        day = start + _dt.timedelta(days=d)
        for h in range(24):
            row = np.full(24, -999.0)
            row[0], row[1], row[2], row[3] = day.year, day.timetuple().tm_yday, h, 0
            phase = np.sin(2 * np.pi * (h - 9) / 24)
            row[11] = 16 + 6 * phase
            row[10] = 72.5 - 12.5 * phase
            row[9] = rng.uniform(1, 5)
            row[12] = 101.3
            row[13] = 0.0
            row[15] = 0.0
            rows.append(row)
    met = np.asarray(rows)
    sol = _sun.metdata(met, latitude, longitude, site_altitude, utc)
    for i in range(met.shape[0]):
        s = rng.uniform(0.6, 1.0)
        if sol.altitude[i] > 0:
            i0, *_ = _sun.clearness_index(sol.zen[i], sol.jday[i], met[i, 11], met[i, 10] / 100., 0.0,
                                          latitude, met[i, 12])
            met[i, 14] = s * max(float(i0), 0.0)
        else:
            met[i, 14] = 0.0
    return met
