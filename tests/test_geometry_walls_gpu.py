"""The geometry wall method on the GPU (src/walls.py:270-332): the device
burn of footprint edges against the exact oracle (oracle/walls_geometry.py)
and the whole calculate_geometry_walls against the oracle's burn and merge.
Coordinates lie on a binary grid so every cross product of the device walk is
exact: the owners must be identical."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_burn(seg, rows, cols):
    import torch
    from solweig_cuda_b200 import _lib
    from solweig_cuda_b200.engine import device_ptr
    t = torch.from_numpy(np.ascontiguousarray(seg, dtype=np.float64)).cuda()
    owner = torch.empty((rows, cols), dtype=torch.int32, device="cuda")
    _lib.check(_lib.lib().solweig_wall_segments_burn(device_ptr(t), len(seg), rows, cols, device_ptr(owner), None),
               "burn")
    return owner.cpu().numpy()


def test_burn_matches_the_exact_oracle(cuda):
    from oracle import walls_geometry as W
    rng = np.random.default_rng(11)
    rows, cols = 40, 56
    n = 600
    seg = rng.integers(-8 * 6, 8 * (cols + 6), size=(n, 4)).astype(np.float64) / 8.0
    seg[:, 1] = rng.integers(-8 * 6, 8 * (rows + 6), size=n) / 8.0
    seg[:, 3] = seg[:, 1] + rng.integers(-8 * 12, 8 * 12, size=n) / 8.0
    seg[:, 2] = seg[:, 0] + rng.integers(-8 * 12, 8 * 12, size=n) / 8.0
    seg[:100, 3] = seg[:100, 1]                 # horizontal
    seg[100:200, 2] = seg[100:200, 0]           # vertical
    k = np.arange(200, 300)                     # exact diagonals through cell corners
    seg[k, 0:2] = np.floor(seg[k, 0:2])
    d = rng.integers(-9, 10, size=100)
    seg[k, 2] = seg[k, 0] + d
    seg[k, 3] = seg[k, 1] + np.where(rng.random(100) < 0.5, d, -d)
    seg[300:310, 2:4] = seg[300:310, 0:2]       # points
    for shuffle in range(2):
        got = _device_burn(seg, rows, cols)
        want = W.burn(seg, rows, cols)
        assert np.array_equal(got, want), np.argwhere(got != want)[:5]
        seg = seg[rng.permutation(n)]


def test_calculate_geometry_walls_matches_the_oracle(cuda, tmp_path):
    from oracle import walls_geometry as W
    from solweig_cuda_b200 import crs, walls
    rng = np.random.default_rng(5)
    # footprints in lon/lat around 15E 52N (UTM 33N), a 0.5 m raster
    feats = []
    for b in range(40):
        lon0, lat0 = 15.0 + rng.uniform(0, 8e-4), 52.0 + rng.uniform(0, 5e-4)
        w, h = rng.uniform(1e-5, 1.2e-4), rng.uniform(1e-5, 8e-5)
        ring = [[lon0, lat0], [lon0 + w, lat0], [lon0 + w, lat0 + h], [lon0 + w / 2, lat0 + 1.4 * h],
                [lon0, lat0 + h], [lon0, lat0]]
        props = {"height": f"{rng.uniform(3, 30):.1f}"} if b % 3 else {"building:levels": int(rng.integers(1, 8))}
        feats.append({"type": "Feature", "properties": props, "geometry": {"type": "Polygon", "coordinates": [ring]}})
    path = tmp_path / "buildings.geojson"
    path.write_text(json.dumps({"type": "FeatureCollection", "features": feats}), encoding="utf-8")
    e0, n0 = crs.utm_forward(15.0, 52.0, 33)
    rows, cols = 140, 130
    gt = (float(np.floor(e0)), 0.5, 0.0, float(np.floor(n0)) + rows * 0.5 + 10.0, 0.0, -0.5)
    buildings = walls.load_buildings(path, "EPSG:32633")
    ghsl = rng.uniform(0, 25, (rows, cols)).astype(np.float32)
    ghsl[rng.random((rows, cols)) < 0.5] = 0.0
    ghsl[0, :5] = [np.nan, np.inf, -np.inf, 1.99, 2.0]
    got_w, got_a = walls.calculate_geometry_walls(buildings, ghsl, (rows, cols), walls.affine_from_gdal(gt), 2.0)
    # oracle: the same segments in pixel coordinates, burned and merged exactly
    seg, hs, asp = [], [], []
    for g, h in buildings:
        hh, aa = walls.wall_segments(g, max(2.0, h))
        for (s, hv), (_, av) in zip(hh, aa):
            seg.append(list(s[0]) + list(s[1]))
            hs.append(hv)
            asp.append(av)
    seg = np.asarray(seg)
    a, b, c, d, e, f = walls.affine_from_gdal(gt)
    pix = np.column_stack([(seg[:, 0] - c) / a, (seg[:, 1] - f) / e, (seg[:, 2] - c) / a, (seg[:, 3] - f) / e])
    want_w, want_a = W.merge(W.burn(pix, rows, cols), hs, asp, ghsl, 2.0)
    assert got_w.dtype == np.float32 and got_a.dtype == np.float32
    assert (want_w > 0).sum() > 500
    assert np.array_equal(got_w, want_w) and np.array_equal(got_a, want_a)


def test_run_timeseries_geometry_walls(cuda, tmp_path):
    """run_timeseries(wall_method="geometry") builds the scene on the footprint
    walls (src/series.py:218-233): its static walls are calculate_geometry_walls'."""
    from solweig_cuda_b200 import series, synthetic, walls
    sc = synthetic.make_scene(48, seed=2)
    for name, arr in (("dsm", sc.dsm), ("trees", sc.trees), ("dem", sc.dem)):
        np.save(tmp_path / f"{name}.npy", arr)
    ring = [[500010.0, 5760010.0], [500030.0, 5760010.0], [500030.0, 5760030.0], [500010.0, 5760030.0],
            [500010.0, 5760010.0]]
    from solweig_cuda_b200 import crs as C
    # the same square in lon/lat (UTM 33N, central meridian 15E), by fixed-point iteration on the forward map
    def lonlat(e, n):
        lon, lat = 15.0, 52.0
        for _ in range(60):
            ee, nn = C.utm_forward(lon, lat, 33)
            lon += (e - float(ee)) / 68000.0
            lat += (n - float(nn)) / 111000.0
        return [lon, lat]
    geo = {"type": "FeatureCollection", "features": [{"type": "Feature", "properties": {"height": 12},
           "geometry": {"type": "Polygon", "coordinates": [[lonlat(*p) for p in ring]]}}]}
    (tmp_path / "b.geojson").write_text(json.dumps(geo), encoding="utf-8")
    np.save(tmp_path / "ghsl.npy", np.zeros((48, 48), np.float32))
    gt = (500000.0, 1.0, 0.0, 5760048.0, 0.0, -1.0)
    met = synthetic.make_met(doy=172, latitude=52.0, longitude=15.0)
    files = series.run_timeseries(str(tmp_path / "dsm.npy"), str(tmp_path / "trees.npy"), str(tmp_path / "dem.npy"),
                                  met, str(tmp_path / "out"), 15.0, 52.0, utc_offset_hours=1.0,
                                  wall_method="geometry", building_geometry_path=str(tmp_path / "b.geojson"),
                                  building_height_path=str(tmp_path / "ghsl.npy"), crs="EPSG:32633",
                                  geotransform=gt)
    w = np.load(files["static"]["walls"])
    b = walls.load_buildings(tmp_path / "b.geojson", "EPSG:32633")
    want, _ = walls.calculate_geometry_walls(b, np.zeros((48, 48), np.float32), (48, 48), walls.affine_from_gdal(gt), 2.0)
    assert np.array_equal(w, want) and (w == 12.0).sum() >= 4 * 19
    assert len(files["days"]) == 1
