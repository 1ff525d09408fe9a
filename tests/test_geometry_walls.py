"""Host side of the geometry wall method (src/walls.py:145-332): building
heights against the reference's own rules (golden data generated by
tests/golden/make_building_heights.py), the map projections, the wall
segments and their aspects, the GeoJSON loader and the exact burn oracle."""
import json
import math
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "building_heights.json")


def _golden():
    with open(GOLD, encoding="utf-8") as f:
        return json.load(f)


def test_building_height_matches_the_reference_rules():
    from solweig_cuda_b200 import walls
    recs = _golden()["building_height"]
    assert len(recs) > 90
    for r in recs:
        props = {k: (float(v) if v in ("inf", "-inf") else v) for k, v in r["properties"].items()}
        assert walls.building_height(props, **r["options"]) == r["height"], r


def test_length_parsing_matches_the_reference():
    from solweig_cuda_b200 import walls
    for r in _golden()["length_metres"]:
        assert walls._length_metres(r["value"]) == r["metres"], r


def test_utm_matches_the_meridian_arc_and_is_conformal():
    from scipy.integrate import quad
    from solweig_cuda_b200 import crs
    a, f = crs.WGS84_A, crs.WGS84_F
    e2 = f * (2 - f)
    for lat in (0.0, 20.0, 45.0, 67.5):
        arc = quad(lambda p: a * (1 - e2) / (1 - e2 * math.sin(p) ** 2) ** 1.5, 0, math.radians(lat),
                   epsabs=1e-9, epsrel=1e-12)[0]
        e, n = crs.utm_forward(15.0, lat, 33)
        assert float(e) == 500000.0 and abs(float(n) - 0.9996 * arc) < 1e-6
    e, n = crs.utm_forward(15.0, -30.0, 33, south=True)
    e_n, n_n = crs.utm_forward(15.0, 30.0, 33)
    assert abs(float(n) - (1e7 - float(n_n))) < 1e-6
    # equal scale along and across, at right angles (conformal), away from the meridian
    h = 1e-6
    for lon, lat in ((18.0, 45.0), (12.5, 5.0), (19.5, 70.0)):
        phi = math.radians(lat)
        w = math.sqrt(1 - e2 * math.sin(phi) ** 2)
        east = (np.array(crs.utm_forward(lon + h, lat, 33)) - np.array(crs.utm_forward(lon - h, lat, 33))) / (2 * h)
        north = (np.array(crs.utm_forward(lon, lat + h, 33)) - np.array(crs.utm_forward(lon, lat - h, 33))) / (2 * h)
        east /= math.radians(1) * a * math.cos(phi) / w
        north /= math.radians(1) * a * (1 - e2) / w ** 3
        assert abs(np.dot(east, north)) < 1e-7
        assert abs(np.linalg.norm(east) / np.linalg.norm(north) - 1) < 1e-7


def test_epsg_codes_and_web_mercator():
    from solweig_cuda_b200 import crs
    wkt = ('PROJCS["WGS 84 / UTM zone 33N",GEOGCS["WGS 84",AUTHORITY["EPSG","4326"]],'
           'UNIT["metre",1],AUTHORITY["EPSG","32633"]]')
    assert crs.epsg_code(wkt) == 32633 and crs.epsg_code("epsg:3857") == 3857 and crs.epsg_code(4326) == 4326
    x, y = crs.project_lonlat([180.0, 0.0], [0.0, 0.0], "EPSG:3857")
    assert x[0] == pytest.approx(math.pi * 6378137.0, abs=1e-6) and abs(y[1]) < 1e-6
    lon, lat = crs.project_lonlat([1.5], [2.5], "EPSG:4326")
    assert lon[0] == 1.5 and lat[0] == 2.5
    with pytest.raises(NotImplementedError):
        crs.project_lonlat([0.0], [0.0], "EPSG:2154")


def test_wall_segments_orient_rings_and_face_outwards():
    from solweig_cuda_b200 import walls
    outer = [[0, 0], [0, 2], [2, 2], [2, 0], [0, 0]]          # clockwise
    hole = [[0.5, 0.5], [1.5, 0.5], [1.5, 1.5], [0.5, 1.5]]   # counter-clockwise, not closed
    h, a = walls.wall_segments({"type": "Polygon", "coordinates": [outer, hole]}, 7.0)
    assert [v for _, v in h] == [7.0] * 8
    assert [v for _, v in a] == [180.0, 90.0, 0.0, 270.0, 90.0, 180.0, 270.0, 0.0]
    assert a[0][0] == ((0.0, 0.0), (2.0, 0.0)) and a[4][0] == ((0.5, 0.5), (0.5, 1.5))
    # orientation of the input does not matter; repeated vertices give no segment
    outer_ccw = [[0, 0], [2, 0], [2, 0], [2, 2], [0, 2], [0, 0]]
    h2, a2 = walls.wall_segments({"type": "MultiPolygon", "coordinates": [[outer_ccw]]}, 3.0)
    assert [s for s, _ in a2] == [s for s, _ in a[:4]]


def test_load_buildings_projects_and_reads_heights(tmp_path):
    from solweig_cuda_b200 import crs, walls
    ring = [[15.0, 52.0], [15.001, 52.0], [15.001, 52.001], [15.0, 52.001], [15.0, 52.0]]
    data = {"type": "FeatureCollection", "features": [
        {"type": "Feature", "properties": {"height": "21 m"}, "geometry": {"type": "Polygon", "coordinates": [ring]}},
        {"type": "Feature", "properties": {"building:levels": 4},
         "geometry": {"type": "MultiPolygon", "coordinates": [[ring]]}},
        {"type": "Feature", "properties": {}, "geometry": {"type": "LineString", "coordinates": ring}},
        {"type": "Feature", "properties": {}, "geometry": None}]}
    path = tmp_path / "b.geojson"
    path.write_text(json.dumps(data), encoding="utf-8")
    got = walls.load_buildings(path, "EPSG:32633", level_height_m=3.5)
    assert [h for _, h in got] == [21.0, 14.0]
    xy = np.asarray(got[0][0]["coordinates"][0][0])
    e, n = crs.utm_forward(np.array(ring)[:, 0], np.array(ring)[:, 1], 33)
    assert np.array_equal(xy, np.column_stack([e, n]))


def test_burn_oracle_rules():
    from oracle import walls_geometry as W
    assert W.cells_touched(0.5, 2.0, 3.5, 2.0) == [(0, 2), (1, 2), (2, 2), (3, 2)]
    assert sorted(W.cells_touched(0, 0, 2, 2)) == [(0, 0), (1, 1), (2, 2)]
    assert sorted(W.cells_touched(2, 2, 0, 0)) == [(0, 0), (1, 1), (2, 2)]
    assert sorted(W.cells_touched(0, 2, 2, 0)) == [(0, 1), (0, 2), (1, 0), (1, 1), (2, 0)]
    assert sorted(W.cells_touched(1.0, 0.25, 1.0, 1.75)) == [(1, 0), (1, 1)]
    owner = W.burn([[0.5, 0.5, 2.5, 0.5], [1.5, 0.0, 1.5, 1.9]], 3, 3)
    assert owner.tolist() == [[0, 1, 0], [-1, 1, -1], [-1, -1, -1]]
    walls, aspect = W.merge(owner, [5.0, 7.0], [359.99999999, 90.0],
                            np.array([[np.nan, 2.0, 9.0]] * 3, np.float32), 2.0)
    assert walls[0].tolist() == [5.0, 2.0, 9.0] and walls[1].tolist() == [0.0, 2.0, 0.0]
    assert aspect[0].tolist() == [0.0, 90.0, 0.0]
