"""Forcing and case validation (scripts/input_check.py rules of the reference)."""
import json

import numpy as np
import pytest


def _met(rows=24, doy=172):
    from solweig_cuda_b200 import synthetic
    return synthetic.make_met(doy=doy)[:rows].copy()


def test_valid_forcing_groups_days():
    from solweig_cuda_b200 import input_check, synthetic
    met = synthetic.make_met(doy=172, days=2)
    forcing = input_check.check_weather(met)
    assert len(forcing.days) == 2 and forcing.timestep_minutes == 60


@pytest.mark.parametrize("mutate,message", [
    (lambda m: m[:, :22], "23 SOLWEIG columns"),
    (lambda m: np.where(np.arange(m.shape[1]) == 11, np.nan, m), "non-finite"),
    (lambda m: m.__setitem__((0, 2), 1.5) or m, "must be integers"),
    (lambda m: m.__setitem__((0, 1), 367) or m, "day-of-year"),
    (lambda m: m.__setitem__((0, 2), 24) or m, "hour must be between"),
    (lambda m: m.__setitem__((0, 3), 60) or m, "minute must be between"),
    (lambda m: m.__setitem__((3, 10), 101) or m, "relative humidity"),
    (lambda m: m.__setitem__((3, 9), -1) or m, "wind"),
    (lambda m: m.__setitem__((3, 12), 0.0) or m, "pressure"),
    (lambda m: m.__setitem__((3, 14), -5) or m, "global shortwave"),
    (lambda m: m.__setitem__((3, 11), 150) or m, "air temperature"),
    (lambda m: np.delete(m, 5, axis=0), "one constant timestep"),
    (lambda m: np.concatenate([m[:5], m[4:]]), "strictly increasing"),
])
def test_invalid_forcing_is_rejected(mutate, message):
    from solweig_cuda_b200 import input_check
    met = mutate(_met())
    with pytest.raises(ValueError, match=message):
        input_check.check_weather(met)


def test_day_of_year_366_only_in_leap_years():
    from solweig_cuda_b200 import input_check
    met = _met(rows=1)
    met[0, 0], met[0, 1] = 2023, 366
    with pytest.raises(ValueError, match="invalid for calendar year"):
        input_check.check_weather(met)
    met[0, 0] = 2024
    input_check.check_weather(met)


def test_forcing_paths(tmp_path):
    from solweig_cuda_b200 import input_check
    met = _met()
    f = tmp_path / "met.txt"
    np.savetxt(f, met, header=" ".join(f"c{i}" for i in range(met.shape[1])), comments="")
    assert len(input_check.check_weather(str(f)).values) == 24
    with pytest.raises(ValueError, match="duplicate"):
        input_check.check_weather([f, f])
    with pytest.raises(TypeError):
        input_check.check_weather([f, 3])
    with pytest.raises(TypeError):
        input_check.check_weather(42)


@pytest.mark.parametrize("raw,message", [
    ([], "JSON object"),
    ({"case_type": "remote"}, "local or open_data"),
    ({"case_name": " "}, "nonempty string"),
    ({"case_type": "open_data"}, "requires case_size_m"),
    ({"resolution_m": 0}, "positive finite"),
    ({"resolution_m": True}, "positive finite"),
    ({"buffer_area_m": -1, "core_area_m": 10}, "nonnegative finite"),
    ({"core_area_m": 10}, "supplied together"),
    ({"core_area_m": 10.5, "buffer_area_m": 2}, "whole number"),
    ({"start_date": "2024-01-01"}, "supplied together"),
    ({"start_date": "2024-1-1", "end_date": "2024-01-02"}, "YYYY-MM-DD"),
    ({"start_date": "2024-01-03", "end_date": "2024-01-02"}, "must not precede"),
    ({"case_type": "open_data", "case_size_m": 100, "start_date": "2024-01-01", "end_date": "2024-01-02",
      "utc_offset_hours": 1}, "utc_offset_hours=0"),
])
def test_preparation_options_rejected(raw, message):
    from solweig_cuda_b200 import input_check
    with pytest.raises(ValueError, match=message):
        input_check.validate_preparation_options(raw)


def test_preparation_defaults():
    from solweig_cuda_b200 import input_check
    opts = input_check.validate_preparation_options({"core_area_m": 180, "buffer_area_m": 10, "resolution_m": 2})
    assert opts["case_type"] == "local" and opts["resolution_m"] == 2


@pytest.mark.parametrize("case,message", [
    ({"output_chunk_steps": 0}, "positive integer"),
    ({"output_queue_size": True}, "positive integer"),
    ({"async_output": 1}, "boolean"),
    ({"latitude": 95}, "latitude"),
    ({"longitude": None}, "longitude"),
    ({"utc_offset_hours": 30}, "utc_offset_hours"),
    ({"site_altitude_m": float("inf")}, "site_altitude_m"),
    ({"dsm_wall_threshold_m": 0}, "dsm_wall_threshold_m"),
    ({"save_svf": 1}, "true or false"),
    ({"wall_method": "lidar"}, "dsm or geometry"),
    ({"wall_method": "geometry"}, "requires building_geometry_path"),
    ({"output_core": [0, 0, 0, 5]}, "output_core"),
    ({"geotransform": [0, 1, 0, 0, 0]}, "six finite numbers"),
    ({"geotransform": [0, 1, 0, 0, 0, float("nan")]}, "six finite numbers"),
    ({"geotransform": [0, 1, 0, 0, 0, 0]}, "invertible"),
    ({"crs": "EPSG:2154"}, "crs"),
])
def test_run_options_rejected(case, message):
    from solweig_cuda_b200 import input_check
    with pytest.raises(ValueError, match=message):
        input_check.check_options(case)


def test_georeferencing_options_accepted():
    from solweig_cuda_b200 import input_check
    input_check.check_options({"geotransform": [500000.0, 1.0, 0.0, 5760048.0, 0.0, -1.0], "crs": "EPSG:32633"})


def test_output_window_and_mask():
    from solweig_cuda_b200 import input_check
    input_check.check_output_window([1, 2, 3, 4], (10, 10), np.ones((3, 4), bool))
    with pytest.raises(ValueError, match="inside"):
        input_check.check_output_window([8, 8, 3, 3], (10, 10))
    with pytest.raises(TypeError, match="boolean"):
        input_check.check_output_window(None, (3, 3), np.ones((3, 3)))
    with pytest.raises(ValueError, match="match the cropped"):
        input_check.check_output_window([0, 0, 2, 2], (10, 10), np.ones((3, 3), bool))


def test_case_file(tmp_path):
    from solweig_cuda_b200 import input_check
    case = {"case_name": "demo", "building_dsm_path": "dsm.npy", "tree_path": "trees.npy",
            "dem_path": "dem.npy", "met_file": ["a.txt", "b.txt"], "longitude": 0.0, "latitude": 53.0}
    p = tmp_path / "case.json"
    p.write_text(json.dumps(case))
    got, settings = input_check.check_case(p)
    assert got["dem_path"] == str(tmp_path / "dem.npy")
    assert got["met_file"] == [str(tmp_path / "a.txt"), str(tmp_path / "b.txt")]
    assert got["output_chunk_steps"] == 24 and settings["case_name"] == "demo"
    p.write_text(json.dumps({**case, "colour": "red"}))
    with pytest.raises(ValueError, match="Unknown case options"):
        input_check.check_case(p)
    bad = dict(case)
    del bad["dem_path"]
    p.write_text(json.dumps(bad))
    with pytest.raises(ValueError, match="Missing case options: dem_path"):
        input_check.check_case(p)


def test_check_arrays():
    from solweig_cuda_b200 import input_check
    a = np.zeros((4, 5))
    assert input_check.check_arrays(a, a, a) == (4, 5)
    with pytest.raises(ValueError, match="aligned"):
        input_check.check_arrays(a, np.zeros((4, 4)), a)
    with pytest.raises(ValueError, match="non-finite"):
        input_check.check_arrays(a, a, np.full((4, 5), np.nan))
