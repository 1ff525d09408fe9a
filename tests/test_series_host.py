"""Host-side logic of the series driver: forcing grouping, tile windows and the
bounded output writer's failure handling (failures injected on the host)."""
import os
import threading

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_load_meteorology_groups_days():
    from solweig_cuda_b200 import series
    met = np.load(os.path.join(GOLD, "sun.npz"))["met_dublin"]
    m = series.load_meteorology(met)
    assert [d.date for d in m.days] == ["2025-06-01", "2025-06-02"]
    assert all(len(d.values) == 24 for d in m.days)
    assert m.timestep_minutes == 60.0
    assert not m.values.flags.writeable


def test_tile_windows_cover_the_raster():
    from solweig_cuda_b200 import tiling
    t = tiling.tile_windows(50, 70, core=20, halo=6)
    assert len(t) == 3 * 4
    cover = np.zeros((50, 70), int)
    for w in t:
        col, row, cw, ch = w["core_window"]
        cover[row:row + ch, col:col + cw] += 1
        r0, c0, nr, nc = w["output_core"]
        left, top, iw, ih = w["input_window"]
        assert (top + r0, left + c0, nr, nc) == (row, col, ch, cw)
        assert 0 <= left and left + iw <= 70 and 0 <= top and top + ih <= 50
    assert (cover == 1).all()


def test_output_writer_surfaces_worker_failures():
    from solweig_cuda_b200.series import OutputWriter
    w = OutputWriter(enabled=True, max_inflight=1)
    done = threading.Event()
    w.submit(lambda: (_ for _ in ()).throw(OSError("disk full")))
    w.submit(done.set)  # skipped after a failure
    with pytest.raises(RuntimeError, match="output writer failed"):
        w.finish()
    assert not done.is_set()


def test_output_writer_sync_mode_runs_inline():
    from solweig_cuda_b200.series import OutputWriter
    out = []
    w = OutputWriter(enabled=False)
    w.submit(lambda: out.append(1))
    w.finish()
    assert out == [1]


def test_bad_forcing_and_raster_shapes_are_rejected():
    from solweig_cuda_b200 import series
    with pytest.raises(Exception):
        series.load_meteorology(np.zeros((3, 2)))  # fewer than 4 columns
    from solweig_cuda_b200 import engine
    with pytest.raises((ValueError, RuntimeError)):
        engine.Scene(np.zeros((10, 10)), np.zeros((10, 11)), np.zeros((10, 10)))


class StubScene:
    """Host stand-in for engine.Scene: the driver only needs the static planes."""

    def __init__(self, dsm, trees, dem, pixel_size=1.0, landcover=None, wall_threshold=3.0, device="cpu",
                 keep_planes=False):
        self.shape = np.shape(dsm)
        self.device = "cpu"
        self.walls_host = np.zeros(self.shape)
        self.aspect_host = np.zeros(self.shape)


class StubRunner:
    """Day runner whose planes depend on the day's forcing and the pixel, so
    every (day, hour, pixel, variable) value is distinct."""

    def __init__(self, scene, latitude, longitude, site_altitude, utc, hours, outputs, form):
        import torch
        self.outputs = outputs
        r, c = scene.shape
        self.pix = torch.arange(r * c, dtype=torch.float32).reshape(r, c)
        self.buf = {k: torch.empty((hours, r, c)) for k in outputs}

    def run_day(self, values):
        import torch
        for j, k in enumerate(self.outputs):
            for h, row in enumerate(values):
                self.buf[k][h] = float(row[1]) * 1000 + float(row[2]) * 10 + j + self.pix / 1e4
        return self.buf


def _forcing(days=4):
    from solweig_cuda_b200 import synthetic
    return synthetic.make_met(doy=172, latitude=53.0, longitude=0.0, days=days)


def run_stub(tmp, **kw):
    from solweig_cuda_b200 import series
    z = np.zeros((12, 10))
    return series.run_timeseries(z, z, z, _forcing(kw.pop("days", 4)), tmp, 0.0, 53.0, scene_factory=StubScene,
                                 runner_factory=StubRunner, device="cpu", **kw)


def test_run_timeseries_masks_cropped_outputs_after_the_copy(tmp_path):
    """output_valid_mask applies to the cropped output core, after the
    device-to-host copy (src/output.py:205-216): masked files equal the
    unmasked run with NaN outside the mask."""
    core = (2, 3, 7, 5)
    mask = np.ones((7, 5), dtype=bool)
    mask[1:3, 2:4] = False
    a = run_stub(tmp_path / "plain", output_core=core, save_kup=True)
    b = run_stub(tmp_path / "masked", output_core=core, save_kup=True, output_valid_mask=mask)
    assert a["days"].keys() == b["days"].keys() and len(a["days"]) == 4
    for date, rec in a["days"].items():
        for var, paths in rec.items():
            x = np.load(paths[0])
            y = np.load(b["days"][date][var][0])
            assert x.shape == (24, 7, 5)
            assert not np.isnan(x).any()
            want = np.where(mask[None], x, np.nan)
            assert np.array_equal(np.isnan(y), np.isnan(want))
            assert np.array_equal(y[:, mask], x[:, mask])


def test_run_timeseries_rejects_bad_mask_and_dtype(tmp_path):
    with pytest.raises(ValueError, match="cropped output"):
        run_stub(tmp_path / "a", output_core=(0, 0, 4, 4), output_valid_mask=np.ones((12, 10), bool))
    with pytest.raises(NotImplementedError, match="float32 or float64"):
        run_stub(tmp_path / "b", dtype=np.float16)
    # the float64 switch is accepted (the stub runner stands in for the float64 step)
    assert len(run_stub(tmp_path / "c", dtype=np.float64)["days"]) == 4


def test_geometry_wall_method_needs_its_inputs(tmp_path):
    with pytest.raises(ValueError, match="building_geometry_path"):
        run_stub(tmp_path / "g1", wall_method="geometry")
    with pytest.raises(ValueError, match="crs and geotransform"):
        run_stub(tmp_path / "g2", wall_method="geometry", building_geometry_path="b.geojson",
                 building_height_path="h.npy")
    with pytest.raises(ValueError, match="wall_method"):
        run_stub(tmp_path / "g3", wall_method="lidar")


def test_float64_switch_selects_the_float64_step():
    from solweig_cuda_b200 import series
    assert series._check_dtype(np.float64) and not series._check_dtype("float32")
    assert series._make_runner64.__code__.co_varnames[:8] == series._make_runner.__code__.co_varnames[:8]


def test_run_timeseries_rank_shares_cover_all_days(tmp_path):
    whole = run_stub(tmp_path / "one", days=5)
    parts = [run_stub(tmp_path / "two", days=5, rank=r, world_size=2) for r in range(2)]
    assert parts[0]["static"] and not parts[1]["static"]
    got = {**parts[0]["days"], **parts[1]["days"]}
    assert sorted(got) == sorted(whole["days"]) and not set(parts[0]["days"]) & set(parts[1]["days"])
    for date, rec in whole["days"].items():
        for var, paths in rec.items():
            assert np.array_equal(np.load(paths[0]), np.load(got[date][var][0]))


def test_day_error_bits_raise_only_for_invalid_results():
    """The sticky word of the flag pair: bits 1 and 3 (contraction wait timed
    out, overlong ray) raise DayError; bit 2 (window sweep walked from the
    raster, results exact) does not; a cleared pair passes."""
    import torch
    from solweig_cuda_b200 import batched
    work = torch.zeros(64, dtype=torch.uint8)
    batched.clear_day_errors(work)
    assert batched.check_day_errors(work) == 0
    words = work[:8].view(torch.int32)
    words[1] = 1 << 2
    assert batched.check_day_errors(work) == 4
    for bit in (1, 3):
        words[1] = (1 << bit) | (1 << 2)
        with pytest.raises(batched.DayError):
            batched.check_day_errors(work)
    batched.clear_day_errors(work)
    assert int(words[0]) == 0 and int(words[1]) == 0


class FlaggedRunner(StubRunner):
    """A runner whose days left invalid results (as a device flag would say)."""

    def check_errors(self):
        from solweig_cuda_b200 import batched
        raise batched.DayError("batched day: test flag - results invalid")


def test_run_timeseries_raises_when_a_day_left_invalid_results(tmp_path):
    from solweig_cuda_b200 import batched, series
    z = np.zeros((12, 10))
    with pytest.raises(batched.DayError):
        series.run_timeseries(z, z, z, _forcing(2), tmp_path, 0.0, 53.0, scene_factory=StubScene,
                              runner_factory=FlaggedRunner, device="cpu")


def test_cli_refuses_geometry_walls_for_tiled_cases(tmp_path):
    """run.py: a tiled case with wall_method=geometry stops before any device
    work (the reference's tile jobs do not crop the building-height raster)."""
    import importlib.util
    import json
    from solweig_cuda_b200 import synthetic
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    header = "iy id it imin Q* QH QE Qs Qf Wind RH Td press rain Kdn snow ldown fcld wuh xsmd lai_hr Kdiff Kdir Wd"
    np.savetxt(tmp_path / "met.txt", met, header=header, comments="", fmt="%.6f")
    case = {"case_name": "t", "building_dsm_path": "dsm.npy", "tree_path": "trees.npy", "dem_path": "dem.npy",
            "met_file": "met.txt", "output_path": "out", "longitude": 0.0, "latitude": 53.0,
            "core_area_m": 20, "buffer_area_m": 6, "wall_method": "geometry",
            "building_geometry_path": "b.geojson", "building_height_path": "h.npy"}
    (tmp_path / "case.json").write_text(json.dumps(case))
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("solweig_run_cli", os.path.join(root, "run.py"))
    cli = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(cli)
    with pytest.raises(SystemExit, match="geometry"):
        cli.main(["--case", str(tmp_path / "case.json"), "--no-progress"])
