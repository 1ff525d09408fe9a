"""The drop-in modules (svf, walls, utci, model, series, run.py) on the GPU,
against the oracle on seeded scenes, with the reference's names and
return orders."""
import json

import numpy as np
import pytest

from conftest import small_scene

pytestmark = pytest.mark.gpu


def _vegetation(a, t1):
    vegdsm = t1 + a
    vegdsm[vegdsm == a] = 0
    vegdsm2 = t1 * 0.25 + a
    vegdsm2[vegdsm2 == a] = 0
    return vegdsm, vegdsm2, np.logical_not(vegdsm2 * vegdsm) * vegdsm


def test_svf_calculator_matches_oracle(cuda):
    from oracle import geometry as G
    from solweig_cuda_b200 import svf as S
    sc = small_scene(40, seed=8)
    a, t1 = sc.dsm.astype(np.float64), sc.trees.astype(np.float64)
    vegdsm, vegdsm2, bush = _vegetation(a, t1)
    amax = max(a.max() - a.min(), t1.max())
    got = S.svf_calculator(2, amax, a, vegdsm, vegdsm2, bush, 1.0)
    want = G.svf_calculator(2, amax, a, vegdsm, vegdsm2, bush, 1.0)
    assert len(got) == 19
    for i in range(15):
        assert np.max(np.abs(got[i].cpu().numpy() - want[i])) < 1e-12, i
    for i in range(15, 18):
        assert np.array_equal(got[i].cpu().numpy(), want[i]), i
    assert np.max(np.abs(got[18].cpu().numpy() - want[18])) < 1e-12
    d = S.compute_diffsh(got[17], got[15], 0.03).cpu().numpy()
    assert np.max(np.abs(d - G.compute_diffsh(want[17], want[15], 0.03))) < 1e-6


def test_calculate_dsm_walls_matches_oracle(cuda):
    from oracle import geometry as G
    from solweig_cuda_b200 import walls as W
    sc = small_scene(60, seed=1)
    a = sc.dsm.astype(np.float64)
    walls, aspect = W.calculate_dsm_walls(a, 1.0)
    assert np.array_equal(walls, G.wall_heights(a, 3.0))
    assert np.array_equal(aspect, G.wall_aspect(G.wall_heights(a, 3.0), a, 1.0))


def test_utci_calculator_scalar_and_array(cuda):
    from oracle import utci as OU
    from solweig_cuda_b200 import utci as U
    rng = np.random.default_rng(2)
    tmrt = (20 + rng.uniform(-15, 40, (30, 30))).astype(np.float32)
    got = U.utci_calculator(np.float32(20.0), np.float32(60.0), tmrt, np.float32(3.0)).cpu().numpy()
    assert got.dtype == np.float32 and got.shape == tmrt.shape
    assert np.max(np.abs(got - OU.utci(20.0, 60.0, tmrt.astype(np.float64), 3.0))) < 1e-3
    ta = rng.uniform(-5, 35, (30, 30)).astype(np.float32)
    got2 = U.utci_calculator(ta, np.float32(50.0), tmrt, np.float32(2.0)).cpu().numpy()
    assert np.max(np.abs(got2 - OU.utci(ta.astype(np.float64), 50.0, tmrt.astype(np.float64), 2.0))) < 1e-3
    assert U.utci_calculator(np.float32(-999.0), np.float32(50.0), tmrt, np.float32(2.0)).cpu().numpy().max() == -999.0


def test_solweig_2022a_calc_39_tuple_over_a_day(cuda):
    """prepare_model + Solweig_2022a_calc hour by hour, state carried by the
    caller as in src/series.py:445-464, against the oracle hour step."""
    from oracle import step as ST
    from solweig_cuda_b200 import model as M, synthetic, sun
    sc = small_scene(40, seed=3)
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    static = dict(s)
    static.update(dict(albedo_b=0.2, absK=0.7, absL=0.95, ewall=0.9, Fside=0.22, Fup=0.06, Fcyl=0.28,
                       usevegdem=1, onlyglobal=1, location=dict(latitude=53.0, longitude=0.0, altitude=3.0),
                       cyl=1, elvis=0, anisotropic_sky=1, patch_option=2))
    prepared = M.prepare_model(dtype=np.float32, **static)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    sol = sun.metdata(met, 53.0, 0.0, 3.0, 0.0)
    loc = static["location"]
    state = {k: np.zeros((40, 40)) for k in ("Tgmap1", "Tgmap1E", "Tgmap1S", "Tgmap1W", "Tgmap1N", "TgOut1")}
    gstate = dict(state)
    fd, ta_, CI, gfd, gta, gCI = 1., 0., 1., 1., 0., 1.
    step = sol.dectime[1] - sol.dectime[0]
    Twater = float(np.mean(met[:, 11]))
    keys = ("dsm", "scale", "rows", "cols", "svf", "svfN", "svfW", "svfE", "svfS", "svfveg", "svfNveg",
            "svfEveg", "svfSveg", "svfWveg", "svfaveg", "svfEaveg", "svfSaveg", "svfWaveg", "svfNaveg",
            "vegdem", "vegdem2")
    for i in range(24):
        if sol.dectime[i] - np.floor(sol.dectime[i]) == 0:
            CI = gCI = 1.
        want = ST.hour_step(s, loc, sol.altitude[i], sol.azimuth[i], sol.zen[i], sol.jday[i], 0.03,
                            sol.dectime[i], sol.altmax[i], met[i, 11], met[i, 10], met[i, 14], met[i, 21],
                            met[i, 22], met[i, 12], Twater, fd, ta_, step, CI=CI, **state)
        got = M.Solweig_2022a_calc(
            i, *(static[k] for k in keys), 0.2, 0.7, 0.95, 0.9, 0.22, 0.06, 0.28, sol.altitude[i],
            sol.azimuth[i], sol.zen[i], sol.jday[i], 1, 1, s["buildings"], loc, 0.03, 1, s["lc_grid"],
            sol.dectime[i], sol.altmax[i], s["dirwalls"], s["walls"], 1, 0, met[i, 11], met[i, 10],
            met[i, 14], met[i, 21], met[i, 22], met[i, 12], s["amaxvalue"], s["bush"], Twater, s["TgK"],
            s["Tstart"], s["alb_grid"], s["emis_grid"], s["TgK_wall"], s["Tstart_wall"], s["TmaxLST"],
            s["TmaxLST_wall"], 1.0, 22.0, s["svfalfa"], s["svfbuveg"], gfd, gta, step, gstate["Tgmap1"],
            gstate["Tgmap1E"], gstate["Tgmap1S"], gstate["Tgmap1W"], gstate["Tgmap1N"], gCI,
            gstate["TgOut1"], s["diffsh"], s["shmat"], s["vegshmat"], s["vbshvegshmat"], 1, s["asvf"], 2,
            prepared=prepared)
        g = dict(zip(M.OUTPUT_NAMES, got))
        assert len(got) == 39
        for k in ("Tmrt", "Kdown", "Kup", "Ldown", "Lup", "Kside", "Lside", "KsideD", "dRad", "Least",
                  "Lsouth", "Lwest", "Lnorth", "Keast", "Knorth", "KsideI", "Tg", "TgOut", "shadow"):
            x = g[k].cpu().numpy()
            y = np.broadcast_to(np.asarray(want[k], dtype=np.float64), x.shape)
            tol = 0.1 if k == "Tmrt" else 0.05 + 1e-4 * np.abs(y).max()
            assert np.max(np.abs(x - y)) <= tol, (i, k, np.max(np.abs(x - y)))
        for k in ("ea", "esky", "CI", "firstdaytime", "timeadd", "radI", "radD", "CI_Tg", "CI_TgG"):
            assert np.isclose(float(g[k]), float(want[k]), rtol=1e-12, atol=1e-12), (i, k)
        fd, ta_, CI = want["firstdaytime"], want["timeadd"], want["CI"]
        gfd, gta, gCI = g["firstdaytime"], g["timeadd"], g["CI"]
        for k in state:
            state[k] = want[k]
            gstate[k] = g[k]


def test_run_timeseries_and_cli_write_outputs(cuda, tmp_path):
    import subprocess
    import sys
    from oracle import step as ST
    from solweig_cuda_b200 import series, synthetic
    sc = small_scene(36, seed=4)
    for name, arr in (("dsm", sc.dsm), ("trees", sc.trees), ("dem", sc.dem), ("lc", sc.landcover)):
        np.save(tmp_path / f"{name}.npy", arr)
    met = np.concatenate([synthetic.make_met(doy=172, latitude=53.0, longitude=0.0, seed=s, days=1)
                          for s in (0,)] + [synthetic.make_met(doy=173, latitude=53.0, longitude=0.0, seed=1)])
    header = "iy id it imin Q* QH QE Qs Qf Wind RH Td press rain Kdn snow ldown fcld wuh xsmd lai_hr Kdiff Kdir Wd"
    np.savetxt(tmp_path / "met.txt", met, header=header, comments="", fmt="%.6f")
    files = series.run_timeseries(tmp_path / "dsm.npy", tmp_path / "trees.npy", tmp_path / "dem.npy",
                                  tmp_path / "met.txt", tmp_path / "out", 0.0, 53.0,
                                  landcover_path=tmp_path / "lc.npy", utc_offset_hours=0.0)
    assert sorted(files["days"]) == ["2025-06-21", "2025-06-22"]
    tm = np.load(files["days"]["2025-06-21"]["TMRT"][0])
    ut = np.load(files["days"]["2025-06-21"]["UTCI"][0])
    assert tm.shape == (24, 36, 36) and ut.shape == (24, 36, 36)
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    want = ST.run_day(s, met[:24], dict(latitude=53.0, longitude=0.0, altitude=3.0), 0.0)
    for h in (6, 12, 18):
        assert np.max(np.abs(tm[h] - want[h]["Tmrt"])) <= 0.1
        ok = ~np.isnan(want[h]["UTCI"])
        assert np.max(np.abs(ut[h][ok] - want[h]["UTCI"][ok])) <= 0.05
    case = {"case_name": "t", "building_dsm_path": "dsm.npy", "tree_path": "trees.npy", "dem_path": "dem.npy",
            "landcover_path": "lc.npy", "met_file": "met.txt", "output_path": "cli_out", "longitude": 0.0,
            "latitude": 53.0, "utc_offset_hours": 0, "core_area_m": 20, "buffer_area_m": 6}
    (tmp_path / "case.json").write_text(json.dumps(case))
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, os.path.join(root, "run.py"), "--case", str(tmp_path / "case.json"),
                        "--no-progress"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    tiles = sorted(p.name for p in (tmp_path / "cli_out").iterdir())
    assert tiles == ["r000_c000", "r000_c001", "r001_c000", "r001_c001"]


def test_run_tiles_equals_run_timeseries_per_tile(cuda, tmp_path):
    """The tiled driver (every tile of a group in one captured graph per day,
    series.run_tiles, as run.py uses it) writes, for each tile, exactly what
    run_timeseries writes for that tile's input window cropped to its core."""
    from solweig_cuda_b200 import series, synthetic, tiling
    sc = small_scene(52, seed=9)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0, seed=3)
    jobs = []
    for t in tiling.tile_windows(52, 52, core=30, halo=8):
        jobs.append({"tile_id": t["tile_id"], "output_core": t["output_core"],
                     **{k: np.ascontiguousarray(tiling.extract(v, t))
                        for k, v in (("dsm", sc.dsm), ("trees", sc.trees), ("dem", sc.dem),
                                     ("landcover", sc.landcover))}})
    got = series.run_tiles(jobs, met, tmp_path / "tiles", 0.0, 53.0, utc_offset_hours=0.0, save_kdown=True)
    assert sorted(got) == sorted(j["tile_id"] for j in jobs)
    for j in jobs:
        ref = series.run_timeseries(j["dsm"], j["trees"], j["dem"], met, tmp_path / "single" / j["tile_id"],
                                    0.0, 53.0, landcover_path=j["landcover"], utc_offset_hours=0.0,
                                    output_core=j["output_core"], save_kdown=True)
        (date,) = ref["days"]
        for var in ("UTCI", "TMRT", "Kdown"):
            a = np.load(got[j["tile_id"]]["days"][date][var][0])
            b = np.load(ref["days"][date][var][0])
            assert a.shape == (24,) + tuple(j["output_core"][2:])
            assert np.array_equal(a.view(np.int32), b.view(np.int32)), (j["tile_id"], var)
