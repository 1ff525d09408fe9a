"""The float64 switch (the reference's ``dtype=float64``: ``run.py:27``,
``src/runtime.py:43-49``) on the GPU: the float64 hourly step against the
float64 oracle, through ``engine.DayRunner64``, the drop-in
``Solweig_2022a_calc(dtype=float64)`` and ``run_timeseries(dtype=float64)``.

Bars (the float32 step is held to Tmrt 0.1 K): shadow bit-exact, Tmrt within
1e-10 K and every flux plane within 1e-12 relative (of the plane's largest
value) of the oracle over a full day, on a scene with water pixels; UTCI
(float32, from the float32-rounded Tmrt as the reference) within 1e-3 K.
Measured on a B200: Tmrt 5.7e-14 K, fluxes <= 1.6e-15 relative.
"""
import numpy as np
import pytest

from conftest import small_scene

pytestmark = pytest.mark.gpu

TMRT_TOL = 1e-10
REL_TOL = 1e-12
PLANES = {"tmrt": "Tmrt", "kdown": "Kdown", "kup": "Kup", "ldown": "Ldown", "lup": "Lup",
          "shadow": "shadow", "tg": "Tg", "keast": "Keast", "ksouth": "Ksouth", "kwest": "Kwest",
          "knorth": "Knorth", "least": "Least", "lsouth": "Lsouth", "lwest": "Lwest", "lnorth": "Lnorth",
          "kside_i": "KsideI", "kside_d": "KsideD", "kside": "Kside", "lside": "Lside", "d_rad": "dRad",
          "tg_out": "TgOut"}


CONSTANTS = dict(albedo_b=0.2, absK=0.7, absL=0.95, ewall=0.9, Fside=0.22, Fup=0.06, Fcyl=0.28, usevegdem=1,
                 onlyglobal=1, location=dict(latitude=53.0, longitude=0.0, altitude=3.0), cyl=1, elvis=0,
                 anisotropic_sky=1, patch_option=2)


@pytest.fixture(scope="module")
def water48(cuda):
    """A 48 x 48 px scene with a pond: the prepared inputs of the reference
    (src/series.py:350-365) with lc_grid == 3 (water) on some ground pixels, so
    the water branches (first-direction Lup, Twater ground and night Lup) run."""
    from oracle import step as ST
    from solweig_cuda_b200 import engine
    sc = small_scene(48, seed=3)
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    lc = np.array(s["lc_grid"], copy=True)
    pond = np.zeros(lc.shape, dtype=bool)
    pond[24:30, 4:14] = True
    lc[pond & (s["buildings"] == 1)] = 3
    s["lc_grid"] = lc
    static = dict(s, **CONSTANTS)
    scene = engine.Scene.from_inputs(static)
    assert scene.has_water
    return sc, scene, s


def test_float64_day_matches_the_oracle(water48):
    from oracle import step as ST
    from solweig_cuda_b200 import engine, synthetic
    sc, scene, s = water48
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    loc = dict(latitude=53.0, longitude=0.0, altitude=3.0)
    want = ST.run_day(s, met, loc, 0.0, outputs=tuple(PLANES.values()) + ("UTCI",))
    runner = engine.DayRunner64(scene, 53.0, 0.0, 3.0, 0.0)
    got = runner.run_day(met, outputs=tuple(PLANES) + ("utci",))
    assert got["tmrt"].dtype.is_floating_point and got["tmrt"].element_size() == 8
    assert got["utci"].element_size() == 4
    host = {k: v.cpu().numpy() for k, v in got.items()}
    worst = {}
    for h in range(24):
        for k, name in PLANES.items():
            y = np.broadcast_to(np.asarray(want[h][name], dtype=np.float64), host[k][h].shape)
            err = float(np.max(np.abs(host[k][h] - y)))
            scale = 1.0 if k == "tmrt" else max(1.0, float(np.max(np.abs(y))))
            worst[k] = max(worst.get(k, 0.0), err / scale)
        ok = ~np.isnan(want[h]["UTCI"])
        assert np.array_equal(np.isnan(host["utci"][h]), ~ok), h
        worst["utci"] = max(worst.get("utci", 0.0),
                            float(np.max(np.abs(host["utci"][h][ok] - want[h]["UTCI"][ok]))))
        assert np.array_equal(host["shadow"][h], np.asarray(want[h]["shadow"], dtype=np.float64)), h
    print("float64 step, worst error per plane (Tmrt, UTCI absolute K; others relative):", worst)
    assert worst["tmrt"] <= TMRT_TOL, worst
    assert worst["utci"] <= 1e-3, worst
    for k in PLANES:
        if k != "tmrt":
            assert worst[k] <= REL_TOL, (k, worst)


def test_float64_step_is_closer_to_the_oracle_than_float32(water48):
    """The float32 step's Tmrt error over the same day bounds the float64
    step's from above by orders of magnitude."""
    from oracle import step as ST
    from solweig_cuda_b200 import engine, synthetic
    sc, scene, s = water48
    met = synthetic.make_met(doy=200, latitude=53.0, longitude=0.0, seed=4)
    loc = dict(latitude=53.0, longitude=0.0, altitude=3.0)
    want = np.stack([w["Tmrt"] for w in ST.run_day(s, met, loc, 0.0, outputs=("Tmrt",))])
    t64 = engine.DayRunner64(scene, 53.0, 0.0, 3.0, 0.0).run_day(met, outputs=("tmrt",))["tmrt"].cpu().numpy()
    t32 = engine.DayRunner(scene, 53.0, 0.0, 3.0, 0.0).run_day(met, outputs=("tmrt",))["tmrt"].cpu().numpy()
    e64 = float(np.max(np.abs(t64 - want)))
    e32 = float(np.max(np.abs(t32 - want)))
    print(f"Tmrt error: float64 step {e64:.3e} K, float32 step {e32:.3e} K")
    assert e64 <= TMRT_TOL and e32 <= 0.1
    assert e64 * 1e5 <= e32


def test_solweig_2022a_calc_float64_equals_the_day_runner(water48):
    """The drop-in step with dtype=float64, state carried by the caller as in
    src/series.py:445-464, returns float64 planes identical to DayRunner64."""
    import torch
    from solweig_cuda_b200 import engine, model as M, synthetic, sun
    sc, scene, s = water48
    static = dict(s, **CONSTANTS)
    prepared = M.prepare_model(dtype=np.float64, **static)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    sol = sun.metdata(met, 53.0, 0.0, 3.0, 0.0)
    loc = static["location"]
    runner = engine.DayRunner64(prepared.scene, 53.0, 0.0, 3.0, 0.0)
    day = runner.run_day(met, outputs=("tmrt", "kdown", "lside", "least", "tg_out"))
    rows, cols = s["rows"], s["cols"]
    state = {k: np.zeros((rows, cols)) for k in ("Tgmap1", "Tgmap1E", "Tgmap1S", "Tgmap1W", "Tgmap1N", "TgOut1")}
    fd, ta_, CI = 1., 0., 1.
    step = sol.dectime[1] - sol.dectime[0]
    Twater = float(np.mean(met[:, 11]))
    keys = ("dsm", "scale", "rows", "cols", "svf", "svfN", "svfW", "svfE", "svfS", "svfveg", "svfNveg",
            "svfEveg", "svfSveg", "svfWveg", "svfaveg", "svfEaveg", "svfSaveg", "svfWaveg", "svfNaveg",
            "vegdem", "vegdem2")
    for i in range(24):
        if sol.dectime[i] - np.floor(sol.dectime[i]) == 0:
            CI = 1.
        got = M.Solweig_2022a_calc(
            i, *(static[k] for k in keys), 0.2, 0.7, 0.95, 0.9, 0.22, 0.06, 0.28, sol.altitude[i],
            sol.azimuth[i], sol.zen[i], sol.jday[i], 1, 1, s["buildings"], loc, 0.03, 1, s["lc_grid"],
            sol.dectime[i], sol.altmax[i], s["dirwalls"], s["walls"], 1, 0, met[i, 11], met[i, 10],
            met[i, 14], met[i, 21], met[i, 22], met[i, 12], s["amaxvalue"], s["bush"], Twater, s["TgK"],
            s["Tstart"], s["alb_grid"], s["emis_grid"], s["TgK_wall"], s["Tstart_wall"], s["TmaxLST"],
            s["TmaxLST_wall"], 1.0, 22.0, s["svfalfa"], s["svfbuveg"], fd, ta_, step, state["Tgmap1"],
            state["Tgmap1E"], state["Tgmap1S"], state["Tgmap1W"], state["Tgmap1N"], CI,
            state["TgOut1"], s["diffsh"], s["shmat"], s["vegshmat"], s["vbshvegshmat"], 1, s["asvf"], 2,
            dtype=np.float64, prepared=prepared)
        g = dict(zip(M.OUTPUT_NAMES, got))
        for name, key in (("Tmrt", "tmrt"), ("Kdown", "kdown"), ("Lside", "lside"), ("Least", "least"),
                          ("TgOut", "tg_out")):
            assert g[name].dtype == torch.float64, name
            assert torch.equal(g[name], day[key][i]), (i, name)
        fd, ta_, CI = g["firstdaytime"], g["timeadd"], g["CI"]
        for k in state:
            assert g[k].dtype == torch.float64
            state[k] = g[k]


def test_run_timeseries_float64_writes_the_float64_step(water48, tmp_path):
    """run_timeseries(dtype=float64) runs the float64 step: its files hold the
    float32 rounding of DayRunner64's planes (the reference writes float32)."""
    from solweig_cuda_b200 import engine, series, synthetic
    sc = water48[0]
    scene = engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    for name, arr in (("dsm", sc.dsm), ("trees", sc.trees), ("dem", sc.dem), ("lc", sc.landcover)):
        np.save(tmp_path / f"{name}.npy", arr)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    files = series.run_timeseries(str(tmp_path / "dsm.npy"), str(tmp_path / "trees.npy"),
                                  str(tmp_path / "dem.npy"), met, str(tmp_path / "out"), 0.0, 53.0,
                                  landcover_path=str(tmp_path / "lc.npy"), utc_offset_hours=0.0,
                                  dtype=np.float64)
    (rec,) = files["days"].values()
    tm = np.load(rec["TMRT"][0])
    ut = np.load(rec["UTCI"][0])
    ref = engine.DayRunner64(scene, 53.0, 0.0, 3.0, 0.0).run_day(met, outputs=("tmrt", "utci"))
    assert tm.dtype == np.float32 and tm.shape == (24,) + scene.shape
    assert np.array_equal(tm, ref["tmrt"].cpu().numpy().astype(np.float32))
    u = ref["utci"].cpu().numpy()
    assert np.array_equal(np.isnan(ut), np.isnan(u)) and np.array_equal(ut[~np.isnan(u)], u[~np.isnan(u)])


def test_run_tiles_float64_equals_run_timeseries_per_tile(cuda, tmp_path):
    """run_tiles(dtype=float64) writes, for each tile, what run_timeseries
    (dtype=float64) writes for that tile's window cropped to its core."""
    from solweig_cuda_b200 import series, synthetic, tiling
    sc = small_scene(40, seed=6)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0, seed=2)
    jobs = []
    for t in tiling.tile_windows(40, 40, core=24, halo=6):
        jobs.append({"tile_id": t["tile_id"], "output_core": t["output_core"],
                     **{k: np.ascontiguousarray(tiling.extract(v, t))
                        for k, v in (("dsm", sc.dsm), ("trees", sc.trees), ("dem", sc.dem),
                                     ("landcover", sc.landcover))}})
    got = series.run_tiles(jobs, met, tmp_path / "tiles", 0.0, 53.0, utc_offset_hours=0.0, dtype=np.float64)
    for j in jobs:
        ref = series.run_timeseries(j["dsm"], j["trees"], j["dem"], met, tmp_path / "single" / j["tile_id"],
                                    0.0, 53.0, landcover_path=j["landcover"], utc_offset_hours=0.0,
                                    output_core=j["output_core"], dtype=np.float64)
        (date,) = ref["days"]
        for var in ("UTCI", "TMRT"):
            a = np.load(got[j["tile_id"]]["days"][date][var][0])
            b = np.load(ref["days"][date][var][0])
            assert a.shape == (24,) + tuple(j["output_core"][2:])
            assert np.array_equal(a.view(np.int32), b.view(np.int32)), (j["tile_id"], var)


def test_float64_day_matches_umep_itself(cuda):
    """The float64 step against UMEP's own Solweig_2022a_calc over a day
    (tests/golden/day.npz: the reference's numpy path imported in place, on the
    statics of tests/golden/svf.npz and the golden walls), at the bar the
    oracle itself is pinned to (1e-9)."""
    import os
    from oracle import step as ST
    from solweig_cuda_b200 import engine, synthetic
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    g = np.load(os.path.join(gold, "day.npz"))
    sv = np.load(os.path.join(gold, "svf.npz"))
    P = int(sv["patches"])
    cubes = [np.unpackbits(sv[k], axis=2)[:, :, :P].astype(np.float64) for k in ("shmat", "vegmat", "vbmat")]
    order = (0, 10, 1, 11, 6, 4, 14, 9, 2, 12, 7, 5, 3, 13, 8)
    planes = sv["planes"]
    svf = tuple(planes[i] for i in order) + (cubes[1], cubes[2], cubes[0], planes[15])
    sc = synthetic.make_scene(32, seed=6)
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover, walls=g["walls"],
                          aspect=g["aspect"], svf=svf)
    scene = engine.Scene.from_inputs(dict(s, **CONSTANTS))
    names = {"tmrt": "Tmrt", "kdown": "Kdown", "kup": "Kup", "ldown": "Ldown", "lup": "Lup", "kside": "Kside",
             "lside": "Lside", "shadow": "shadow"}
    got = engine.DayRunner64(scene, 53.0, 0.0, 3.0, 0.0).run_day(g["met"], outputs=tuple(names))
    worst = 0.0
    for k, name in names.items():
        worst = max(worst, float(np.max(np.abs(got[k].cpu().numpy() - g[name]))))
    print(f"float64 step vs UMEP day: worst absolute difference {worst:.3e}")
    assert worst < 1e-9
