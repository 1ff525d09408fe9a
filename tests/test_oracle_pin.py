"""Pin the oracle (and the product's FP64 host scalars) to the reference.

Against the committed golden fixtures (generated from the reference by
tests/golden/make_golden.py) on every machine, and against the reference
imported in place when its tree is present.
"""
import os

import numpy as np
import pytest

from conftest import have_reference

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gold(name):
    return np.load(os.path.join(GOLD, name))


def test_spa_matches_reference_bit_for_bit():
    from solweig_cuda_b200 import sun
    g = gold("sun.npz")
    for y, mo, d, h, mi, utc, lat, lon, alt, zen, azi in g["spa"]:
        z, a = sun.sun_position(int(y), int(mo), int(d), int(h), int(mi), 0, utc, lat, lon, alt)
        assert z == zen and a == azi


@pytest.mark.parametrize("tag,lat,lon", [("dublin", 53.3473, -6.2591), ("synthetic", 53.0, 0.0)])
def test_metdata_matches_reference(tag, lat, lon):
    from solweig_cuda_b200 import sun
    g = gold("sun.npz")
    met = g["met_" + tag]
    s = sun.metdata(met, lat, lon, 3.0, 0.0)
    for n in ("altitude", "azimuth", "zen", "jday", "dectime", "altmax"):
        assert np.array_equal(getattr(s, n), g[f"{tag}_{n}"]), n


def test_host_scalars_match_reference():
    from solweig_cuda_b200 import sky, sun
    g = gold("scalars.npz")
    met = g["met"]
    s = sun.metdata(met, 53.0, 0.0, 3.0, 0.0)
    L = sky.patch_layout(2)
    for (i, I0, CI, Kt, radI, radD, snup), lv in zip(g["rec"], g["lv"]):
        i = int(i)
        ta, rh, rad_g, pk = met[i, 11], met[i, 10], met[i, 14], met[i, 12]
        mI0, mCI, mKt, _, _ = sun.clearness_index(s.zen[i], s.jday[i], ta, rh / 100., rad_g, 53.0, pk)
        assert (mI0, mCI, mKt) == (I0, CI, Kt)
        mradI, mradD = sun.diffuse_fraction(rad_g, s.altitude[i], mKt, ta, rh)
        assert (mradI, mradD) == (radI, radD)
        assert sun.daylen(s.jday[i], 53.0)[3] == snup
        assert np.array_equal(sky.perez(s.zen[i] * 180 / np.pi, s.azimuth[i], radD, radI, s.jday[i], L), lv)


def test_oracle_shadows_bit_exact():
    from oracle import geometry as G
    g = gold("shadow.npz")
    a, t1 = g["dsm"], g["trees"]
    vegdsm = t1 + a
    vegdsm[vegdsm == a] = 0
    vegdsm2 = t1 * 0.25 + a
    vegdsm2[vegdsm2 == a] = 0
    bush = np.logical_not(vegdsm2 * vegdsm) * vegdsm
    assert np.array_equal(G.wall_heights(a, 3.0), g["walls"])
    asp = g["aspect"] * np.pi / 180.
    for (azi, alt), want, want13 in zip(g["suns"], g["planes"], g["planes13"]):
        got = G.shadow_sweep(a, vegdsm, vegdsm2, azi, alt, 1.0, float(g["amax"]), bush, g["walls"], asp)
        for i in range(8):
            assert np.array_equal(np.asarray(got[i], float), want[i]), (azi, alt, i)
        got13 = G.shadow_sweep_buildings(a, azi, alt, 1.0, g["walls"], asp)
        for i in range(5):
            assert np.array_equal(np.asarray(got13[i], float), want13[i]), (azi, alt, i)


def test_oracle_svf_matches_reference_kernels():
    from oracle import geometry as G
    g = gold("svf.npz")
    a, t1 = g["dsm"], g["trees"]
    vegdsm = t1 + a
    vegdsm[vegdsm == a] = 0
    vegdsm2 = t1 * 0.25 + a
    vegdsm2[vegdsm2 == a] = 0
    bush = np.logical_not(vegdsm2 * vegdsm) * vegdsm
    P = int(g["patches"])
    shm, vegm, vbm = G.svf_patch_masks(a, vegdsm, vegdsm2, bush, 1.0, float(g["amax"]), 2)
    for mine, key in ((shm, "shmat"), (vegm, "vegmat"), (vbm, "vbmat")):
        want = np.unpackbits(g[key], axis=2)[:, :, :P]
        assert np.array_equal(mine.astype(np.uint8), want), key
    red = G.svf_reduce(shm, vegm, vbm, vegdsm2)
    for i in range(16):
        assert np.max(np.abs(red[i] - g["planes"][i])) < 1e-12, i


def test_oracle_utci_matches_reference_kernel():
    from oracle import utci as OU
    rows = gold("utci.npz")["rows"]
    for r in rows:
        ta, rh, va = r[:3]
        tmrt, ref, coef = r[3:19], r[19:35], r[35:42]
        mine = OU.utci(ta, rh, tmrt, va)
        # the reference evaluates the vapour pressure and powers in float32
        assert np.max(np.abs(mine - ref)) < 2e-3
        c = OU.utci_collapsed(ta, rh, va)
        assert np.allclose(c, coef, rtol=2e-3, atol=1e-9)


def test_oracle_day_matches_umep():
    """The oracle hour loop against UMEP's Solweig_2022a_calc on the same statics."""
    from oracle import step as ST
    from solweig_cuda_b200 import synthetic
    g = gold("day.npz")
    sv = gold("svf.npz")
    P = int(sv["patches"])
    cubes = [np.unpackbits(sv[k], axis=2)[:, :, :P].astype(np.float64) for k in ("shmat", "vegmat", "vbmat")]
    order = (0, 10, 1, 11, 6, 4, 14, 9, 2, 12, 7, 5, 3, 13, 8)
    planes = sv["planes"]
    svf = tuple(planes[i] for i in order) + (cubes[1], cubes[2], cubes[0], planes[15])
    sc = synthetic.make_scene(32, seed=6)
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover, walls=g["walls"],
                          aspect=g["aspect"], svf=svf)
    res = ST.run_day(s, g["met"], dict(latitude=53.0, longitude=0.0, altitude=3.0), 0.0,
                     outputs=("Tmrt", "Kdown", "Kup", "Ldown", "Lup", "Kside", "Lside", "shadow"))
    for h in range(24):
        for k in ("Tmrt", "Kdown", "Kup", "Ldown", "Lup", "Kside", "Lside", "shadow"):
            assert np.max(np.abs(res[h][k] - g[k][h])) < 1e-9, (h, k)


@pytest.mark.skipif(not have_reference(), reason="reference tree not present")
def test_oracle_gvf_matches_umep_live(umep):
    from oracle import geometry as G, ground as GR
    from solweig_cuda_b200 import synthetic
    sc = synthetic.make_scene(40, seed=2)
    a = sc.dsm.astype(np.float64)
    t1 = sc.trees.astype(np.float64)
    vegdsm = t1 + a
    vegdsm[vegdsm == a] = 0
    vegdsm2 = t1 * 0.25 + a
    vegdsm2[vegdsm2 == a] = 0
    bush = np.logical_not(vegdsm2 * vegdsm) * vegdsm
    walls = G.wall_heights(a, 3.0)
    aspect = G.wall_aspect(walls, a, 1.0)
    amax = max(a.max() - a.min(), t1.max())
    rng = np.random.default_rng(0)
    buildings = (a < 2).astype(float)
    vegsh, sh, _, _, wallsun, *_ = G.shadow_sweep(a, vegdsm, vegdsm2, 135., 35., 1.0, amax, bush,
                                                  walls, aspect * np.pi / 180.)
    shadow = sh - (1 - vegsh) * (1 - 0.03)
    Tg = rng.uniform(0, 10, a.shape)
    emis = rng.uniform(0.9, 0.98, a.shape)
    alb = rng.uniform(0.1, 0.3, a.shape)
    lc = np.where(rng.uniform(size=a.shape) < 0.05, 3.0, 1.0)
    with np.errstate(all="ignore"):
        ref = umep.gvf_2018a(wallsun.copy(), walls.copy(), buildings.copy(), 1.0, shadow.copy(), 1.0,
                             22.0, aspect.copy(), Tg.copy(), 5.0, 20.0, emis, 0.9, alb, 5.67051e-8, 0.2,
                             40, 40, 18.0, lc, 1)
    mine, _ = GR.gvf(wallsun, walls, buildings, 1.0, shadow, 1.0, 22.0, aspect, Tg, 5.0, 20.0, emis,
                     0.9, alb, 5.67051e-8, 0.2, 18.0, lc, 1)
    for x, y in zip(ref, mine):
        assert np.array_equal(np.asarray(x, float), np.asarray(y, float))


def test_oracle_c1_day_matches_umep_200():
    """The oracle at the CPU-baseline configuration (200 x 200 px, seed 0,
    53 N, DOY 172), with its own walls, aspect and 153-patch SVF, against UMEP's
    Solweig_2022a_calc fed by the reference's compiled wall and SVF kernels
    (day200.npz, float32-rounded): Tmrt within 1e-4 K, the shadow plane
    exact to float32, UTCI within the 2e-3 K of the float32 reference UTCI."""
    from oracle import step as ST
    from solweig_cuda_b200 import synthetic
    g = gold("day200.npz")
    sc = synthetic.make_scene(200, seed=0)
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    hours = [int(h) for h in g["hours"]]
    res = ST.run_day(s, g["met"], dict(latitude=53.0, longitude=0.0, altitude=3.0), 0.0,
                     outputs=("Tmrt", "UTCI", "shadow"))
    for j, h in enumerate(hours):
        assert np.max(np.abs(res[h]["Tmrt"] - g["Tmrt"][j])) < 1e-4, h
        sh = np.broadcast_to(res[h]["shadow"], (200, 200)).astype(np.float32)
        assert np.array_equal(sh, g["shadow"][j]), h
        want = g["UTCI"][j]
        assert np.array_equal(np.isnan(res[h]["UTCI"]), np.isnan(want)), h
        ok = ~np.isnan(want)
        assert np.max(np.abs(res[h]["UTCI"][ok] - want[ok])) < 2e-3, h
