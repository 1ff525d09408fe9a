"""GPU parity at the configured sizes.

C1: the CPU-baseline configuration, 200 x 200 px (synthetic scene seed 0,
53 N, DOY 172, 24 hourly steps), through the batched form (ChosenDay) and the
per-hour form (DayRunner) against (i) the float64 oracle run over the same
day and (ii) UMEP's Solweig_2022a_calc imported in place (tests/golden/
day200.npz, made by tests/golden/make_golden.py with the reference's
compiled wall, SVF and UTCI kernels).  Bars: Tmrt <= 0.1 K and UTCI <= 0.05 K
every hour, identical NaN roofs, the shadow plane and the 8 shadow planes of
the sweep bit-exact (float32 / float64 as produced).

C2: the benched 2000 x 2000 px scene (seed 0): the sweep's planes bit-exact
against the oracle's sweep for the 6.0 degree morning hour and the 60 degree
midday hour, through both the per-hour sweep (8 planes) and the batched
day's sweep (shadow value and sunlit-wall bit of every pixel).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TMRT_TOL = 0.1   # K
UTCI_TOL = 0.05  # K
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
LOC = dict(latitude=53.0, longitude=0.0, altitude=3.0)


def _vegetation(a, t1):
    vegdsm = t1 + a
    vegdsm[vegdsm == a] = 0
    vegdsm2 = t1 * 0.25 + a
    vegdsm2[vegdsm2 == a] = 0
    bush = np.logical_not(vegdsm2 * vegdsm) * vegdsm
    return vegdsm, vegdsm2, bush


def _sun(met):
    from solweig_cuda_b200 import sun
    return sun.metdata(met, 53.0, 0.0, 3.0, 0.0)


@pytest.fixture(scope="module")
def c1(cuda):
    from oracle import step as ST
    from solweig_cuda_b200 import engine, synthetic
    sc = synthetic.make_scene(200, seed=0)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    scene = engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    want = ST.run_day(s, met, LOC, 0.0, outputs=("Tmrt", "UTCI", "shadow"))
    return sc, scene, met, want


@pytest.fixture(scope="module")
def c1_forms(c1):
    import torch
    from solweig_cuda_b200 import batched, engine
    sc, scene, met, _ = c1
    chosen = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0, outputs=("tmrt", "utci", "shadow"))
    got_c = {k: v.cpu().numpy() for k, v in chosen.run_day(met).items()}
    quads = chosen.quads().cpu().numpy()
    torch.cuda.synchronize()
    assert chosen.error_flag() == 0
    plain = engine.DayRunner(scene, 53.0, 0.0, 3.0, 0.0)
    got_p = {k: v.cpu().numpy() for k, v in plain.run_day(met, outputs=("tmrt", "utci", "shadow")).items()}
    return {"chosen": got_c, "plain": got_p, "quads": quads}


@pytest.mark.parametrize("form", ["chosen", "plain"])
def test_c1_day_matches_oracle_every_hour(c1, c1_forms, form):
    _, _, _, want = c1
    got = c1_forms[form]
    for h in range(24):
        d_t = np.max(np.abs(got["tmrt"][h] - want[h]["Tmrt"]))
        assert d_t <= TMRT_TOL, (form, h, d_t)
        ok = ~np.isnan(want[h]["UTCI"])
        assert np.array_equal(np.isnan(got["utci"][h]), ~ok), (form, h)
        d_u = np.max(np.abs(got["utci"][h][ok] - want[h]["UTCI"][ok]))
        assert d_u <= UTCI_TOL, (form, h, d_u)
        sh = np.broadcast_to(want[h]["shadow"], got["shadow"][h].shape).astype(np.float32)
        assert np.array_equal(got["shadow"][h], sh), (form, h)


@pytest.mark.parametrize("form", ["chosen", "plain"])
def test_c1_day_matches_umep_golden(c1_forms, form):
    """Against UMEP itself (imported in place when the fixture was made)."""
    g = np.load(os.path.join(GOLD, "day200.npz"))
    got = c1_forms[form]
    for j, h in enumerate(int(x) for x in g["hours"]):
        assert np.max(np.abs(got["tmrt"][h] - g["Tmrt"][j])) <= TMRT_TOL, (form, h)
        want = g["UTCI"][j]
        ok = ~np.isnan(want)
        assert np.array_equal(np.isnan(got["utci"][h]), ~ok), (form, h)
        assert np.max(np.abs(got["utci"][h][ok] - want[ok])) <= UTCI_TOL, (form, h)
        assert np.array_equal(got["shadow"][h], g["shadow"][j]), (form, h)


def _oracle_planes(sc, scene, azi, alt):
    from oracle import geometry as G
    a = sc.dsm.astype(np.float64)
    t1 = sc.trees.astype(np.float64)
    vegdsm, vegdsm2, bush = _vegetation(a, t1)
    return G.shadow_sweep(a, vegdsm, vegdsm2, azi, alt, 1.0, scene.amaxvalue, bush, scene.walls_host,
                          scene.aspect_host * np.pi / 180.)


def _check_quads(quad, want, walls, ground, psi):
    """The batched sweep's per-pixel outputs against the oracle's planes:
    shadow = sh - (1 - vegsh)(1 - psi) in float32, and the sunlit-wall bit
    (wallsun / walls * buildings == 1, src/umep_solweig.py:606)."""
    vegsh, sh, _, _, wallsun = (np.asarray(want[i], dtype=np.float64) for i in range(5))
    shadow = (sh - (1 - vegsh) * (1 - psi)).astype(np.float32)
    assert np.array_equal(quad[..., 0], shadow)
    bits = quad[..., 3].copy().view(np.int32)
    with np.errstate(all="ignore"):
        sunwall = (wallsun / walls * ground) == 1
    assert np.array_equal((bits & 2) != 0, sunwall)
    assert np.array_equal((bits & 1) != 0, ground == 1)


@pytest.mark.parametrize("hour", [5, 9, 13, 20])
def test_c1_shadow_planes_bit_exact(c1, c1_forms, hour):
    """Hours 5 and 20 have the sun at 6.0 and 6.5 degrees."""
    from solweig_cuda_b200 import ops
    sc, scene, met, _ = c1
    sol = _sun(met)
    azi, alt = float(sol.azimuth[hour]), float(sol.altitude[hour])
    want = _oracle_planes(sc, scene, azi, alt)
    got = ops.cast_shadow(scene, azi, alt).cpu().numpy()
    for i in range(8):
        assert np.array_equal(got[i], np.asarray(want[i], dtype=np.float64)), (hour, i)
    ground = (sc.dsm.astype(np.float64) - sc.dem < 2).astype(np.float64)
    _check_quads(c1_forms["quads"][hour], want, scene.walls_host, ground, 0.03)


@pytest.fixture(scope="module")
def c2(cuda):
    from solweig_cuda_b200 import batched, engine, synthetic
    sc = synthetic.make_scene(2000, seed=0)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    scene = engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    chosen = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0, outputs=("tmrt",))
    chosen.run_day(met)
    quads = chosen.quads()
    return sc, scene, met, {h: quads[h].cpu().numpy() for h in (5, 13)}


@pytest.mark.parametrize("hour", [5, 13])
def test_c2_2000_shadow_planes_bit_exact(c2, hour):
    from solweig_cuda_b200 import ops
    sc, scene, met, quads = c2
    sol = _sun(met)
    azi, alt = float(sol.azimuth[hour]), float(sol.altitude[hour])
    want = _oracle_planes(sc, scene, azi, alt)
    got = ops.cast_shadow(scene, azi, alt).cpu().numpy()
    for i in range(8):
        assert np.array_equal(got[i], np.asarray(want[i], dtype=np.float64)), (hour, i)
    ground = (sc.dsm.astype(np.float64) - sc.dem < 2).astype(np.float64)
    _check_quads(quads[hour], want, scene.walls_host, ground, 0.03)
