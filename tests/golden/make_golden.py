"""Generate the golden fixtures in this directory from the reference itself.

Run in a checkout that has the reference tree (default ``/root/reference``,
override with SOLWEIG_REFERENCE_TREE) and the compiled reference kernels
(``make -C oracle``):

    python tests/golden/make_golden.py            # every fixture
    python tests/golden/make_golden.py day200     # only day200.npz

Every value stored here is computed by reference code: the UMEP numpy
routines of ``src/umep_solweig.py`` imported in place, the ray setup of
``src/svf.py`` imported in place, and the reference's CUDA kernels
``src/kernels/geometry.cu`` / ``utci.cu`` compiled for the CPU into
``oracle/_ref/libsolweig_ref.so``.  Inputs come from the seeded synthetic
generator of the package.  The fixtures pin the oracle (tests/test_oracle_pin.py)
and, through it, the GPU parity tests on machines without the reference.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("SOLWEIG_REFERENCE_TREE", "/root/reference")
sys.path.insert(0, ROOT)
sys.path.insert(0, REF)

import src.umep_solweig as U  # noqa: E402  (reference, imported in place)
import src.svf as RS  # noqa: E402

from solweig_cuda_b200 import synthetic  # noqa: E402
from oracle import geometry as G  # noqa: E402

LIB = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libsolweig_ref.so"))
VP = ctypes.c_void_p


def p(a):
    return ctypes.c_void_p(a.ctypes.data)


def sun_fixture():
    rng = np.random.default_rng(11)
    rows = []
    for _ in range(64):
        y, mo, d = int(rng.integers(1990, 2040)), int(rng.integers(1, 13)), int(rng.integers(1, 29))
        h, mi, utc = int(rng.integers(0, 24)), int(rng.integers(0, 60)), float(rng.integers(-10, 11))
        lat, lon, alt = float(rng.uniform(-60, 70)), float(rng.uniform(-180, 180)), float(rng.uniform(0, 2000))
        r = U.sun_position(dict(year=y, month=mo, day=d, hour=h, min=mi, sec=0, UTC=utc),
                           dict(latitude=lat, longitude=lon, altitude=alt))
        rows.append([y, mo, d, h, mi, utc, lat, lon, alt, float(np.ravel(r["zenith"])[0]),
                     float(np.ravel(r["azimuth"])[0])])
    met_dublin = np.loadtxt(os.path.join(REF, "examples", "data", "met.txt"), skiprows=1)
    loc = dict(latitude=53.3473, longitude=-6.2591, altitude=3.0)
    md = U.Solweig_2015a_metdata_noload(met_dublin, loc, 0.0)
    met_syn = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    ms = U.Solweig_2015a_metdata_noload(met_syn, dict(latitude=53.0, longitude=0.0, altitude=3.0), 0.0)
    names = ("year", "altitude", "azimuth", "zen", "jday", "leafon", "dectime", "altmax")
    out = {"spa": np.asarray(rows), "met_dublin": met_dublin, "met_synthetic": met_syn}
    for tag, res in (("dublin", md), ("synthetic", ms)):
        for n, v in zip(names, res):
            out[f"{tag}_{n}"] = np.ravel(v)
    np.savez_compressed(os.path.join(HERE, "sun.npz"), **out)


def scalars_fixture():
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    loc = dict(latitude=53.0, longitude=0.0, altitude=3.0)
    s = U.Solweig_2015a_metdata_noload(met, loc, 0.0)
    alt, azi, zen, jday = (np.ravel(x) for x in (s[1], s[2], s[3], s[4]))
    rec = []
    lvs = []
    for i in range(24):
        if alt[i] <= 0:
            continue
        ta, rh, rad_g, pk = met[i, 11], met[i, 10], met[i, 14], met[i, 12]
        I0, CI, Kt, I0et, CIu = U.clearnessindex_2013b(zen[i], jday[i], ta, rh / 100., rad_g, loc, pk)
        radI, radD = U.diffusefraction(rad_g, alt[i], Kt, ta, rh)
        lv, _, _ = U.Perez_v3(zen[i] * 180 / np.pi, azi[i], radD, radI, jday[i], 1, 2)
        _, _, _, snup = U.daylen(jday[i], 53.0)
        rec.append([i, I0, CI, Kt, radI, radD, snup])
        lvs.append(lv)
    np.savez_compressed(os.path.join(HERE, "scalars.npz"), rec=np.asarray(rec, dtype=np.float64),
                        lv=np.asarray(lvs), met=met)


def _scene(n, seed):
    sc = synthetic.make_scene(n, seed=seed)
    a = sc.dsm.astype(np.float64)
    t1 = sc.trees.astype(np.float64)
    vegdsm = t1 + a
    vegdsm[vegdsm == a] = 0
    vegdsm2 = t1 * 0.25 + a
    vegdsm2[vegdsm2 == a] = 0
    bush = np.logical_not(vegdsm2 * vegdsm) * vegdsm
    amax = max(a.max() - a.min(), t1.max())
    return sc, a, t1, vegdsm, vegdsm2, bush, amax


def ref_walls(a):
    rows, cols = a.shape
    walls = np.empty_like(a)
    LIB.ref_wall_heights(p(a), p(walls), rows, cols, ctypes.c_double(3.0))
    return walls


def shadow_fixture():
    sc, a, t1, vegdsm, vegdsm2, bush, amax = _scene(40, 4)
    walls = ref_walls(a)
    aspect = G.wall_aspect(walls, a, 1.0)
    suns = np.array([[45., 30.], [100.3, 12.5], [180., 58.8], [200., 6.], [271.7, 3.2],
                     [350., 20.], [90., 45.], [315., 60.]])
    planes = []
    planes13 = []
    for azi, alt in suns:
        r = U.shadowingfunction_wallheight_23(a.copy(), vegdsm.copy(), vegdsm2.copy(), azi, alt, 1.0,
                                              amax, bush.copy(), walls.copy(), aspect * np.pi / 180.)
        planes.append(np.stack([np.asarray(x, dtype=np.float64) for x in r]))
        r13 = U.shadowingfunction_wallheight_13(a.copy(), azi, alt, 1.0, walls.copy(),
                                                aspect * np.pi / 180.)
        planes13.append(np.stack([np.asarray(x, dtype=np.float64) for x in r13]))
    np.savez_compressed(os.path.join(HERE, "shadow.npz"), dsm=a, trees=t1, walls=walls,
                        aspect=aspect, suns=suns, planes=np.asarray(planes),
                        planes13=np.asarray(planes13), amax=amax)


def svf_fixture():
    sc, a, t1, vegdsm, vegdsm2, bush, amax = _scene(32, 6)
    rows, cols = a.shape
    md = RS._prepare_rays_numpy(2, rows, cols, amax, 1.0)
    P = md["patches"]
    sh = np.empty((rows, cols, P), np.float32)
    veg = np.empty_like(sh)
    vb = np.empty_like(sh)
    af, tf, bf = (x.astype(np.float32) for x in (a, vegdsm, vegdsm2))
    bp = (bush > 1).astype(np.uint8)
    offs = np.ascontiguousarray(md["offsets"], dtype=np.int32)
    h32 = np.ascontiguousarray(md["heights32"])
    h64 = np.ascontiguousarray(md["heights"])
    ln = np.ascontiguousarray(md["lengths"], dtype=np.int32)
    LIB.ref_svf_visibility(p(af), p(tf), p(bf), p(a), p(vegdsm), p(vegdsm2), p(bp), rows, cols, P,
                           int(md["capacity"]), p(offs), p(h32), p(h64), p(ln), p(sh), p(veg), p(vb))
    out = np.empty((16, rows * cols))
    LIB.ref_svf_reduce.argtypes = [VP] * 7 + [ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_double, VP]
    sec = np.ascontiguousarray(md["sectors"], np.uint8)
    bo = np.ascontiguousarray(md["band_offsets"], np.int32)
    w = np.ascontiguousarray(md["weights"])
    LIB.ref_svf_reduce(sh.ctypes.data, veg.ctypes.data, vb.ctypes.data, vegdsm2.ctypes.data,
                       sec.ctypes.data, bo.ctypes.data, w.ctypes.data, rows * cols, P, int(md["bands"]),
                       0.03, out.ctypes.data)
    np.savez_compressed(os.path.join(HERE, "svf.npz"), dsm=a, trees=t1, amax=amax,
                        shmat=np.packbits(sh.astype(np.uint8), axis=2),
                        vegmat=np.packbits(veg.astype(np.uint8), axis=2),
                        vbmat=np.packbits(vb.astype(np.uint8), axis=2), patches=P,
                        planes=out.reshape(16, rows, cols))


def utci_fixture():
    rng = np.random.default_rng(3)
    f = ctypes.c_float
    LIB.ref_utci_scalar.argtypes = [f, f, f, VP, VP, ctypes.c_longlong, VP]
    rows = []
    for _ in range(40):
        ta = np.float32(rng.uniform(-20, 40))
        rh = np.float32(rng.uniform(10, 100))
        va = np.float32(rng.uniform(0.5, 15))
        tmrt = (ta + rng.uniform(-20, 60, 16)).astype(np.float32)
        out = np.empty(16, np.float32)
        co = np.empty(7)
        LIB.ref_utci_scalar(ta, rh, va, tmrt.ctypes.data, out.ctypes.data, 16, co.ctypes.data)
        rows.append(np.concatenate([[ta, rh, va], tmrt, out, co]))
    np.savez_compressed(os.path.join(HERE, "utci.npz"), rows=np.asarray(rows, dtype=np.float64))


def day_fixture():
    """24 hours of UMEP Solweig_2022a_calc on a 32 x 32 scene whose SVF comes
    from the reference's own visibility kernel and ray setup."""
    from oracle import step as ST
    sc = synthetic.make_scene(32, seed=6)
    d = np.load(os.path.join(HERE, "svf.npz"))
    P = int(d["patches"])
    cubes = [np.unpackbits(d[k], axis=2)[:, :, :P].astype(np.float64) for k in ("shmat", "vegmat", "vbmat")]
    order = (0, 10, 1, 11, 6, 4, 14, 9, 2, 12, 7, 5, 3, 13, 8)
    planes = d["planes"]
    svf = tuple(planes[i] for i in order) + (cubes[1], cubes[2], cubes[0], planes[15])
    a = sc.dsm.astype(np.float64)
    walls = ref_walls(a)
    aspect = G.wall_aspect(walls, a, 1.0)
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover, walls=walls,
                          aspect=aspect, svf=svf)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    loc = dict(latitude=53.0, longitude=0.0, altitude=3.0)
    sol = U.Solweig_2015a_metdata_noload(met, loc, 0.0)
    alt, azi, zen, jday, dectime, altmax = (np.ravel(sol[k]) for k in (1, 2, 3, 4, 6, 7))
    names = ("Tmrt", "Kdown", "Kup", "Ldown", "Lup", "Kside", "Lside", "shadow")
    keep = {k: [] for k in names}
    state = {k: np.zeros((32, 32)) for k in ("Tgmap1", "Tgmap1E", "Tgmap1S", "Tgmap1W", "Tgmap1N", "TgOut1")}
    fd, ta_, CI = 1., 0., 1.
    Twater = float(np.mean(met[:, 11]))
    step = dectime[1] - dectime[0]
    for i in range(24):
        if dectime[i] - np.floor(dectime[i]) == 0:
            CI = 1.
        r = U.Solweig_2022a_calc(
            i, s["dsm"], 1.0, 32, 32, s["svf"], s["svfN"], s["svfW"], s["svfE"], s["svfS"], s["svfveg"],
            s["svfNveg"], s["svfEveg"], s["svfSveg"], s["svfWveg"], s["svfaveg"], s["svfEaveg"],
            s["svfSaveg"], s["svfWaveg"], s["svfNaveg"], s["vegdem"], s["vegdem2"], 0.2, 0.7, 0.95, 0.9,
            0.22, 0.06, 0.28, alt[i], azi[i], zen[i], jday[i], 1, 1, s["buildings"], loc, 0.03, 1,
            s["lc_grid"], dectime[i], altmax[i], s["dirwalls"], s["walls"], 1, 0, met[i, 11],
            met[i, 10], met[i, 14], met[i, 21], met[i, 22], met[i, 12], s["amaxvalue"], s["bush"],
            Twater, s["TgK"].copy(), s["Tstart"], s["alb_grid"], s["emis_grid"], s["TgK_wall"],
            s["Tstart_wall"], s["TmaxLST"], s["TmaxLST_wall"], 1.0, 22.0, s["svfalfa"], s["svfbuveg"],
            fd, ta_, step, state["Tgmap1"], state["Tgmap1E"], state["Tgmap1S"], state["Tgmap1W"],
            state["Tgmap1N"], CI, state["TgOut1"], s["diffsh"], s["shmat"], s["vegshmat"],
            s["vbshvegshmat"], 1, s["asvf"], 2)
        o = dict(zip(ST.OUTPUT_NAMES, r))
        fd, ta_, CI = o["firstdaytime"], o["timeadd"], o["CI"]
        for k in state:
            state[k] = o[k]
        for k in names:
            keep[k].append(np.broadcast_to(np.asarray(o[k], dtype=np.float64), (32, 32)))
    np.savez_compressed(os.path.join(HERE, "day.npz"), met=met, walls=walls, aspect=aspect,
                        **{k: np.asarray(v) for k, v in keep.items()})


def _ref_svf(a, vegdsm, vegdsm2, bush, amax):
    """Visibility cubes and the 16 reduced planes of the reference's own SVF
    kernels (``src/kernels/geometry.cu:77-159``, compiled for the CPU) with the
    ray setup of ``src/svf.py`` imported in place."""
    rows, cols = a.shape
    md = RS._prepare_rays_numpy(2, rows, cols, amax, 1.0)
    P = md["patches"]
    sh = np.empty((rows, cols, P), np.float32)
    veg = np.empty_like(sh)
    vb = np.empty_like(sh)
    af, tf, bf = (np.ascontiguousarray(x, dtype=np.float32) for x in (a, vegdsm, vegdsm2))
    bp = (bush > 1).astype(np.uint8)
    offs = np.ascontiguousarray(md["offsets"], dtype=np.int32)
    h32 = np.ascontiguousarray(md["heights32"])
    h64 = np.ascontiguousarray(md["heights"])
    ln = np.ascontiguousarray(md["lengths"], dtype=np.int32)
    LIB.ref_svf_visibility(p(af), p(tf), p(bf), p(a), p(vegdsm), p(vegdsm2), p(bp), rows, cols, P,
                           int(md["capacity"]), p(offs), p(h32), p(h64), p(ln), p(sh), p(veg), p(vb))
    out = np.empty((16, rows * cols))
    LIB.ref_svf_reduce.argtypes = [VP] * 7 + [ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_double, VP]
    sec = np.ascontiguousarray(md["sectors"], np.uint8)
    bo = np.ascontiguousarray(md["band_offsets"], np.int32)
    w = np.ascontiguousarray(md["weights"])
    LIB.ref_svf_reduce(sh.ctypes.data, veg.ctypes.data, vb.ctypes.data, vegdsm2.ctypes.data,
                       sec.ctypes.data, bo.ctypes.data, w.ctypes.data, rows * cols, P, int(md["bands"]),
                       0.03, out.ctypes.data)
    return P, (sh, veg, vb), out.reshape(16, rows, cols)


# Hours of the 200 x 200 day stored in day200.npz: a night hour, both
# low-sun hours (6.0 and 6.5 degrees), a morning and the midday sun.
DAY200_HOURS = (2, 5, 9, 13, 20)


def day200_fixture():
    """24 hours of UMEP ``Solweig_2022a_calc`` (imported in place) on the
    200 x 200 px synthetic scene (seed 0, 53 N, DOY 172): walls and SVF from
    the reference's compiled kernels, UTCI from the reference's compiled
    ``utci.cu`` on the float32 Tmrt, roofs NaN (``src/series.py:466-469``).
    Tmrt, UTCI and the shadow plane of DAY200_HOURS are stored as float32."""
    from oracle import step as ST
    n = 200
    sc, a, t1, vegdsm, vegdsm2, bush, amax = _scene(n, 0)
    P, cubes, planes = _ref_svf(a, vegdsm, vegdsm2, bush, amax)
    order = (0, 10, 1, 11, 6, 4, 14, 9, 2, 12, 7, 5, 3, 13, 8)
    cubes64 = [c.astype(np.float64) for c in cubes]
    svf = tuple(planes[i] for i in order) + (cubes64[1], cubes64[2], cubes64[0], planes[15])
    walls = ref_walls(a)
    aspect = G.wall_aspect(walls, a, 1.0)
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover, walls=walls,
                          aspect=aspect, svf=svf)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    loc = dict(latitude=53.0, longitude=0.0, altitude=3.0)
    sol = U.Solweig_2015a_metdata_noload(met, loc, 0.0)
    alt, azi, zen, jday, dectime, altmax = (np.ravel(sol[k]) for k in (1, 2, 3, 4, 6, 7))
    state = {k: np.zeros((n, n)) for k in ("Tgmap1", "Tgmap1E", "Tgmap1S", "Tgmap1W", "Tgmap1N", "TgOut1")}
    fd, ta_, CI = 1., 0., 1.
    Twater = float(np.mean(met[:, 11]))
    step = dectime[1] - dectime[0]
    f = ctypes.c_float
    LIB.ref_utci_scalar.argtypes = [f, f, f, VP, VP, ctypes.c_longlong, VP]
    keep = {"Tmrt": [], "UTCI": [], "shadow": []}
    for i in range(24):
        if dectime[i] - np.floor(dectime[i]) == 0:
            CI = 1.
        r = U.Solweig_2022a_calc(
            i, s["dsm"], 1.0, n, n, s["svf"], s["svfN"], s["svfW"], s["svfE"], s["svfS"], s["svfveg"],
            s["svfNveg"], s["svfEveg"], s["svfSveg"], s["svfWveg"], s["svfaveg"], s["svfEaveg"],
            s["svfSaveg"], s["svfWaveg"], s["svfNaveg"], s["vegdem"], s["vegdem2"], 0.2, 0.7, 0.95, 0.9,
            0.22, 0.06, 0.28, alt[i], azi[i], zen[i], jday[i], 1, 1, s["buildings"], loc, 0.03, 1,
            s["lc_grid"], dectime[i], altmax[i], s["dirwalls"], s["walls"], 1, 0, met[i, 11],
            met[i, 10], met[i, 14], met[i, 21], met[i, 22], met[i, 12], s["amaxvalue"], s["bush"],
            Twater, s["TgK"].copy(), s["Tstart"], s["alb_grid"], s["emis_grid"], s["TgK_wall"],
            s["Tstart_wall"], s["TmaxLST"], s["TmaxLST_wall"], 1.0, 22.0, s["svfalfa"], s["svfbuveg"],
            fd, ta_, step, state["Tgmap1"], state["Tgmap1E"], state["Tgmap1S"], state["Tgmap1W"],
            state["Tgmap1N"], CI, state["TgOut1"], s["diffsh"], s["shmat"], s["vegshmat"],
            s["vbshvegshmat"], 1, s["asvf"], 2)
        o = dict(zip(ST.OUTPUT_NAMES, r))
        fd, ta_, CI = o["firstdaytime"], o["timeadd"], o["CI"]
        for k in state:
            state[k] = o[k]
        if i not in DAY200_HOURS:
            continue
        tm = np.ascontiguousarray(np.broadcast_to(np.asarray(o["Tmrt"], dtype=np.float64), (n, n)))
        tm32 = tm.astype(np.float32)
        ut = np.empty(n * n, np.float32)
        co = np.empty(7)
        LIB.ref_utci_scalar(np.float32(met[i, 11]), np.float32(met[i, 10]), np.float32(met[i, 9]),
                            tm32.ctypes.data, ut.ctypes.data, n * n, co.ctypes.data)
        ut = np.where(s["buildings"] == 1, ut.reshape(n, n), np.nan).astype(np.float32)
        keep["Tmrt"].append(tm32)
        keep["UTCI"].append(ut)
        keep["shadow"].append(np.broadcast_to(np.asarray(o["shadow"], dtype=np.float64), (n, n)).astype(np.float32))
    np.savez_compressed(os.path.join(HERE, "day200.npz"), hours=np.asarray(DAY200_HOURS), met=met,
                        **{k: np.asarray(v) for k, v in keep.items()})


if __name__ == "__main__":
    if len(sys.argv) > 1:
        for name in sys.argv[1:]:
            globals()[f"{name}_fixture"]()
        raise SystemExit(0)
    sun_fixture()
    scalars_fixture()
    shadow_fixture()
    svf_fixture()
    utci_fixture()
    day_fixture()
    day200_fixture()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
