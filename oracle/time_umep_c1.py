"""Time the reference's UMEP numpy path, imported in place, on the CPU
configuration of the benchmark (200 x 200 px synthetic scene, seed 0, 53 N,
DOY 172, 24 hourly steps), beside this repository's float64 port of the same
path (oracle/step.py), on the same host (test infrastructure: it needs the
reference tree, so it runs where that tree is, not on the GPU machines).

    python oracle/time_umep_c1.py [--hours 12] [--workers N]

Walls come from the reference's compiled wall kernel and the 153-patch SVF
from its compiled visibility/reduce kernels (oracle/_ref, `make -C oracle`);
the reference has no numpy code for those two stages, so they are prepared
once, untimed, for both arms.  Timed: the first `--hours` hourly steps of the
day (thermal state carried), UMEP's `Solweig_2022a_calc` plus the compiled
reference UTCI for the reference arm; `oracle.step.day_hours` for the port.
With `--workers N > 1` every process runs its own copy of the day at once
and the figure is the aggregate pixel-hours/s.  Prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def _statics():
    import numpy as np
    import make_golden as MG
    from oracle import geometry as G
    from oracle import step as ST
    from solweig_cuda_b200 import synthetic
    n = 200
    sc, a, t1, vegdsm, vegdsm2, bush, amax = MG._scene(n, 0)
    P, cubes, planes = MG._ref_svf(a, vegdsm, vegdsm2, bush, amax)
    order = (0, 10, 1, 11, 6, 4, 14, 9, 2, 12, 7, 5, 3, 13, 8)
    cubes64 = [c.astype(np.float64) for c in cubes]
    svf = tuple(planes[i] for i in order) + (cubes64[1], cubes64[2], cubes64[0], planes[15])
    walls = MG.ref_walls(a)
    aspect = G.wall_aspect(walls, a, 1.0)
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover, walls=walls, aspect=aspect,
                          svf=svf)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    return n, s, met


def _umep_hours(hours):
    import ctypes
    import numpy as np
    import make_golden as MG
    U = MG.U
    n, s, met = _statics()
    loc = dict(latitude=53.0, longitude=0.0, altitude=3.0)
    sol = U.Solweig_2015a_metdata_noload(met, loc, 0.0)
    alt, azi, zen, jday, dectime, altmax = (np.ravel(sol[k]) for k in (1, 2, 3, 4, 6, 7))
    state = {k: np.zeros((n, n)) for k in ("Tgmap1", "Tgmap1E", "Tgmap1S", "Tgmap1W", "Tgmap1N", "TgOut1")}
    fd, ta_, CI = 1., 0., 1.
    Twater = float(np.mean(met[:, 11]))
    step = dectime[1] - dectime[0]
    f = ctypes.c_float
    MG.LIB.ref_utci_scalar.argtypes = [f, f, f, MG.VP, MG.VP, ctypes.c_longlong, MG.VP]
    t0 = time.perf_counter()
    with np.errstate(all="ignore"):
        for i in range(hours):
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
            tmrt, fd, ta_, CI = r[0], r[11], r[13], r[9]
            for k, j in zip(("Tgmap1", "Tgmap1E", "Tgmap1S", "Tgmap1W", "Tgmap1N", "TgOut1"), (14, 15, 16, 17, 18, 28)):
                state[k] = r[j]
            tm = np.ascontiguousarray(np.broadcast_to(np.asarray(tmrt, np.float64), (n, n))).astype(np.float32)
            ut = np.empty(n * n, np.float32)
            co = np.empty(7)
            MG.LIB.ref_utci_scalar(np.float32(met[i, 11]), np.float32(met[i, 10]), np.float32(met[i, 9]),
                                   tm.ctypes.data, ut.ctypes.data, n * n, co.ctypes.data)
    return n * n * hours, time.perf_counter() - t0


def _port_hours(hours):
    from oracle import step as ST
    n, s, met = _statics()
    gen = ST.day_hours(s, met, dict(latitude=53.0, longitude=0.0, altitude=3.0), 0.0)
    t0 = time.perf_counter()
    for _ in range(hours):
        next(gen)
    return n * n * hours, time.perf_counter() - t0


def _pool(fn, hours, workers):
    if workers <= 1:
        work, sec = fn(hours)
        return work / sec, sec
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        t0 = time.perf_counter()
        res = pool.map(fn, [hours] * workers, chunksize=1)
        wall = time.perf_counter() - t0
    # the statics are prepared inside each task: rate = work / the slowest task's timed part
    return sum(r[0] for r in res) / max(r[1] for r in res), wall


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--hours", type=int, default=12)
    ap.add_argument("--workers", type=int, default=1)
    a = ap.parse_args()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    out = {"config": "200x200 px, seed 0, 53N, DOY 172", "hours": a.hours, "workers": a.workers,
           "os_cpu_count": os.cpu_count(), "affinity_cores": cores}
    for name, fn in (("umep_numpy_in_place", _umep_hours), ("port_oracle_step", _port_hours)):
        v, sec = _pool(fn, a.hours, a.workers)
        out[name] = {"pixel_hours_per_s": v, "seconds": sec}
    out["umep_over_port"] = out["umep_numpy_in_place"]["pixel_hours_per_s"] / out["port_oracle_step"]["pixel_hours_per_s"]
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
