"""Oracle restatement of the hourly SOLWEIG step and its static inputs
(test infrastructure).

* :func:`prepare_static` restates ``_prepare_spatial`` (``src/series.py:197-382``)
  for in-memory rasters (walls, SVF, land-cover maps, derived SVF fields);
* :func:`hour_step` restates ``Solweig_2022a_calc`` (``src/umep_solweig.py:50-372``);
* :func:`run_day` restates the hour loop of ``_run_day`` (``src/series.py:396-495``)
  including the UTCI and the NaN roof mask.

Per-hour FP64 scalars (sun position, clearness index, diffuse split, Perez
luminance) come from the product's host modules ``sun`` and ``sky``; those are
pinned bit-exactly against the reference by ``tests/test_host_scalars.py``.
Everything per pixel is restated here in float64 numpy.
"""
from __future__ import annotations

import numpy as np

from . import geometry as G
from . import ground as GR
from . import radiation as R
from . import utci as U
from ._host import sky, sun

SBC = 5.67051e-8
LANDCOVER_CLASSES = np.array([  # code, albedo, emissivity, TgK, Tstart, TmaxLST
    [2, 0.18, 0.95, 0.58, -9.78, 15.0],
    [1, 0.18, 0.95, 0.58, -9.78, 15.0],
    [0, 0.20, 0.95, 0.37, -3.41, 15.0],
    [7, 0.05, 0.98, 0.00, 0.00, 12.0],
    [5, 0.16, 0.94, 0.21, -3.38, 14.0],
    [6, 0.25, 0.94, 0.33, -3.01, 14.0],
    [99, 0.20, 0.90, 0.58, -3.41, 15.0],
])

CONSTANTS = dict(albedo_b=0.2, albedo_g=0.15, ewall=0.9, eground=0.95, absK=0.7, absL=0.95,
                 Fside=0.22, Fup=0.06, Fcyl=0.28, cyl=1, elvis=0, usevegdem=1, onlyglobal=1,
                 transVeg=0.03, anisotropic_sky=1, patch_option=2, firstdayleaf=97, lastdayleaf=300)


def normalise_landcover(values):
    """``_normalise_landcover_grid`` (``src/series.py:505-513``)."""
    src = np.asarray(values, dtype=float)
    r = np.rint(src)
    bad = (~np.isfinite(src)) | (~np.isclose(src, r)) | (r < 1) | (r > 7)
    r[bad] = 6
    r[(r == 3) | (r == 4)] = 5
    return r.astype(np.float32)


def landcover_maps(lc):
    """``Tgmaps_v1`` (``src/umep_solweig.py:1603-1628``)."""
    maps = {k: np.array(lc, dtype=np.float64, copy=True) for k in ("TgK", "Tstart", "alb", "emis", "TmaxLST")}
    cols = {"alb": 1, "emis": 2, "TgK": 3, "Tstart": 4, "TmaxLST": 5}
    for code in np.unique(lc):
        row = LANDCOVER_CLASSES[:, 0] == code
        for k, c in cols.items():
            m = maps[k]
            m[m == code] = LANDCOVER_CLASSES[row, c]
    wall = LANDCOVER_CLASSES[LANDCOVER_CLASSES[:, 0] == 99][0]
    return maps, float(wall[3]), float(wall[4]), float(wall[5])


def prepare_static(dsm, trees, dem, pixel_size=1.0, landcover=None, wall_threshold=3.0,
                   walls=None, aspect=None, svf=None):
    """Static inputs of the hourly step from in-memory rasters (float64).

    ``walls``/``aspect`` and ``svf`` (the 19-tuple of :func:`geometry.svf_calculator`)
    may be supplied to skip their computation.
    """
    a = np.asarray(dsm, dtype=np.float64).copy()
    t1 = np.asarray(trees, dtype=np.float64).copy()
    t2 = np.asarray(dem, dtype=np.float64).copy()
    if walls is None:
        walls = G.wall_heights(a, wall_threshold)
        aspect = G.wall_aspect(walls, a, pixel_size)
    walls = walls.astype(np.float32).astype(np.float64)
    aspect = aspect.astype(np.float32).astype(np.float64)
    raise_a = max(0.0, -float(a.min()))
    raise_d = max(0.0, -float(t2.min()))
    a = a + raise_a if raise_a else a
    t2 = t2 + raise_d if raise_d else t2
    rows, cols = a.shape
    scale = 1 / pixel_size
    t1[t1 < 0.] = 0.
    vegdsm = t1 + a
    vegdsm[vegdsm == a] = 0
    vegdsm2 = t1 * 0.25 + a
    vegdsm2[vegdsm2 == a] = 0
    bush = np.logical_not(vegdsm2 * vegdsm) * vegdsm
    amaxvalue = max(a.max() - a.min(), t1.max())
    buildings = a - t2
    buildings[buildings < 2.] = 1.
    buildings[buildings >= 2.] = 0.
    if landcover is not None:
        lc = normalise_landcover(landcover).astype(np.float64)
        maps, TgK_wall, Tstart_wall, TmaxLST_wall = landcover_maps(lc)
        maps = {k: v.astype(np.float32).astype(np.float64) for k, v in maps.items()}
        lc_flag = 1
    else:
        z = np.zeros((rows, cols))
        maps = {"TgK": z + 0.37, "Tstart": z - 3.41, "alb": z + CONSTANTS["albedo_g"],
                "emis": z + CONSTANTS["eground"], "TmaxLST": z + 15.}
        maps = {k: v.astype(np.float32).astype(np.float64) for k, v in maps.items()}
        TgK_wall, Tstart_wall, TmaxLST_wall = 0.37, -3.41, 15.
        lc = z
        lc_flag = 0
    if svf is None:
        svf = G.svf_calculator(2, amaxvalue, a, vegdsm, vegdsm2, bush, scale)
    svf = tuple(v.astype(np.float32).astype(np.float64) for v in svf[:15]) + tuple(svf[15:])
    (svf_, svfaveg, svfE, svfEaveg, svfEveg, svfN, svfNaveg, svfNveg, svfS, svfSaveg, svfSveg,
     svfveg, svfW, svfWaveg, svfWveg, vegmat, vbmat, shmat, _) = svf
    tv = CONSTANTS["transVeg"]
    svfbuveg = svf_ - (1.0 - svfveg) * (1.0 - tv)
    asvf = np.arccos(np.sqrt(svf_))
    diffsh = G.compute_diffsh(shmat.astype(np.float32), vegmat.astype(np.float32), np.float32(tv)).astype(np.float64)
    tmp = svf_ + svfveg - 1.0
    tmp[tmp < 0.0] = 0.0
    with np.errstate(divide='ignore'):
        svfalfa = np.arcsin(np.exp(np.log(1.0 - tmp) / 2.0))
    return dict(dsm=a, scale=scale, rows=rows, cols=cols, svf=svf_, svfN=svfN, svfW=svfW, svfE=svfE,
                svfS=svfS, svfveg=svfveg, svfNveg=svfNveg, svfEveg=svfEveg, svfSveg=svfSveg,
                svfWveg=svfWveg, svfaveg=svfaveg, svfEaveg=svfEaveg, svfSaveg=svfSaveg,
                svfWaveg=svfWaveg, svfNaveg=svfNaveg, vegdem=vegdsm, vegdem2=vegdsm2, bush=bush,
                amaxvalue=amaxvalue, buildings=buildings, walls=walls, dirwalls=aspect,
                landcover=lc_flag, lc_grid=lc, TgK=maps["TgK"], Tstart=maps["Tstart"],
                alb_grid=maps["alb"], emis_grid=maps["emis"], TmaxLST=maps["TmaxLST"],
                TgK_wall=TgK_wall, Tstart_wall=Tstart_wall, TmaxLST_wall=TmaxLST_wall,
                svfalfa=svfalfa, svfbuveg=svfbuveg, asvf=asvf, diffsh=diffsh, shmat=shmat,
                vegshmat=vegmat, vbshvegshmat=vbmat, first=1.0, second=22.0)


OUTPUT_NAMES = ('Tmrt', 'Kdown', 'Kup', 'Ldown', 'Lup', 'Tg', 'ea', 'esky', 'I0', 'CI', 'shadow',
                'firstdaytime', 'timestepdec', 'timeadd', 'Tgmap1', 'Tgmap1E', 'Tgmap1S', 'Tgmap1W',
                'Tgmap1N', 'Keast', 'Ksouth', 'Kwest', 'Knorth', 'Least', 'Lsouth', 'Lwest', 'Lnorth',
                'KsideI', 'TgOut1', 'TgOut', 'radI', 'radD', 'Lside', 'L_patches', 'CI_Tg', 'CI_TgG',
                'KsideD', 'dRad', 'Kside')


def hour_step(s, location, altitude, azimuth, zen, jday, psi, dectime, altmax, Ta, RH, radG, radD,
              radI, P, Twater, firstdaytime, timeadd, timestepdec, Tgmap1, Tgmap1E, Tgmap1S, Tgmap1W,
              Tgmap1N, CI, TgOut1, cyl=1, anisotropic_sky=1):
    """One hour, ``Solweig_2022a_calc`` (usevegdem=1, onlyglobal=1); returns a dict
    keyed by :data:`OUTPUT_NAMES`."""
    C = CONSTANTS
    rows, cols = s["rows"], s["cols"]
    layout = sky.patch_layout(2)
    t = 0.
    _, _, _, SNUP = sun.daylen(jday, location["latitude"])
    ea = 6.107 * 10 ** ((7.5 * Ta) / (237.3 + Ta)) * (RH / 100.)
    msteg = 46.5 * (ea / (Ta + 273.15))
    esky = (1 - (1 + msteg) * np.exp(-((1.2 + 3.0 * msteg) ** 0.5))) + C["elvis"]
    zeros = np.zeros((rows, cols))
    lv = None
    if altitude > 0:
        I0, CI, Kt, _, _ = sun.clearness_index(zen, jday, Ta, RH / 100., radG, location["latitude"], P)
        if CI > 1 or CI == np.inf:
            CI = 1
        radI, radD = sun.diffuse_fraction(radG, altitude, Kt, Ta, RH)
        if anisotropic_sky:
            lv = sky.perez(zen * (180 / np.pi), azimuth, radD, radI, jday, layout)
            lum = np.zeros((rows, cols))
            for k in range(lv.shape[0]):
                lum += s["diffsh"][:, :, k] * lv[k, 2]
            dRad = lum * radD
        else:
            dRad = radD * s["svfbuveg"]
        vegsh, sh, _, wallsh, wallsun, wallshve, _, facesun = G.shadow_sweep(
            s["dsm"], s["vegdem"], s["vegdem2"], azimuth, altitude, s["scale"], s["amaxvalue"],
            s["bush"], s["walls"], s["dirwalls"] * np.pi / 180.)
        shadow = sh - (1 - vegsh) * (1 - psi)
        Tgamp = s["TgK"] * altmax + s["Tstart"]
        Tgampwall = s["TgK_wall"] * altmax + s["Tstart_wall"]
        frac = dectime - np.floor(dectime)
        Tg = Tgamp * np.sin(((frac - SNUP / 24) / (s["TmaxLST"] / 24 - SNUP / 24)) * np.pi / 2)
        Tgwall = Tgampwall * np.sin(((frac - SNUP / 24) / (s["TmaxLST_wall"] / 24 - SNUP / 24)) * np.pi / 2)
        if Tgwall < 0:
            Tgwall = 0
        radI0, radD0 = sun.diffuse_fraction(I0, altitude, 1., Ta, RH)
        corr = 0.1473 * np.log(90 - (zen / np.pi * 180)) + 0.3454
        CI_Tg = (radG / radI0) + (1 - corr)
        if CI_Tg > 1 or CI_Tg == np.inf:
            CI_Tg = 1
        radG0 = radI0 * (np.sin(altitude * (np.pi / 180))) + radD0
        CI_TgG = (radG / radG0) + (1 - corr)
        if CI_TgG > 1 or CI_TgG == np.inf:
            CI_TgG = 1
        Tg = Tg * CI_TgG
        Tgwall = Tgwall * CI_TgG
        if s["landcover"] == 1:
            Tg[Tg < 0] = 0
        planes, Tg = GR.gvf(wallsun, s["walls"], s["buildings"], s["scale"], shadow, s["first"],
                            s["second"], s["dirwalls"], Tg, Tgwall, Ta, s["emis_grid"], C["ewall"],
                            s["alb_grid"], SBC, C["albedo_b"], Twater, s["lc_grid"], s["landcover"])
        (gvfLup, gvfalb, gvfalbnosh, gvfLupE, gvfalbE, gvfalbnoshE, gvfLupS, gvfalbS, gvfalbnoshS,
         gvfLupW, gvfalbW, gvfalbnoshW, gvfLupN, gvfalbN, gvfalbnoshN, _, _) = planes
        Lup, _, Tgmap1 = R.wave_delay(gvfLup, firstdaytime, timeadd, timestepdec, Tgmap1)
        LupE, _, Tgmap1E = R.wave_delay(gvfLupE, firstdaytime, timeadd, timestepdec, Tgmap1E)
        LupS, _, Tgmap1S = R.wave_delay(gvfLupS, firstdaytime, timeadd, timestepdec, Tgmap1S)
        LupW, _, Tgmap1W = R.wave_delay(gvfLupW, firstdaytime, timeadd, timestepdec, Tgmap1W)
        LupN, _, Tgmap1N = R.wave_delay(gvfLupN, firstdaytime, timeadd, timestepdec, Tgmap1N)
        TgOut, timeadd, TgOut1 = R.wave_delay(Tg * shadow + Ta, firstdaytime, timeadd, timestepdec, TgOut1)
        F_sh = R.cylindric_wedge(zen, s["svfalfa"])
        F_sh[np.isnan(F_sh)] = 0.5
        Kdown = (radI * shadow * np.sin(altitude * (np.pi / 180)) + dRad
                 + C["albedo_b"] * (1 - s["svfbuveg"]) * (radG * (1 - F_sh) + radD * F_sh))
        Kup, KupE, KupS, KupW, KupN = R.kup(
            radI, radD, radG, altitude, s["svfbuveg"], C["albedo_b"], F_sh,
            (gvfalb, gvfalbE, gvfalbS, gvfalbW, gvfalbN),
            (gvfalbnosh, gvfalbnoshE, gvfalbnoshS, gvfalbnoshW, gvfalbnoshN))
        Keast, Ksouth, Kwest, Knorth, KsideI, KsideD, Kside = R.kside(
            radI, radD, radG, shadow, s["svfS"], s["svfW"], s["svfN"], s["svfE"], s["svfEveg"],
            s["svfSveg"], s["svfWveg"], s["svfNveg"], azimuth, altitude, psi, t, C["albedo_b"], F_sh,
            KupE, KupS, KupW, KupN, cyl, lv, anisotropic_sky, s["diffsh"], s["asvf"], s["shmat"],
            s["vegshmat"], s["vbshvegshmat"])
        firstdaytime = 0
    else:
        Tgwall = 0
        Kdown = Kwest = Kup = Keast = Ksouth = Knorth = KsideI = KsideD = F_sh = Tg = shadow = zeros
        CI_Tg = CI_TgG = CI
        dRad = Kside = zeros
        Lup = SBC * s["emis_grid"] * ((zeros + Ta + Tg + 273.15) ** 4)
        if s["landcover"] == 1:
            Lup = np.where(s["lc_grid"] == 3, SBC * 0.98 * (Twater + 273.15) ** 4, Lup)
        LupE = LupS = LupW = LupN = Lup
        TgOut = Ta + Tg
        I0 = 0
        timeadd = 0
        firstdaytime = 1
    L_patches = None
    if anisotropic_sky:
        if lv is not None:
            L_patches = lv.copy()
        else:
            L_patches = np.column_stack((layout.altitude, layout.azimuth, np.zeros(layout.count)))
        if CI < 0.95:
            esky = CI * esky + (1 - CI) * 1.
        Ldown, Lside, Least_, Lwest_, Lnorth_, Lsouth_ = R.lcyl(
            esky, L_patches, Ta, Tgwall, C["ewall"], Lup, s["shmat"], s["vegshmat"], s["vbshvegshmat"],
            altitude, azimuth, s["asvf"])
    else:
        base = SBC * ((Ta + 273.15) ** 4)
        svf, svfveg, svfaveg = s["svf"], s["svfveg"], s["svfaveg"]
        Ldown = ((svf + svfveg - 1) * esky * base + (2 - svfveg - svfaveg) * C["ewall"] * base
                 + (svfaveg - svf) * C["ewall"] * SBC * ((Ta + 273.15 + Tgwall) ** 4)
                 + (2 - svf - svfveg) * (1 - C["ewall"]) * esky * base)
        Lside = zeros
        if CI < 0.95:
            c = 1 - CI
            Ldown = Ldown * (1 - c) + c * ((svf + svfveg - 1) * base + (2 - svfveg - svfaveg) * C["ewall"] * base
                                           + (svfaveg - svf) * C["ewall"] * SBC * ((Ta + 273.15 + Tgwall) ** 4)
                                           + (2 - svf - svfveg) * (1 - C["ewall"]) * base)
        Least_ = Lwest_ = Lnorth_ = Lsouth_ = 0
    Least, Lsouth, Lwest, Lnorth = R.lside(
        s["svfS"], s["svfW"], s["svfN"], s["svfE"], s["svfEveg"], s["svfSveg"], s["svfWveg"], s["svfNveg"],
        s["svfEaveg"], s["svfSaveg"], s["svfWaveg"], s["svfNaveg"], azimuth, altitude, Ta, Tgwall,
        C["ewall"], Ldown, esky, t, F_sh, CI, LupE, LupS, LupW, LupN, anisotropic_sky)
    if cyl == 0 and anisotropic_sky == 1:
        Least, Lsouth, Lwest, Lnorth = Least + Least_, Lsouth + Lsouth_, Lwest + Lwest_, Lnorth + Lnorth_
    Tmrt, _ = R.tmrt(Kdown, Kup, Knorth, Keast, Ksouth, Kwest, Ldown, Lup, Lnorth, Least, Lsouth, Lwest,
                     KsideI, Kside, Lside, C["absK"], C["absL"], C["Fside"], C["Fup"], C["Fcyl"], cyl,
                     anisotropic_sky)
    if cyl == 1 and anisotropic_sky == 1:
        Least, Lsouth, Lwest, Lnorth = Least + Least_, Lsouth + Lsouth_, Lwest + Lwest_, Lnorth + Lnorth_
    values = (Tmrt, Kdown, Kup, Ldown, Lup, Tg, ea, esky, I0, CI, shadow, firstdaytime, timestepdec,
              timeadd, Tgmap1, Tgmap1E, Tgmap1S, Tgmap1W, Tgmap1N, Keast, Ksouth, Kwest, Knorth, Least,
              Lsouth, Lwest, Lnorth, KsideI, TgOut1, TgOut, radI, radD, Lside, L_patches, CI_Tg,
              CI_TgG, KsideD, dRad, Kside)
    return dict(zip(OUTPUT_NAMES, values))


def day_hours(s, met, location, utc, hours=None, outputs=("Tmrt", "UTCI"), psi=None):
    """The hour loop of one calendar day (``src/series.py:396-495``) as a
    generator: one dict of the requested outputs per hour, the thermal state
    carried from hour to hour.  ``UTCI`` has NaN on roofs (``buildings != 1``).
    ``psi`` (scalar or per-pixel array), when given, replaces the
    leaf-on/off transmissivity of every hour."""
    sol = sun.metdata(met, location["latitude"], location["longitude"], location["altitude"], utc)
    doy = met[:, 1]
    leaf = (doy > CONSTANTS["firstdayleaf"]) & (doy < CONSTANTS["lastdayleaf"])
    if psi is None:
        psi = np.where(leaf, 3. / 100., .5)
    else:
        psi = [psi] * len(met)
    shape = (s["rows"], s["cols"])
    state = {k: np.zeros(shape) for k in ("Tgmap1", "Tgmap1E", "Tgmap1S", "Tgmap1W", "Tgmap1N", "TgOut1")}
    dectime = sol.dectime
    timestepdec = (dectime[1] - dectime[0]) if len(met) > 1 else 1 / 24.
    timeadd, firstdaytime, CI = 0., 1., 1.
    Twater = float(np.mean(met[:, 11])) if s["landcover"] else None
    for i in range(len(met)) if hours is None else hours:
        if dectime[i] - np.floor(dectime[i]) == 0:
            CI = 1.
        o = hour_step(s, location, sol.altitude[i], sol.azimuth[i], sol.zen[i], sol.jday[i], psi[i],
                      dectime[i], sol.altmax[i], met[i, 11], met[i, 10], met[i, 14], met[i, 21],
                      met[i, 22], met[i, 12], Twater, firstdaytime, timeadd, timestepdec, CI=CI, **state)
        firstdaytime, timeadd, CI = o["firstdaytime"], o["timeadd"], o["CI"]
        for k in state:
            state[k] = o[k]
        rec = {}
        for name in outputs:
            if name == "UTCI":
                u = U.utci(np.float32(met[i, 11]), np.float32(met[i, 10]), o["Tmrt"], np.float32(met[i, 9]))
                rec["UTCI"] = np.where(s["buildings"] == 1, u, np.nan)
            else:
                rec[name] = o[name]
        yield rec


def run_day(s, met, location, utc, hours=None, outputs=("Tmrt", "UTCI"), psi=None):
    """Hour loop of one calendar day (``src/series.py:396-495``).

    ``met`` is the (rows, 24) forcing table of one day.  Returns a list (one
    entry per hour) of dicts with the requested outputs (see :func:`day_hours`).
    """
    return list(day_hours(s, met, location, utc, hours, outputs, psi))
