"""Oracle restatement of the hourly radiation fluxes and Tmrt (test infrastructure).

float64 numpy restatements of the reference routines named in each docstring.
Patch masks are float arrays ``[rows, cols, P]`` (1 = visible through that
class), as produced by :func:`oracle.geometry.svf_patch_masks`.
"""
from __future__ import annotations

import numpy as np

SBC = 5.67051e-8
_D2R = np.pi / 180


def cylindric_wedge(zen, svfalfa):
    """Fraction of shaded wall (F_sh), ``src/umep_solweig.py:383-426``."""
    beta = zen
    alfa = np.asarray(svfalfa, dtype=np.float64)
    with np.errstate(divide='ignore', invalid='ignore'):
        xa = 1 - 2. / (np.tan(alfa) * np.tan(beta))
        ha = 2. / (np.tan(alfa) * np.tan(beta))
        ba = 1. / np.tan(alfa)
        hkil = 2. * ba * ha
        neg = xa < 0
        qa = np.where(neg, np.tan(beta) / 2, 0.0)
        za = np.where(neg, np.sqrt(np.where(neg, ba ** 2 - qa ** 2 / 4, 0.0)), 0.0)
        phi = np.where(neg, np.arctan(za / np.where(neg, qa, 1.0)), 0.0)
        area = np.where(neg, (np.sin(phi) - phi * np.cos(phi)) / (1 - np.cos(np.where(neg, phi, 1.0))), 0.0)
        ukil = np.where(neg, 2 * ba * xa * area, 0.0)
        return (2 * np.pi * ba - (hkil + ukil)) / (2 * np.pi * ba)


def wave_delay(current, firstdaytime, timeadd, timestepdec, previous):
    """Surface temperature lag, ``TsWaveDelay_2015a`` (``src/umep_solweig.py:1633-1652``).

    Returns ``(delayed, timeadd_next, state_next)``.
    """
    state = current if firstdaytime == 1 else previous
    if timeadd >= (59 / 1440):
        w = np.exp(-33.27 * timeadd)
        state = current * (1 - w) + state * w
        out = state
        timeadd = timestepdec if timestepdec > (59 / 1440) else 0
    else:
        timeadd = timeadd + timestepdec
        w = np.exp(-33.27 * timeadd)
        out = current * (1 - w) + state * w
    return out, timeadd, state


def kup(radI, radD, radG, altitude, svfbuveg, albedo_b, F_sh, alb5, nosh5):
    """Upwelling shortwave (all, E, S, W, N), ``Kup_veg_2015a`` (``:915-927``)."""
    base = radD * svfbuveg + albedo_b * (1 - svfbuveg) * (radG * (1 - F_sh) + radD * F_sh)
    s = np.sin(altitude * (np.pi / 180.))
    return [a * radI * s + base * n for a, n in zip(alb5, nosh5)]


def _weight_poly(x):
    return 63.227 * x ** 6 - 161.51 * x ** 5 + 156.91 * x ** 4 - 70.424 * x ** 3 + 16.773 * x ** 2 - 0.4863 * x


def shaded_or_sunlit(solar_altitude, solar_azimuth, patch_altitude, patch_azimuth, asvf):
    """``src/umep_solweig.py:1362-1397``: (sunlit, shaded) boolean pixel maps."""
    xi = np.cos(np.abs(solar_azimuth - patch_azimuth) * _D2R)
    yi = 2 * xi * np.tan(solar_altitude * _D2R)
    yi_ = 0 if yi > 0 else yi
    deg = np.arctan(np.tan(asvf) + yi_) * (180 / np.pi)
    return deg < patch_altitude, deg > patch_altitude


def _steradians(alt):
    uniq, counts = np.unique(alt, return_counts=True)
    out = np.zeros(alt.size)
    for i in range(alt.size):
        n = int(counts[uniq == alt[i]][0])
        if n > 1:
            out[i] = ((360 / n) * _D2R) * (np.sin((alt[i] + alt[0]) * _D2R) - np.sin((alt[i] - alt[0]) * _D2R))
        else:
            out[i] = ((360 / n) * _D2R) * (np.sin(alt[i] * _D2R) - np.sin((alt[i - 1] + alt[0]) * _D2R))
    return out


def kside(radI, radD, radG, shadow, svfS, svfW, svfN, svfE, svfEveg, svfSveg, svfWveg, svfNveg,
          azimuth, altitude, psi, t, albedo, F_sh, KupE, KupS, KupW, KupN, cyl, lv,
          anisotropic, diffsh, asvf, shmat, vegshmat, vbshvegshmat):
    """Side shortwave, ``Kside_veg_v2022a`` (``src/umep_solweig.py:666-911``).

    Returns ``(Keast, Ksouth, Kwest, Knorth, KsideI, KsideD, Kside)``.
    """
    shape = np.shape(shadow)
    zeros = np.zeros(shape)
    if cyl == 1:
        KsideI = shadow * radI * np.cos(altitude * _D2R)
        direct = [0, 0, 0, 0]
    else:
        direct = []
        for rot, active in ((0, azimuth > (360 - t) or azimuth <= (180 - t)),
                            (90, (90 - t) < azimuth <= (270 - t)),
                            (180, (180 - t) < azimuth <= (360 - t)),
                            (270, azimuth <= (90 - t) or azimuth > (270 - t))):
            direct.append(radI * shadow * np.cos(altitude * _D2R) * np.sin((azimuth - rot + t) * _D2R)
                          if active else 0)
        KsideI = shadow * 0
    if anisotropic != 1:
        out = []
        for svf, svfveg, kup_, d in ((svfE, svfEveg, KupE, direct[0]), (svfS, svfSveg, KupS, direct[1]),
                                     (svfW, svfWveg, KupW, direct[2]), (svfN, svfNveg, KupN, direct[3])):
            wall = (4.4897 - _weight_poly(svf)) / 4.4897
            vegw = (4.4897 - _weight_poly(svfveg + svf - 1)) / 4.4897 - wall
            w = wall + vegw * (1 - psi)
            out.append(d + (radD * (1 - w) + albedo * (w * (radG * (1 - F_sh) + radD * F_sh)) + kup_) * 0.5)
        return out[0], out[1], out[2], out[3], KsideI, zeros, zeros
    p_alt, p_azi, lum = lv[:, 0], lv[:, 1], lv[:, 2]
    omega = _steradians(p_alt)
    rad_tot = 0.0
    for i in range(p_alt.size):
        rad_tot += lum[i] * omega[i] * np.sin(p_alt[i] * _D2R)
    lum_chi = (lum * radD) / rad_tot
    sun_surf = (albedo * (radI * np.cos(altitude * _D2R)) + (radD * 0.5)) / np.pi
    shade_surf = (albedo * radD * 0.5) / np.pi
    KsideD = np.zeros(shape)
    ref_sun = np.zeros(shape)
    ref_sh = np.zeros(shape)
    ref_veg = np.zeros(shape)
    card = {k: np.zeros(shape) for k in ("dE", "dS", "dW", "dN", "vE", "vS", "vW", "vN",
                                          "uE", "uS", "uW", "uN", "hE", "hS", "hW", "hN")}
    for k in range(p_alt.size):
        ca = np.cos(p_alt[k] * _D2R)
        vegmask = (vegshmat[:, :, k] == 0) | (vbshvegshmat[:, :, k] == 0)
        bmask = ((1 - shmat[:, :, k]) * vbshvegshmat[:, :, k]) == 1
        ref_veg += shade_surf * vegmask * omega[k] * ca
        if cyl == 1:
            KsideD += diffsh[:, :, k] * lum_chi[k] * ca * omega[k]
            sunlit, shaded = shaded_or_sunlit(altitude, azimuth, p_alt[k], p_azi[k], asvf)
            ref_sun += sun_surf * sunlit * bmask * omega[k] * ca
            ref_sh += shade_surf * shaded * bmask * omega[k] * ca
            continue
        a = p_azi[k]
        for key, ok, rot in (("E", a > 360 or a <= 180, 90), ("S", 90 < a <= 270, 180),
                             ("W", 180 < a <= 360, 270), ("N", a > 270 or a <= 90, 0)):
            if ok:
                card["d" + key] += diffsh[:, :, k] * lum_chi[k] * (ca * np.cos((rot - a + t) * _D2R)) * omega[k]
        strict = (("E", a > 360 or a < 180, 90), ("S", 90 < a < 270, 180),
                  ("W", 180 < a < 360, 270), ("N", a > 270 or a < 90, 0))
        for key, ok, rot in strict:
            if ok:
                card["v" + key] += shade_surf * omega[k] * ca * vegmask * np.cos((rot - a + t) * _D2R)
        diff = np.abs(azimuth - a)
        if 90 < diff < 270:
            sunlit, shaded = shaded_or_sunlit(altitude, azimuth, p_alt[k], a, asvf)
            ref_sun += sun_surf * sunlit * bmask * omega[k] * ca
            ref_sh += shade_surf * shaded * bmask * omega[k] * ca
            for key, ok, rot in strict:
                if ok:
                    c = np.cos((rot - a + t) * _D2R)
                    card["u" + key] += sun_surf * sunlit * omega[k] * ca * bmask * c
                    card["h" + key] += shade_surf * shaded * omega[k] * ca * bmask * c
        else:
            ref_sh += shade_surf * bmask * omega[k] * ca
            for key, ok, rot in strict:
                if ok:
                    card["h" + key] += shade_surf * omega[k] * ca * bmask * np.cos((rot - a + t) * _D2R)
    if cyl == 1:
        Kside = KsideI + KsideD + ref_sun + ref_sh + ref_veg
        return KupE * 0.5, KupS * 0.5, KupW * 0.5, KupN * 0.5, KsideI, KsideD, Kside
    outs = []
    for key, d, kup_ in (("E", direct[0], KupE), ("S", direct[1], KupS), ("W", direct[2], KupW),
                         ("N", direct[3], KupN)):
        outs.append(d + card["d" + key] + card["u" + key] + card["h" + key] + card["v" + key] + kup_ * 0.5)
    return outs[0], outs[1], outs[2], outs[3], KsideI, KsideD, zeros


def lcyl(esky, sky_patches, Ta, Tgwall, ewall, Lup, shmat, vegshmat, vbshvegshmat,
         solar_altitude, solar_azimuth, asvf):
    """Anisotropic sky longwave, ``Lcyl_v2022a`` + ``define_patch_characteristics``
    (``src/umep_solweig.py:946-1028``, ``:1205-1356``).

    Returns ``(Ldown, Lside, Least_, Lwest_, Lnorth_, Lsouth_)``.
    """
    p_alt, p_azi = sky_patches[:, 0], sky_patches[:, 1]
    omega = _steradians(p_alt)
    uniq = np.unique(p_alt)
    band = 1 - (1 - esky) * np.exp(0.308 * (1.7 - (1 / np.cos((90 - uniq) * _D2R))))
    emis = np.zeros(p_alt.size)
    for a, e in zip(uniq, band):
        emis[p_alt == a] = e
    base = SBC * ((Ta + 273.15) ** 4)
    sky_down = ((emis * base) / np.pi) * omega * np.sin(p_alt * _D2R)
    sky_side = ((emis * base) / np.pi) * omega * np.cos(p_alt * _D2R)
    shape = np.shape(Lup)
    z = lambda: np.zeros(shape)  # noqa: E731
    d_sky, d_veg, d_sun, d_sh, d_ref = z(), z(), z(), z(), z()
    s_sky, s_veg, s_sun, s_sh, s_ref = z(), z(), z(), z(), z()
    card = {k: z() for k in "ESWN"}
    veg_surf = (ewall * SBC * ((Ta + 273.15) ** 4)) / np.pi
    sun_surf = (ewall * SBC * ((Ta + Tgwall + 273.15) ** 4)) / np.pi
    shade_surf = (ewall * SBC * ((Ta + 273.15) ** 4)) / np.pi
    dirs = (("E", lambda a: a > 360 or a < 180, 90), ("S", lambda a: 90 < a < 270, 180),
            ("W", lambda a: 180 < a < 360, 270), ("N", lambda a: a > 270 or a < 90, 0))
    for k in range(p_alt.size):
        ca, sa = np.cos(p_alt[k] * _D2R), np.sin(p_alt[k] * _D2R)
        sky = (shmat[:, :, k] == 1) & (vegshmat[:, :, k] == 1)
        vegm = (vegshmat[:, :, k] == 0) | (vbshvegshmat[:, :, k] == 0)
        bm = ((1 - shmat[:, :, k]) * vbshvegshmat[:, :, k]) == 1
        d_sky += sky * sky_down[k]
        s_sky += sky * sky_side[k]
        s_veg += veg_surf * omega[k] * ca * vegm
        d_veg += veg_surf * omega[k] * sa * vegm
        a = p_azi[k]
        for key, ok, rot in dirs:
            if ok(a):
                c = np.cos((rot - a) * _D2R)
                card[key] += sky * sky_side[k] * c
                card[key] += veg_surf * omega[k] * ca * vegm * c
        diff = np.abs(solar_azimuth - a)
        if 90 < diff < 270 and solar_altitude > 0:
            sunlit, shaded = shaded_or_sunlit(solar_altitude, solar_azimuth, p_alt[k], a, asvf)
            s_sun += sun_surf * sunlit * omega[k] * ca * bm
            s_sh += shade_surf * shaded * omega[k] * ca * bm
            d_sun += sun_surf * sunlit * omega[k] * sa * bm
            d_sh += shade_surf * shaded * omega[k] * sa * bm
            for key, ok, rot in dirs:
                if ok(a):
                    c = np.cos((rot - a) * _D2R)
                    card[key] += sun_surf * sunlit * omega[k] * ca * bm * c
                    card[key] += shade_surf * shaded * omega[k] * ca * bm * c
        else:
            s_sh += shade_surf * omega[k] * ca * bm
            d_sh += shade_surf * omega[k] * sa * bm
            for key, ok, rot in dirs:
                if ok(a):
                    card[key] += shade_surf * omega[k] * ca * bm * np.cos((rot - a) * _D2R)
    refl = ((d_sky + Lup) * (1 - ewall) * 0.5) / np.pi
    for k in range(p_alt.size):
        ca, sa = np.cos(p_alt[k] * _D2R), np.sin(p_alt[k] * _D2R)
        om = (shmat[:, :, k] == 0) | (vegshmat[:, :, k] == 0) | (vbshvegshmat[:, :, k] == 0)
        s_ref += refl * omega[k] * ca * om
        d_ref += refl * omega[k] * sa * om
        a = p_azi[k]
        for key, ok, rot in dirs:
            if ok(a):
                card[key] += refl * omega[k] * ca * om * np.cos((rot - a) * _D2R)
    Lside = s_sky + s_veg + s_sh + s_sun + s_ref
    Ldown = d_sky + d_veg + d_sh + d_sun + d_ref
    return Ldown, Lside, card["E"], card["W"], card["N"], card["S"]


def lside(svfS, svfW, svfN, svfE, svfEveg, svfSveg, svfWveg, svfNveg, svfEaveg, svfSaveg, svfWaveg,
          svfNaveg, azimuth, altitude, Ta, Tw, ewall, Ldown, esky, t, F_sh, CI, LupE, LupS, LupW, LupN,
          anisotropic):
    """Cardinal longwave, ``Lside_veg_v2022a`` (``src/umep_solweig.py:1032-1181``).

    Returns ``(Least, Lsouth, Lwest, Lnorth)``.
    """
    if anisotropic == 1:
        return LupE * 0.5, LupS * 0.5, LupW * 0.5, LupN * 0.5
    F = 2 * F_sh - 1
    c = 1 - CI
    base = (Ta + 273.15) ** 4
    allsky = esky * SBC * base * (1 - c) + c * SBC * base
    out = []
    specs = ((svfE, svfEveg, svfEaveg, LupE, azimuth - 180 + t, (180 - t) < azimuth <= (360 - t)),
             (svfS, svfSveg, svfSaveg, LupS, azimuth - 270 + t, azimuth <= (90 - t) or azimuth > (270 - t)),
             (svfW, svfWveg, svfWaveg, LupW, azimuth + t, azimuth > (360 - t) or azimuth <= (180 - t)),
             (svfN, svfNveg, svfNaveg, LupN, azimuth - 90 + t, (90 - t) < azimuth <= (270 - t)))
    for svf, svfveg, svfaveg, lup_, azi_d, lit in specs:
        onlywall = (4.4897 - _weight_poly(svf)) / 4.4897
        aveg = (4.4897 - _weight_poly(svfaveg)) / 4.4897
        wwall = onlywall - aveg
        comb = svfveg + svf - 1
        wsky = _weight_poly(comb) / 4.4897
        wrefl = (4.4897 - _weight_poly(comb)) / 4.4897
        wveg = (4.4897 - _weight_poly(comb)) / 4.4897 - wwall
        if altitude > 0 and lit:
            svfalfa = np.arcsin(np.exp((np.log(1 - svf)) / 2))
            alfaB = np.arctan(svfalfa)
            betaB = np.arctan(np.tan(svfalfa * F))
            betasun = ((alfaB - betaB) / 2) + betaB
            wallsun = SBC * ewall * ((Ta + 273.15 + Tw * np.sin(azi_d * (np.pi / 180))) ** 4) * \
                wwall * (1 - F) * np.cos(betasun) * 0.5
            wallsh = SBC * ewall * base * wwall * F * 0.5
        else:
            wallsun = 0
            wallsh = SBC * ewall * base * wwall * 0.5
        sky = ((svf + svfveg - 1) * allsky) * wsky * 0.5
        veg = SBC * ewall * base * wveg * 0.5
        out.append(sky + wallsun + wallsh + veg + lup_ * 0.5 + (Ldown + lup_) * wrefl * (1 - ewall) * 0.5)
    return tuple(out)


def tmrt(Kdown, Kup, Knorth, Keast, Ksouth, Kwest, Ldown, Lup, Lnorth, Least, Lsouth, Lwest,
         KsideI, Kside, Lside, absK, absL, Fside, Fup, Fcyl, cyl, anisotropic):
    """Absorbed flux and mean radiant temperature, ``src/umep_solweig.py:345-360``."""
    ksum = Knorth + Keast + Ksouth + Kwest
    lsum = Lnorth + Least + Lsouth + Lwest
    if cyl == 1 and anisotropic == 0:
        sstr = absK * (KsideI * Fcyl + (Kdown + Kup) * Fup + ksum * Fside) + absL * ((Ldown + Lup) * Fup + lsum * Fside)
    elif cyl == 1 and anisotropic == 1:
        sstr = absK * (Kside * Fcyl + (Kdown + Kup) * Fup + ksum * Fside) + \
            absL * ((Ldown + Lup) * Fup + Lside * Fcyl + lsum * Fside)
    else:
        sstr = absK * ((Kdown + Kup) * Fup + ksum * Fside) + absL * ((Ldown + Lup) * Fup + lsum * Fside)
    return np.sqrt(np.sqrt((sstr / (absL * SBC)))) - 273.2, sstr
