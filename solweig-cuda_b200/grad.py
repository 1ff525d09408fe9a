"""Gradients of a day's mean UTCI (or Tmrt) with the shadow and SVF masks fixed.

``DayGradient`` drives the hand-written reverse pass of the batched day
(``solweig_day_grad_forward`` / ``solweig_day_grad_backward``): per-pixel
ground albedo, ground emissivity and the direct-beam transmissivity of
vegetation (which replaces the hour's psi in the shadow value), and the
hourly forcing Ta, RH and wind speed.

The device returns the partials of J with respect to the per-hour scalars it
consumes (Ta, direct / diffuse radiation, their normaliser, CI_TgG, the wall
temperature, the band sky emittances, the UTCI coefficients, the Perez
luminances).  Those scalars come from the host's FP64 hour plan; its Jacobian
with respect to each hour's Ta, RH and wind is taken by central differences
of the FP64 plan (the whole day is re-planned, so quantities carried from
hour to hour, such as the clearness index, are included), and the UTCI
coefficients by central differences of their FP64 collapse.

:class:`DailyUTCI` wraps it as a ``torch.autograd.Function``.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .engine import HourBuffers, device_ptr, plan_day, stream_handle

__all__ = ["DayGradient", "DailyUTCI", "HOUR_FIELDS", "FORCING_COLUMNS"]

HOUR_FIELDS = ("ta", "rad_i", "rad_d", "rad_tot", "ci_tgg", "tgwall") + tuple(f"band_lsky{b}" for b in range(8)) \
    + tuple(f"utci{i}" for i in range(7))
FORCING_COLUMNS = {"ta": 11, "rh": 10, "ws": 9}  # UMEP forcing table columns
_OBJECTIVES = {"utci": 0, "tmrt": 1}


def _hour_vector(h, scal, patches):
    """FP64 values of the hour scalars the device consumes (HOUR_FIELDS + lum[P])."""
    band = scal.band_lsky if scal.band_lsky is not None else np.zeros(8)
    v = [h.ta, h.rad_i, h.rad_d, h.rad_tot, h.ci_tgg, h.tgwall] + list(np.resize(band, 8)) + list(h.utci)
    lum = scal.lv[:, 2] if (h.daytime and scal.lv is not None) else np.zeros(patches)
    return np.asarray(v, dtype=np.float64), np.asarray(lum, dtype=np.float64)


def _utci_coefficients(ta, rh, ws):
    coef = (ctypes.c_double * 7)()
    _lib.check(_lib.lib().solweig_utci_collapse(float(ta), float(rh), float(ws), coef), "solweig_utci_collapse")
    return np.array(coef[:], dtype=np.float64)


class DayGradient:
    """Forward and reverse pass of one day on one tile."""

    def __init__(self, scene, latitude, longitude, site_altitude=3.0, utc=0.0, hours=24, objective="utci"):
        self.scene = scene
        self.latitude, self.longitude, self.site_altitude, self.utc = latitude, longitude, site_altitude, utc
        self.hours = hours
        self.objective = _OBJECTIVES[objective]
        dev = scene.device
        self.buffers = HourBuffers(scene, hours)
        self.layout_dev = scene.layout.device(dev)
        self.work_bytes = int(_lib.lib().solweig_day_grad_work_bytes(scene.rows, scene.cols, hours))
        self.work = torch.empty(self.work_bytes, dtype=torch.uint8, device=dev)
        L = scene.layout.host
        self.patches = L.count
        # luminance weight factor of the contraction's second column (float32 as on the device)
        self.cw = (L.cos_alt.astype(np.float32) * L.steradian.astype(np.float32)).astype(np.float64)

    # ---------------------------------------------------------------- plan
    def _plan(self, met):
        met = np.asarray(met, dtype=np.float64)
        if len(met) != self.hours:
            raise ValueError(f"expected {self.hours} forcing rows, got {len(met)}")
        plan = plan_day(self.scene, met, self.latitude, self.longitude, self.site_altitude, self.utc)
        self.buffers.wait_free()
        for i, (h, ray, _) in enumerate(plan):
            self.buffers.put(i, h, ray)
        self.buffers.upload(0, self.hours, self.buffers.kmax)
        return plan

    def _params(self, albedo, emissivity, transmissivity):
        sc = self.scene
        ts = [torch.as_tensor(x, dtype=torch.float32, device=sc.device).reshape(sc.shape).contiguous()
              for x in (albedo, emissivity, transmissivity)]
        p = _lib.SolweigGradParams(ts[0].data_ptr(), ts[1].data_ptr(), ts[2].data_ptr())
        return p, ts

    # ---------------------------------------------------------------- passes
    def forward(self, albedo, emissivity, transmissivity, met):
        """Daily mean objective per pixel, [rows, cols] float64 (NaN on roofs for UTCI)."""
        sc = self.scene
        self._plan(met)
        prm, keep = self._params(albedo, emissivity, transmissivity)
        daily = torch.empty(sc.shape, dtype=torch.float64, device=sc.device)
        _lib.check(_lib.lib().solweig_day_grad_forward(
            ctypes.byref(sc.struct), device_ptr(self.layout_dev), self.buffers.ptr(), self.hours,
            sc.gvf_host_ptr, sc.first_steps, sc.second_steps, ctypes.byref(prm), self.objective,
            device_ptr(daily), device_ptr(self.work), self.work_bytes, stream_handle()),
            "solweig_day_grad_forward")
        self.buffers.mark()
        torch.cuda.current_stream().synchronize()
        del keep
        return daily

    def backward(self, albedo, emissivity, transmissivity, met, weights):
        """Gradients of J = sum(weights * daily): (d_albedo, d_emissivity,
        d_transmissivity) [rows, cols] float32 tensors and the host arrays
        hour_grad [H, 21] and lum_grad [H, 4, 160] (float64)."""
        sc = self.scene
        self._plan(met)
        prm, keep = self._params(albedo, emissivity, transmissivity)
        w = torch.as_tensor(weights, dtype=torch.float32, device=sc.device).reshape(sc.shape).contiguous()
        w = torch.nan_to_num(w, nan=0.0)
        outs = [torch.empty(sc.shape, dtype=torch.float32, device=sc.device) for _ in range(3)]
        hour_grad = torch.zeros((self.hours, len(HOUR_FIELDS)), dtype=torch.float64, device=sc.device)
        lum_grad = torch.zeros((self.hours, 4, _lib.MAX_PATCHES), dtype=torch.float64, device=sc.device)
        _lib.check(_lib.lib().solweig_day_grad_backward(
            ctypes.byref(sc.struct), device_ptr(self.layout_dev), self.buffers.ptr(), self.hours,
            sc.gvf_host_ptr, sc.first_steps, sc.second_steps, ctypes.byref(prm), self.objective,
            device_ptr(w), device_ptr(outs[0]), device_ptr(outs[1]), device_ptr(outs[2]),
            device_ptr(hour_grad), device_ptr(lum_grad), device_ptr(self.work), self.work_bytes,
            stream_handle()), "solweig_day_grad_backward")
        self.buffers.mark()
        torch.cuda.current_stream().synchronize()
        del keep
        return outs[0], outs[1], outs[2], hour_grad.cpu().numpy(), lum_grad.cpu().numpy()

    # ---------------------------------------------------------------- forcing
    def scalar_partials(self, hour_grad, lum_grad):
        """dJ/d(HOUR_FIELDS) [H, 21] and dJ/d lum [H, P] from the device partials."""
        P = self.patches
        lg = lum_grad[:, :, :P]
        dlum = lg[:, 0] + lg[:, 2] + self.cw[None, :] * (lg[:, 1] + lg[:, 3])
        return hour_grad, dlum

    def forcing_jacobian(self, met, delta=None):
        """{var: (d fields [H(src), H, 21], d lum [H(src), H, P])}: central
        differences of the FP64 plan with respect to each hour's forcing."""
        met = np.asarray(met, dtype=np.float64)
        delta = delta or {"ta": 1e-4, "rh": 1e-3, "ws": 1e-4}
        H, P = self.hours, self.patches
        out = {}
        for var, col in FORCING_COLUMNS.items():
            dF = np.zeros((H, H, len(HOUR_FIELDS)))
            dL = np.zeros((H, H, P))
            d = delta[var]
            for src in range(H):
                vecs = []
                for sgn in (1.0, -1.0):
                    m = met.copy()
                    m[src, col] += sgn * d
                    plan = plan_day(self.scene, m, self.latitude, self.longitude, self.site_altitude, self.utc)
                    vecs.append([_hour_vector(h, s, P) for h, _, s in plan])
                for hh in range(H):
                    dF[src, hh] = (vecs[0][hh][0] - vecs[1][hh][0]) / (2 * d)
                    dL[src, hh] = (vecs[0][hh][1] - vecs[1][hh][1]) / (2 * d)
                # UTCI coefficients: FP64 collapse (the plan rounds its inputs to float32)
                ta, rh, ws = met[src, 11], met[src, 10], met[src, 9]
                args = {"ta": [ta, rh, ws], "rh": [ta, rh, ws], "ws": [ta, rh, ws]}[var]
                k = {"ta": 0, "rh": 1, "ws": 2}[var]
                a_p, a_m = list(args), list(args)
                a_p[k] += d
                a_m[k] -= d
                dF[src, :, 14:21] = 0.0
                dF[src, src, 14:21] = (_utci_coefficients(*a_p) - _utci_coefficients(*a_m)) / (2 * d)
            out[var] = (dF, dL)
        return out

    def forcing_grad(self, met, hour_grad, lum_grad, jacobian=None):
        """{var: dJ/d forcing [H]} for var in ta, rh, ws."""
        jac = jacobian if jacobian is not None else self.forcing_jacobian(met)
        gF, gL = self.scalar_partials(hour_grad, lum_grad)
        return {var: np.einsum("shf,hf->s", dF, gF) + np.einsum("shk,hk->s", dL, gL)
                for var, (dF, dL) in jac.items()}


class DailyUTCI(torch.autograd.Function):
    """daily = DailyUTCI.apply(albedo, emissivity, transmissivity, ta, rh, ws, day_gradient, met)

    albedo / emissivity / transmissivity: [rows, cols] tensors (any device);
    ta / rh / ws: [H] float64 CPU tensors replacing the forcing table's
    columns; met: the day's forcing table (numpy).  Returns the daily mean
    UTCI (or Tmrt, by the DayGradient's objective) per pixel; roofs are NaN
    for UTCI and receive no gradient."""

    @staticmethod
    def _met(met, ta, rh, ws):
        m = np.array(met, dtype=np.float64, copy=True)
        for col, v in ((11, ta), (10, rh), (9, ws)):
            m[:, col] = v.detach().cpu().numpy().astype(np.float64)
        return m

    @staticmethod
    def forward(ctx, albedo, emissivity, transmissivity, ta, rh, ws, day, met):
        m = DailyUTCI._met(met, ta, rh, ws)
        ctx.day, ctx.met = day, m
        ctx.save_for_backward(albedo, emissivity, transmissivity, ta, rh, ws)
        return day.forward(albedo, emissivity, transmissivity, m).to(device=albedo.device, dtype=albedo.dtype)

    @staticmethod
    def backward(ctx, grad):
        albedo, emissivity, transmissivity, ta, rh, ws = ctx.saved_tensors
        day, met = ctx.day, ctx.met
        da, de, dt, hg, lg = day.backward(albedo, emissivity, transmissivity, met, grad)
        fg = day.forcing_grad(met, hg, lg)
        conv = lambda g, like: torch.as_tensor(g, dtype=like.dtype, device=like.device)  # noqa: E731
        return (da.to(albedo.device), de.to(emissivity.device), dt.to(transmissivity.device),
                conv(fg["ta"], ta), conv(fg["rh"], rh), conv(fg["ws"], ws), None, None)
