"""Drop-in for the reference's ``src/model.py`` step: ``prepare_model`` and
``Solweig_2022a_calc`` with the same names, arguments and 39-tuple result.

``prepare_model(**inputs)`` packs the static inputs (the ``static`` dict of
``src/series.py:350-365``) into a device :class:`engine.Scene`;
``Solweig_2022a_calc`` runs one hour through the CUDA step (shadow sweep,
ground view factors, anisotropic K/L fluxes, Tmrt) and returns the tuple of
``src/model.py:253-256`` (names in :data:`OUTPUT_NAMES`).  Planes are torch
CUDA tensors, scalars are Python floats.

Supported configuration: cylinder (``cyl=1``), anisotropic sky
(``anisotropic_sky=1``), vegetation scheme on (``usevegdem=1``), global-only
radiation (``onlyglobal=1``) -- the configuration the reference's series
driver uses (``src/series.py:48-51``, ``:319``).  Other switches raise
``NotImplementedError``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib, engine
from .engine import _as_device, device_ptr, stream_handle

__all__ = ["prepare_model", "Solweig_2022a_calc", "PreparedModel", "OUTPUT_NAMES", "STATE_NAMES",
           "FIELD_NAMES", "SBC"]

SBC = 5.67051e-8

OUTPUT_NAMES = ('Tmrt', 'Kdown', 'Kup', 'Ldown', 'Lup', 'Tg', 'ea', 'esky', 'I0', 'CI',
                'shadow', 'firstdaytime', 'timestepdec', 'timeadd', 'Tgmap1', 'Tgmap1E', 'Tgmap1S',
                'Tgmap1W', 'Tgmap1N', 'Keast', 'Ksouth', 'Kwest', 'Knorth', 'Least', 'Lsouth', 'Lwest',
                'Lnorth', 'KsideI', 'TgOut1', 'TgOut', 'radI', 'radD', 'Lside', 'L_patches', 'CI_Tg',
                'CI_TgG', 'KsideD', 'dRad', 'Kside')
STATE_NAMES = ('CI', 'firstdaytime', 'timeadd', 'Tgmap1', 'Tgmap1E', 'Tgmap1S', 'Tgmap1W', 'Tgmap1N',
               'TgOut1')
FIELD_NAMES = ('svf', 'svfN', 'svfW', 'svfE', 'svfS', 'svfveg', 'svfNveg', 'svfEveg', 'svfSveg',
               'svfWveg', 'svfaveg', 'svfEaveg', 'svfSaveg', 'svfWaveg', 'svfNaveg', 'lc_grid', 'TgK',
               'Tstart', 'alb_grid', 'emis_grid', 'TmaxLST', 'svfbuveg', 'asvf', 'svfalfa')

_STATE_ARGS = ("Tgmap1", "Tgmap1E", "Tgmap1S", "Tgmap1W", "Tgmap1N", "TgOut1")
_STATE_ABI = ("tgmap1", "tgmap1e", "tgmap1s", "tgmap1w", "tgmap1n", "tgout1")
_PLANES = {  # 39-tuple name -> ABI output plane
    'Tmrt': 'tmrt', 'Kdown': 'kdown', 'Kup': 'kup', 'Ldown': 'ldown', 'Lup': 'lup', 'Tg': 'tg',
    'shadow': 'shadow', 'Keast': 'keast', 'Ksouth': 'ksouth', 'Kwest': 'kwest', 'Knorth': 'knorth',
    'Least': 'least', 'Lsouth': 'lsouth', 'Lwest': 'lwest', 'Lnorth': 'lnorth', 'KsideI': 'kside_i',
    'TgOut': 'tg_out', 'Lside': 'lside', 'KsideD': 'kside_d', 'dRad': 'd_rad', 'Kside': 'kside'}


@dataclass(frozen=True)
class PreparedModel:
    """Device-resident static geometry of one tile (see ``src/model.py:973-984``)."""
    scene: object
    dtype: np.dtype
    shape: tuple
    inputs: dict

    @property
    def fields(self):
        return {n: self.inputs.get(n) for n in FIELD_NAMES}


def _check_switches(inputs):
    for key, want in (("cyl", 1), ("anisotropic_sky", 1), ("usevegdem", 1), ("onlyglobal", 1)):
        if key in inputs and int(inputs[key]) != want:
            raise NotImplementedError(f"{key}={inputs[key]} is not supported (only {key}={want})")


def prepare_model(*, dtype=np.float32, **inputs):
    """Prepared geometry for :func:`Solweig_2022a_calc` (``src/model.py:987-1016``)."""
    _check_switches(inputs)
    scene = engine.Scene.from_inputs(inputs)
    return PreparedModel(scene, np.dtype(dtype), scene.shape, dict(inputs))


class _StepRunner:
    """Per-scene buffers for single-hour calls (the float32 or float64 step's
    scratch is allocated on first use)."""

    def __init__(self, scene):
        self.scene = scene
        self.buffers = engine.HourBuffers(scene, 1)
        self.layout_dev = scene.layout.device(scene.device)
        self._scratch = {}
        self.h64_host = self.h64_dev = None

    def scratch(self, dtype):
        if dtype not in self._scratch:
            planes = _lib.SCRATCH64_PLANES if dtype == torch.float64 else _lib.SCRATCH_PLANES
            self._scratch[dtype] = torch.empty((planes,) + self.scene.shape, dtype=dtype, device=self.scene.device)
        return self._scratch[dtype]

    def put64(self, hour, scal):
        """Stage and upload the hour's float64 patch weights (after ``buffers.put``)."""
        raw = np.frombuffer(_lib.struct_bytes(engine.hour64_record(self.scene, hour, scal)), dtype=np.uint8)
        if self.h64_host is None:
            self.h64_host = torch.empty(raw.size, dtype=torch.uint8, pin_memory=True)
            self.h64_dev = torch.empty(raw.size, dtype=torch.uint8, device=self.scene.device)
        self.h64_host.numpy()[:] = raw
        self.h64_dev.copy_(self.h64_host, non_blocking=True)


_RUNNERS = {}

# prepare_model results of calls without ``prepared``, keyed by the identity
# of the static inputs (the arrays are held here, so their ids stay unique).
_STATIC_ARGS = ("dsm", "svf", "svfN", "svfW", "svfE", "svfS", "svfveg", "svfNveg", "svfEveg", "svfSveg",
                "svfWveg", "svfaveg", "svfEaveg", "svfSaveg", "svfWaveg", "svfNaveg", "vegdem", "vegdem2",
                "buildings", "lc_grid", "dirwalls", "walls", "bush", "TgK", "Tstart", "alb_grid",
                "emis_grid", "TmaxLST", "svfalfa", "svfbuveg", "diffsh", "shmat", "vegshmat",
                "vbshvegshmat", "asvf")
_STATIC_SCALARS = ("scale", "amaxvalue", "landcover", "patch_option", "first", "second")
_PREPARED = []  # [(key, held arrays, PreparedModel)], most recent last
_PREPARED_MAX = 2


def _prepared_for(args, dtype):
    key = tuple(id(args[k]) for k in _STATIC_ARGS) + tuple(
        float(args[k]) if np.ndim(args[k]) == 0 else id(args[k]) for k in _STATIC_SCALARS) + (str(np.dtype(dtype)),)
    for i, (k, _, prep) in enumerate(_PREPARED):
        if k == key:
            _PREPARED.append(_PREPARED.pop(i))
            return prep
    inputs = {k: v for k, v in args.items() if k not in ("prepared", "dtype")}
    prep = prepare_model(dtype=dtype, **inputs)
    _PREPARED.append((key, tuple(args[k] for k in _STATIC_ARGS), prep))
    while len(_PREPARED) > _PREPARED_MAX:
        old = _PREPARED.pop(0)
        _RUNNERS.pop(id(old[2].scene), None)
    return prep


def Solweig_2022a_calc(i, dsm, scale, rows, cols, svf, svfN, svfW, svfE, svfS, svfveg, svfNveg, svfEveg, svfSveg,
                       svfWveg, svfaveg, svfEaveg, svfSaveg, svfWaveg, svfNaveg, vegdem, vegdem2, albedo_b, absK, absL,
                       ewall, Fside, Fup, Fcyl, altitude, azimuth, zen, jday, usevegdem, onlyglobal, buildings, location, psi,
                       landcover, lc_grid, dectime, altmax, dirwalls, walls, cyl, elvis, Ta, RH, radG, radD, radI, P,
                       amaxvalue, bush, Twater, TgK, Tstart, alb_grid, emis_grid, TgK_wall, Tstart_wall, TmaxLST,
                       TmaxLST_wall, first, second, svfalfa, svfbuveg, firstdaytime, timeadd, timestepdec, Tgmap1,
                       Tgmap1E, Tgmap1S, Tgmap1W, Tgmap1N, CI, TgOut1, diffsh, shmat, vegshmat, vbshvegshmat,
                       anisotropic_sky, asvf, patch_option, *, dtype=np.float32, prepared=None):
    """One SOLWEIG 2022a hour on the device; returns the reference's 39-tuple.

    Without ``prepared`` the device geometry is built on the first call and
    reused by later calls given the same static array objects (the two most
    recent sets are kept); arrays changed in place between calls need a new
    ``prepare_model``.  ``dtype`` float64 runs the float64 step
    (``solweig_step64``: the reference's float64 radiation switch) and returns
    float64 planes and state."""
    args = dict(locals())
    _check_switches(args)
    constants = dict(albedo_b=0.2, absK=0.7, absL=0.95, ewall=0.9, Fside=0.22, Fup=0.06, Fcyl=0.28,
                     elvis=0)
    for k, v in constants.items():
        if abs(float(args[k]) - v) > 1e-12:
            raise NotImplementedError(f"{k}={args[k]} differs from the compiled constant {v}")
    if prepared is None:
        prepared = _prepared_for(args, dtype)
    scene = prepared.scene
    key = id(scene)
    if key not in _RUNNERS:
        _RUNNERS[key] = _StepRunner(scene)
    run = _RUNNERS[key]
    dt = np.dtype(dtype)
    h, ray, scal, (fd_next, timeadd_next, ci_next) = engine.hour_plan(
        scene, float(location["latitude"]), float(altitude), float(azimuth), float(zen), float(jday),
        float(dectime), float(altmax), float(Ta), float(RH), float(radG), float(radD), float(radI),
        float(P), 0.0, float(psi), float(CI), int(firstdaytime), float(timeadd), float(timestepdec),
        None if Twater is None else float(Twater))
    f64 = dt == np.float64
    tdt = torch.float64 if f64 else torch.float32
    run.buffers.wait_free()
    run.buffers.put(0, h, ray)
    run.buffers.upload(0, 1, ray.steps if ray is not None else 1)
    if f64:
        run.put64(h, scal)
    state = {}
    st = _lib.SolweigState64() if f64 else _lib.SolweigState()
    for arg, abi in zip(_STATE_ARGS, _STATE_ABI):
        t = _as_device(args[arg], tdt, scene.device, scene.shape).clone()
        state[arg] = t
        setattr(st, abi, t.data_ptr())
    planes = {name: torch.empty(scene.shape, dtype=tdt, device=scene.device) for name in _PLANES}
    out = _lib.SolweigOutputs64() if f64 else _lib.SolweigOutputs()
    for name, abi in _PLANES.items():
        setattr(out, abi, planes[name].data_ptr())
    if f64:
        _lib.check(_lib.lib().solweig_step64(
            ctypes.byref(scene.struct), device_ptr(scene.svfbuveg64()), device_ptr(run.layout_dev),
            device_ptr(scene.layout.device64(scene.device)), run.buffers.ptr(), device_ptr(run.h64_dev), 0,
            ctypes.byref(st), ctypes.byref(out), scene.gvf_host_ptr, scene.first_steps, scene.second_steps,
            device_ptr(run.scratch(torch.float64)), stream_handle()), "solweig_step64")
    else:
        _lib.check(_lib.lib().solweig_step(
            ctypes.byref(scene.struct), device_ptr(run.layout_dev), run.buffers.ptr(), 0, ctypes.byref(st),
            ctypes.byref(out), scene.gvf_host_ptr, scene.first_steps, scene.second_steps,
            device_ptr(run.scratch(torch.float32)), stream_handle()), "solweig_step")
    run.buffers.mark()
    torch.cuda.current_stream().synchronize()
    if altitude > 0:
        L_patches = scal.lv.copy()
    else:
        lay = scene.layout.host
        L_patches = np.column_stack((lay.altitude, lay.azimuth, np.zeros(lay.count)))
    values = {
        'ea': float(scal.ea), 'esky': float(scal.esky), 'I0': float(scal.I0), 'CI': float(ci_next),
        'firstdaytime': fd_next, 'timestepdec': float(timestepdec), 'timeadd': timeadd_next,
        'radI': float(scal.radI), 'radD': float(scal.radD), 'L_patches': L_patches,
        'CI_Tg': float(scal.CI_Tg), 'CI_TgG': float(scal.CI_TgG),
    }
    for name in _PLANES:
        values[name] = planes[name]
    for arg in _STATE_ARGS:
        values[arg] = state[arg]
    return tuple(values[n] for n in OUTPUT_NAMES)
