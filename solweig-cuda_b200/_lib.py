"""ctypes binding of ``libsolweig_b200.so`` (the C ABI of ``include/solweig_b200.h``).

The structs below mirror the header field by field.  The library is loaded
lazily on first use; if it is missing or cannot be loaded this raises -- the
package has no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

__all__ = ["lib", "check", "SolweigScene", "SolweigSkyLayout", "SolweigHour", "SolweigOutputs",
           "SolweigState", "SolweigSky64", "SolweigHour64", "SolweigOutputs64", "SolweigState64", "MAX_PATCHES", "MASK_WORDS", "MAX_BANDS", "GVF_DIRECTIONS",
           "GVF_MAX_STEPS", "EXPORTED_SYMBOLS", "library_path"]

MAX_PATCHES = 160
MASK_WORDS = 5
MAX_BANDS = 8
GVF_DIRECTIONS = 18
GVF_MAX_STEPS = 64
SCRATCH_PLANES = 20  # quad (4) + first-direction Lup (1) + 15 GVF planes
SCRATCH64_PLANES = 20  # float64 step: 5 per-pixel GVF inputs + 15 GVF planes
STATIC_SCRATCH_MAX_PIXELS = 512 * 512  # capacity of solweig_step_static_scratch

_c_double_p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p


class SolweigScene(ctypes.Structure):
    _fields_ = [
        ("rows", ctypes.c_int32), ("cols", ctypes.c_int32), ("scale", ctypes.c_double),
        ("dsm", _vp), ("vegdem", _vp), ("vegdem2", _vp), ("walls", _vp), ("aspect", _vp),
        ("flags", _vp), ("alb", _vp), ("emis", _vp), ("tgk", _vp), ("tstart", _vp),
        ("tmaxlst", _vp), ("svfbuveg", _vp), ("svfalfa", _vp), ("tan_asvf", _vp), ("masks", _vp),
        ("veg_sums", _vp), ("sky_band_counts", _vp), ("gvf_face", _vp), ("svf_dir", _vp),
        ("patches", ctypes.c_int32), ("nbands", ctypes.c_int32), ("landcover", ctypes.c_int32),
        ("has_water", ctypes.c_int32), ("hmax", ctypes.c_double), ("geo32", _vp),
        ("gvf_hits", _vp), ("gvf_nosh", _vp),
    ]


class SolweigSkyLayout(ctypes.Structure):
    _fields_ = [
        ("patches", ctypes.c_int32), ("nbands", ctypes.c_int32),
        ("band_of_patch", ctypes.c_int32 * MAX_PATCHES),
        ("omega", ctypes.c_float * MAX_PATCHES), ("cos_alt", ctypes.c_float * MAX_PATCHES),
        ("sin_alt", ctypes.c_float * MAX_PATCHES),
        ("band_omega", ctypes.c_float * MAX_BANDS), ("band_cos", ctypes.c_float * MAX_BANDS),
        ("band_sin", ctypes.c_float * MAX_BANDS),
        ("sunlit_below", ctypes.c_double * MAX_PATCHES),
        ("shaded_above", ctypes.c_double * MAX_PATCHES),
        ("cardinal", (ctypes.c_float * MAX_PATCHES) * 4),
    ]


class SolweigHour(ctypes.Structure):
    _fields_ = [
        ("daytime", ctypes.c_int32),
        ("altitude", ctypes.c_double), ("azimuth", ctypes.c_double), ("zen", ctypes.c_double),
        ("ta", ctypes.c_double), ("rh", ctypes.c_double), ("ws", ctypes.c_double),
        ("rad_g", ctypes.c_double), ("rad_d", ctypes.c_double), ("rad_i", ctypes.c_double),
        ("psi", ctypes.c_double), ("cos_alt", ctypes.c_double), ("sin_alt", ctypes.c_double),
        ("tan_zen", ctypes.c_double), ("esky", ctypes.c_double), ("ci_tgg", ctypes.c_double),
        ("tg_phase", ctypes.c_double), ("altmax", ctypes.c_double),
        ("dectime_frac", ctypes.c_double), ("snup", ctypes.c_double), ("tgwall", ctypes.c_double),
        ("twater", ctypes.c_double),
        ("firstdaytime", ctypes.c_int32), ("wave_update", ctypes.c_int32),
        ("wave_weight", ctypes.c_double),
        ("steps", ctypes.c_int32), ("ray_dxdy", _vp), ("ray_dz", _vp),
        ("ray_low", ctypes.c_double), ("ray_high", ctypes.c_double), ("ray_middle", ctypes.c_int32),
        ("lum", ctypes.c_float * MAX_PATCHES), ("yi", ctypes.c_double * MAX_PATCHES),
        ("lw_sun_test", ctypes.c_uint8 * MAX_PATCHES), ("band_lsky", ctypes.c_float * MAX_BANDS),
        ("rad_tot", ctypes.c_double), ("utci", ctypes.c_double * 7), ("utci_valid", ctypes.c_int32),
    ]


OUTPUT_FIELDS = ("tmrt", "utci", "kdown", "kup", "ldown", "lup", "shadow", "tg", "keast", "ksouth",
                 "kwest", "knorth", "least", "lsouth", "lwest", "lnorth", "kside_i", "kside_d",
                 "kside", "lside", "d_rad", "tg_out")


class SolweigOutputs(ctypes.Structure):
    _fields_ = [(name, _vp) for name in OUTPUT_FIELDS]


STATE_FIELDS = ("tgmap1", "tgmap1e", "tgmap1s", "tgmap1w", "tgmap1n", "tgout1")


class SolweigState(ctypes.Structure):
    _fields_ = [(name, _vp) for name in STATE_FIELDS]


class SolweigSky64(ctypes.Structure):
    """Float64 per-patch constants of the float64 step (device copy per layout)."""
    _fields_ = [("omega", ctypes.c_double * MAX_PATCHES), ("cos_alt", ctypes.c_double * MAX_PATCHES),
                ("sin_alt", ctypes.c_double * MAX_PATCHES),
                ("cardinal", (ctypes.c_double * MAX_PATCHES) * 4), ("diffsh_veg", ctypes.c_double)]


class SolweigHour64(ctypes.Structure):
    """Float64 per-patch weights of one hour (beside its SolweigHour)."""
    _fields_ = [("lum", ctypes.c_double * MAX_PATCHES), ("band_lsky", ctypes.c_double * MAX_BANDS)]


class SolweigOutputs64(ctypes.Structure):
    """SolweigOutputs of the float64 step: float64 planes, float32 UTCI."""
    _fields_ = [(name, _vp) for name in OUTPUT_FIELDS]


class SolweigState64(ctypes.Structure):
    _fields_ = [(name, _vp) for name in STATE_FIELDS]


class SolweigGradParams(ctypes.Structure):
    """Per-pixel parameters of the day gradient (device float32 pointers)."""
    _fields_ = [("albedo", _vp), ("emissivity", _vp), ("transmissivity", _vp)]


class SolweigDayConfig(ctypes.Structure):
    """Launch shapes of the batched day (``solweig_day_batched_ex``)."""
    _fields_ = [("shadow_bx", ctypes.c_int32), ("shadow_by", ctypes.c_int32),
                ("gvf_rows", ctypes.c_int32), ("rad_threads", ctypes.c_int32),
                ("gemm_ctas_per_sm", ctypes.c_int32), ("gvf_hours", ctypes.c_int32),
                ("no_ceiling", ctypes.c_int32), ("sweep_window", ctypes.c_int32)]

    def astuple(self):
        return tuple(getattr(self, f) for f, _ in self._fields_)

    @classmethod
    def default(cls):
        return cls(16, 16, 8, 256, 0, 1, 0, 0)


EXPORTED_SYMBOLS = (
    "solweig_last_error", "solweig_version", "solweig_wall_heights", "solweig_wall_aspect",
    "solweig_shadow", "solweig_svf", "solweig_svf_unpack", "solweig_diffsh", "solweig_gvf",
    "solweig_step", "solweig_utci", "solweig_utci_collapse", "solweig_scene_build",
    "solweig_scene_finalize", "solweig_struct_sizes", "solweig_step_shadow",
    "solweig_step_radiation", "solweig_day", "solweig_step_gvf", "solweig_utci_scalar",
    "solweig_svf_pack", "solweig_svf_reduce", "solweig_step_static_scratch",
    "solweig_day_batched", "solweig_day_batched_work_bytes", "solweig_day_batched_error",
    "solweig_patch_sums", "solweig_day_batched_timed", "solweig_day_batched_ex", "solweig_day_batched_part",
    "solweig_day_batched_layout", "solweig_day_grad_work_bytes", "solweig_day_grad_forward",
    "solweig_day_grad_backward", "solweig_svf_ex", "solweig_svf_ex2", "solweig_svf_work_bytes",
    "solweig_gvf_statics", "solweig_step64", "solweig_struct_sizes64", "solweig_wall_segments_burn",
    "solweig_geometry_walls",
)

_lock = threading.Lock()
_lib = None


def library_path():
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsolweig_b200.so")


def _declare(lib):
    i32, i64, dbl, fl, P = ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_float, _vp
    sig = {
        "solweig_last_error": (ctypes.c_char_p, []),
        "solweig_version": (i32, []),
        "solweig_wall_heights": (i32, [P, P, i32, i32, dbl, P]),
        "solweig_wall_aspect": (i32, [P, P, P, i32, i32, i32, P, P, P, P, P, P, P]),
        "solweig_wall_segments_burn": (i32, [P, i64, i32, i32, P, P]),
        "solweig_geometry_walls": (i32, [P, P, P, P, i64, dbl, P, P, P]),
        "solweig_shadow": (i32, [P, P, P, i32, dbl, dbl, i32, i32, P, P]),
        "solweig_svf": (i32, [P, P, P, P, i32, i32, i32, i32, P, P, P, dbl, P, P, P, dbl, P, P, P, P,
                              P]),
        "solweig_svf_ex": (i32, [P, P, P, P, P, i32, i32, i32, i32, P, P, P, dbl, P, P, P, dbl, P, P, P,
                                 P, P]),
        "solweig_svf_ex2": (i32, [P, P, P, P, P, i32, i32, i32, i32, P, P, P, dbl, P, P, P, dbl, P, P, P,
                                  P, P, i64, P]),
        "solweig_svf_work_bytes": (i64, [i32, i32]),
        "solweig_svf_unpack": (i32, [P, i64, i32, P, P, P, P]),
        "solweig_diffsh": (i32, [P, P, P, i64, fl, P]),
        "solweig_gvf": (i32, [P, P, P, P, dbl, dbl, dbl, dbl, dbl, P, i32, i32, P, P, P]),
        "solweig_step": (i32, [P, P, P, i32, P, P, P, i32, i32, P, P]),
        "solweig_step_static_scratch": (i32, [P, P, P, i32, P, P, P, i32, i32, P]),
        "solweig_step64": (i32, [P, P, P, P, P, P, i32, P, P, P, i32, i32, P, P]),
        "solweig_day_batched": (i32, [P, P, P, i32, P, P, i64, P, i32, i32, P, i64, P]),
        "solweig_day_batched_work_bytes": (i64, [i32, i32, i32, i32]),
        "solweig_day_batched_timed": (i32, [P, P, P, i32, P, P, i64, P, i32, i32, P, i64, P, P, P]),
        "solweig_day_batched_ex": (i32, [P, P, P, i32, P, P, i64, P, i32, i32, P, i64, P, P]),
        "solweig_day_batched_part": (i32, [P, P, P, i32, P, P, i64, P, i32, i32, P, i64, P, i32, i32, i32, P]),
        "solweig_day_batched_layout": (i32, [i32, i32, i32, i32, P]),
        "solweig_gvf_statics": (i32, [P, P, i32, i32, P, P, P]),
        "solweig_day_grad_work_bytes": (i64, [i32, i32, i32]),
        "solweig_day_grad_forward": (i32, [P, P, P, i32, P, i32, i32, P, i32, P, P, i64, P]),
        "solweig_day_grad_backward": (i32, [P, P, P, i32, P, i32, i32, P, i32, P, P, P, P, P, P, P, i64, P]),
        "solweig_day_batched_error": (i32, [P, i32, i32, i32, i32, P, P]),
        "solweig_patch_sums": (i32, [P, i64, i32, P, i32, P, P, i64, P]),
        "solweig_day": (i32, [P, P, P, i32, P, P, i64, P, i32, i32, P, P]),
        "solweig_utci": (i32, [P, P, P, P, i32, i32, i32, P, i64, P]),
        "solweig_utci_collapse": (i32, [dbl, dbl, dbl, P]),
        "solweig_scene_build": (i32, [P, P, P, P, i64, dbl, dbl, P, i32, P, P, P, P, P, P, P, P, P,
                                      P, P, P]),
        "solweig_scene_finalize": (i32, [P, P, P, i64, dbl, P, P, P, P, P, P, P, P, P]),
        "solweig_struct_sizes": (i32, [P]),
        "solweig_struct_sizes64": (i32, [P]),
        "solweig_utci_scalar": (i32, [dbl, dbl, dbl, P, P, i64, P]),
        "solweig_svf_pack": (i32, [P, P, P, i64, i32, P, P]),
        "solweig_svf_reduce": (i32, [P, P, i64, P, P, P, dbl, P, P, P, P]),
        "solweig_step_shadow": (i32, [P, P, i32, P, P]),
        "solweig_step_gvf": (i32, [P, P, i32, P, i32, i32, P, i32, P]),
        "solweig_step_radiation": (i32, [P, P, P, i32, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def lib():
    """The loaded library (loaded once, thread-safe)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                path = library_path()
                if not os.path.exists(path):
                    raise RuntimeError(
                        f"libsolweig_b200.so not found at {path}; build it with "
                        "`python __graft_entry__.py` or `make -C solweig-cuda_b200/csrc`")
                handle = ctypes.CDLL(path)
                _declare(handle)
                sizes = (ctypes.c_int64 * 5)()
                handle.solweig_struct_sizes(sizes)
                mine = [ctypes.sizeof(t) for t in (SolweigScene, SolweigSkyLayout, SolweigHour,
                                                  SolweigOutputs, SolweigState)]
                sizes64 = (ctypes.c_int64 * 4)()
                handle.solweig_struct_sizes64(sizes64)
                mine64 = [ctypes.sizeof(t) for t in (SolweigSky64, SolweigHour64, SolweigOutputs64,
                                                    SolweigState64)]
                if list(sizes) != mine or list(sizes64) != mine64:
                    raise RuntimeError(f"ABI struct size mismatch: library {list(sizes)} {list(sizes64)} "
                                       f"vs binding {mine} {mine64}")
                _lib = handle
    return _lib


def check(status, what="solweig"):
    """Raise ``RuntimeError`` with the library's message on a non-zero status."""
    if status != 0:
        msg = lib().solweig_last_error()
        raise RuntimeError(f"{what} failed ({status}): {msg.decode() if msg else ''}")


def struct_bytes(obj):
    """Raw bytes of a ctypes struct (for upload to device memory)."""
    return ctypes.string_at(ctypes.addressof(obj), ctypes.sizeof(obj))
