"""Drop-in for the reference's ``src/svf.py``: the 153-patch sky view factor.

``svf_calculator`` and ``compute_diffsh`` keep the reference's names,
arguments and return order; arrays come back as torch CUDA tensors (the
reference returns CuPy arrays).  The visibility is computed bit-packed on the
device and only expanded to the reference's [rows, cols, P] float32 cubes for
the return value.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib, rays
from .engine import CONSTANTS, SkyLayout, _as_device, _upload, device_ptr, stream_handle

__all__ = ["svf_calculator", "compute_diffsh", "DEFAULT_ANGLE_BATCH"]

DEFAULT_ANGLE_BATCH = 32
# reduce-plane index of each returned SVF plane (src/svf.py:113-114)
_ORDER = (0, 10, 1, 11, 6, 4, 14, 9, 2, 12, 7, 5, 3, 13, 8)


def svf_calculator(patch_option, amaxvalue, a, vegdem, vegdem2, bush, scale,
                   angle_batch=DEFAULT_ANGLE_BATCH, transmissivity=0.03, device="cuda"):
    """19-tuple (svf, svfaveg, svfE, svfEaveg, svfEveg, svfN, svfNaveg, svfNveg, svfS,
    svfSaveg, svfSveg, svfveg, svfW, svfWaveg, svfWveg, vegmat, vbmat, shmat, svftotal),
    as ``src/svf.py:81-114``.  ``angle_batch`` is accepted for compatibility; the
    device kernel batches patches itself."""
    del angle_batch
    dev = torch.device(device)
    a = torch.as_tensor(np.asarray(a) if not isinstance(a, torch.Tensor) else a)
    rows, cols = a.shape
    shape = (rows, cols)
    a, top, bot, bu = (_as_device(x, torch.float64, dev, shape) for x in (a, vegdem, vegdem2, bush))
    flags = ((bu > 1).to(torch.uint8) << 1).contiguous()
    hmax = float(max(a.max().item(), top.max().item(), bot.max().item()))
    layout = SkyLayout(patch_option)
    dxdy, dz, lengths, cap = rays.svf_rays(patch_option, shape, float(amaxvalue), float(scale))
    t_dxdy, t_dz, t_len = (_upload(dxdy, np.int32, dev), _upload(dz, np.float64, dev),
                           _upload(lengths, np.int32, dev))
    P = layout.struct.patches
    masks = torch.empty((2 * _lib.MASK_WORDS, rows, cols), dtype=torch.int32, device=dev)
    planes = torch.empty((16, rows, cols), dtype=torch.float64, device=dev)
    veg_sums = torch.empty((4, rows, cols), dtype=torch.float32, device=dev)
    counts = torch.empty((layout.struct.nbands, rows, cols), dtype=torch.uint8, device=dev)
    st = stream_handle()
    L = _lib.lib()
    _lib.check(L.solweig_svf(
        device_ptr(a), device_ptr(top), device_ptr(bot), device_ptr(flags), rows, cols, P, cap,
        device_ptr(t_dxdy), device_ptr(t_dz), device_ptr(t_len), hmax, ctypes.byref(layout.struct),
        layout.band_weights.ctypes.data_as(ctypes.c_void_p),
        layout.sectors.ctypes.data_as(ctypes.c_void_p), float(transmissivity), device_ptr(masks),
        device_ptr(planes), device_ptr(veg_sums), device_ptr(counts), st), "solweig_svf")
    cubes = [torch.empty((rows, cols, P), dtype=torch.float32, device=dev) for _ in range(3)]
    _lib.check(L.solweig_svf_unpack(device_ptr(masks), rows * cols, P, device_ptr(cubes[0]),
                                    device_ptr(cubes[1]), device_ptr(cubes[2]), st), "solweig_svf_unpack")
    torch.cuda.current_stream().synchronize()
    shmat, vegmat, vbmat = cubes
    return tuple(planes[i] for i in _ORDER) + (vegmat, vbmat, shmat, planes[15])


def compute_diffsh(shmat, vegshmat, transmissivity, device="cuda"):
    """``diffsh = shmat - (1 - vegshmat)(1 - transmissivity)`` in float32 (``src/svf.py:117-131``)."""
    sh = torch.as_tensor(shmat, dtype=torch.float32, device=device).contiguous()
    veg = torch.as_tensor(vegshmat, dtype=torch.float32, device=device).contiguous()
    out = torch.empty_like(sh)
    _lib.check(_lib.lib().solweig_diffsh(device_ptr(sh), device_ptr(veg), device_ptr(out), sh.numel(),
                                         float(np.float32(transmissivity)), stream_handle()),
               "solweig_diffsh")
    torch.cuda.current_stream().synchronize()
    return out
