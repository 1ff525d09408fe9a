"""Drop-in for the reference's ``src/utci.py``: ``utci_calculator(Ta, RH, Tmrt, va10m)``.

Scalar weather (Ta, RH and wind as scalars, the series path) folds the
6th-order UTCI polynomial into seven coefficients in (Tmrt - Ta) on the host
and evaluates them per pixel; per-pixel weather evaluates the full
polynomial per pixel.  Returns a float32 CUDA tensor shaped like ``Tmrt``;
-999 marks inputs at the -999 sentinel, as in the reference.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .engine import device_ptr, stream_handle

__all__ = ["utci_calculator"]


def _is_scalar(x):
    return np.ndim(x) == 0 or (isinstance(x, torch.Tensor) and x.numel() == 1)


def utci_calculator(Ta, RH, Tmrt, va10m, device="cuda"):
    tm = torch.as_tensor(Tmrt, dtype=torch.float32, device=device).contiguous()
    out = torch.empty_like(tm)
    if tm.numel() == 0:
        return out
    if all(_is_scalar(x) for x in (Ta, RH, va10m)):
        ta, rh, va = (float(np.float32(torch.as_tensor(x).item() if isinstance(x, torch.Tensor) else x))
                      for x in (Ta, RH, va10m))
        _lib.check(_lib.lib().solweig_utci_scalar(ta, rh, va, device_ptr(tm), device_ptr(out),
                                                  tm.numel(), stream_handle()), "solweig_utci_scalar")
    else:
        args, flags = [], []
        for x in (Ta, RH, va10m):
            t = torch.as_tensor(x, dtype=torch.float32, device=tm.device)
            scalar = t.numel() == 1
            args.append(t.reshape(-1).contiguous() if scalar else torch.broadcast_to(t, tm.shape).contiguous())
            flags.append(int(scalar))
        _lib.check(_lib.lib().solweig_utci(device_ptr(args[0]), device_ptr(args[1]), device_ptr(tm),
                                           device_ptr(args[2]), flags[0], flags[1], flags[2],
                                           device_ptr(out), tm.numel(), stream_handle()), "solweig_utci")
    torch.cuda.current_stream().synchronize()
    return out
