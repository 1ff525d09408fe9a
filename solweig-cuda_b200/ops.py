"""Thin wrappers of single C-ABI calls on a prepared :class:`engine.Scene`.

Each returns torch tensors on the scene's device; launches go to torch's
current CUDA stream.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib, rays
from .engine import _upload, device_ptr, stream_handle

__all__ = ["cast_shadow", "unpack_masks", "gvf_planes", "utci"]


def cast_shadow(scene, azimuth, altitude, vegetation=True, stream=None):
    """Eight shadow planes [8, rows, cols] float64 for one sun position
    (``src/model.py:689-708``; order vegsh, sh, vbshvegsh, wallsh, wallsun,
    wallshve, facesh, facesun)."""
    maximum = scene.amaxvalue if vegetation else scene.dsm_max
    ray = rays.shadow_ray(float(azimuth), float(altitude), scene.scale, maximum, scene.shape,
                          vegetation)
    out = torch.empty((8,) + scene.shape, dtype=torch.float64, device=scene.device)
    dxdy = _upload(ray.dxdy if ray.steps else np.zeros((1, 2), np.int32), np.int32, scene.device)
    dz = _upload(ray.dz if ray.steps else np.zeros(1), np.float64, scene.device)
    _lib.check(_lib.lib().solweig_shadow(
        ctypes.byref(scene.struct), device_ptr(dxdy), device_ptr(dz), ray.steps, ray.low, ray.high,
        ray.middle, int(bool(vegetation)), device_ptr(out), stream_handle(stream)), "solweig_shadow")
    torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
    return out


def unpack_masks(scene, which=("sh", "veg", "vb"), stream=None):
    """The reference's float32 cubes [rows, cols, P] from the packed masks."""
    P = scene.layout.struct.patches
    outs = {k: torch.empty(scene.shape + (P,), dtype=torch.float32, device=scene.device)
            for k in which}
    _lib.check(_lib.lib().solweig_svf_unpack(
        device_ptr(scene.masks), scene.pixels, P, device_ptr(outs.get("sh")),
        device_ptr(outs.get("veg")), device_ptr(outs.get("vb")), stream_handle(stream)),
        "solweig_svf_unpack")
    return tuple(outs[k] for k in which)


def gvf_planes(scene, shadow, wallsun, tg, tgwall, ta, twater=0.0, ewall=0.9, albedo_b=0.2,
               stream=None):
    """17 GVF planes [17, rows, cols] float32 (``src/model.py:569-622``)."""
    dev = scene.device
    sh = torch.as_tensor(shadow, dtype=torch.float32, device=dev).contiguous()
    ws = torch.as_tensor(wallsun, dtype=torch.float64, device=dev).contiguous()
    t = torch.as_tensor(tg, dtype=torch.float32, device=dev).contiguous()
    scratch = torch.empty((5,) + scene.shape, dtype=torch.float32, device=dev)
    planes = torch.empty((17,) + scene.shape, dtype=torch.float32, device=dev)
    _lib.check(_lib.lib().solweig_gvf(
        ctypes.byref(scene.struct), device_ptr(sh), device_ptr(ws), device_ptr(t), float(tgwall),
        float(ta), float(ewall), float(albedo_b), float(twater), device_ptr(scene.gvf_dxdy),
        scene.first_steps, scene.second_steps, device_ptr(scratch), device_ptr(planes),
        stream_handle(stream)), "solweig_gvf")
    return planes


def utci(ta, rh, tmrt, va, stream=None):
    """UTCI per pixel; ``ta``/``rh``/``va`` may be scalars or arrays shaped like ``tmrt``."""
    tm = torch.as_tensor(tmrt, dtype=torch.float32, device="cuda").contiguous()
    args, flags = [], []
    for x in (ta, rh, va):
        t = torch.as_tensor(x, dtype=torch.float32, device=tm.device)
        scalar = t.numel() == 1
        args.append(t.reshape(-1).contiguous() if scalar else torch.broadcast_to(t, tm.shape).contiguous())
        flags.append(int(scalar))
    out = torch.empty_like(tm)
    _lib.check(_lib.lib().solweig_utci(
        device_ptr(args[0]), device_ptr(args[1]), device_ptr(tm), device_ptr(args[2]), flags[0],
        flags[1], flags[2], device_ptr(out), tm.numel(), stream_handle(stream)), "solweig_utci")
    return out
