"""Host orchestration of the B200 SOLWEIG engine.

``Scene``      static geometry of one raster tile on the device: walls and
               aspect, the bit-packed 153-patch visibility, SVF planes and the
               derived per-pixel statics (``src/series.py:197-382``);
``hour_plan``  the FP64 host scalars of one forcing hour turned into the
               ``SolweigHour`` struct (``src/model.py:79-216``);
``DayRunner``  the hour loop of one calendar day with the thermal state
               carried on the device (``src/series.py:396-495``).

Device memory is owned by torch tensors; kernels are launched through the C
ABI on torch's current CUDA stream.  There is no CPU fallback: without the
CUDA library or a GPU every entry point raises.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from . import rays
from . import sky as _sky
from . import sun as _sun

__all__ = ["Scene", "SkyLayout", "hour_plan", "DayRunner", "LANDCOVER_CLASSES", "CONSTANTS",
           "stream_handle", "device_ptr"]

SBC = 5.67051e-8

# src/landcoverclasses_2016a.txt: code, albedo, emissivity, TgK, Tstart, TmaxLST
LANDCOVER_CLASSES = np.array([
    [2, 0.18, 0.95, 0.58, -9.78, 15.0],
    [1, 0.18, 0.95, 0.58, -9.78, 15.0],
    [0, 0.20, 0.95, 0.37, -3.41, 15.0],
    [7, 0.05, 0.98, 0.00, 0.00, 12.0],
    [5, 0.16, 0.94, 0.21, -3.38, 14.0],
    [6, 0.25, 0.94, 0.33, -3.01, 14.0],
    [99, 0.20, 0.90, 0.58, -3.41, 15.0],
])

# src/series.py:35-55, :318-325
CONSTANTS = dict(albedo_b=0.2, albedo_g=0.15, ewall=0.9, eground=0.95, absK=0.7, absL=0.95,
                 Fside=0.22, Fup=0.06, Fcyl=0.28, transVeg=0.03, firstdayleaf=97, lastdayleaf=300,
                 elvis=0.0)


def stream_handle(stream=None):
    s = torch.cuda.current_stream() if stream is None else stream
    return ctypes.c_void_p(s.cuda_stream)


def device_ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("solweig_cuda_b200 needs a CUDA device (sm_100a); none is available")


class SkyLayout:
    """Host + ABI view of one sky-vault layout (``patch_option``)."""

    def __init__(self, patch_option=2):
        L = _sky.patch_layout(patch_option)
        self.host = L
        s = _lib.SolweigSkyLayout()
        s.patches = L.count
        s.nbands = L.band_counts.size
        if L.count > _lib.MAX_PATCHES or s.nbands > _lib.MAX_BANDS:
            raise ValueError(f"patch_option {patch_option}: {L.count} patches / {s.nbands} bands "
                             f"exceed the library limits")
        for k in range(L.count):
            s.band_of_patch[k] = int(L.band_of_patch[k])
            s.omega[k] = L.steradian[k]
            s.cos_alt[k] = L.cos_alt[k]
            s.sin_alt[k] = L.sin_alt[k]
            s.sunlit_below[k] = L.sunlit_below[k]
            s.shaded_above[k] = L.shaded_above[k]
            for d in range(4):
                s.cardinal[d][k] = L.cardinal[k, d]
        self.band_omega = np.zeros(s.nbands)
        for b in range(s.nbands):
            k = int(L.band_offsets[b])
            s.band_omega[b] = L.steradian[k]
            s.band_cos[b] = L.cos_alt[k]
            s.band_sin[b] = L.sin_alt[k]
            self.band_omega[b] = L.steradian[k]
        self.struct = s
        # SVF annulus weights and sector bits (src/svf.py:36-46)
        azimuth, altitude, counts = rays.svf_patch_directions(patch_option)
        edges = (0, 12, 24, 36, 48, 60, 72, 84, 90)
        w = np.zeros((len(counts), 2))
        for b, n in enumerate(counts):
            for k in np.arange(edges[b] + 1, edges[b + 1] + 1):
                ring = 91. - k
                x = (1. / (2. * np.pi)) * np.sin(np.pi / 180.) * np.sin((np.pi * (2. * ring - 1.)) / 180.)
                w[b, 0] += ((360. / n) * (np.pi / 180.)) * x
                w[b, 1] += ((360. / np.ceil(n / 2.)) * (np.pi / 180.)) * x
        self.band_weights = np.ascontiguousarray(w)
        sec = ((azimuth >= 0) & (azimuth < 180)).astype(np.uint8)
        sec |= (((azimuth >= 90) & (azimuth < 270)).astype(np.uint8) << 1)
        sec |= (((azimuth >= 180) & (azimuth < 360)).astype(np.uint8) << 2)
        sec |= (((azimuth >= 270) | (azimuth < 90)).astype(np.uint8) << 3)
        self.sectors = np.ascontiguousarray(sec)
        self._device = {}

    def device(self, dev):
        """The layout struct in device memory (uploaded once per device)."""
        key = str(dev)
        if key not in self._device:
            raw = np.frombuffer(_lib.struct_bytes(self.struct), dtype=np.uint8)
            self._device[key] = torch.from_numpy(raw.copy()).to(dev)
        return self._device[key]

    def struct64(self):
        """The float64 per-patch constants of the float64 step (``SolweigSky64``)."""
        L = self.host
        s = _lib.SolweigSky64()
        P = L.count
        np.ctypeslib.as_array(s.omega)[:P] = L.steradian
        np.ctypeslib.as_array(s.cos_alt)[:P] = L.cos_alt
        np.ctypeslib.as_array(s.sin_alt)[:P] = L.sin_alt
        card = np.ctypeslib.as_array(s.cardinal)
        for d in range(4):
            card[d, :P] = L.cardinal[:, d]
        # diffsh of a vegetation patch (shmat 1, vegshmat 0) in float32, as
        # compute_diffsh evaluates it (src/svf.py:117-131)
        one, tv = np.float32(1.0), np.float32(CONSTANTS["transVeg"])
        s.diffsh_veg = float(one - (one - np.float32(0.0)) * (one - tv))
        return s

    def device64(self, dev):
        """``struct64`` in device memory (uploaded once per device)."""
        key = "f64:" + str(dev)
        if key not in self._device:
            raw = np.frombuffer(_lib.struct_bytes(self.struct64()), dtype=np.uint8)
            self._device[key] = torch.from_numpy(raw.copy()).to(dev)
        return self._device[key]


def _upload(arr, dtype, device):
    return torch.from_numpy(np.ascontiguousarray(arr, dtype=dtype)).to(device, non_blocking=False)


def _raster_to_device(x, device):
    """A 2-D raster (numpy in any real dtype, torch tensor, or anything with
    __cuda_array_interface__) as a contiguous float64 device tensor; host
    arrays are copied in their own dtype and widened on the device."""
    if isinstance(x, torch.Tensor):
        t = x.to(device=device)
    elif hasattr(x, "__cuda_array_interface__"):
        t = torch.as_tensor(x, device=device)
    else:
        t = torch.from_numpy(np.ascontiguousarray(x)).to(device)
    return t.to(torch.float64).contiguous()


def _as_device(x, dtype, device, shape):
    """Any array-like (numpy, torch, __cuda_array_interface__, scalar) as a
    contiguous device tensor of ``shape`` (scalars are broadcast)."""
    if isinstance(x, torch.Tensor):
        t = x.to(device=device, dtype=dtype)
    elif hasattr(x, "__cuda_array_interface__"):
        t = torch.as_tensor(x, device=device).to(dtype)
    else:
        t = torch.as_tensor(np.asarray(x), dtype=dtype).to(device)
    if t.dim() == 0 or t.numel() == 1:
        t = t.reshape(()).expand(shape)
    return t.reshape(shape).contiguous()


def _aspect_templates(pixel_size):
    """Flattened template offset lists for ``solweig_wall_aspect`` (``src/walls.py:24-56``)."""
    from scipy.ndimage import rotate
    size = int(np.floor((1.0 / pixel_size + 1e-10) * 9))
    if size <= 2:
        size = 3
    elif size != 9 and size % 2 == 0:
        size += 1
    radius = size // 2
    line = np.zeros((size, size))
    line[:, radius] = 1
    sides = np.zeros((size, size))
    sides[radius, :radius] = 1
    sides[radius, radius + 1:] = 2
    lists = ([], [], [])
    for angle in range(180):
        rl = np.round(rotate(line, angle, order=1, reshape=False, mode="nearest"))
        rs = np.round(rotate(sides, angle, order=0, reshape=False, mode="nearest"))
        if angle in (150, 30):
            rs[:, size - 1] = 0
        if 270 - angle == 225:
            rl[0, 0] = rl[size - 1, size - 1] = 1
        if 270 - angle == 135:
            rl[0, size - 1] = rl[size - 1, 0] = 1
        for lst, m in zip(lists, (rl != 0, rs == 1, rs == 2)):
            lst.append(np.argwhere(m).astype(np.int32) - radius)
    packed = []
    for lst in lists:
        starts = np.concatenate(([0], np.cumsum([a.shape[0] for a in lst]))).astype(np.int32)
        offs = np.concatenate(lst).astype(np.int32).reshape(-1, 2)
        packed.append((np.ascontiguousarray(offs), starts))
    return radius, size, packed


_TEMPLATE_CACHE = {}


def wall_heights_device(dsm_dev, threshold, stream=None):
    rows, cols = dsm_dev.shape
    walls = torch.empty_like(dsm_dev)
    _lib.check(_lib.lib().solweig_wall_heights(device_ptr(dsm_dev), device_ptr(walls), rows, cols,
                                                float(threshold), stream_handle(stream)),
               "solweig_wall_heights")
    return walls


def wall_aspect(dsm_host, dsm_dev, walls_dev, pixel_size, stream=None):
    """Wall aspect (degrees, float64 host array), ``src/walls.py:83-129``."""
    rows, cols = dsm_host.shape
    key = float(pixel_size)
    if key not in _TEMPLATE_CACHE:
        _TEMPLATE_CACHE[key] = _aspect_templates(pixel_size)
    radius, size, packed = _TEMPLATE_CACHE[key]
    walls = walls_dev.cpu().numpy()
    mask = walls > 0
    aspect = np.zeros((rows, cols))
    if not mask.any():
        return aspect, walls
    if rows > 2 * radius + 2 and cols > 2 * radius + 2:
        dev = dsm_dev.device
        t = [(_upload(o, np.int32, dev), _upload(s, np.int32, dev)) for o, s in packed]
        out = torch.empty_like(dsm_dev)
        _lib.check(_lib.lib().solweig_wall_aspect(
            device_ptr(dsm_dev), device_ptr(walls_dev), device_ptr(out), rows, cols, radius,
            device_ptr(t[0][0]), device_ptr(t[0][1]), device_ptr(t[1][0]), device_ptr(t[1][1]),
            device_ptr(t[2][0]), device_ptr(t[2][1]), stream_handle(stream)), "solweig_wall_aspect")
        aspect = out.cpu().numpy()
    unresolved = np.flatnonzero(mask & (aspect == 0))
    if unresolved.size:
        aspect.ravel()[unresolved] += _gradient_aspect(dsm_host, pixel_size, unresolved)
    return aspect, walls


def wall_aspect_device(dsm_host, dsm_dev, walls_dev, pixel_size, stream=None, host_work=None):
    """Wall aspect in degrees as a float64 device tensor (``src/walls.py:83-129``):
    the template kernel on the device, the gradient fall-back only at the few
    wall pixels the templates leave unresolved (from ``dsm_host`` when given).
    ``host_work`` (optional) runs on the host while the template kernel runs."""
    rows, cols = dsm_dev.shape
    key = float(pixel_size)
    if key not in _TEMPLATE_CACHE:
        _TEMPLATE_CACHE[key] = _aspect_templates(pixel_size)
    radius, size, packed = _TEMPLATE_CACHE[key]
    mask = walls_dev > 0
    aspect = torch.zeros_like(dsm_dev)
    if not bool(mask.any()):
        if host_work is not None:
            host_work()
        return aspect
    if rows > 2 * radius + 2 and cols > 2 * radius + 2:
        dev = dsm_dev.device
        t = [(_upload(o, np.int32, dev), _upload(s, np.int32, dev)) for o, s in packed]
        _lib.check(_lib.lib().solweig_wall_aspect(
            device_ptr(dsm_dev), device_ptr(walls_dev), device_ptr(aspect), rows, cols, radius,
            device_ptr(t[0][0]), device_ptr(t[0][1]), device_ptr(t[1][0]), device_ptr(t[1][1]),
            device_ptr(t[2][0]), device_ptr(t[2][1]), stream_handle(stream)), "solweig_wall_aspect")
    if host_work is not None:
        host_work()
    unresolved = torch.nonzero((mask & (aspect == 0)).flatten()).flatten()
    if unresolved.numel():
        host = dsm_host if dsm_host is not None else dsm_dev.cpu().numpy()
        fix = _gradient_aspect(host, pixel_size, unresolved.cpu().numpy())
        flat = aspect.view(-1)
        flat[unresolved] = flat[unresolved] + torch.from_numpy(fix).to(aspect.device)
    return aspect


def _gradient_aspect(dsm, pixel_size, flat_idx):
    """``-arctan2(fx, fy)`` in degrees at selected pixels, numpy.gradient semantics."""
    rows, cols = dsm.shape
    step = 1.0 / (1.0 / pixel_size)
    r, c = np.divmod(flat_idx, cols)

    def grad(axis_len, idx, get):
        out = np.empty(idx.size)
        if axis_len < 2:
            out[:] = 0.0
            return out
        inner = (idx > 0) & (idx < axis_len - 1)
        lo = idx == 0
        hi = idx == axis_len - 1
        out[inner] = (get(idx[inner] + 1, inner) - get(idx[inner] - 1, inner)) / (2. * step)
        out[lo] = (get(idx[lo] + 1, lo) - get(idx[lo], lo)) / step
        out[hi] = (get(idx[hi], hi) - get(idx[hi] - 1, hi)) / step
        return out

    fy = grad(rows, r, lambda ri, sel: np.asarray(dsm[ri, c[sel]], dtype=np.float64))
    fx = grad(cols, c, lambda ci, sel: np.asarray(dsm[r[sel], ci], dtype=np.float64))
    g = -np.arctan2(fx, fy)
    g[g < 0] += 2 * np.pi
    return 1 * (g / (math.pi / 180.0))


class Scene:
    """Static geometry and per-pixel statics of one tile, resident on the device."""

    def __init__(self, dsm, trees, dem, pixel_size=1.0, landcover=None, wall_threshold=3.0,
                 patch_option=2, device="cuda", walls=None, aspect=None, stream=None,
                 keep_planes=False):
        _require_cuda()
        self.device = torch.device(device)
        dev = self.device
        # Rasters go to the device in their own dtype and are widened there.
        dsm_in = _raster_to_device(dsm, dev)
        trees_in = _raster_to_device(trees, dev)
        dem_in = _raster_to_device(dem, dev)
        if dsm_in.dim() != 2 or dsm_in.shape != trees_in.shape or dsm_in.shape != dem_in.shape:
            raise ValueError("dsm, trees and dem must be 2-D arrays of the same shape")
        if landcover is not None and tuple(np.shape(landcover)) != tuple(dsm_in.shape):
            raise ValueError("landcover must have the raster's shape")
        self.shape = tuple(dsm_in.shape)
        self.rows, self.cols = self.shape
        self.pixels = self.rows * self.cols
        self.pixel_size = float(pixel_size)
        self.scale = 1 / self.pixel_size
        self.layout = SkyLayout(patch_option)
        self.patch_option = int(patch_option)
        L = _lib.lib()
        st = stream_handle(stream)
        n = self.pixels
        # Raise / clip semantics of src/series.py:252-291 (host syncs, so before
        # the wall kernels: the SVF rays are built on the host while they run).
        raise_dsm = max(0.0, -float(dsm_in.min()))
        raise_dem = max(0.0, -float(dem_in.min()))
        a_min, a_max = float(dsm_in.min()) + raise_dsm, float(dsm_in.max()) + raise_dsm
        t1_max = float(trees_in.clamp_min(0.).max())
        self.amaxvalue = float(max(a_max - a_min, t1_max))
        self.dsm_max = a_max
        self.hmax = float(a_max + max(t1_max, 0.0))
        svf_ray_tables = []

        def build_svf_rays():
            svf_ray_tables.append(rays.svf_rays(patch_option, self.shape, self.amaxvalue, self.scale))

        # Walls from the unraised DSM, rounded through float32 (src/series.py:213-236).
        if walls is None:
            walls_dev = wall_heights_device(dsm_in, wall_threshold, stream)
            aspect_dev = wall_aspect_device(dsm if isinstance(dsm, np.ndarray) else None, dsm_in, walls_dev,
                                            pixel_size, stream, host_work=build_svf_rays)
        else:
            walls_dev = _raster_to_device(walls, dev)
            aspect_dev = _raster_to_device(aspect, dev)
        self.walls = walls_dev.to(torch.float32).to(torch.float64)
        self._aspect_deg = aspect_dev.to(torch.float32).to(torch.float64)
        self.aspect = ((self._aspect_deg * math.pi) / 180.).contiguous()
        del walls_dev, aspect_dev
        lc_in = _raster_to_device(landcover, dev) if landcover is not None else None
        self.landcover = 1 if landcover is not None else 0
        f64 = dict(dtype=torch.float64, device=dev)
        f32 = dict(dtype=torch.float32, device=dev)
        self.dsm = torch.empty(self.shape, **f64)
        self.vegdem = torch.empty(self.shape, **f64)
        self.vegdem2 = torch.empty(self.shape, **f64)
        self.flags = torch.empty(self.shape, dtype=torch.uint8, device=dev)
        self.alb = torch.empty(self.shape, **f32)
        self.emis = torch.empty(self.shape, **f32)
        self.tgk = torch.empty(self.shape, **f32)
        self.tstart = torch.empty(self.shape, **f32)
        self.tmaxlst = torch.empty(self.shape, **f32)
        self.lc_grid = torch.empty(self.shape, **f32)
        classes = np.ascontiguousarray(LANDCOVER_CLASSES, dtype=np.float64)
        defaults = np.array([CONSTANTS["albedo_g"], CONSTANTS["eground"], 0.37, -3.41, 15.0])
        _lib.check(L.solweig_scene_build(
            device_ptr(dsm_in), device_ptr(trees_in), device_ptr(dem_in), device_ptr(lc_in), n,
            raise_dsm, raise_dem, classes.ctypes.data_as(ctypes.c_void_p), classes.shape[0],
            defaults.ctypes.data_as(ctypes.c_void_p), device_ptr(self.dsm), device_ptr(self.vegdem),
            device_ptr(self.vegdem2), device_ptr(self.flags), device_ptr(self.alb),
            device_ptr(self.emis), device_ptr(self.tgk), device_ptr(self.tstart),
            device_ptr(self.tmaxlst), device_ptr(self.lc_grid), st), "solweig_scene_build")
        if landcover is not None:
            wall_row = LANDCOVER_CLASSES[LANDCOVER_CLASSES[:, 0] == 99][0]
            self.tgk_wall, self.tstart_wall, self.tmaxlst_wall = (float(wall_row[3]),
                                                                  float(wall_row[4]),
                                                                  float(wall_row[5]))
        else:
            self.tgk_wall, self.tstart_wall, self.tmaxlst_wall = 0.37, -3.41, 15.
        del dsm_in, trees_in, dem_in, lc_in
        self.has_water = int(bool(((self.flags & 4) != 0).any().item())) if landcover is not None else 0
        # Sky view factor: bit-packed visibility + the 16 reduce planes.
        if not svf_ray_tables:
            build_svf_rays()
        dxdy, dz, lengths, cap = svf_ray_tables[0]
        self.svf_steps = int(lengths.sum())
        t_dxdy = _upload(dxdy, np.int32, dev)
        t_dz = _upload(dz, np.float64, dev)
        t_len = _upload(lengths, np.int32, dev)
        nb = self.layout.struct.nbands
        self.masks = torch.empty((2 * _lib.MASK_WORDS, self.rows, self.cols), dtype=torch.int32,
                                 device=dev)
        planes = torch.empty((16, self.rows, self.cols), **f64)
        self.veg_sums = torch.empty((4, self.rows, self.cols), **f32)
        self.sky_band_counts = torch.empty((nb, self.rows, self.cols), dtype=torch.uint8, device=dev)
        lay = self.layout
        self.geo32 = self._packed_geometry()
        self._geo_checked = True
        # GVF step offsets, uploaded before the SVF launch: nothing after it
        # waits for the device, so the host returns (and can plan the day)
        # while the SVF runs
        self.gvf_dxdy_host, self.first_steps, self.second_steps = rays.gvf_offsets(self.scale)
        self.gvf_dxdy = _upload(self.gvf_dxdy_host, np.int32, dev)
        self.gvf_host_ptr = self.gvf_dxdy_host.ctypes.data_as(ctypes.c_void_p)
        # ray ceilings and exit tables of one patch word (solweig_svf_ex2)
        svf_work = torch.empty(int(L.solweig_svf_work_bytes(self.rows, self.cols)), dtype=torch.uint8, device=dev)
        _lib.check(L.solweig_svf_ex2(
            device_ptr(self.dsm), device_ptr(self.vegdem), device_ptr(self.vegdem2), device_ptr(self.geo32),
            device_ptr(self.flags), self.rows, self.cols, lay.struct.patches, cap,
            device_ptr(t_dxdy), device_ptr(t_dz), device_ptr(t_len), self.hmax,
            ctypes.byref(lay.struct), lay.band_weights.ctypes.data_as(ctypes.c_void_p),
            lay.sectors.ctypes.data_as(ctypes.c_void_p), CONSTANTS["transVeg"],
            device_ptr(self.masks), device_ptr(planes), device_ptr(self.veg_sums),
            device_ptr(self.sky_band_counts), device_ptr(svf_work), svf_work.numel(), st), "solweig_svf")
        del t_dxdy, t_dz, t_len, svf_work
        # Derived statics after the float32 round trip of the SVF planes.
        self.svf32 = torch.empty((15, self.rows, self.cols), **f32)
        self.svfbuveg = torch.empty(self.shape, **f32)
        self.svfalfa = torch.empty(self.shape, **f64)
        self.tan_asvf = torch.empty(self.shape, **f64)
        self.gvf_face = torch.empty(self.shape, dtype=torch.int32, device=dev)
        lo, hi, mid = rays.gvf_face_windows()
        _lib.check(L.solweig_scene_finalize(
            device_ptr(planes), device_ptr(self.walls), device_ptr(self.aspect), n,
            CONSTANTS["transVeg"], lo.ctypes.data_as(ctypes.c_void_p),
            hi.ctypes.data_as(ctypes.c_void_p), mid.ctypes.data_as(ctypes.c_void_p),
            device_ptr(self.svf32), device_ptr(self.svfbuveg), device_ptr(self.svfalfa),
            device_ptr(self.tan_asvf), device_ptr(self.gvf_face), st), "solweig_scene_finalize")
        self.planes = planes if keep_planes else None
        self.struct = self._make_struct()
        self._gvf_statics(st)

    @classmethod
    def from_inputs(cls, inputs, device="cuda", stream=None):
        """Build a scene from the reference's prepared inputs (the ``static``
        dict of ``src/series.py:350-365`` handed to ``prepare_model``): DSM
        fields, walls/aspect, land-cover grids, the derived SVF fields and the
        three [rows, cols, P] visibility cubes."""
        _require_cuda()
        self = cls.__new__(cls)
        dev = torch.device(device)
        self.device = dev
        rows, cols = int(inputs["rows"]), int(inputs["cols"])
        self.shape = (rows, cols)
        self.rows, self.cols = rows, cols
        self.pixels = rows * cols
        self.scale = float(inputs["scale"])
        self.pixel_size = 1.0 / self.scale
        self.patch_option = int(inputs.get("patch_option", 2))
        self.layout = SkyLayout(self.patch_option)
        L = _lib.lib()
        st = stream_handle(stream)

        def f64(x):
            return _as_device(x, torch.float64, dev, self.shape)

        def f32(x):
            return _as_device(x, torch.float32, dev, self.shape)

        self.dsm = f64(inputs["dsm"])
        self.vegdem = f64(inputs["vegdem"])
        self.vegdem2 = f64(inputs["vegdem2"])
        self.walls = f64(inputs["walls"])
        dirwalls = f64(inputs["dirwalls"])
        self.aspect = (dirwalls * np.pi / 180.).contiguous()
        self._aspect_deg = dirwalls
        bush = f64(inputs["bush"])
        buildings = f64(inputs["buildings"])
        lc = f64(inputs.get("lc_grid", 0.0))
        self.flags = ((buildings == 1).to(torch.uint8) | ((bush > 1).to(torch.uint8) << 1)
                      | ((lc == 3).to(torch.uint8) << 2)).contiguous()
        self.landcover = int(inputs.get("landcover", 0))
        self.has_water = int(bool(((self.flags & 4) != 0).any().item())) if self.landcover else 0
        self.alb = f32(inputs["alb_grid"])
        self.emis = f32(inputs["emis_grid"])
        self.tgk = f32(inputs["TgK"])
        self.tstart = f32(inputs["Tstart"])
        self.tmaxlst = f32(inputs["TmaxLST"])
        self.lc_grid = f32(lc)
        self.tgk_wall = float(inputs["TgK_wall"])
        self.tstart_wall = float(inputs["Tstart_wall"])
        self.tmaxlst_wall = float(inputs["TmaxLST_wall"])
        self.amaxvalue = float(inputs["amaxvalue"])
        self.dsm_max = float(self.dsm.max().item())
        self.hmax = float(max(self.dsm_max, self.vegdem.max().item(), self.vegdem2.max().item()))
        self.svfbuveg = f32(inputs["svfbuveg"])
        self._svfbuveg64 = f64(inputs["svfbuveg"])
        self.svfalfa = f64(inputs["svfalfa"])
        self.tan_asvf = torch.tan(f64(inputs["asvf"])).contiguous()
        P = self.layout.struct.patches
        cubes = [_as_device(inputs[k], torch.float32, dev, self.shape + (P,))
                 for k in ("shmat", "vegshmat", "vbshvegshmat")]
        self.masks = torch.empty((2 * _lib.MASK_WORDS, rows, cols), dtype=torch.int32, device=dev)
        _lib.check(L.solweig_svf_pack(device_ptr(cubes[0]), device_ptr(cubes[1]), device_ptr(cubes[2]),
                                      self.pixels, P, device_ptr(self.masks), st), "solweig_svf_pack")
        nb = self.layout.struct.nbands
        planes = torch.empty((16, rows, cols), dtype=torch.float64, device=dev)
        self.veg_sums = torch.empty((4, rows, cols), dtype=torch.float32, device=dev)
        self.sky_band_counts = torch.empty((nb, rows, cols), dtype=torch.uint8, device=dev)
        lay = self.layout
        _lib.check(L.solweig_svf_reduce(
            device_ptr(self.masks), device_ptr(self.vegdem2), self.pixels, ctypes.byref(lay.struct),
            lay.band_weights.ctypes.data_as(ctypes.c_void_p), lay.sectors.ctypes.data_as(ctypes.c_void_p),
            CONSTANTS["transVeg"], device_ptr(planes), device_ptr(self.veg_sums),
            device_ptr(self.sky_band_counts), st), "solweig_svf_reduce")
        self.planes = None
        svf_names = cls.SVF_ORDER
        self.svf32 = torch.stack([f32(inputs[k]) for k in svf_names])
        # GVF wall-face bits (finalize computes them together with SVF-derived
        # fields; only the face bits are kept here, the fields come from inputs)
        scratch = {k: torch.empty(self.shape, dtype=t, device=dev) for k, t in
                   (("svfbuveg", torch.float32), ("svfalfa", torch.float64), ("tan", torch.float64))}
        self.gvf_face = torch.empty(self.shape, dtype=torch.int32, device=dev)
        lo, hi, mid = rays.gvf_face_windows()
        _lib.check(L.solweig_scene_finalize(
            device_ptr(planes), device_ptr(self.walls), device_ptr(self.aspect), self.pixels,
            CONSTANTS["transVeg"], lo.ctypes.data_as(ctypes.c_void_p), hi.ctypes.data_as(ctypes.c_void_p),
            mid.ctypes.data_as(ctypes.c_void_p), None, device_ptr(scratch["svfbuveg"]),
            device_ptr(scratch["svfalfa"]), device_ptr(scratch["tan"]), device_ptr(self.gvf_face), st),
            "solweig_scene_finalize")
        first, second = float(inputs.get("first", 1.0)), float(inputs.get("second", 22.0))
        self.gvf_dxdy_host, self.first_steps, self.second_steps = rays.gvf_offsets(self.scale, first, second)
        self.gvf_dxdy = _upload(self.gvf_dxdy_host, np.int32, dev)
        self.gvf_host_ptr = self.gvf_dxdy_host.ctypes.data_as(ctypes.c_void_p)
        self.struct = self._make_struct()
        self._gvf_statics(st)
        return self

    def _gvf_statics(self, st):
        """The hour-independent part of the batched day's GVF (walk length of
        every direction, albedo-without-shadow plane) for the 1 m walk of a
        scene without water, prepared once here (``solweig_gvf_statics``) so
        the days skip that walk; other scenes leave the pointers NULL."""
        self.gvf_hits = self.gvf_nosh = None
        if self.first_steps != 1 or self.second_steps != 22 or self.has_water:
            return
        dev = self.dsm.device
        self.gvf_hits = torch.empty((4,) + self.shape, dtype=torch.int32, device=dev)
        self.gvf_nosh = torch.empty(self.shape, dtype=torch.float32, device=dev)
        _lib.check(_lib.lib().solweig_gvf_statics(
            ctypes.byref(self.struct), self.gvf_host_ptr, self.first_steps, self.second_steps,
            device_ptr(self.gvf_hits), device_ptr(self.gvf_nosh), st), "solweig_gvf_statics")
        self.struct.gvf_hits = self.gvf_hits.data_ptr()
        self.struct.gvf_nosh = self.gvf_nosh.data_ptr()

    def _make_struct(self):
        s = _lib.SolweigScene()
        s.rows, s.cols, s.scale = self.rows, self.cols, self.scale
        for name in ("dsm", "vegdem", "vegdem2", "walls", "aspect", "flags", "alb", "emis", "tgk",
                     "tstart", "tmaxlst", "svfbuveg", "svfalfa", "tan_asvf", "masks", "veg_sums",
                     "sky_band_counts", "gvf_face"):
            setattr(s, name, getattr(self, name).data_ptr())
        s.svf_dir = None
        s.patches = self.layout.struct.patches
        s.nbands = self.layout.struct.nbands
        s.landcover = self.landcover
        s.has_water = self.has_water
        s.hmax = self.hmax
        if getattr(self, "geo32", None) is None and not getattr(self, "_geo_checked", False):
            self.geo32 = self._packed_geometry()
        self._geo_checked = True
        s.geo32 = self.geo32.data_ptr() if self.geo32 is not None else None
        return s

    def _packed_geometry(self):
        """(dsm, vegdem, vegdem2, 0) as float4 per pixel when all three rasters
        are exactly representable in float32 (the sweep then loads one sample
        per step); None otherwise."""
        stack = torch.stack((self.dsm, self.vegdem, self.vegdem2), dim=-1)
        packed = stack.to(torch.float32)
        if not bool(torch.equal(packed.to(torch.float64), stack)):
            return None
        geo = torch.zeros(self.shape + (4,), dtype=torch.float32, device=self.dsm.device)
        geo[..., :3] = packed
        return geo

    def svfbuveg64(self):
        """svf - (1 - svfveg)(1 - transVeg) in float64 from the float32-rounded
        SVF planes (``src/series.py:337-341``), for the float64 step."""
        t = getattr(self, "_svfbuveg64", None)
        if t is None:
            svf = self.svf32[self.SVF_ORDER.index("svf")].to(torch.float64)
            veg = self.svf32[self.SVF_ORDER.index("svfveg")].to(torch.float64)
            t = (svf - (1.0 - veg) * (1.0 - CONSTANTS["transVeg"])).contiguous()
            self._svfbuveg64 = t
        return t

    @property
    def walls_host(self):
        """Wall heights, float64 host array (float32-rounded values)."""
        return self.walls.cpu().numpy()

    @property
    def aspect_host(self):
        """Wall aspect in degrees, float64 host array (float32-rounded values)."""
        return self._aspect_deg.cpu().numpy()

    # The 15 SVF planes in the reference's svf_calculator order, float32-rounded.
    SVF_ORDER = ("svf", "svfE", "svfS", "svfW", "svfN", "svfveg", "svfEveg", "svfSveg", "svfWveg",
                 "svfNveg", "svfaveg", "svfEaveg", "svfSaveg", "svfWaveg", "svfNaveg")

    def svf_plane(self, name):
        return self.svf32[self.SVF_ORDER.index(name)]


def _leaf_psi(doy):
    first, last = CONSTANTS["firstdayleaf"], CONSTANTS["lastdayleaf"]
    if first > last:
        leaf = (doy > first) | (doy < last)
    else:
        leaf = (doy > first) & (doy < last)
    return 3. / 100. if leaf else .5


@dataclass
class HourScalars:
    """Host-side FP64 results of one hour that the step also returns."""
    ea: float
    esky: float
    I0: float
    CI: float
    radI: float
    radD: float
    CI_Tg: float
    CI_TgG: float
    Tgwall: float
    lv: object
    band_lsky: object = None  # float64 band sky emittances (the record holds float32)


def _ster_sin(L):
    """(steradian, sin(altitude)) of every patch as Python floats, cached per layout."""
    cached = getattr(L, "_ster_sin", None)
    if cached is None:
        cached = [(float(L.steradian[k]), float(np.sin(L.altitude[k] * (np.pi / 180))))
                  for k in range(L.count)]
        L._ster_sin = cached
    return cached


def hour_plan(scene, latitude, altitude, azimuth, zen, jday, dectime, altmax, ta, rh, rad_g, rad_d,
              rad_i, p_kpa, ws, psi, ci_prev, firstdaytime, timeadd, timestepdec, twater):
    """FP64 host scalars of one hour (``src/umep_solweig.py:122-232``).

    Returns ``(SolweigHour, ShadowRay or None, HourScalars, next_state)`` where
    next_state = (firstdaytime, timeadd, CI).
    """
    L = scene.layout.host
    h = _lib.SolweigHour()
    _, _, _, snup = _sun.daylen(jday, latitude)
    ea = 6.107 * 10 ** ((7.5 * ta) / (237.3 + ta)) * (rh / 100.)
    msteg = 46.5 * (ea / (ta + 273.15))
    esky = (1 - (1 + msteg) * np.exp(-((1.2 + 3.0 * msteg) ** 0.5))) + CONSTANTS["elvis"]
    day = altitude > 0
    CI = ci_prev
    ray = None
    lv = None
    I0 = 0
    CI_Tg = CI_TgG = None
    tgwall = 0.0
    if day:
        I0, CI, Kt, _, _ = _sun.clearness_index(zen, jday, ta, rh / 100., rad_g, latitude, p_kpa)
        if CI > 1 or CI == np.inf:
            CI = 1
        rad_i, rad_d = _sun.diffuse_fraction(rad_g, altitude, Kt, ta, rh)
        lv = _sky.perez(zen * (180 / np.pi), azimuth, rad_d, rad_i, jday, L)
        tgamp_wall = scene.tgk_wall * altmax + scene.tstart_wall
        frac = dectime - np.floor(dectime)
        tgwall = tgamp_wall * np.sin((((frac) - snup / 24) / (scene.tmaxlst_wall / 24 - snup / 24)) * np.pi / 2)
        if tgwall < 0:
            tgwall = 0
        radI0, radD0 = _sun.diffuse_fraction(I0, altitude, 1., ta, rh)
        corr = 0.1473 * np.log(90 - (zen / np.pi * 180)) + 0.3454
        CI_Tg = (rad_g / radI0) + (1 - corr)
        if CI_Tg > 1 or CI_Tg == np.inf:
            CI_Tg = 1
        radG0 = radI0 * (np.sin(altitude * (np.pi / 180))) + radD0
        CI_TgG = (rad_g / radG0) + (1 - corr)
        if CI_TgG > 1 or CI_TgG == np.inf:
            CI_TgG = 1
        tgwall = tgwall * CI_TgG
        ray = rays.shadow_ray(azimuth, altitude, scene.scale, scene.amaxvalue, scene.shape, True)
        # wave delay flags (all six TsWaveDelay calls share them)
        if timeadd >= (59 / 1440):
            weight = math.exp(-33.27 * timeadd)
            update = 1
            next_timeadd = timestepdec if timestepdec > (59 / 1440) else 0
        else:
            next_timeadd = timeadd + timestepdec
            weight = math.exp(-33.27 * next_timeadd)
            update = 0
        h.firstdaytime = int(firstdaytime)
        h.wave_update = update
        h.wave_weight = weight
        next_state = (0, next_timeadd, CI)
    else:
        CI_Tg = CI_TgG = CI
        next_state = (1, 0, CI)
    if CI < 0.95:
        esky = CI * esky + (1 - CI) * 1.
    h.daytime = int(day)
    h.altitude, h.azimuth, h.zen = altitude, azimuth, zen
    h.ta, h.rh, h.ws = ta, rh, ws
    h.rad_g, h.rad_d, h.rad_i = rad_g, rad_d, rad_i
    h.psi = psi
    h.cos_alt = np.cos(altitude * (np.pi / 180))
    h.sin_alt = np.sin(altitude * (np.pi / 180))
    h.tan_zen = np.tan(zen)
    h.esky = esky
    h.ci_tgg = CI_TgG if day else 0.0
    h.altmax = altmax
    h.dectime_frac = dectime - math.floor(dectime)
    h.snup = snup
    h.tgwall = tgwall
    h.twater = twater if twater is not None else 0.0
    if ray is not None:
        h.steps = ray.steps
        h.ray_low, h.ray_high, h.ray_middle = ray.low, ray.high, ray.middle
    # per-patch weights
    band_e = _sky.band_emissivity(esky, L)
    base = SBC * ((ta + 273.15) ** 4)
    band_lsky = np.zeros(L.band_counts.size)
    for b in range(L.band_counts.size):
        k = int(L.band_offsets[b])
        band_lsky[b] = (band_e[k] * base) / np.pi
        h.band_lsky[b] = band_lsky[b]
    if day:
        lum = lv[:, 2]
        # sequential float64 sum in patch order, as the reference loop
        ster_sin = _ster_sin(L)
        rad_tot = 0.0
        for lk, w in zip(lum.tolist(), ster_sin):
            rad_tot += lk * w[0] * w[1]
        h.rad_tot = rad_tot
        tan_alt = np.tan(altitude * (np.pi / 180))
        diff = np.abs(azimuth - L.azimuth)
        yi = 2 * np.cos(diff * (np.pi / 180)) * tan_alt
        P = L.count
        np.ctypeslib.as_array(h.lum)[:P] = lum.astype(np.float32)
        np.ctypeslib.as_array(h.yi)[:P] = np.where(yi > 0, 0.0, yi)
        np.ctypeslib.as_array(h.lw_sun_test)[:P] = ((diff > 90) & (diff < 270)).astype(np.uint8)
    else:
        h.rad_tot = 1.0
    coef = (ctypes.c_double * 7)()
    _lib.check(_lib.lib().solweig_utci_collapse(float(np.float32(ta)), float(np.float32(rh)),
                                                float(np.float32(ws)), coef), "solweig_utci_collapse")
    for i in range(7):
        h.utci[i] = coef[i]
    h.utci_valid = int(not (np.float32(ta) <= -999 or np.float32(rh) <= -999 or np.float32(ws) <= -999))
    scal = HourScalars(ea=ea, esky=esky, I0=I0, CI=CI, radI=rad_i, radD=rad_d, CI_Tg=CI_Tg,
                       CI_TgG=CI_TgG, Tgwall=tgwall, lv=lv, band_lsky=band_lsky)
    return h, ray, scal, next_state


STEP_OUTPUTS = ("tmrt", "utci", "kdown", "kup", "ldown", "lup", "shadow", "tg", "keast", "ksouth",
                "kwest", "knorth", "least", "lsouth", "lwest", "lnorth", "kside_i", "kside_d",
                "kside", "lside", "d_rad", "tg_out")


class HourBuffers:
    """Pinned host + device slots for H hour records and their sun rays."""

    def __init__(self, scene, hours=24):
        self.hours = hours
        self.kmax = max(scene.shape) + 2
        self.hsize = ctypes.sizeof(_lib.SolweigHour)
        dev = scene.device
        self.h_host = torch.empty(hours * self.hsize, dtype=torch.uint8, pin_memory=True)
        self.h_dev = torch.empty(hours * self.hsize, dtype=torch.uint8, device=dev)
        self.r_host = torch.empty((hours, self.kmax, 2), dtype=torch.int32, pin_memory=True)
        self.z_host = torch.empty((hours, self.kmax), dtype=torch.float64, pin_memory=True)
        self.r_dev = torch.zeros((hours, self.kmax, 2), dtype=torch.int32, device=dev)
        self.z_dev = torch.zeros((hours, self.kmax), dtype=torch.float64, device=dev)
        self.done = None

    def wait_free(self):
        if self.done is not None:
            self.done.synchronize()
            self.done = None

    def put(self, slot, hour, ray):
        """Write hour record ``slot`` (pointing at its device ray slot) into pinned memory."""
        if ray is not None and ray.steps:
            k = ray.steps
            if k > self.kmax:
                raise ValueError("sun ray longer than the ray buffer")
            self.r_host[slot, :k].numpy()[:] = ray.dxdy
            self.z_host[slot, :k].numpy()[:] = ray.dz
            hour.ray_dxdy = self.r_dev[slot].data_ptr()
            hour.ray_dz = self.z_dev[slot].data_ptr()
        raw = np.frombuffer(_lib.struct_bytes(hour), dtype=np.uint8)
        self.h_host.numpy()[slot * self.hsize:(slot + 1) * self.hsize] = raw

    def upload(self, first, count, steps):
        """Async copy of slots [first, first + count) to the device."""
        hs = self.hsize
        self.h_dev[first * hs:(first + count) * hs].copy_(self.h_host[first * hs:(first + count) * hs],
                                                          non_blocking=True)
        k = max(1, int(steps))
        self.r_dev[first:first + count, :k].copy_(self.r_host[first:first + count, :k], non_blocking=True)
        self.z_dev[first:first + count, :k].copy_(self.z_host[first:first + count, :k], non_blocking=True)

    def mark(self):
        self.done = torch.cuda.Event()
        self.done.record()

    def ptr(self):
        return ctypes.c_void_p(self.h_dev.data_ptr())


def plan_hours(scene, met, latitude, longitude, site_altitude, utc):
    """FP64 host plan of the rows of one day, yielded row by row as
    (SolweigHour, ShadowRay|None, HourScalars): the sun positions of all rows
    first, then each row's scalars (the clearness index and the wave-delay
    clock carry from row to row)."""
    met = np.asarray(met, dtype=np.float64)
    sol = _sun.metdata(met, latitude, longitude, site_altitude, utc)
    dectime = sol.dectime
    timestepdec = (dectime[1] - dectime[0]) if len(met) > 1 else 1 / 24.
    twater = float(np.mean(met[:, 11])) if scene.landcover else None
    firstdaytime, timeadd, CI = 1, 0.0, 1.0
    for i in range(len(met)):
        if dectime[i] - np.floor(dectime[i]) == 0:
            CI = 1.
        psi = _leaf_psi(met[i, 1])
        h, ray, scal, (firstdaytime, timeadd, CI) = hour_plan(
            scene, latitude, sol.altitude[i], sol.azimuth[i], sol.zen[i], sol.jday[i], dectime[i],
            sol.altmax[i], met[i, 11], met[i, 10], met[i, 14], met[i, 21], met[i, 22], met[i, 12],
            met[i, 9], psi, CI, firstdaytime, timeadd, timestepdec, twater)
        yield h, ray, scal


def plan_day(scene, met, latitude, longitude, site_altitude, utc):
    """FP64 host plan of every row of one day: [(SolweigHour, ShadowRay|None, HourScalars)]."""
    return list(plan_hours(scene, met, latitude, longitude, site_altitude, utc))


def outputs_struct(outputs, index=None):
    out = _lib.SolweigOutputs()
    for k, t in outputs.items():
        setattr(out, k, (t[index] if index is not None else t).data_ptr())
    return out


class DayRunner:
    """Plain form: one host plan, one hour-record upload and one kernel pair
    per hour, launched as the hours are planned (the host plans hour h+1
    while the GPU runs hour h)."""

    def __init__(self, scene, latitude, longitude, site_altitude=3.0, utc=0.0):
        self.scene = scene
        self.latitude, self.longitude, self.site_altitude, self.utc = latitude, longitude, site_altitude, utc
        dev = scene.device
        self.state = {k: torch.zeros(scene.shape, dtype=torch.float32, device=dev)
                      for k in _lib.STATE_FIELDS}
        self.scratch = torch.empty((_lib.SCRATCH_PLANES, scene.rows, scene.cols), dtype=torch.float32,
                                   device=dev)
        self.buffers = HourBuffers(scene, 24)
        self.layout_dev = scene.layout.device(dev)
        self.gvf_tile_rows = 8

    def state_struct(self):
        s = _lib.SolweigState()
        for k in _lib.STATE_FIELDS:
            setattr(s, k, self.state[k].data_ptr())
        return s

    def reset_state(self):
        for t in self.state.values():
            t.zero_()

    def _launch(self, slot, out_struct, stream=None):
        sc = self.scene
        _lib.check(_lib.lib().solweig_step(
            ctypes.byref(sc.struct), device_ptr(self.layout_dev), self.buffers.ptr(), slot,
            ctypes.byref(self.state_struct()), ctypes.byref(out_struct), sc.gvf_host_ptr,
            sc.first_steps, sc.second_steps, device_ptr(self.scratch), stream_handle(stream)),
            "solweig_step")

    def _alloc_outputs(self, outputs, nrows):
        return {k: torch.empty((nrows,) + self.scene.shape, dtype=torch.float32, device=self.scene.device)
                for k in outputs}

    def _put(self, slot, hour, ray, scal):
        """Stage hour record ``slot`` and copy it to the device."""
        self.buffers.put(slot, hour, ray)
        self.buffers.upload(slot, 1, ray.steps if ray is not None else 1)

    def _outputs_struct(self, res, index):
        return outputs_struct(res, index)

    def run_day(self, met, outputs=("tmrt", "utci"), stream=None):
        """Run the rows of one calendar day; returns {name: tensor [H, rows, cols]}."""
        met = np.asarray(met, dtype=np.float64)
        if len(met) > self.buffers.hours:
            raise ValueError(f"at most {self.buffers.hours} rows per day")
        sol = _sun.metdata(met, self.latitude, self.longitude, self.site_altitude, self.utc)
        dectime = sol.dectime
        timestepdec = (dectime[1] - dectime[0]) if len(met) > 1 else 1 / 24.
        twater = float(np.mean(met[:, 11])) if self.scene.landcover else None
        res = self._alloc_outputs(outputs, len(met))
        self.buffers.wait_free()
        self.reset_state()
        firstdaytime, timeadd, CI = 1, 0.0, 1.0
        scalars = []
        for i in range(len(met)):
            if dectime[i] - np.floor(dectime[i]) == 0:
                CI = 1.
            psi = _leaf_psi(met[i, 1])
            h, ray, scal, (firstdaytime, timeadd, CI) = hour_plan(
                self.scene, self.latitude, sol.altitude[i], sol.azimuth[i], sol.zen[i], sol.jday[i],
                dectime[i], sol.altmax[i], met[i, 11], met[i, 10], met[i, 14], met[i, 21],
                met[i, 22], met[i, 12], met[i, 9], psi, CI, firstdaytime, timeadd, timestepdec,
                twater)
            self._put(i, h, ray, scal)
            self._launch(i, self._outputs_struct(res, i), stream)
            scalars.append(scal)
        self.buffers.mark()
        self.last_scalars = scalars
        return res

    def profile_day(self, met):
        """Per-kernel device time of one day: {kernel: {ms, launches, bytes_per_launch}}."""
        sc = self.scene
        plan = plan_day(sc, met, self.latitude, self.longitude, self.site_altitude, self.utc)
        self.buffers.wait_free()
        for i, (h, ray, _) in enumerate(plan):
            self.buffers.put(i, h, ray)
        self.buffers.upload(0, len(plan), self.buffers.kmax)
        self.reset_state()
        out = {k: torch.empty(sc.shape, dtype=torch.float32, device=sc.device) for k in ("tmrt", "utci")}
        o = outputs_struct(out)
        st = self.state_struct()
        L = _lib.lib()
        names = ("step_shadow_kernel", "step_gvf_kernel", "step_radiation_kernel")
        times = {k: [] for k in names}
        for i, (h, ray, _) in enumerate(plan):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            ev[0].record()
            if h.daytime:
                _lib.check(L.solweig_step_shadow(ctypes.byref(sc.struct), self.buffers.ptr(), i,
                                                 device_ptr(self.scratch), stream_handle()), "shadow")
            ev[1].record()
            if h.daytime:
                _lib.check(L.solweig_step_gvf(ctypes.byref(sc.struct), self.buffers.ptr(), i,
                                              sc.gvf_host_ptr, sc.first_steps, sc.second_steps,
                                              device_ptr(self.scratch), self.gvf_tile_rows,
                                              stream_handle()), "gvf")
            ev[2].record()
            _lib.check(L.solweig_step_radiation(
                ctypes.byref(sc.struct), device_ptr(self.layout_dev), self.buffers.ptr(), i,
                ctypes.byref(st), ctypes.byref(o), device_ptr(self.scratch), stream_handle()),
                "radiation")
            ev[3].record()
            times["step_shadow_kernel"].append((ev, 0, 1, bool(h.daytime)))
            times["step_gvf_kernel"].append((ev, 1, 2, bool(h.daytime)))
            times["step_radiation_kernel"].append((ev, 2, 3, True))
        self.buffers.mark()
        torch.cuda.synchronize()
        n = sc.pixels
        bytes_per = {"step_shadow_kernel": n * SHADOW_BYTES_PER_PIXEL,
                     "step_gvf_kernel": n * GVF_BYTES_PER_PIXEL,
                     "step_radiation_kernel": n * RADIATION_BYTES_PER_PIXEL}
        res = {}
        for k, lst in times.items():
            ms = sum(e[a].elapsed_time(e[b]) for e, a, b, used in lst if used)
            launches = sum(1 for *_, used in lst if used)
            res[k] = {"ms": ms, "launches": launches, "bytes_per_launch": bytes_per[k]}
        return res


# Algorithmic HBM bytes per pixel and launch (each input and output once):
# shadow: own dsm/vegdem/vegdem2/walls/aspect (40) + flags (1) + tgk/tstart/tmaxlst/emis/alb (20)
#         + quad written (16);
# gvf: quad (16) + wall-face bits (4) + emissivity (4) + 15 planes written (60);
# radiation: shadow from the quad (4) + 15 GVF planes (60) + flags (1) + emis/tgk/tstart/tmaxlst
#         (16) + svfbuveg (4) + svfalfa and tan(asvf) (16) + masks (40) + vegetation/obstruction
#         sums (16) + sky band counts (8) + thermal state read+write (48) + Tmrt and UTCI (8).
SHADOW_BYTES_PER_PIXEL = 77
GVF_BYTES_PER_PIXEL = 84
RADIATION_BYTES_PER_PIXEL = 221


def hour64_record(scene, hour, scal):
    """The float64 per-patch weights of one hour (``SolweigHour64``): the Perez
    luminances (daytime) and the band sky emittances of ``hour_plan``."""
    h64 = _lib.SolweigHour64()
    if hour.daytime:
        np.ctypeslib.as_array(h64.lum)[:scene.layout.host.count] = scal.lv[:, 2]
    np.ctypeslib.as_array(h64.band_lsky)[:len(scal.band_lsky)] = scal.band_lsky
    return h64


class DayRunner64(DayRunner):
    """Plain form with float64 radiation, the reference's ``dtype=float64``
    (``run.py:27``, ``src/runtime.py:43-49``): one ``solweig_step64`` per hour
    (shadow fields, ground view factors and radiation in float64), float64
    thermal state and output planes; UTCI stays float32."""

    def __init__(self, scene, latitude, longitude, site_altitude=3.0, utc=0.0, hours=24):
        self.scene = scene
        self.latitude, self.longitude, self.site_altitude, self.utc = latitude, longitude, site_altitude, utc
        dev = scene.device
        self.state = {k: torch.zeros(scene.shape, dtype=torch.float64, device=dev)
                      for k in _lib.STATE_FIELDS}
        self.scratch = torch.empty((_lib.SCRATCH64_PLANES, scene.rows, scene.cols), dtype=torch.float64,
                                   device=dev)
        slots = max(24, int(hours))
        self.buffers = HourBuffers(scene, slots)
        self.h64size = ctypes.sizeof(_lib.SolweigHour64)
        self.h64_host = torch.empty(slots * self.h64size, dtype=torch.uint8, pin_memory=True)
        self.h64_dev = torch.empty(slots * self.h64size, dtype=torch.uint8, device=dev)
        self.layout_dev = scene.layout.device(dev)
        self.sky64_dev = scene.layout.device64(dev)
        self.svfbuveg = scene.svfbuveg64()

    def state_struct(self):
        s = _lib.SolweigState64()
        for k in _lib.STATE_FIELDS:
            setattr(s, k, self.state[k].data_ptr())
        return s

    def _alloc_outputs(self, outputs, nrows):
        return {k: torch.empty((nrows,) + self.scene.shape,
                               dtype=torch.float32 if k == "utci" else torch.float64, device=self.scene.device)
                for k in outputs}

    def _outputs_struct(self, res, index):
        out = _lib.SolweigOutputs64()
        for k, t in res.items():
            setattr(out, k, (t[index] if index is not None else t).data_ptr())
        return out

    def _put(self, slot, hour, ray, scal):
        super()._put(slot, hour, ray, scal)
        n = self.h64size
        raw = np.frombuffer(_lib.struct_bytes(hour64_record(self.scene, hour, scal)), dtype=np.uint8)
        self.h64_host.numpy()[slot * n:(slot + 1) * n] = raw
        self.h64_dev[slot * n:(slot + 1) * n].copy_(self.h64_host[slot * n:(slot + 1) * n], non_blocking=True)

    def _launch(self, slot, out_struct, stream=None):
        sc = self.scene
        _lib.check(_lib.lib().solweig_step64(
            ctypes.byref(sc.struct), device_ptr(self.svfbuveg), device_ptr(self.layout_dev),
            device_ptr(self.sky64_dev), self.buffers.ptr(), device_ptr(self.h64_dev), slot,
            ctypes.byref(self.state_struct()), ctypes.byref(out_struct), sc.gvf_host_ptr,
            sc.first_steps, sc.second_steps, device_ptr(self.scratch), stream_handle(stream)),
            "solweig_step64")

    def profile_day(self, met):
        raise NotImplementedError("profile_day times the float32 kernels; time a DayRunner64 day with events")
