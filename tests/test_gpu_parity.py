"""GPU parity of each CUDA stage against the float64 oracle on seeded scenes.

Bars: shadow and wall masks bit-exact; SVF planes within 1e-12 (float64
annulus sums in the same band order) and masks identical; GVF within float32
rounding; Tmrt within 0.1 K and UTCI within 0.05 K over a full day.
"""
import numpy as np
import pytest

from conftest import small_scene

pytestmark = pytest.mark.gpu


def _vegetation(a, t1):
    vegdsm = t1 + a
    vegdsm[vegdsm == a] = 0
    vegdsm2 = t1 * 0.25 + a
    vegdsm2[vegdsm2 == a] = 0
    bush = np.logical_not(vegdsm2 * vegdsm) * vegdsm
    return vegdsm, vegdsm2, bush


@pytest.fixture(scope="module")
def scene48(cuda):
    from solweig_cuda_b200 import engine
    sc = small_scene(48, seed=3)
    return sc, engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover, keep_planes=True)


def test_walls_match_oracle(scene48):
    from oracle import geometry as G
    sc, scene = scene48
    a = sc.dsm.astype(np.float64)
    walls = G.wall_heights(a, 3.0)
    aspect = G.wall_aspect(walls, a, 1.0)
    assert np.array_equal(scene.walls_host, walls.astype(np.float32).astype(np.float64))
    assert np.array_equal(scene.aspect_host, aspect.astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("azi,alt", [(45., 30.), (100.3, 12.5), (180., 58.8), (200., 6.),
                                     (271.7, 3.2), (350., 20.), (90., 45.), (315., 60.)])
def test_shadow_planes_bit_exact(scene48, azi, alt):
    import torch
    from oracle import geometry as G
    from solweig_cuda_b200 import ops
    sc, scene = scene48
    a = sc.dsm.astype(np.float64)
    t1 = sc.trees.astype(np.float64)
    vegdsm, vegdsm2, bush = _vegetation(a, t1)
    want = G.shadow_sweep(a, vegdsm, vegdsm2, azi, alt, 1.0, scene.amaxvalue, bush,
                          scene.walls_host, scene.aspect_host * np.pi / 180.)
    got = ops.cast_shadow(scene, azi, alt).cpu().numpy()
    for i in range(8):
        assert np.array_equal(got[i], np.asarray(want[i], dtype=np.float64)), f"plane {i}"


def test_svf_masks_and_planes(scene48):
    from oracle import geometry as G
    from solweig_cuda_b200 import ops
    sc, scene = scene48
    a = sc.dsm.astype(np.float64)
    t1 = sc.trees.astype(np.float64)
    vegdsm, vegdsm2, bush = _vegetation(a, t1)
    shm, vegm, vbm = G.svf_patch_masks(a, vegdsm, vegdsm2, bush, 1.0, scene.amaxvalue, 2)
    red = G.svf_reduce(shm, vegm, vbm, vegdsm2)
    cubes = ops.unpack_masks(scene)
    assert np.array_equal(cubes[0].cpu().numpy(), shm)
    assert np.array_equal(cubes[1].cpu().numpy(), vegm)
    assert np.array_equal(cubes[2].cpu().numpy(), vbm)
    planes = scene.planes.cpu().numpy()
    for i in range(16):
        assert np.max(np.abs(planes[i] - red[i])) < 1e-12, f"plane {i}"


def test_day_tmrt_utci(scene48):
    from oracle import step as ST
    from solweig_cuda_b200 import engine, synthetic
    sc, scene = scene48
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    loc = dict(latitude=53.0, longitude=0.0, altitude=3.0)
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    want = ST.run_day(s, met, loc, 0.0, outputs=("Tmrt", "UTCI"))
    runner = engine.DayRunner(scene, 53.0, 0.0, 3.0, 0.0)
    got = runner.run_day(met, outputs=("tmrt", "utci"))
    tm = got["tmrt"].cpu().numpy()
    ut = got["utci"].cpu().numpy()
    for h in range(24):
        d_t = np.max(np.abs(tm[h] - want[h]["Tmrt"]))
        ok = ~np.isnan(want[h]["UTCI"])
        d_u = np.max(np.abs(ut[h][ok] - want[h]["UTCI"][ok]))
        assert d_t <= 0.1, f"hour {h}: Tmrt error {d_t}"
        assert d_u <= 0.05, f"hour {h}: UTCI error {d_u}"
        assert np.array_equal(np.isnan(ut[h]), ~ok)


def test_batched_graph_matches_plain_and_replays(scene48):
    """The graph-captured day equals the plain per-hour loop bit for bit, and a
    second replay with another day's forcing still matches the oracle."""
    import torch
    from oracle import step as ST
    from solweig_cuda_b200 import batched, engine, synthetic
    sc, scene = scene48
    loc = dict(latitude=53.0, longitude=0.0, altitude=3.0)
    plain = engine.DayRunner(scene, 53.0, 0.0, 3.0, 0.0)
    day = batched.BatchedDay(scene, 53.0, 0.0, 3.0, 0.0)
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    for doy, seed in ((172, 0), (200, 5)):
        met = synthetic.make_met(doy=doy, latitude=53.0, longitude=0.0, seed=seed)
        a = {k: v.clone() for k, v in plain.run_day(met).items()}
        b = day.run_day(met)
        torch.cuda.synchronize()
        assert torch.equal(a["tmrt"], b["tmrt"])
        assert torch.equal(torch.nan_to_num(a["utci"], nan=-1e9), torch.nan_to_num(b["utci"], nan=-1e9))
        want = ST.run_day(s, met, loc, 0.0)
        tm = b["tmrt"].cpu().numpy()
        for h in range(24):
            assert np.max(np.abs(tm[h] - want[h]["Tmrt"])) <= 0.1, (doy, h)


@pytest.mark.parametrize("tile_rows", [4, 8, 16])
def test_step_gvf_planes_match_oracle(cuda, tile_rows):
    """The hourly GVF kernel (interior fast path and border path) against the
    oracle's gvf_2018a restatement for the same shadow and surface temperature."""
    import ctypes
    import torch
    from oracle import geometry as G, ground as GR
    from solweig_cuda_b200 import _lib, engine, synthetic
    from solweig_cuda_b200.engine import device_ptr, stream_handle
    sc = synthetic.make_scene(100, seed=9)
    scene = engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    runner = engine.DayRunner(scene, 53.0, 0.0, 3.0, 0.0)
    runner.gvf_tile_rows = tile_rows
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    plan = engine.plan_day(scene, met, 53.0, 0.0, 3.0, 0.0)
    i = 13
    h, ray, scal = plan[i]
    runner.buffers.put(0, h, ray)
    runner.buffers.upload(0, 1, runner.buffers.kmax)
    L = _lib.lib()
    _lib.check(L.solweig_step_shadow(ctypes.byref(scene.struct), runner.buffers.ptr(), 0,
                                     device_ptr(runner.scratch), stream_handle()), "shadow")
    _lib.check(L.solweig_step_gvf(ctypes.byref(scene.struct), runner.buffers.ptr(), 0,
                                  scene.gvf_host_ptr, scene.first_steps, scene.second_steps,
                                  device_ptr(runner.scratch), tile_rows, stream_handle()), "gvf")
    torch.cuda.synchronize()
    got = runner.scratch[5:20].cpu().numpy()
    n = scene.pixels
    quad = runner.scratch.reshape(-1)[:4 * n].reshape(scene.rows, scene.cols, 4).permute(2, 0, 1).cpu().numpy()
    # oracle with the GPU's own shadow value (float32) and the oracle's Tg
    s = __import__("oracle.step", fromlist=["prepare_static"]).prepare_static(
        sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover,
        walls=scene.walls_host, aspect=scene.aspect_host,
        svf=None)
    a = s["dsm"]
    vegsh, sh, _, wallsh, wallsun, wallshve, _, _ = G.shadow_sweep(
        a, s["vegdem"], s["vegdem2"], h.azimuth, h.altitude, 1.0, s["amaxvalue"], s["bush"],
        s["walls"], s["dirwalls"] * np.pi / 180.)
    shadow = sh - (1 - vegsh) * (1 - h.psi)
    assert np.max(np.abs(quad[0] - shadow)) < 1e-6
    frac = h.dectime_frac
    Tg = (s["TgK"] * h.altmax + s["Tstart"]) * np.sin(((frac - h.snup / 24) / (s["TmaxLST"] / 24 - h.snup / 24)) * np.pi / 2)
    Tg = Tg * h.ci_tgg
    Tg[Tg < 0] = 0
    planes, _ = GR.gvf(wallsun, s["walls"], s["buildings"], 1.0, shadow, 1.0, 22.0, s["dirwalls"], Tg,
                       h.tgwall, h.ta, s["emis_grid"], 0.9, s["alb_grid"], 5.67051e-8, 0.2)
    order = [0, 3, 6, 9, 12, 1, 4, 7, 10, 13, 2, 5, 8, 11, 14]
    for k, j in enumerate(order):
        err = np.max(np.abs(got[k] - planes[j]) / (np.abs(planes[j]) + 1.0))
        assert err < 2e-5, (k, err)


@pytest.mark.parametrize("packed", [True, False])
def test_svf_ray_ceilings_are_bit_identical(cuda, packed):
    """solweig_svf_ex2 (ray ceilings + exit tables, one launch per patch word)
    against solweig_svf_ex (every ray walked to its clearance): identical
    masks, planes and band counts on a 150 x 134 city, packed and float64
    geometry."""
    import ctypes
    import torch
    from solweig_cuda_b200 import _lib, engine, rays, synthetic
    from solweig_cuda_b200.engine import device_ptr, stream_handle
    s = synthetic.make_scene(150, 134, seed=11)
    scene = engine.Scene(s.dsm, s.trees, s.dem, 1.0, landcover=s.landcover)
    L = _lib.lib()
    dxdy, dz, lengths, cap = rays.svf_rays(2, scene.shape, scene.amaxvalue, scene.scale)
    t_dxdy = torch.from_numpy(np.ascontiguousarray(dxdy, dtype=np.int32)).to(cuda)
    t_dz = torch.from_numpy(np.ascontiguousarray(dz, dtype=np.float64)).to(cuda)
    t_len = torch.from_numpy(np.ascontiguousarray(lengths, dtype=np.int32)).to(cuda)
    lay = scene.layout
    nb = lay.struct.nbands
    geo = scene.geo32 if packed else None
    if packed:
        assert geo is not None
    out = {}
    for ex2 in (False, True):
        masks = torch.zeros((2 * _lib.MASK_WORDS, scene.rows, scene.cols), dtype=torch.int32, device=cuda)
        planes = torch.zeros((16, scene.rows, scene.cols), dtype=torch.float64, device=cuda)
        veg = torch.zeros((4, scene.rows, scene.cols), dtype=torch.float32, device=cuda)
        cnt = torch.zeros((nb, scene.rows, scene.cols), dtype=torch.uint8, device=cuda)
        args = [device_ptr(scene.dsm), device_ptr(scene.vegdem), device_ptr(scene.vegdem2), device_ptr(geo),
                device_ptr(scene.flags), scene.rows, scene.cols, lay.struct.patches, cap, device_ptr(t_dxdy),
                device_ptr(t_dz), device_ptr(t_len), scene.hmax, ctypes.byref(lay.struct),
                lay.band_weights.ctypes.data_as(ctypes.c_void_p), lay.sectors.ctypes.data_as(ctypes.c_void_p),
                0.03, device_ptr(masks), device_ptr(planes), device_ptr(veg), device_ptr(cnt)]
        if ex2:
            work = torch.empty(int(L.solweig_svf_work_bytes(scene.rows, scene.cols)), dtype=torch.uint8,
                               device=cuda)
            _lib.check(L.solweig_svf_ex2(*args, device_ptr(work), work.numel(), stream_handle()), "svf_ex2")
        else:
            _lib.check(L.solweig_svf_ex(*args, stream_handle()), "svf_ex")
        torch.cuda.synchronize()
        out[ex2] = (masks, planes, veg, cnt)
    for a, b in zip(out[False], out[True]):
        assert torch.equal(a.view(torch.uint8), b.view(torch.uint8))
    assert torch.equal(out[True][0], scene.masks)
