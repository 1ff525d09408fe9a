"""The batched form (``solweig_day_batched``): the BF16 tensor-core patch
contraction against an FP64 reference of the same sums, and whole days
against the oracle and the per-hour form."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# Patch sums: BF16 hi + lo weights carry ~16 significant bits, FP32 accumulation.
SUM_RTOL = 2e-5
TMRT_TOL = 0.1    # K, against the oracle (UMEP restatement)
UTCI_TOL = 0.05   # K
FORM_TOL = 0.02   # K, batched vs per-hour form


def _sums_reference(S, V, P, W):
    """FP64 sums of W over the sky (S & ~V) and vegetation (S & V) patches."""
    px = S.shape[1]
    bits = np.zeros((px, 160), dtype=np.float64)
    vbits = np.zeros((px, 160), dtype=np.float64)
    for w in range(5):
        for b in range(32):
            k = 32 * w + b
            if k >= P:
                continue
            s = (S[w] >> b) & 1
            v = (V[w] >> b) & 1
            bits[:, k] = s & (1 - v)
            vbits[:, k] = s & v
    return bits @ W.T.astype(np.float64), vbits @ W.T.astype(np.float64)


@pytest.mark.parametrize("px,ncols", [(128 * 37, 48), (1000, 16), (5 * 128 + 77, 96)])
def test_patch_sums_match_fp64(cuda, px, ncols):
    import torch
    from solweig_cuda_b200 import _lib
    from solweig_cuda_b200.engine import device_ptr, stream_handle
    rng = np.random.default_rng(px + ncols)
    P = 153
    words = rng.integers(0, 2**32, size=(10, px), dtype=np.uint64).astype(np.uint32)
    W = rng.uniform(0.0, 0.02, size=(ncols, 160)).astype(np.float32)
    W[:, P:] = 0
    masks = torch.from_numpy(words.view(np.int32)).to(cuda)
    wt = torch.from_numpy(W).to(cuda)
    out = torch.full((2 * ncols, px), np.nan, dtype=torch.float32, device=cuda)
    nb = (ncols + 15) // 16 * 16
    work = torch.empty(4 * nb * 160 + 16, dtype=torch.uint8, device=cuda)
    L = _lib.lib()
    _lib.check(L.solweig_patch_sums(device_ptr(masks), px, P, device_ptr(wt), ncols, device_ptr(out),
                                    device_ptr(work), work.numel(), stream_handle()), "solweig_patch_sums")
    torch.cuda.synchronize()
    err = int(work[4 * nb * 160:4 * nb * 160 + 4].view(torch.int32).item())
    assert err == 0
    got = out.cpu().numpy().astype(np.float64)
    sky, veg = _sums_reference(words[:5].astype(np.int64), words[5:].astype(np.int64), P, W)
    scale = np.abs(W).sum(axis=1)[None, :]  # bound of every sum
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got[:ncols].T - sky) / scale) < SUM_RTOL
    assert np.max(np.abs(got[ncols:].T - veg) / scale) < SUM_RTOL


def test_day_patch_sums_match_fp64(cuda):
    """The batched day's contraction (pipelined tcgen05 kernel: two operand
    stages, two tensor-memory accumulators, several tiles per CTA and a
    partial last tile) against FP64 sums of the same masks and the day's
    FP64 weights: sky + 0.03 x vegetation, every pixel and hour."""
    import torch
    from solweig_cuda_b200 import batched, engine, synthetic
    sc = synthetic.make_scene(300, 260, seed=9)
    scene = engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0, seed=1)
    day = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0)
    day.run_day(met)
    torch.cuda.synchronize()
    assert day.error_flag() == 0
    sums = day.patch_sums().to(torch.float64)
    L = scene.layout.host
    P = L.count
    words = scene.masks.view(torch.int32).view(10, -1).to(torch.int64) & 0xFFFFFFFF
    bit = torch.arange(P, device=words.device)
    Sb = (words[bit // 32] >> (bit % 32)[:, None]) & 1
    Vb = (words[5 + bit // 32] >> (bit % 32)[:, None]) & 1
    sky = (Sb * (1 - Vb)).to(torch.float64).T
    veg = (Sb * Vb).to(torch.float64).T
    W = np.zeros((2 * 24, P))
    for h, s_ in enumerate(day.last_scalars):
        if s_.lv is not None:
            lum = s_.lv[:, 2]
            W[2 * h] = lum
            W[2 * h + 1] = lum * L.cos_alt * L.steradian
    Wt = torch.from_numpy(W).to(words.device)
    want = sky @ Wt.T + 0.03 * (veg @ Wt.T)
    scale = Wt.abs().sum(dim=1).clamp_min(1e-30)
    assert torch.isfinite(sums).all()
    assert ((sums.T - want).abs() / scale).max().item() < SUM_RTOL


@pytest.fixture(scope="module")
def scene64():
    from solweig_cuda_b200 import engine, synthetic
    sc = synthetic.make_scene(64, 56, seed=4)
    return sc, engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)


def test_chosen_day_matches_oracle_and_plain(scene64):
    import torch
    from oracle import step as ST
    from solweig_cuda_b200 import batched, engine, synthetic
    sc, scene = scene64
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    outs = ("tmrt", "utci", "kdown", "ldown", "lup", "kup", "kside", "lside")
    chosen = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0, outputs=outs)
    got = {k: v.clone() for k, v in chosen.run_day(met).items()}
    torch.cuda.synchronize()
    assert chosen.error_flag() == 0
    plain = engine.DayRunner(scene, 53.0, 0.0, 3.0, 0.0)
    ref = plain.run_day(met, outputs=outs)
    for k in outs:
        a = got[k].cpu().numpy()
        b = ref[k].cpu().numpy()
        assert np.array_equal(np.isnan(a), np.isnan(b)), k
        tol = FORM_TOL if k in ("tmrt", "utci") else 0.05  # W/m2 for the fluxes
        d = np.nanmax(np.abs(a - b))
        assert d <= tol, (k, d)
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    want = ST.run_day(s, met, dict(latitude=53.0, longitude=0.0, altitude=3.0), 0.0, outputs=("Tmrt", "UTCI"))
    tm = got["tmrt"].cpu().numpy()
    ut = got["utci"].cpu().numpy()
    for h in range(24):
        assert np.max(np.abs(tm[h] - want[h]["Tmrt"])) <= TMRT_TOL, h
        ok = ~np.isnan(want[h]["UTCI"])
        assert np.max(np.abs(ut[h][ok] - want[h]["UTCI"][ok])) <= UTCI_TOL, h


def test_chosen_day_graph_replays_new_forcing(scene64):
    import torch
    from solweig_cuda_b200 import batched, engine, synthetic
    sc, scene = scene64
    chosen = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0)
    plain = engine.DayRunner(scene, 53.0, 0.0, 3.0, 0.0)
    for doy, seed in ((172, 0), (200, 5), (350, 2)):
        met = synthetic.make_met(doy=doy, latitude=53.0, longitude=0.0, seed=seed)
        b = {k: v.clone() for k, v in chosen.run_day(met).items()}
        a = plain.run_day(met)
        torch.cuda.synchronize()
        d = torch.max(torch.abs(a["tmrt"] - b["tmrt"])).item()
        assert d <= FORM_TOL, (doy, d)
    assert chosen.error_flag() == 0


def test_multiday_graph_equals_day_by_day(scene64):
    """Two days in one captured graph equal the single-day batched form."""
    import torch
    from solweig_cuda_b200 import batched, synthetic
    sc, scene = scene64
    met = synthetic.make_met(doy=180, latitude=53.0, longitude=0.0, days=2, seed=3)
    md = batched.MultiDay(scene, 53.0, 0.0, 3.0, 0.0, days=2)
    out = {k: v.clone() for k, v in md.run(met).items()}
    one = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0)
    for d in range(2):
        ref = one.run_day(met[24 * d:24 * (d + 1)])
        torch.cuda.synchronize()
        assert torch.equal(out["tmrt"][24 * d:24 * (d + 1)], ref["tmrt"]), d
    # replaying the captured graph again gives the same result
    again = md.replay()
    torch.cuda.synchronize()
    assert torch.equal(again["tmrt"], out["tmrt"])


def test_tile_batch_and_autotuner(cuda, tmp_path, monkeypatch):
    """Uneven tiles in one graph equal each tile run alone; the autotuner picks
    a config from its search space and caches it."""
    import torch
    from solweig_cuda_b200 import batched, engine, synthetic, tune
    monkeypatch.setenv("SOLWEIG_TUNE_CACHE", str(tmp_path / "tune.json"))
    specs = [(40, 33, 1, 40.0), (57, 64, 2, 52.5), (72, 50, 3, 59.0)]
    scenes, mets, lats = [], [], []
    for r, c, seed, lat in specs:
        s = synthetic.make_scene(r, c, seed=seed)
        scenes.append(engine.Scene(s.dsm, s.trees, s.dem, 1.0, landcover=s.landcover))
        mets.append(synthetic.make_met(doy=150, latitude=lat, longitude=0.0, seed=seed))
        lats.append(lat)
    day = batched.ChosenDay(scenes[2], lats[2], 0.0, 3.0, 0.0)
    cfg, stages = tune.tune(day, mets[2], repeats=1)
    assert (cfg.shadow_bx, cfg.shadow_by) in tune.SHADOW_BLOCKS
    assert cfg.gvf_rows in tune.GVF_ROWS and cfg.rad_threads in tune.RAD_THREADS
    assert cfg.gvf_hours in tune.GVF_HOURS
    assert set(stages) >= {"day_shadow_kernel", "day_gvf_kernel", "day_radiation_kernel"}
    assert tune.lookup(day).astuple() == cfg.astuple()
    tb = batched.TileBatch(scenes, lats, [0.0] * 3, configs=[cfg] * 3)
    outs = tb.run(mets)
    outs = [{k: v.clone() for k, v in o.items()} for o in outs]
    for s, met, lat, o in zip(scenes, mets, lats, outs):
        alone = batched.ChosenDay(s, lat, 0.0, 3.0, 0.0)
        alone.set_config(cfg)
        ref = alone.run_day(met)
        torch.cuda.synchronize()
        assert torch.equal(o["tmrt"], ref["tmrt"])


# hour-vectorized GVF against the per-hour kernel: (Lup W/m2, albedo) absolute
# tolerances and the day's Tmrt (K)
HV_TOL = {1: (1e-3, 1e-6, 1e-3)}


@pytest.mark.parametrize("hv_kind", [1])
def test_hour_vectorized_gvf_matches_per_hour_kernel(cuda, hv_kind):
    """Interior tiles through the hour-vectorized GVF kernel (float32, 4-hour
    passes) against the per-hour kernel everywhere: GVF planes of every
    daytime hour and the day's Tmrt.  The scene is large enough for interior
    32 x 32 tiles."""
    import torch
    from solweig_cuda_b200 import _lib, batched, engine, synthetic
    s = synthetic.make_scene(150, 134, seed=17)
    scene = engine.Scene(s.dsm, s.trees, s.dem, 1.0, landcover=s.landcover)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0, seed=2)
    res = {}
    lup_tol, alb_tol, tmrt_tol = HV_TOL[hv_kind]
    for hv in (0, hv_kind):
        day = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0)
        cfg = _lib.SolweigDayConfig.default()
        cfg.gvf_hours = hv
        day.set_config(cfg)
        out = {k: v.clone() for k, v in day.run_day(met).items()}
        torch.cuda.synchronize()
        o = day.work_offsets()
        n = scene.pixels
        gvf = day.work[o["gvf"]:o["gvf"] + 12 * 24 * n].view(torch.float32).view(24, 3, n).clone()
        nosh = day.work[o["nosh"]:o["nosh"] + 4 * n].view(torch.float32).clone()
        res[hv] = (out, gvf, nosh, [h.daytime for h, _, _ in day.plan(met)])
    (o0, g0, n0, dayflags), (o1, g1, n1, _) = res[0], res[hv_kind]
    torch.testing.assert_close(n1, n0, rtol=1e-6, atol=1e-6)
    for h, d in enumerate(dayflags):
        if d:
            # Lup (W/m2): float32 sums in another order; albedo: albedo*shadow rounded per sample
            torch.testing.assert_close(g1[h, 0], g0[h, 0], rtol=1e-5, atol=lup_tol)
            torch.testing.assert_close(g1[h, 1], g0[h, 1], rtol=1e-5, atol=alb_tol)
            assert torch.equal(g1[h, 2], g0[h, 2])
    assert torch.max(torch.abs(o1["tmrt"] - o0["tmrt"])).item() <= tmrt_tol


def test_packed_float32_geometry_is_bit_identical(scene64):
    """The sweep's packed float4 geometry (used when the three height rasters
    are exact in float32) gives the same shadow quads, bit for bit, as the
    float64 rasters."""
    import torch
    from solweig_cuda_b200 import batched, synthetic
    sc, scene = scene64
    assert scene.geo32 is not None  # the generator's heights are float32 values
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    quads = {}
    saved = scene.struct.geo32
    try:
        for packed in (True, False):
            scene.struct.geo32 = saved if packed else None
            day = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0, use_graph=False)
            day.run_day(met)
            torch.cuda.synchronize()
            o = day.work_offsets()
            quads[packed] = day.work[o["quads"]:o["quads"] + 16 * 24 * scene.pixels].clone()
    finally:
        scene.struct.geo32 = saved
    flags = [h.daytime for h, _, _ in day.plan(met)]
    q1 = quads[True].view(torch.int32).view(24, -1)
    q0 = quads[False].view(torch.int32).view(24, -1)
    for h, d in enumerate(flags):
        if d:
            assert torch.equal(q1[h], q0[h]), h


@pytest.mark.parametrize("doy,lat,shift", [(172, 53.0, 0.0), (355, 60.0, 0.0), (80, 10.0, -3.0)])
def test_ray_ceiling_exit_is_bit_identical(cuda, doy, lat, shift):
    """The sweep's early exit on the per-hour ray ceilings changes no bit of the
    shadow quads (shadow, Lup, albedo, ground/sunlit-wall bits) nor of the
    day's outputs, for packed and float64 geometry, low winter sun (long
    rays) and a terrain partly below zero (where the exit is never taken)."""
    import torch
    from solweig_cuda_b200 import _lib, batched, engine, synthetic
    s = synthetic.make_scene(150, 134, seed=17)
    dsm = (s.dsm + np.float32(shift)).astype(np.float32)
    scene = engine.Scene(dsm, s.trees, s.dem + np.float32(shift), 1.0, landcover=s.landcover)
    met = synthetic.make_met(doy=doy, latitude=lat, longitude=0.0, seed=5)
    saved = scene.struct.geo32
    res = {}
    try:
        for packed in (True, False):
            scene.struct.geo32 = saved if packed else None
            for no_ceiling in (0, 1):
                day = batched.ChosenDay(scene, lat, 0.0, 3.0, 0.0, outputs=("tmrt", "utci", "shadow"),
                                        use_graph=False)
                cfg = _lib.SolweigDayConfig.default()
                cfg.no_ceiling = no_ceiling
                day.set_config(cfg)
                out = {k: v.clone() for k, v in day.run_day(met).items()}
                torch.cuda.synchronize()
                assert day.error_flag() == 0
                o = day.work_offsets()
                q = day.work[o["quads"]:o["quads"] + 16 * 24 * scene.pixels].clone()
                res[packed, no_ceiling] = (out, q.view(torch.int32).view(24, -1))
    finally:
        scene.struct.geo32 = saved
    flags = [h.daytime for h, _, _ in day.plan(met)]
    for packed in (True, False):
        (o1, q1), (o0, q0) = res[packed, 0], res[packed, 1]
        for h, d in enumerate(flags):
            if d:
                assert torch.equal(q1[h], q0[h]), (packed, h)
        for k in o0:  # bit patterns: UTCI is NaN on building pixels
            assert torch.equal(o1[k].view(torch.int32), o0[k].view(torch.int32)), (packed, k)


@pytest.mark.parametrize("ranges", [5, (1, 2, 3, 7)])
def test_pipelined_sweep_ranges_match_whole_day(scene64, ranges):
    """Sweep ranges launched as their hours are planned (eager first day, then
    graph replays) give the whole-day results bit for bit, on two forcings."""
    import torch
    from solweig_cuda_b200 import batched, synthetic
    sc, scene = scene64
    outs = ("tmrt", "utci", "shadow", "kdown")
    whole = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0, outputs=outs, pipeline_hours=0)
    piped = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0, outputs=outs, pipeline_hours=ranges)
    assert piped.launches_per_day > whole.launches_per_day
    for doy, seed in ((172, 0), (200, 3), (172, 0)):
        met = synthetic.make_met(doy=doy, latitude=53.0, longitude=0.0, seed=seed)
        ref = {k: v.clone() for k, v in whole.run_day(met).items()}
        got = {k: v.clone() for k, v in piped.run_day(met).items()}
        torch.cuda.synchronize()
        for k in outs:
            assert torch.equal(got[k].view(torch.int32), ref[k].view(torch.int32)), (doy, k)
    assert piped.error_flag() == 0


@pytest.mark.parametrize("shape,doy,lat,shift", [((150, 134), 172, 53.0, 0.0), ((150, 134), 355, 60.0, 0.0),
                                                 ((97, 203), 80, 10.0, -3.0), ((40, 36), 172, 53.0, 0.0)])
def test_window_sweep_is_bit_identical(cuda, shape, doy, lat, shift):
    """The sweep on TMA-staged shared-memory windows with the warp-vote exit
    (sweep_window = 1: 48 x 48 px, 2: 40 x 40 px) gives the quads and the
    day's outputs of the sweep that
    reads every step from the raster, bit for bit: with and without the ray
    ceilings, low winter sun, tiles cut by the raster edge, a raster smaller
    than one window and terrain partly below zero (vote never taken there)."""
    import torch
    from solweig_cuda_b200 import _lib, batched, engine, synthetic
    s = synthetic.make_scene(*shape, seed=23)
    dsm = (s.dsm + np.float32(shift)).astype(np.float32)
    scene = engine.Scene(dsm, s.trees, s.dem + np.float32(shift), 1.0, landcover=s.landcover)
    assert scene.geo32 is not None
    met = synthetic.make_met(doy=doy, latitude=lat, longitude=0.0, seed=7)
    res = {}
    for window in (0, 1, 2):
        for no_ceiling in (0, 1):
            day = batched.ChosenDay(scene, lat, 0.0, 3.0, 0.0, outputs=("tmrt", "utci", "shadow"),
                                    use_graph=False)
            cfg = _lib.SolweigDayConfig.default()
            cfg.no_ceiling = no_ceiling
            cfg.sweep_window = window
            day.set_config(cfg)
            out = {k: v.clone() for k, v in day.run_day(met).items()}
            torch.cuda.synchronize()
            assert day.error_flag() == 0
            q = day.quads().clone().view(torch.int32).view(24, -1)
            res[window, no_ceiling] = (out, q)
    flags = [h.daytime for h, _, _ in day.plan(met)]
    for window in (1, 2):
        for no_ceiling in (0, 1):
            (o1, q1), (o0, q0) = res[window, no_ceiling], res[0, no_ceiling]
            for h, d in enumerate(flags):
                if d:
                    assert torch.equal(q1[h], q0[h]), (window, no_ceiling, h)
            for k in o0:
                assert torch.equal(o1[k].view(torch.int32), o0[k].view(torch.int32)), (window, no_ceiling, k)


def test_gvf_statics_prepared_with_the_scene_are_identical(cuda):
    """Days that read the GVF walk lengths and albedo-without-shadow plane
    prepared with the scene (solweig_gvf_statics) equal, bit for bit, days
    that walk them from the first daytime hour's quads (border and interior
    tiles)."""
    import torch
    from solweig_cuda_b200 import batched, engine, synthetic
    s = synthetic.make_scene(150, 134, seed=17)
    scene = engine.Scene(s.dsm, s.trees, s.dem, 1.0, landcover=s.landcover)
    assert scene.gvf_hits is not None and scene.struct.gvf_hits
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0, seed=2)
    outs = ("tmrt", "utci", "kup", "lup")
    res = []
    for with_statics in (True, False):
        if not with_statics:
            scene.struct.gvf_hits = None
            scene.struct.gvf_nosh = None
        day = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0, outputs=outs)
        out = {k: v.clone() for k, v in day.run_day(met).items()}
        torch.cuda.synchronize()
        o = day.work_offsets()
        n = scene.pixels
        gvf = day.work[o["gvf"]:o["gvf"] + 12 * 24 * n].view(torch.float32).view(24, 3, n).clone()
        nosh = day.work[o["nosh"]:o["nosh"] + 4 * n].view(torch.float32).clone()
        res.append((out, gvf, nosh, [h.daytime for h, _, _ in day.plan(met)]))
    scene.struct.gvf_hits = scene.gvf_hits.data_ptr()
    scene.struct.gvf_nosh = scene.gvf_nosh.data_ptr()
    (a, ga, na, flags), (b, gb, nb, _) = res
    assert torch.equal(na, nb)
    for h, d in enumerate(flags):  # the GVF planes of daytime hours (night ones are not written)
        if d:
            assert torch.equal(ga[h], gb[h]), h
    for k in outs:
        torch.testing.assert_close(a[k], b[k], rtol=0, atol=0, equal_nan=True)
