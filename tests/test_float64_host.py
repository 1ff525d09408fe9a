"""Host side of the float64 step: the float64 patch constants and hour
weights handed to solweig_step64 keep the host plan's float64 values (the
float32 step's records round them), and the library's struct sizes agree
with the bindings."""
import types

import numpy as np


def _scene_stub():
    from solweig_cuda_b200 import engine
    return types.SimpleNamespace(layout=engine.SkyLayout(2), tgk_wall=0.37, tstart_wall=-3.41, tmaxlst_wall=15.0,
                                 scale=1.0, amaxvalue=20.0, shape=(40, 40), landcover=0)


def test_sky64_keeps_the_float64_layout():
    from solweig_cuda_b200 import engine
    lay = engine.SkyLayout(2)
    s = lay.struct64()
    L = lay.host
    P = L.count
    assert np.array_equal(np.ctypeslib.as_array(s.omega)[:P], L.steradian)
    assert np.array_equal(np.ctypeslib.as_array(s.cos_alt)[:P], L.cos_alt)
    assert np.array_equal(np.ctypeslib.as_array(s.sin_alt)[:P], L.sin_alt)
    assert np.array_equal(np.ctypeslib.as_array(s.cardinal)[:, :P], L.cardinal.T)
    # float32 diffsh of a vegetation patch, as compute_diffsh evaluates it
    from oracle import geometry as G
    want = G.compute_diffsh(np.float32([1.0]), np.float32([0.0]), np.float32(0.03))[0]
    assert want.dtype == np.float32 and s.diffsh_veg == float(want)
    assert s.diffsh_veg != 0.03 and abs(s.diffsh_veg - 0.03) < 1e-7


def test_hour64_records_carry_the_float64_plan():
    from solweig_cuda_b200 import _lib, engine, sun, synthetic
    scene = _scene_stub()
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    sol = sun.metdata(met, 53.0, 0.0, 3.0, 0.0)
    P = scene.layout.host.count
    seen_day = seen_night = False
    for i in (2, 12):
        h, ray, scal, _ = engine.hour_plan(scene, 53.0, sol.altitude[i], sol.azimuth[i], sol.zen[i], sol.jday[i],
                                           sol.dectime[i], sol.altmax[i], met[i, 11], met[i, 10], met[i, 14],
                                           met[i, 21], met[i, 22], met[i, 12], met[i, 9], 0.03, 1.0, 1, 0.0,
                                           1 / 24, None)
        r = engine.hour64_record(scene, h, scal)
        lum = np.ctypeslib.as_array(r.lum)
        assert np.array_equal(np.ctypeslib.as_array(r.band_lsky)[:len(scal.band_lsky)], scal.band_lsky)
        if h.daytime:
            seen_day = True
            assert np.array_equal(lum[:P], scal.lv[:, 2])
            # the float32 record rounds the same luminances
            assert np.array_equal(np.ctypeslib.as_array(h.lum)[:P], scal.lv[:, 2].astype(np.float32))
            assert not np.array_equal(lum[:P], lum[:P].astype(np.float32).astype(np.float64))
        else:
            seen_night = True
            assert not lum.any()
    assert seen_day and seen_night
    import ctypes
    sizes = (ctypes.c_int64 * 4)()
    assert _lib.lib().solweig_struct_sizes64(sizes) == 0
    assert list(sizes) == [ctypes.sizeof(t) for t in (_lib.SolweigSky64, _lib.SolweigHour64,
                                                      _lib.SolweigOutputs64, _lib.SolweigState64)]
