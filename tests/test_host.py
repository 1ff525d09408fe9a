"""CPU tests of the host logic and of the C-ABI library surface (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "solweig_b200.h")).read()
    return sorted(set(re.findall(r"\b(?:int|const char\*)\s+(solweig_\w+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    from solweig_cuda_b200 import _lib
    L = _lib.lib()
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
        assert n in _lib.EXPORTED_SYMBOLS, n


def test_null_arguments_are_rejected_without_a_gpu():
    from solweig_cuda_b200 import _lib
    L = _lib.lib()
    assert L.solweig_wall_heights(None, None, 10, 10, 3.0, None) == 1
    assert b"null" in L.solweig_last_error()
    assert L.solweig_shadow(None, None, None, 0, 0.0, 0.0, 0, 1, None, None) == 1
    assert L.solweig_utci_collapse(20.0, 50.0, 2.0, None) == 1
    scene = _lib.SolweigScene()
    assert L.solweig_step_shadow(ctypes.byref(scene), None, 0, None, None) == 1
    assert b"scene" in L.solweig_last_error()


def test_utci_collapse_matches_oracle():
    from oracle import utci as OU
    from solweig_cuda_b200 import _lib
    L = _lib.lib()
    rng = np.random.default_rng(0)
    for _ in range(50):
        ta, rh, va = rng.uniform(-30, 45), rng.uniform(5, 100), rng.uniform(0.5, 17)
        c = (ctypes.c_double * 7)()
        assert L.solweig_utci_collapse(ta, rh, va, c) == 0
        assert np.allclose(np.array(c), OU.utci_collapsed(ta, rh, va), rtol=1e-12, atol=1e-15)
    c = (ctypes.c_double * 7)()
    assert L.solweig_utci_collapse(-999.0, 50.0, 2.0, c) == 0 and not any(c)


def test_shadow_ray_matches_oracle_walk():
    from oracle.geometry import _ray_step
    from solweig_cuda_b200 import rays
    for azi, alt in ((45., 30.), (100.3, 12.5), (200., 6.), (271.7, 3.2), (359.9, 50.)):
        r = rays.shadow_ray(azi, alt, 1.0, 40.0, (300, 250))
        az = azi * np.pi / 180
        for k in range(r.steps):
            dx, dy, ds = _ray_step(az, k)
            assert (r.dxdy[k, 0], r.dxdy[k, 1]) == (int(dx), int(dy))
            assert r.dz[k] == (ds * k) * (np.tan(alt * (np.pi / 180.)) / 1.0)
        assert np.all(np.diff(np.abs(r.dxdy[:, 0])) >= 0) and np.all(np.diff(np.abs(r.dxdy[:, 1])) >= 0)
        assert np.all(np.diff(r.dz) >= 0)
        last = r.dz[-1] > 40.0 or abs(r.dxdy[-1, 0]) >= 300 or abs(r.dxdy[-1, 1]) >= 250
        assert last and not (r.dz[:-1] > 40.0).any()


def test_svf_rays_match_reference_setup():
    from solweig_cuda_b200 import rays
    dxdy, dz, lengths, cap = rays.svf_rays(2, (40, 50), 30.0, 1.0)
    assert dxdy.shape[0] == 153 and lengths.max() == cap
    assert lengths.min() >= 1


def test_gvf_offsets_stay_inside_halo():
    from solweig_cuda_b200 import rays
    offs, first, second = rays.gvf_offsets(1.0)
    assert (first, second) == (1, 22)
    assert np.abs(offs).max() <= second - 1
    assert tuple(offs[0, 0]) == (0, 0)


def test_arctan_thresholds_are_exact():
    from solweig_cuda_b200 import sky
    L = sky.patch_layout(2)
    rng = np.random.default_rng(1)
    for a in np.unique(L.altitude):
        k = int(np.flatnonzero(L.altitude == a)[0])
        lo, hi = L.sunlit_below[k], L.shaded_above[k]
        xs = np.concatenate([rng.uniform(-5, 50, 2000), [lo, hi], np.nextafter(lo, [-np.inf, np.inf]),
                             np.nextafter(hi, [-np.inf, np.inf]), [1.633123935319537e16]])
        xs = xs[np.isfinite(xs)]  # tan(asvf) <= tan(pi/2) is always finite
        deg = np.arctan(xs) * (180 / np.pi)
        assert np.array_equal(deg < a, xs < lo)
        assert np.array_equal(deg > a, xs > hi)


def test_synthetic_scene_statistics_and_determinism():
    from solweig_cuda_b200 import synthetic
    a = synthetic.make_scene(200, seed=0)
    b = synthetic.make_scene(200, seed=0)
    assert np.array_equal(a.dsm, b.dsm) and np.array_equal(a.trees, b.trees)
    roof = a.dsm > 0
    assert 0.28 <= roof.mean() <= 0.40
    assert 0.08 <= (a.trees > 0).mean() <= 0.16
    assert not (roof & (a.trees > 0)).any()
    assert a.dsm.max() <= 40 and a.dsm[roof].min() >= 5
    assert set(np.unique(a.landcover)) <= {1.0, 2.0, 5.0}
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    assert met.shape == (24, 24)
    assert 9.9 <= met[:, 11].min() and met[:, 11].max() <= 22.1
    assert (met[:, 14] >= 0).all() and met[:, 14].max() > 300


def test_shard_split_is_a_partition():
    from solweig_cuda_b200 import shard
    units = list(range(30))
    for world in (1, 2, 3, 4, 8):
        parts = [shard.split(units, r, world) for r in range(world)]
        assert sum(parts, []) == units
        assert max(map(len, parts)) - min(map(len, parts)) <= 1


def test_pipelined_sweep_ranges_cover_the_day():
    """Hour ranges of the pipelined batched day: consecutive, covering every
    hour once, the last length repeating; 0 turns pipelining off."""
    from solweig_cuda_b200.batched import ChosenDay
    assert ChosenDay._ranges(24, 0) is None
    for hours, spec in ((24, (2, 2, 2, 2, 4, 4, 8)), (24, 5), (7, (1, 2)), (30, (3, 9)), (1, 4)):
        r = ChosenDay._ranges(hours, spec)
        assert r[0][0] == 0 and r[-1][1] == hours
        assert all(a[1] == b[0] and a[0] < a[1] for a, b in zip(r, r[1:]))
    assert ChosenDay._ranges(24, (2, 2, 2, 2, 4, 4, 8)) == [(0, 2), (2, 4), (4, 6), (6, 8), (8, 12), (12, 16),
                                                             (16, 24)]
    with pytest.raises(ValueError):
        ChosenDay._ranges(24, (2, 0))


@pytest.mark.parametrize("shape,amax,scale", [((2000, 2000), 40.0, 1.0), ((150, 134), 25.3, 1.0),
                                               ((64, 200), 12.0, 0.5), ((37, 41), 60.0, 2.0),
                                               ((500, 480), 0.0, 1.0), ((30, 20), -1.0, 1.0)])
def test_svf_rays_prefix_equals_full_tables(shape, amax, scale):
    """The SVF ray tables evaluated on each patch's prefix of steps equal the
    tables evaluated on every step (offsets, heights, lengths, capacity)."""
    from solweig_cuda_b200 import rays
    for po in (1, 2, 3):
        a = rays.svf_rays(po, shape, amax, scale)
        b = rays._svf_rays_per_patch(po, shape, amax, scale)
        assert a[3] == b[3]
        assert np.array_equal(a[2], b[2]) and np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
