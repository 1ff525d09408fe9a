"""Ray ceilings of the batched shadow sweep (``csrc/ceiling.cuh``).

A numpy restatement of the construction (frame from the ray table, integer
shear, dilation by the measured band, discounted backward maximum along each
sheared line) checked against the property the sweep's early exit relies on:
for every pixel p, every step k >= 1 of its ray inside the raster and every
later step j,  H(q_j) - dz_{j-1} <= C(q_k) - dz_{k-1};  and the window
maximum M (the largest sampled dilated height at X .. X + 7 of the line)
against the property of the 8-step skip:  H(q_j) - dz_{j-1} <= M(q_k) -
dz_{k-1}  for k <= j < k + 8.
"""
SKIP = 8
import numpy as np
import pytest


def _frame(dxdy, dz, rows, cols):
    K = len(dz)
    i = np.arange(K)
    last = dxdy[K - 1]
    sr = -1 if last[0] < 0 else 1
    sc = -1 if last[1] < 0 else 1
    rows_ok = bool(np.all(dxdy[:, 0] == sr * i))
    cols_ok = bool(np.all(dxdy[:, 1] == sc * i))
    assert rows_ok or cols_ok, "a sun ray has a major axis"
    s_major, s_minor = (sr, sc) if rows_ok else (sc, sr)
    minor = (dxdy[:, 1] if rows_ok else dxdy[:, 0]).astype(np.int64) * s_minor
    d, m = K - 1, int(minor[-1])
    e = minor * d - i.astype(np.int64) * m
    band = int(e.max() - e.min()) // d + 1
    delta = np.float32(np.diff(dz).min())
    if float(delta) > np.diff(dz).min():
        delta = np.nextafter(delta, np.float32(-np.inf))
    return dict(rows_major=rows_ok, s_major=s_major, s_minor=s_minor, m=m, d=d, band=band,
                delta=float(delta))


def _dilate_minor(Hm, w):
    """max over +-w along axis 1 (neighbours outside the raster ignored)."""
    out = Hm.copy()
    for d in range(1, w + 1):
        out[:, :-d] = np.maximum(out[:, :-d], Hm[:, d:])
        out[:, d:] = np.maximum(out[:, d:], Hm[:, :-d])
    return out


def ceiling_planes(H, dxdy, dz):
    """Ceiling plane of one hour, restating the kernels: H dilated by +-W
    along the minor axis (the dilation kernel's planes), sampled along each
    sheared line with the centre clamped to the raster when it lies within W
    of it, and the discounted backward maximum."""
    rows, cols = H.shape
    f = _frame(dxdy, dz, rows, cols)
    W = f["band"]
    Hm = H if f["rows_major"] else H.T          # [major][minor] in raster order
    plane = _dilate_minor(Hm, W)
    nx, nb = Hm.shape
    R = np.arange(nx) * f["m"] // f["d"]
    roff = int(R[-1])
    lines = nb + roff
    line = np.arange(lines) - roff               # sheared line N of each lane
    G = np.full(lines, -np.inf)
    win = np.full((SKIP - 1, lines), -np.inf)    # samples at x + 1 .. x + SKIP - 1
    Co = np.empty_like(Hm)
    Mo = np.empty_like(Hm)
    for x in range(nx - 1, -1, -1):
        a = x if f["s_major"] > 0 else nx - 1 - x
        y = line + R[x]
        near = (y >= -W) & (y < nb + W)
        yc = np.clip(y, 0, nb - 1)
        b = yc if f["s_minor"] > 0 else nb - 1 - yc
        v = np.where(near, plane[a, b], -np.inf)
        G = np.maximum(v, G - f["delta"])
        M = np.maximum(v, win.max(axis=0))
        win = np.vstack([v[None], win[:-1]])
        inside = (y >= 0) & (y < nb)
        col = np.where(f["s_minor"] > 0, y, nb - 1 - y)[inside]
        Co[a, col] = G[inside]
        Mo[a, col] = M[inside]
    if not f["rows_major"]:
        Co, Mo = Co.T, Mo.T
    return Co, f, Mo


def _check_bound(H, C, ray):
    rows, cols = H.shape
    rr, cc = np.meshgrid(np.arange(rows), np.arange(cols), indexing="ij")
    K = ray.steps
    hs, inside = [], []
    for j in range(K):
        r2, c2 = rr + ray.dxdy[j][0], cc + ray.dxdy[j][1]
        ok = (r2 >= 0) & (r2 < rows) & (c2 >= 0) & (c2 < cols)
        if j:
            ok &= inside[-1]
        inside.append(ok)
        hs.append((np.where(ok, H[np.clip(r2, 0, rows - 1), np.clip(c2, 0, cols - 1)], -np.inf),
                   np.where(ok, C[np.clip(r2, 0, rows - 1), np.clip(c2, 0, cols - 1)], np.inf)))
    suffix = np.full(H.shape, -np.inf)
    slack = np.inf
    for k in range(K - 1, 0, -1):
        suffix = np.maximum(suffix, hs[k][0] - ray.dz[k - 1])
        rhs = hs[k][1] - ray.dz[k - 1]
        m = inside[k]
        if m.any():
            slack = min(slack, float(np.min(rhs[m] - suffix[m])))
    return slack


@pytest.mark.parametrize("seed", range(6))
def test_ceiling_bounds_every_later_sample(seed):
    from solweig_cuda_b200 import rays
    rng = np.random.default_rng(seed)
    rows, cols = int(rng.integers(24, 64)), int(rng.integers(24, 64))
    H = rng.uniform(0, 35, (rows, cols)) * (rng.random((rows, cols)) < 0.35)
    azimuths = [0.0, 45.0, 90.0, 135.0, 180.0, 225.0, 270.0, 315.0] if seed == 0 else rng.uniform(0, 360, 8)
    for az in azimuths:
        alt = float(rng.uniform(4, 75))
        ray = rays.shadow_ray(float(az), alt, 1.0, float(H.max()), (rows, cols), True)
        if ray.steps < 5:
            continue
        C, f, M = ceiling_planes(H, ray.dxdy, ray.dz)
        assert f["band"] <= 2 and f["m"] <= f["d"]
        assert np.all(C >= H)            # the sample itself is in its own bound
        assert _check_bound(H, C, ray) >= 0.0, (az, alt)
        assert _check_window(H, M, ray) >= 0.0, (az, alt)


def _check_window(H, M, ray):
    """Smallest slack of M(q_k) - dz_{k-1} - (H(q_j) - dz_{j-1}) over every
    pixel, step k >= 1 inside the raster and k <= j < k + SKIP inside."""
    rows, cols = H.shape
    rr, cc = np.meshgrid(np.arange(rows), np.arange(cols), indexing="ij")
    K = ray.steps
    hv, mv, inside = [], [], []
    for j in range(K):
        r2, c2 = rr + ray.dxdy[j][0], cc + ray.dxdy[j][1]
        ok = (r2 >= 0) & (r2 < rows) & (c2 >= 0) & (c2 < cols)
        if j:
            ok &= inside[-1]
        inside.append(ok)
        R2, C2 = np.clip(r2, 0, rows - 1), np.clip(c2, 0, cols - 1)
        hv.append(np.where(ok, H[R2, C2], -np.inf))
        mv.append(np.where(ok, M[R2, C2], np.inf))
    slack = np.inf
    for k in range(1, K):
        rhs = mv[k] - ray.dz[k - 1]
        for j in range(k, min(K, k + SKIP)):
            m = inside[j]
            if m.any():
                slack = min(slack, float(np.min(rhs[m] - (hv[j][m] - ray.dz[j - 1]))))
    return slack


def test_ceiling_cuts_the_walk_on_a_city():
    """On the synthetic city the bound lets most rays stop far before the
    global clearance (the reason for the plane)."""
    from solweig_cuda_b200 import rays, synthetic
    sc = synthetic.make_scene(96, seed=3)
    dsm = sc.dsm.astype(np.float64)
    H = np.maximum(dsm, np.where(sc.trees > 0, sc.trees + dsm, 0.0))
    ray = rays.shadow_ray(200.0, 35.0, 1.0, float(H.max()), H.shape, True)
    C, _, _ = ceiling_planes(H, ray.dxdy, ray.dz)
    # steps needed by the global clearance vs by the ceiling at step 4, for ground pixels
    ground = dsm == 0
    clear_global = np.searchsorted(ray.dz, H.max())
    r4, c4 = ray.dxdy[4]
    rr, cc = np.nonzero(ground)
    ok = (rr + r4 >= 0) & (rr + r4 < 96) & (cc + c4 >= 0) & (cc + c4 < 96)
    stop = C[rr[ok] + r4, cc[ok] + c4] - ray.dz[3] < dsm[rr[ok], cc[ok]]
    assert clear_global > 40 and stop.mean() > 0.4
