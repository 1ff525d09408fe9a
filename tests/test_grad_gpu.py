"""The day gradient (hand-written reverse pass): forward against the batched
form, directional derivatives against central finite differences of the GPU
forward and of the FP64 oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FD_RTOL = 1e-3      # adjoint vs central differences of the same (GPU) forward
ORACLE_RTOL = 1e-3  # adjoint vs central differences of the FP64 oracle
FORWARD_TOL = 2e-3  # K, gradient forward vs the batched form (daily mean UTCI)

STEPS = {"albedo": 1e-2, "emissivity": 1e-2, "transmissivity": 1e-2, "ta": 1e-2, "rh": 1e-1, "ws": 1e-2}


@pytest.fixture(scope="module")
def setup():
    import torch
    from solweig_cuda_b200 import engine, grad, synthetic
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    sc = synthetic.make_scene(40, 36, seed=21)
    scene = engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0, seed=4)
    rng = np.random.default_rng(5)
    shape = scene.shape
    params = {
        "albedo": rng.uniform(0.1, 0.4, shape).astype(np.float32),
        "emissivity": rng.uniform(0.9, 0.98, shape).astype(np.float32),
        "transmissivity": rng.uniform(0.02, 0.2, shape).astype(np.float32),
    }
    weights = rng.uniform(0.5, 1.5, shape).astype(np.float32)
    dg = grad.DayGradient(scene, 53.0, 0.0, 3.0, 0.0)
    return sc, scene, met, params, weights, dg


def _J(dg, params, met, weights):
    import torch
    daily = dg.forward(params["albedo"], params["emissivity"], params["transmissivity"], met).cpu().numpy()
    return float(np.nansum(daily * weights))


def _directions(shape, rng):
    return {
        "albedo": rng.uniform(-1, 1, shape), "emissivity": rng.uniform(-1, 1, shape),
        "transmissivity": rng.uniform(-1, 1, shape),
        "ta": rng.uniform(-1, 1, 24), "rh": rng.uniform(-1, 1, 24), "ws": rng.uniform(-1, 1, 24),
    }


def _perturb(params, met, name, v, h):
    p = {k: v_.copy() for k, v_ in params.items()}
    m = met.copy()
    if name in p:
        p[name] = (p[name].astype(np.float64) + h * v).astype(np.float32)
    else:
        col = {"ta": 11, "rh": 10, "ws": 9}[name]
        m[:, col] = m[:, col] + h * v
    return p, m


def _adjoint(dg, params, met, weights):
    da, de, dt, hg, lg = dg.backward(params["albedo"], params["emissivity"], params["transmissivity"], met, weights)
    fg = dg.forcing_grad(met, hg, lg)
    return {"albedo": da.cpu().numpy().astype(np.float64), "emissivity": de.cpu().numpy().astype(np.float64),
            "transmissivity": dt.cpu().numpy().astype(np.float64), "ta": fg["ta"], "rh": fg["rh"],
            "ws": fg["ws"]}


def test_gradient_forward_matches_batched_form(setup):
    import torch
    from solweig_cuda_b200 import batched
    sc, scene, met, params, weights, dg = setup
    base = {"albedo": scene.alb.cpu().numpy(), "emissivity": scene.emis.cpu().numpy(),
            "transmissivity": np.full(scene.shape, 0.03, np.float32)}
    daily = dg.forward(base["albedo"], base["emissivity"], base["transmissivity"], met).cpu().numpy()
    day = batched.ChosenDay(scene, 53.0, 0.0, 3.0, 0.0)
    ut = day.run_day(met)["utci"]
    torch.cuda.synchronize()
    want = ut.cpu().numpy().astype(np.float64).mean(axis=0)
    assert np.array_equal(np.isnan(daily), np.isnan(want))
    assert np.nanmax(np.abs(daily - want)) <= FORWARD_TOL


def test_adjoint_matches_central_differences(setup):
    sc, scene, met, params, weights, dg = setup
    g = _adjoint(dg, params, met, weights)
    rng = np.random.default_rng(11)
    dirs = _directions(scene.shape, rng)
    for name, v in dirs.items():
        h = STEPS[name]
        jp = _J(dg, *_perturb(params, met, name, v, h), weights)
        jm = _J(dg, *_perturb(params, met, name, v, -h), weights)
        fd = (jp - jm) / (2 * h)
        ad = float(np.sum(g[name] * v))
        assert abs(ad - fd) <= FD_RTOL * max(abs(fd), 1e-9), (name, ad, fd)


def _oracle_objective(sc, weights):
    """J of the FP64 oracle (UMEP restatement, masks from its own shadow sweep)."""
    from oracle import step as ST
    s = ST.prepare_static(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    loc = dict(latitude=53.0, longitude=0.0, altitude=3.0)

    def J(p, m):
        s2 = dict(s)
        s2["alb_grid"] = p["albedo"].astype(np.float64)
        s2["emis_grid"] = p["emissivity"].astype(np.float64)
        res = ST.run_day(s2, m, loc, 0.0, outputs=("UTCI",), psi=p["transmissivity"].astype(np.float64))
        daily = np.mean([r["UTCI"] for r in res], axis=0)
        return float(np.nansum(daily * weights))
    return J


def _check_against_oracle(sc, shape, met, params, weights, g, seeds):
    J = _oracle_objective(sc, weights)
    worst = {}
    for seed in seeds:
        dirs = _directions(shape, np.random.default_rng(seed))
        for name in ("albedo", "emissivity", "transmissivity", "ta", "rh", "ws"):
            v = dirs[name]
            h = STEPS[name]
            fd = (J(*_perturb(params, met, name, v, h)) - J(*_perturb(params, met, name, v, -h))) / (2 * h)
            ad = float(np.sum(g[name] * v))
            rel = abs(ad - fd) / max(abs(fd), 1e-9)
            worst[name] = max(worst.get(name, 0.0), rel)
            assert rel <= ORACLE_RTOL, (name, seed, ad, fd)
    return worst


def test_adjoint_matches_fp64_oracle(setup):
    """Directional derivatives of the FP64 oracle by central differences, three
    random directions per parameter group."""
    sc, scene, met, params, weights, dg = setup
    g = _adjoint(dg, params, met, weights)
    _check_against_oracle(sc, scene.shape, met, params, weights, g, seeds=(13, 100, 101))


def test_adjoint_matches_fp64_oracle_second_scene():
    """The same check on a larger scene (64 x 56 px, another city and other
    parameter fields), two directions per group."""
    import torch
    from solweig_cuda_b200 import engine, grad, synthetic
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    sc = synthetic.make_scene(64, 56, seed=5)
    scene = engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0, seed=4)
    rng = np.random.default_rng(5)
    params = {
        "albedo": rng.uniform(0.1, 0.4, scene.shape).astype(np.float32),
        "emissivity": rng.uniform(0.9, 0.98, scene.shape).astype(np.float32),
        "transmissivity": rng.uniform(0.02, 0.2, scene.shape).astype(np.float32),
    }
    weights = rng.uniform(0.5, 1.5, scene.shape).astype(np.float32)
    dg = grad.DayGradient(scene, 53.0, 0.0, 3.0, 0.0)
    g = _adjoint(dg, params, met, weights)
    _check_against_oracle(sc, scene.shape, met, params, weights, g, seeds=(100, 101))
