"""solweig_step_static_scratch (scratch in a static device array, nothing
allocated) against solweig_step with a caller scratch buffer.

The file name sorts last so that, in a full run, the entry point is also
exercised after every other GPU test has used the library."""
import ctypes

import numpy as np
import pytest

# Identical kernels run on both sides, so the results should agree bit for
# bit; the tolerance only guards against reassociation in a future kernel.
ATOL = 1e-5
PLANES = ("tmrt", "utci", "kdown", "kup", "ldown", "lup", "shadow", "tg_out")


def _step(scene, plan, hour_indices, static):
    import torch
    from solweig_cuda_b200 import _lib, engine
    from solweig_cuda_b200.engine import device_ptr, stream_handle
    dev = scene.device
    buffers = engine.HourBuffers(scene, len(plan))
    for i, (h, ray, _) in enumerate(plan):
        buffers.put(i, h, ray)
    buffers.upload(0, len(plan), buffers.kmax)
    layout = scene.layout.device(dev)
    state = {k: torch.zeros(scene.shape, dtype=torch.float32, device=dev) for k in _lib.STATE_FIELDS}
    st = _lib.SolweigState()
    for k in _lib.STATE_FIELDS:
        setattr(st, k, state[k].data_ptr())
    scratch = None if static else torch.empty((_lib.SCRATCH_PLANES,) + scene.shape,
                                              dtype=torch.float32, device=dev)
    L = _lib.lib()
    results = []
    for i in hour_indices:
        out = {k: torch.full(scene.shape, -7.0, dtype=torch.float32, device=dev) for k in PLANES}
        o = engine.outputs_struct(out)
        if static:
            rc = L.solweig_step_static_scratch(
                ctypes.byref(scene.struct), device_ptr(layout), buffers.ptr(), i, ctypes.byref(st),
                ctypes.byref(o), scene.gvf_host_ptr, scene.first_steps, scene.second_steps,
                stream_handle())
            _lib.check(rc, "solweig_step_static_scratch")
        else:
            rc = L.solweig_step(
                ctypes.byref(scene.struct), device_ptr(layout), buffers.ptr(), i, ctypes.byref(st),
                ctypes.byref(o), scene.gvf_host_ptr, scene.first_steps, scene.second_steps,
                device_ptr(scratch), stream_handle())
            _lib.check(rc, "solweig_step")
        torch.cuda.synchronize()
        results.append({k: v.cpu().numpy() for k, v in out.items()})
    return results, {k: v.cpu().numpy() for k, v in state.items()}


@pytest.mark.gpu
def test_static_scratch_step_matches_solweig_step(cuda):
    from solweig_cuda_b200 import engine, synthetic
    sc = synthetic.make_scene(72, 56, seed=11)
    scene = engine.Scene(sc.dsm, sc.trees, sc.dem, 1.0, landcover=sc.landcover)
    met = synthetic.make_met(doy=172, latitude=53.0, longitude=0.0)
    plan = engine.plan_day(scene, met, 53.0, 0.0, 3.0, 0.0)
    hours = [12, 13]  # two calls in a row; the second reads the state the first wrote
    assert all(plan[i][0].daytime for i in hours)
    want, want_state = _step(scene, plan, hours, static=False)
    got, got_state = _step(scene, plan, hours, static=True)
    for k, (w, g) in enumerate(zip(want, got)):
        for name in PLANES:
            np.testing.assert_allclose(g[name], w[name], rtol=0, atol=ATOL, equal_nan=True,
                                       err_msg=f"call {k}: {name}")
    for name in want_state:
        np.testing.assert_allclose(got_state[name], want_state[name], rtol=0, atol=ATOL,
                                   err_msg=f"state {name}")


def test_static_scratch_rejects_large_tiles():
    """A tile above the static capacity fails with SOLWEIG_ERR_INVALID before
    any CUDA call (so this runs without a GPU)."""
    from solweig_cuda_b200 import _lib
    L = _lib.lib()
    s = _lib.SolweigScene()
    s.rows, s.cols = 513, 512
    assert s.rows * s.cols > _lib.STATIC_SCRATCH_MAX_PIXELS
    rc = L.solweig_step_static_scratch(ctypes.byref(s), None, None, 0, None, None, None, 1, 22, None)
    assert rc == 1
    msg = L.solweig_last_error().decode()
    assert "exceeds the static scratch capacity of 262144 pixels" in msg
