"""Host-side logic of the series driver: forcing grouping, tile windows and the
bounded output writer's failure handling (failures injected on the host)."""
import os
import threading

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_load_meteorology_groups_days():
    from solweig_cuda_b200 import series
    met = np.load(os.path.join(GOLD, "sun.npz"))["met_dublin"]
    m = series.load_meteorology(met)
    assert [d.date for d in m.days] == ["2025-06-01", "2025-06-02"]
    assert all(len(d.values) == 24 for d in m.days)
    assert m.timestep_minutes == 60.0
    assert not m.values.flags.writeable


def test_tile_windows_cover_the_raster():
    from solweig_cuda_b200 import tiling
    t = tiling.tile_windows(50, 70, core=20, halo=6)
    assert len(t) == 3 * 4
    cover = np.zeros((50, 70), int)
    for w in t:
        col, row, cw, ch = w["core_window"]
        cover[row:row + ch, col:col + cw] += 1
        r0, c0, nr, nc = w["output_core"]
        left, top, iw, ih = w["input_window"]
        assert (top + r0, left + c0, nr, nc) == (row, col, ch, cw)
        assert 0 <= left and left + iw <= 70 and 0 <= top and top + ih <= 50
    assert (cover == 1).all()


def test_output_writer_surfaces_worker_failures():
    from solweig_cuda_b200.series import OutputWriter
    w = OutputWriter(enabled=True, max_inflight=1)
    done = threading.Event()
    w.submit(lambda: (_ for _ in ()).throw(OSError("disk full")))
    w.submit(done.set)  # skipped after a failure
    with pytest.raises(RuntimeError, match="output writer failed"):
        w.finish()
    assert not done.is_set()


def test_output_writer_sync_mode_runs_inline():
    from solweig_cuda_b200.series import OutputWriter
    out = []
    w = OutputWriter(enabled=False)
    w.submit(lambda: out.append(1))
    w.finish()
    assert out == [1]


def test_bad_forcing_and_raster_shapes_are_rejected():
    from solweig_cuda_b200 import series
    with pytest.raises(Exception):
        series.load_meteorology(np.zeros((3, 2)))  # fewer than 4 columns
    from solweig_cuda_b200 import engine
    with pytest.raises((ValueError, RuntimeError)):
        engine.Scene(np.zeros((10, 10)), np.zeros((10, 11)), np.zeros((10, 10)))
