"""Batched sub-swath pairs (tops_batch) and the per-burst launch loop.

Three small pairs with different burst sizes -- like the three sub-swaths of
a product -- run as one batch (one launch per stage for all bursts), with
the grid-sized and the persistent work-queue kernels, and each pair also runs
alone and through the per-burst launch loop.  With the same tiles the outputs
are bit-identical (the per-item work does not depend on which launch or CTA
runs it); other tiles move the ring window and with it the deramp reference
column, so they agree to FP32 rounding.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_rms

pytestmark = pytest.mark.gpu

SHAPES = [dict(n_bursts=2, lines_per_burst=200, samples_per_burst=512, overlap_lines=20,
               dem_lines=160, dem_pixels=160, seed=31),
          dict(n_bursts=3, lines_per_burst=180, samples_per_burst=384, overlap_lines=18,
               dem_lines=160, dem_pixels=160, seed=32),
          dict(n_bursts=2, lines_per_burst=240, samples_per_burst=640, overlap_lines=24,
               dem_lines=192, dem_pixels=192, seed=33)]


@pytest.fixture(scope="module")
def scenes(T):
    return [T.Scene(**s) for s in SHAPES]


def _plan(T, S, opts=None):
    P = T.Pair(S.swath[0], S.swath[1], S.dem.shape, opts)
    di = S.dem_info
    P.set_dem(S.dem, di.lat0, di.lon0, di.dlat, di.dlon, T.scene_windows(S))
    P.upload(S.slc[0], S.slc[1])
    return P


def _outputs(P):
    return P.download()


def _same(a, b):
    for k in ("reslave", "reslave_esd", "coh", "cpm", "shifts"):
        assert np.array_equal(a[k], b[k]), k


def test_batch_equals_single_pairs(T, scenes):
    alone = []
    for S in scenes:
        P = _plan(T, S)
        P.run()
        alone.append(_outputs(P))
        P.close()
    plans = [_plan(T, S) for S in scenes]
    B = T.Batch(plans)
    B.run(graph=True)
    # 2 geocoreg + 2 resample + 2 ESD + 1 coherence launches for all 7 bursts,
    # and 1 copy of the 3 first bursts' ReSlave into ReSlaveESD
    assert B.launches() == 8
    for P, ref in zip(plans, alone):
        _same(_outputs(P), ref)
    B.close()


def test_persistent_queue_equals_grid_launch(T, scenes):
    plans = [_plan(T, S) for S in scenes]
    B = T.Batch(plans)
    B.run()
    ref = [_outputs(P) for P in plans]
    B.tune(T.Tune(252, 1, 128, 1))
    B.run(graph=True)
    for P, r in zip(plans, ref):
        _same(_outputs(P), r)
    B.close()


def test_per_burst_loop_equals_batched(T, scenes):
    S = scenes[1]
    P = _plan(T, S)
    P.run()
    ref = _outputs(P)
    P.run_per_burst()
    _same(_outputs(P), ref)
    P.close()


def test_autotune_picks_a_valid_tile(T, scenes):
    plans = [_plan(T, S) for S in scenes]
    B = T.Batch(plans)
    B.run()
    ref = [_outputs(P) for P in plans]
    best, ms = B.autotune()
    assert best.rs_seg_rows in (84, 168, 252) and best.rs_persistent in (0, 1)
    assert best.coh_seg_rows in (64, 128, 256, 512) and best.coh_persistent in (0, 1)
    assert np.all(ms > 0)
    t = B.tune()
    assert (t.rs_seg_rows, t.coh_seg_rows) == (best.rs_seg_rows, best.coh_seg_rows)
    B.run(graph=True)
    for P, r in zip(plans, ref):
        o = _outputs(P)
        assert rel_rms(o["reslave_esd"], r["reslave_esd"]) < 1e-6
        assert np.abs(o["coh"] - r["coh"]).max() < 1e-5
        assert np.abs(o["shifts"] - r["shifts"]).max() < 1e-6
    B.close()


def test_batch_rejects_mixed_options(T, scenes):
    a = _plan(T, scenes[0])
    b = _plan(T, scenes[1], T.pair_opts(win_rg=24, win_az=6))
    arr = (C.c_void_p * 2)(a._h.value, b._h.value)
    h = C.c_void_p()
    assert T.lib.tops_batch_create(arr, 2, C.byref(h)) == T.TOPS_E_INVALID
    arr = (C.c_void_p * 2)(a._h.value, a._h.value)
    assert T.lib.tops_batch_create(arr, 2, C.byref(h)) == T.TOPS_E_INVALID
