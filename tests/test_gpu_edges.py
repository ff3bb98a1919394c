"""Edge cases on the GPU: images smaller than the coherence window, ESD
windows without a compile-time kernel (the generic path), a one-burst pair
(no overlap, so no ESD), and stage calls with nothing to do."""
import ctypes as C

import numpy as np
import pytest

from conftest import c64, rel_rms
from test_gpu_stages import _esd_bands

pytestmark = pytest.mark.gpu
COH_TOL, ESD_TOL, RS_TOL = 1e-5, 1e-5, 1e-4


@pytest.mark.parametrize("shape", [(1, 1), (5, 3), (7, 40), (40, 7)])
@pytest.mark.parametrize("win", [(10, 3), (24, 6), (3, 1)])
def test_coherence_image_smaller_than_window(T, O, shape, win):
    rng = np.random.default_rng(shape[0] * 100 + shape[1] + win[0])
    h, w = shape
    m = rng.integers(-900, 900, (h, w, 2), dtype=np.int16)
    s = (rng.standard_normal((h, w, 2)) * 500).astype(np.float32)
    d = T.resample_first_burst(s.view(np.complex64).reshape(h, w))
    gpu = T.coherence_est(m, d, *win)
    ref = O.coherence(m, s, *win)
    assert gpu.shape == (h, w)
    assert np.abs(gpu - ref).max() < COH_TOL


# (az, rg): windows without a compile-time kernel.  A 1 x 1 window is no
# parity case: every pixel's coherence is 1 up to rounding, and the mask
# drops coherences >= 1 (MaskOut, EstESD.cu:130-161), so which pixels count
# depends on the last bit of each implementation's arithmetic.
@pytest.mark.parametrize("win", [(2, 7), (1, 3), (5, 31)])
def test_esd_generic_windows(T, O, scene_esd, win):
    S = scene_esd
    mF, mB, sF, sB, ov, ss, dt = _esd_bands(O, S)
    waz, wrg = win
    ref, _, _ = O.esd(mF, mB, sF, sB, ov, waz, wrg, 0.3, ss, dt)
    gpu = T.est_esd_shifts(mF, mB, sF.view(np.complex64)[..., 0], sB.view(np.complex64)[..., 0],
                           ov, waz, wrg, 0.3, ss, dt)
    assert np.abs(gpu - ref).max() < ESD_TOL, (win, gpu, ref)


def test_single_burst_pair(T, O, scene_esd):
    """One burst: nothing overlaps, so no ESD; ReSlaveESD is the uncorrected
    ReSlave and the coherence is that of master and ReSlave."""
    S = scene_esd
    m, s = T.sub_swath(S.swath[0], 1, 1), T.sub_swath(S.swath[1], 1, 1)
    P = T.Pair(m, s, S.dem.shape, T.pair_opts())
    di = S.dem_info
    P.set_dem(S.dem, di.lat0, di.lon0, di.dlat, di.dlon,
              (T.DemWindow * 1)(T.DemWindow(*S.dem_window(1))))
    L = S.cfg.lines_per_burst
    P.upload(np.ascontiguousarray(S.slc[0][L:2 * L]), np.ascontiguousarray(S.slc[1][L:2 * L]))
    P.run()
    out = P.download()
    P.close()
    assert len(out["shifts"]) == 0
    assert np.array_equal(out["reslave_esd"], out["reslave"])
    ref = O.coherence(S.slc[0][L:2 * L], c64(out["reslave"].astype(np.complex128)), 10, 3)
    assert np.abs(out["coh"] - ref).max() < COH_TOL
    assert rel_rms(out["reslave"], out["reslave_esd"]) == 0.0


def test_empty_calls_do_nothing(T):
    """Zero jobs, zero overlaps and zero rows are accepted and launch nothing."""
    assert T.lib.tops_coherence(None, 0, 10, 3, None) == T.TOPS_OK
    assert T.lib.tops_geocoreg(None, 0, None, 0, None) == T.TOPS_OK
    assert T.lib.tops_stitch(C.c_void_p(16), 64, C.c_void_p(16), 64, C.c_void_p(16), 0, 64,
                             None) == T.TOPS_OK
