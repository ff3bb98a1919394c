"""The CUDA path against the reference's own CUDA stages.

Same fixtures as test_golden_oracle.py (tests/golden/ref_stages{,2}.npz: the
reference's outputs on two seeded scenes of 3 and 4 bursts).  Each stage is
called through the reference-compatible C ABI with the inputs the reference
got; then the whole device-resident pipeline runs on the fixture's SLCs and
DEM windows and every output is compared with the reference's chained
outputs.  Bounds are the task's tolerances: offsets 1e-4 px, resampled SLC
1e-4 relative complex RMS, ESD shift 1e-5 px, coherence 1e-5 (on pixels whose
box touches no pad; the reference's CoherenceEst pads are uninitialised).
"""
import numpy as np
import pytest

from golden_io import SCENES, WINDOWS, scene, scene_bursts, swath_info
from conftest import rel_rms

pytestmark = pytest.mark.gpu

OFF_TOL, RS_TOL, ESD_TOL, COH_TOL = 1e-4, 1e-4, 1e-5, 1e-5


@pytest.mark.parametrize("sfx,b", scene_bursts())
def test_geocoreg_matches_reference(T, sfx, b):
    S = scene(sfx)
    G, L, W = S.G, S.L, S.W
    a = S.geo_args(b)
    az, rg = T.geocoreg_warp(G[f"dem{b}"], a["lat0"], a["lon0"], a["dlat"], a["dlon"], a["xmin"],
                             a["xmax"], a["ymin"], a["ymax"], b, b, L, a["dt"],
                             a["first_line_time"], a["slr_time"], a["range_spacing"],
                             (G["m_sv"][0], G["s_sv"][0]), a["coefs"], a["azi_init"], W)
    daz = np.abs(S.poly_grid(az, b) - S.poly_grid(G["cpm_az"][b], b)).max()
    drg = np.abs(S.poly_grid(rg, b) - S.poly_grid(G["cpm_rg"][b], b)).max()
    assert daz < OFF_TOL and drg < OFF_TOL, (daz, drg)


@pytest.mark.parametrize("sfx,b", scene_bursts())
def test_resample_matches_reference(T, sfx, b):
    S = scene(sfx)
    for key, shift, dt in S.resample_cases(b):
        ref = S.G[key][b]
        gpu = T.deramp_demod_resample(**S.rs_kwargs(b, shift, dt))
        assert rel_rms(gpu, ref) < RS_TOL, (key, rel_rms(gpu, ref))
        assert np.array_equal(gpu == 0, ref == 0)


@pytest.mark.parametrize("sfx", SCENES)
@pytest.mark.parametrize("wr,wa", WINDOWS)
def test_esd_matches_reference(T, sfx, wr, wa):
    S = scene(sfx)
    mF, mB, sF, sB, ov = S.esd_bands(S.G["reslave"])
    gpu = T.est_esd_shifts(mF, mB, sF, sB, ov, wa, wr, 0.3, float(S.H["m_spec_sep"]),
                           float(S.G["m_reals"][0]))
    ref = S.G[f"esd_shift_{wr}x{wa}"]
    assert np.abs(gpu - ref).max() < ESD_TOL, (gpu, ref)


@pytest.mark.parametrize("sfx", SCENES)
@pytest.mark.parametrize("wr,wa", WINDOWS)
def test_coherence_matches_reference(T, sfx, wr, wa):
    """Burst 0 through CoherenceEst_ESD, later bursts through CoherenceEst,
    as the reference's driver calls them (Func.cpp:2653-2702)."""
    S = scene(sfx)
    G, L = S.G, S.L
    inner = S.interior(wr, wa)
    for b in range(S.NB):
        sl = np.ascontiguousarray(G[f"reslave_esd_{wr}x{wa}"][b])
        d = T.resample_first_burst(sl)
        gpu = T.coherence_est(G["master_slc"][b * L:(b + 1) * L], d, wr, wa,
                              esd_variant=(b == 0))
        err = np.abs(gpu - G[f"coh_{wr}x{wa}"][b])[inner].max()
        assert err < COH_TOL, (b, err)


@pytest.mark.parametrize("sfx", SCENES)
@pytest.mark.parametrize("wr,wa", WINDOWS)
@pytest.mark.parametrize("precision", ["split", "fp64"])
def test_pipeline_matches_reference(T, sfx, wr, wa, precision):
    S = scene(sfx)
    G, H, NB, L = S.G, S.H, S.NB, S.L
    m = swath_info(T, H, "m")
    s = swath_info(T, H, "s")
    dem, lat0, lon0, dlat, dlon, wins = S.dem_canvas()
    opts = T.pair_opts(win_rg=wr, win_az=wa,
                       precision=T.PREC_SPLIT if precision == "split" else T.PREC_FP64)
    P = T.Pair(m, s, dem.shape, opts)
    w = (T.DemWindow * NB)(*[T.DemWindow(*x) for x in wins])
    P.set_dem(dem, lat0, lon0, dlat, dlon, w)
    ms = np.ascontiguousarray(G["master_slc"])
    ss = np.ascontiguousarray(G["slave_slc"])
    P.upload(ms, ss)
    P.run(graph=True)
    out = P.download()
    P.close()
    for b in range(NB):
        daz = np.abs(S.poly_grid(out["cpm"][b, :6], b) - S.poly_grid(G["cpm_az"][b], b)).max()
        drg = np.abs(S.poly_grid(out["cpm"][b, 6:], b) - S.poly_grid(G["cpm_rg"][b], b)).max()
        assert daz < OFF_TOL and drg < OFF_TOL, (b, daz, drg)
    assert np.abs(out["shifts"] - G[f"esd_shift_{wr}x{wa}"]).max() < ESD_TOL
    inner = S.interior(wr, wa)
    for b in range(NB):
        rows = slice(b * L, (b + 1) * L)
        assert rel_rms(out["reslave"][rows], G["reslave"][b]) < RS_TOL
        assert rel_rms(out["reslave_esd"][rows], G[f"reslave_esd_{wr}x{wa}"][b]) < RS_TOL
        err = np.abs(out["coh"][rows] - G[f"coh_{wr}x{wa}"][b])[inner].max()
        assert err < COH_TOL, (b, err)
