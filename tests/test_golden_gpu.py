"""The CUDA path against the reference's own CUDA stages.

Same fixture as test_golden_oracle.py (tests/golden/ref_stages.npz: the
reference's outputs on a seeded 3-burst scene).  Each stage is called through
the reference-compatible C ABI with the inputs the reference got; then the
whole device-resident pipeline runs on the fixture's SLCs and DEM windows and
every output is compared with the reference's chained outputs.  Bounds are
the task's tolerances: offsets 1e-4 px, resampled SLC 1e-4 relative complex
RMS, ESD shift 1e-5 px, coherence 1e-5 (on pixels whose box touches no pad;
the reference's CoherenceEst pads are uninitialised).
"""
import numpy as np
import pytest

from golden_io import load, swath_info
from test_golden_oracle import (G, H, L, NB, W, WINDOWS, esd_bands, geo_args, interior,
                                poly_grid, rs_kwargs)
from conftest import rel_rms

pytestmark = pytest.mark.gpu

OFF_TOL, RS_TOL, ESD_TOL, COH_TOL = 1e-4, 1e-4, 1e-5, 1e-5


@pytest.mark.parametrize("b", range(NB))
def test_geocoreg_matches_reference(T, b):
    a = geo_args(b)
    az, rg = T.geocoreg_warp(G[f"dem{b}"], a["lat0"], a["lon0"], a["dlat"], a["dlon"], a["xmin"],
                             a["xmax"], a["ymin"], a["ymax"], b, b, L, a["dt"],
                             a["first_line_time"], a["slr_time"], a["range_spacing"],
                             (G["m_sv"][0], G["s_sv"][0]), a["coefs"], a["azi_init"], W)
    daz = np.abs(poly_grid(az, b) - poly_grid(G["cpm_az"][b], b)).max()
    drg = np.abs(poly_grid(rg, b) - poly_grid(G["cpm_rg"][b], b)).max()
    assert daz < OFF_TOL and drg < OFF_TOL, (daz, drg)


@pytest.mark.parametrize("b", range(NB))
def test_resample_matches_reference(T, b):
    s_dt, m_dt = G["s_reals"][0], G["m_reals"][0]
    cases = [("reslave", 0.0, s_dt)]
    if b > 0:
        cases.append(("reslave_esd_24x6", G["esd_shift_24x6"][b - 1], m_dt))
    for key, shift, dt in cases:
        ref = G[key][b]
        kw = rs_kwargs(b, shift, dt)
        gpu = T.deramp_demod_resample(**kw)
        assert rel_rms(gpu, ref) < RS_TOL, (key, rel_rms(gpu, ref))
        assert np.array_equal(gpu == 0, ref == 0)


@pytest.mark.parametrize("wr,wa", WINDOWS)
def test_esd_matches_reference(T, wr, wa):
    mF, mB, sF, sB, ov = esd_bands(G["reslave"])
    gpu = T.est_esd_shifts(mF, mB, sF, sB, ov, wa, wr, 0.3, float(H["m_spec_sep"]),
                           float(G["m_reals"][0]))
    ref = G[f"esd_shift_{wr}x{wa}"]
    assert np.abs(gpu - ref).max() < ESD_TOL, (gpu, ref)


@pytest.mark.parametrize("wr,wa", WINDOWS)
def test_coherence_matches_reference(T, wr, wa):
    """Burst 0 through CoherenceEst_ESD, later bursts through CoherenceEst,
    as the reference's driver calls them (Func.cpp:2653-2702)."""
    inner = interior(wr, wa)
    for b in range(NB):
        sl = np.ascontiguousarray(G[f"reslave_esd_{wr}x{wa}"][b])
        d = T.resample_first_burst(sl)
        gpu = T.coherence_est(G["master_slc"][b * L:(b + 1) * L], d, wr, wa,
                              esd_variant=(b == 0))
        err = np.abs(gpu - G[f"coh_{wr}x{wa}"][b])[inner].max()
        assert err < COH_TOL, (b, err)


def _dem_canvas():
    """The per-burst DEM windows of the fixture placed on one grid, with
    their offsets (the pipeline takes one DEM and a window per burst)."""
    dlat, dlon = G["dem_geo0"][2], G["dem_geo0"][3]
    offs = []
    for b in range(NB):
        lat0, lon0 = G[f"dem_geo{b}"][:2]
        offs.append((int(round((G["dem_geo0"][0] - lat0) / dlat)),
                     int(round((lon0 - G["dem_geo0"][1]) / dlon))))
    r_min = min(r for r, _ in offs)
    c_min = min(c for _, c in offs)
    rows = max(r - r_min + G[f"dem{b}"].shape[0] for b, (r, _) in enumerate(offs))
    cols = max(c - c_min + G[f"dem{b}"].shape[1] for b, (_, c) in enumerate(offs))
    dem = np.full((rows, cols), -32768.0, np.float32)
    wins = []
    for b, (r, c) in enumerate(offs):
        d = G[f"dem{b}"]
        r0, c0 = r - r_min, c - c_min
        dem[r0:r0 + d.shape[0], c0:c0 + d.shape[1]] = d
        wins.append((r0, c0, d.shape[0], d.shape[1]))
    lat0 = G["dem_geo0"][0] - r_min * dlat
    lon0 = G["dem_geo0"][1] + c_min * dlon
    return dem, lat0, lon0, dlat, dlon, wins


@pytest.mark.parametrize("wr,wa", WINDOWS)
@pytest.mark.parametrize("precision", ["split", "fp64"])
def test_pipeline_matches_reference(T, wr, wa, precision):
    m = swath_info(T, H, "m")
    s = swath_info(T, H, "s")
    dem, lat0, lon0, dlat, dlon, wins = _dem_canvas()
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
        daz = np.abs(poly_grid(out["cpm"][b, :6], b) - poly_grid(G["cpm_az"][b], b)).max()
        drg = np.abs(poly_grid(out["cpm"][b, 6:], b) - poly_grid(G["cpm_rg"][b], b)).max()
        assert daz < OFF_TOL and drg < OFF_TOL, (b, daz, drg)
    assert np.abs(out["shifts"] - G[f"esd_shift_{wr}x{wa}"]).max() < ESD_TOL
    inner = interior(wr, wa)
    for b in range(NB):
        rows = slice(b * L, (b + 1) * L)
        assert rel_rms(out["reslave"][rows], G["reslave"][b]) < RS_TOL
        assert rel_rms(out["reslave_esd"][rows], G[f"reslave_esd_{wr}x{wa}"][b]) < RS_TOL
        err = np.abs(out["coh"][rows] - G[f"coh_{wr}x{wa}"][b])[inner].max()
        assert err < COH_TOL, (b, err)
