"""GPU tests of the burst-pair pipeline (tops_pipeline.h).

The device-resident plan is checked end to end against the oracle chain
(geocoreg -> resample -> ESD -> shifted resample -> coherence), and its
forms against each other: CUDA-graph replay == eager launches, overlap-band
dataflow == full ReSlave dataflow, and the reference-shaped plain per-burst
form == the batched form (bit-for-bit)."""
import numpy as np
import pytest

from chain import (TOL_ESD_PX, TOL_OFFSETS_PX, TOL_SLC_REL_RMS, check_burst_parity,
                   oracle_chain, run_pair)
from conftest import rel_rms

pytestmark = pytest.mark.gpu


def test_pipeline_vs_oracle(T, O, scene_esd):
    S = scene_esd
    gpu = run_pair(T, S)
    ref = oracle_chain(O, S, coherence=True)
    nb, L, W = S.cfg.n_bursts, S.cfg.lines_per_burst, S.cfg.samples_per_burst
    # offsets: polynomials evaluated over each burst box
    y = np.linspace(-2, 2, 21)
    Lh, Ph = np.meshgrid(y, y, indexing="ij")
    A = np.stack([np.ones_like(Lh), Lh, Ph, Lh * Lh, Lh * Ph, Ph * Ph], -1)
    assert np.abs(A @ gpu["cpm"][:, :6].T - A @ ref["cpm"][:, :6].T).max() < TOL_OFFSETS_PX
    assert np.abs(A @ gpu["cpm"][:, 6:].T - A @ ref["cpm"][:, 6:].T).max() < TOL_OFFSETS_PX
    assert rel_rms(gpu["reslave"], ref["reslave"]) < TOL_SLC_REL_RMS
    assert np.abs(gpu["shifts"] - ref["shifts"]).max() < TOL_ESD_PX
    assert rel_rms(gpu["reslave_esd"], ref["reslave_esd"]) < TOL_SLC_REL_RMS
    # coherence within 1e-5 of the oracle's, but for boxes holding a pixel
    # whose kernel bin flips (the LUT-bin rule of chain.py)
    for b in range(nb):
        check_burst_parity(S, gpu, ref, b)
    # known answers: high coherence, ESD sees the injected 0.05-line shift
    assert gpu["coh"][:, 20:-20].mean() > 0.9
    expect = -0.05 * (L - S.cfg.overlap_lines - 1) / L
    assert np.all(np.abs(gpu["shifts"] - expect) < 0.01)


def test_compensated_sums_vs_oracle(T, O, scene_esd):
    """tops_pair_opts.compensated: Kahan-compensated ESD phasor sums and
    pairwise coherence window sums, at the same tolerances against the FP64
    oracle chain; the option changes no resampling before ESD (ReSlave equal
    to the default plan's bit for bit)."""
    S = scene_esd
    gpu = run_pair(T, S, compensated=1)
    ref = oracle_chain(O, S, coherence=True)
    assert np.abs(gpu["shifts"] - ref["shifts"]).max() < TOL_ESD_PX
    for b in range(S.cfg.n_bursts):
        check_burst_parity(S, gpu, ref, b)
    plain = run_pair(T, S)
    assert np.array_equal(gpu["reslave"], plain["reslave"])
    assert np.abs(gpu["shifts"] - plain["shifts"]).max() < 1e-9


def test_pipeline_graph_equals_eager(T, scene_small):
    a = run_pair(T, scene_small)
    b = run_pair(T, scene_small, graph=True)
    for k in ("reslave", "reslave_esd", "coh", "cpm", "shifts"):
        assert np.array_equal(a[k], b[k]), k


def test_pipeline_overlap_bands_only(T, scene_esd):
    a = run_pair(T, scene_esd)
    b = run_pair(T, scene_esd, reslave_full=0)
    for k in ("reslave_esd", "coh", "cpm", "shifts"):
        assert np.array_equal(a[k], b[k]), k
    # the first burst's ReSlaveESD is its ReSlave: copied in a, resampled with
    # the slave's interval in b
    L = scene_esd.swath[0].lines_per_burst
    assert np.array_equal(a["reslave_esd"][:L], a["reslave"][:L])


@pytest.mark.parametrize("graph", [False, True])
def test_coherence_overlap_equals_one_launch(T, scene_esd, graph):
    """coh_overlap: each chunk's coherence on a second stream right after its
    ReSlaveESD resample gives the one-launch outputs bit for bit, eager and
    captured in a CUDA graph."""
    a = run_pair(T, scene_esd)
    b = run_pair(T, scene_esd, graph=graph, coh_overlap=1)
    for k in ("reslave", "reslave_esd", "coh", "cpm", "shifts"):
        assert np.array_equal(a[k], b[k]), k
    # up to 3 chunks of bursts, each a resample launch (none for a chunk that
    # holds only the copied first burst) and a coherence launch
    n = scene_esd.cfg.n_bursts
    per = (n + 2) // 3
    chunks = -(-n // per)
    extra = (chunks - (1 if per == 1 else 0)) + chunks - 2
    assert b["launches"] == a["launches"] + extra


def test_plain_form_equals_pipeline(T, scene_esd):
    S = scene_esd
    dem_int = np.rint(S.dem).astype(np.int32)
    plain = T.plain_pair(S, dem_int=dem_int)
    pipe = run_pair(T, S, dem=dem_int.astype(np.float32))
    for k in ("cpm", "shifts", "reslave", "reslave_esd", "coh"):
        assert np.array_equal(plain[k], pipe[k]), k


def test_pipeline_reference_window(T, O, scene_small):
    """The reference's own 24 x 6 window and per-burst deramp rows."""
    a = run_pair(T, scene_small, win_rg=24, win_az=6, burst0_deramp_rows=0)
    assert a["coh"].mean() > 0.8


@pytest.mark.parametrize("reslave_full", [1, 0])
def test_process_equals_upload_run_download(T, scene_esd, reslave_full):
    """The pipelined host-to-host call (per-burst copies beside the kernels,
    per-overlap ESD) gives the batched run's outputs bit for bit, and a
    second call on the same plan the same again."""
    S = scene_esd
    a = run_pair(T, S, reslave_full=reslave_full)
    o = T.pair_opts(reslave_full=reslave_full)
    di = S.dem_info
    P = T.Pair(S.swath[0], S.swath[1], S.dem.shape, o)
    P.set_dem(S.dem, di.lat0, di.lon0, di.dlat, di.dlon, T.scene_windows(S))
    for _ in range(2):
        b = P.process(S.slc[0], S.slc[1], reslave=bool(reslave_full))
        for k in ("reslave_esd", "coh", "cpm", "shifts") + (("reslave",) if reslave_full else ()):
            assert np.array_equal(a[k], b[k]), k
    P.close()
