"""GPU tests of the burst-pair pipeline (tops_pipeline.h).

The device-resident plan is checked end to end against the oracle chain
(geocoreg -> resample -> ESD -> shifted resample -> coherence), and its
forms against each other: CUDA-graph replay == eager launches, overlap-band
dataflow == full ReSlave dataflow, and the reference-shaped plain per-burst
form == the batched form (bit-for-bit)."""
import numpy as np
import pytest

from conftest import c64, rel_rms

pytestmark = pytest.mark.gpu


def run_pair(T, S, dem=None, graph=False, **opts):
    o = T.pair_opts(**opts)
    di = S.dem_info
    dem = S.dem if dem is None else dem
    P = T.Pair(S.swath[0], S.swath[1], dem.shape, o)
    P.set_dem(dem, di.lat0, di.lon0, di.dlat, di.dlon, T.scene_windows(S))
    P.upload(S.slc[0], S.slc[1])
    P.run(graph=graph)
    out = P.download(reslave=bool(o.reslave_full))
    out["launches"] = P.buffers().n_launches
    P.close()
    return out


def oracle_chain(O, S, win_rg=10, win_az=3, thr=0.3):
    nb, L, W = S.cfg.n_bursts, S.cfg.lines_per_burst, S.cfg.samples_per_burst
    m, s = S.swath
    cpm, rs, re = [], [], []
    d = S.deramp[1]
    for b in range(nb):
        g = S.geo_args(b)
        az, rg, st, _ = O.geocoreg(g["dem"], g["lat0"], g["lon0"], g["dlat"], g["dlon"], g["xmin"],
                                   g["xmax"], g["ymin"], g["ymax"], g["dt"], g["first_line_time"],
                                   g["slr_time"], g["range_spacing"], g["mid_time"],
                                   g["azi_init"], g["line_offset"], g["coefs"])
        assert st == 0
        cpm.append(np.concatenate([az, rg]))
    kw = lambda b, sh, dt: dict(slave=S.burst(1, b), cpm_az=cpm[b][:6], cpm_rg=cpm[b][6:],
                                az_shift=sh, kaz=S.kaz, krg=S.krg, s_burst_idx=b,
                                mbox=S.boxes(b)[0], sbox=S.boxes(b)[1], lines_per_burst=L, dt=dt,
                                kt=d["kt"][0], tref=d["tref"][0], fdc=d["dc"][0])
    for b in range(nb):
        rs.append(O.resample(**kw(b, 0.0, s.dt))[0])
    ov, _, _ = O.overlap_size(np.array(m.burst_first_line_time[:nb]),
                              np.array(m.burst_last_line_time[:nb]), m.dt)
    mF = np.concatenate([S.slc[0][(i + 1) * L - ov[i]:(i + 1) * L] for i in range(nb - 1)])
    mB = np.concatenate([S.slc[0][(i + 1) * L:(i + 1) * L + ov[i]] for i in range(nb - 1)])
    sF = c64(np.concatenate([rs[i][L - ov[i]:] for i in range(nb - 1)]))
    sB = c64(np.concatenate([rs[i + 1][:ov[i]] for i in range(nb - 1)]))
    ss = O.spectral_sep(S.deramp[0]["kt"], L, m.dt)
    shifts, _, _ = O.esd(mF, mB, sF, sB, ov, win_az, win_rg, thr, ss, m.dt)
    shifts = np.where(np.abs(shifts) > 100, 0.0, shifts)
    for b in range(nb):
        re.append(rs[0] if b == 0 else O.resample(**kw(b, shifts[b - 1], m.dt))[0])
    return dict(cpm=np.array(cpm), reslave=np.concatenate(rs), reslave_esd=np.concatenate(re),
                shifts=shifts)


def test_pipeline_vs_oracle(T, O, scene_esd):
    S = scene_esd
    gpu = run_pair(T, S)
    ref = oracle_chain(O, S)
    nb, L, W = S.cfg.n_bursts, S.cfg.lines_per_burst, S.cfg.samples_per_burst
    # offsets: polynomials evaluated over each burst box
    y = np.linspace(-2, 2, 21)
    Lh, Ph = np.meshgrid(y, y, indexing="ij")
    A = np.stack([np.ones_like(Lh), Lh, Ph, Lh * Lh, Lh * Ph, Ph * Ph], -1)
    assert np.abs(A @ gpu["cpm"][:, :6].T - A @ ref["cpm"][:, :6].T).max() < 1e-4
    assert np.abs(A @ gpu["cpm"][:, 6:].T - A @ ref["cpm"][:, 6:].T).max() < 1e-4
    assert rel_rms(gpu["reslave"], ref["reslave"]) < 1e-4
    assert np.abs(gpu["shifts"] - ref["shifts"]).max() < 1e-5
    assert rel_rms(gpu["reslave_esd"], ref["reslave_esd"]) < 1e-4
    coh_ref = O.coherence(S.slc[0][:L], c64(ref["reslave_esd"][:L]), 10, 3)
    assert np.abs(gpu["coh"][:L] - coh_ref).max() < 1e-4
    for b in range(1, nb):
        sl = slice(b * L, (b + 1) * L)
        coh_ref = O.coherence(S.slc[0][sl], c64(ref["reslave_esd"][sl]), 10, 3)
        assert np.abs(gpu["coh"][sl] - coh_ref).max() < 1e-4
    # known answers: high coherence, ESD sees the injected 0.05-line shift
    assert gpu["coh"][:, 20:-20].mean() > 0.9
    expect = -0.05 * (L - S.cfg.overlap_lines - 1) / L
    assert np.all(np.abs(gpu["shifts"] - expect) < 0.01)


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
