"""GPU parity of the four stages through the reference-compatible C ABI.

Each test runs the CUDA path (libtops_b200.so) and the FP64 oracle on the
same seeded synthetic inputs and compares at the tolerances of the task:
resampled SLC within 1e-4 relative complex RMS, coherence within 1e-5
absolute, ESD shift within 1e-5 px, offsets within 1e-4 px.
"""
import numpy as np
import pytest

from conftest import c64, rel_rms

pytestmark = pytest.mark.gpu

RS_TOL = 1e-4      # relative complex RMS of the resampled SLC
COH_TOL = 1e-5     # absolute coherence
ESD_TOL = 1e-5     # pixels
OFF_TOL = 1e-4     # pixels


def oracle_cpm(O, S, b):
    g = S.geo_args(b)
    az, rg, st, nv = O.geocoreg(g["dem"], g["lat0"], g["lon0"], g["dlat"], g["dlon"], g["xmin"],
                                g["xmax"], g["ymin"], g["ymax"], g["dt"], g["first_line_time"],
                                g["slr_time"], g["range_spacing"], g["mid_time"], g["azi_init"],
                                g["line_offset"], g["coefs"])
    assert st == 0 and nv > 100
    return az, rg


def rs_inputs(S, b, cpm, shift=0.0):
    mb, sb = S.boxes(b)
    d = S.deramp[1]
    L = S.cfg.lines_per_burst
    # the reference passes the burst-0 rows for every burst (Func.cpp:2383)
    return dict(slave=S.burst(1, b), cpm_az=cpm[0], cpm_rg=cpm[1], az_shift=shift, kaz=S.kaz,
                krg=S.krg, s_burst_idx=b, mbox=mb, sbox=sb, lines_per_burst=L, dt=S.swath[1].dt,
                kt=d["kt"][0], tref=d["tref"][0], fdc=d["dc"][0])


@pytest.mark.parametrize("b,shift", [(0, 0.0), (1, 0.0), (1, 0.0371)])
def test_resample_parity(T, O, scene_small, b, shift):
    S = scene_small
    cpm = oracle_cpm(O, S, b)
    kw = rs_inputs(S, b, cpm, shift)
    gpu = T.deramp_demod_resample(**kw)
    ref, cnt = O.resample(**kw)
    assert cnt[2] > 0.9 * ref.size
    err = rel_rms(gpu, ref)
    assert err < RS_TOL, err


def test_resample_regions(T, O, scene_small):
    """Polynomial pushing the grid off the slave box: outside -> 0, edge ->
    the nearest sample, interior -> interpolated (DerampAndResample.cu:383-404)."""
    S = scene_small
    az, rg = oracle_cpm(O, S, 0)
    az = az.copy()
    rg = rg.copy()
    az[0] += 120.0   # shift down by 120 lines and right by 200 samples
    rg[0] += 200.0
    kw = rs_inputs(S, 0, (az, rg))
    gpu = T.deramp_demod_resample(**kw)
    ref, cnt = O.resample(**kw)
    assert cnt[0] > 1000 and cnt[1] > 1000 and cnt[2] > 1000
    assert rel_rms(gpu, ref) < RS_TOL
    zero = np.abs(ref) == 0
    assert np.all(gpu[zero] == 0)


def test_resample_nonuniform_bins(T, O, scene_small):
    """Azimuth offset varying quickly across range: the LUT bin changes
    inside row segments, exercising the per-pixel paths."""
    S = scene_small
    az, rg = oracle_cpm(O, S, 1)
    az = az.copy()
    az[2] += 0.9      # ~1.8 lines across the burst width
    az[5] += 0.35
    kw = rs_inputs(S, 1, (az, rg))
    gpu = T.deramp_demod_resample(**kw)
    ref, _ = O.resample(**kw)
    assert rel_rms(gpu, ref) < RS_TOL


def test_resample_steep_polynomial(T, O, scene_small):
    """Strongly rotated/scaled mapping: ring window misses, HBM fallback."""
    S = scene_small
    az, rg = oracle_cpm(O, S, 0)
    az = az.copy()
    rg = rg.copy()
    az[2] += 25.0     # azimuth position moves 50 lines across the width
    rg[1] += 12.0     # range position moves 24 samples along azimuth
    kw = rs_inputs(S, 0, (az, rg))
    gpu = T.deramp_demod_resample(**kw)
    ref, cnt = O.resample(**kw)
    assert rel_rms(gpu, ref) < RS_TOL


@pytest.mark.parametrize("prec", ["split", "fp64"])
def test_resample_azimuth_scale(T, O, scene_small, prec):
    """An azimuth scale of 1.01 lines per row: the row-to-line map skips a
    line every ~100 rows, so rows inside a group leave the register window's
    line (their sums are formed directly from the staged lines), and the LUT
    bin changes every row (more bins per item than the tap table holds).
    Against the FP64 oracle, and row subsets bit for bit."""
    S = scene_small
    az, rg = oracle_cpm(O, S, 1)
    az = np.array(az, np.float64)
    az[1] *= 1.01
    kw = rs_inputs(S, 1, (az, rg), 0.02)
    mode = T.PREC_SPLIT if prec == "split" else T.PREC_FP64
    gpu = _resample_device(T, kw, mode)
    ref, _ = O.resample(**kw)
    assert rel_rms(gpu, ref) < RS_TOL
    for r0, n in ((95, 30), (13, 250)):
        part = _resample_device(T, kw, mode, rows=(r0, n))
        bad = np.argwhere(part != gpu[r0:r0 + n])
        assert bad.size == 0, (r0, n, bad[:8].tolist(), bad.shape[0])


def _resample_device(T, kw, precision, out_offset=0, slave_offset=0, rows=None):
    """tops_resample_ex on device buffers; out_offset / slave_offset (bytes)
    misalign the output and slave bases to force the scalar-access paths;
    rows = (row0, n) produces only master rows row0 .. row0 + n - 1."""
    import ctypes as C
    import torch
    slave = np.ascontiguousarray(kw["slave"], np.int16)
    L, W = slave.shape[0], slave.shape[1]
    s_dev = torch.zeros(slave.nbytes + 64, dtype=torch.uint8, device="cuda")
    s_dev[slave_offset:slave_offset + slave.nbytes].copy_(
        torch.from_numpy(slave.view(np.uint8).reshape(-1)))
    o_dev = torch.zeros(L * W * 8 + 64, dtype=torch.uint8, device="cuda")
    par = [torch.from_numpy(np.ascontiguousarray(kw[k], np.float64)).cuda()
           for k in ("kt", "tref", "fdc")]
    lut = C.c_void_p()
    kaz = np.ascontiguousarray(kw["kaz"], np.float32)
    krg = np.ascontiguousarray(kw["krg"], np.float32)
    T.check(T.lib.tops_lut_create(T.ptr(kaz, C.c_float), T.ptr(krg, C.c_float), C.byref(lut)),
            "lut")
    j = T.ResampleJob()
    j.slave, j.slave_pitch = s_dev.data_ptr() + slave_offset, W * 4
    j.out, j.out_pitch = o_dev.data_ptr() + out_offset, W * 8
    j.kt, j.tref, j.fdc = (t.data_ptr() for t in par)
    for i in range(4):
        j.mbox[i], j.sbox[i] = int(kw["mbox"][i]), int(kw["sbox"][i])
    for i in range(6):
        j.cpm_az[i], j.cpm_rg[i] = kw["cpm_az"][i], kw["cpm_rg"][i]
    j.az_shift = kw["az_shift"]
    j.s_first_line = kw["s_burst_idx"] * kw["lines_per_burst"]
    j.dt = kw["dt"]
    j.out_row0, j.out_rows = (0, -1) if rows is None else rows
    stream = torch.cuda.current_stream().cuda_stream
    T.check(T.lib.tops_resample_ex(lut, C.byref(j), 1, precision, C.c_void_p(stream)),
            "tops_resample_ex")
    torch.cuda.synchronize()
    T.lib.tops_lut_destroy(lut)
    out = o_dev[out_offset:out_offset + L * W * 8].cpu().numpy().view(np.complex64)
    out = out.reshape(L, W)
    return out if rows is None else out[:rows[1]]


@pytest.mark.parametrize("prec", ["split", "fp64"])
def test_resample_precision_modes(T, O, scene_small, prec):
    """Both deramp-phase precisions against the FP64 oracle; the FP64 mode
    also agrees with the reference's phase sum to FP32 rounding."""
    S = scene_small
    cpm = oracle_cpm(O, S, 1)
    kw = rs_inputs(S, 1, cpm, 0.0371)
    mode = T.PREC_SPLIT if prec == "split" else T.PREC_FP64
    gpu = _resample_device(T, kw, mode)
    ref, _ = O.resample(**kw)
    err = rel_rms(gpu, ref)
    assert err < RS_TOL, err
    if prec == "fp64":
        assert err < 1e-5, err


def _two_bin_share(cpm_az, mbox, shift, strip=112):
    """Share of (row, 112-column strip) pieces whose azimuth keys are two
    adjacent LUT bins of one line."""
    from chain import positions
    y = positions(np.asarray(cpm_az), mbox, shift)
    line = np.trunc(y)
    b = np.clip(np.trunc((y - line) * 2047.0 + 0.5), 0, 2047)
    n = two = 0
    for c in range(0, y.shape[1], strip):
        bb, ll = b[:, c:c + strip], line[:, c:c + strip]
        one_line = ll.min(1) == ll.max(1)
        two += int(np.sum(one_line & (bb.max(1) - bb.min(1) == 1)))
        n += y.shape[0]
    return two / n


@pytest.mark.parametrize("prec", ["split", "fp64"])
def test_resample_two_bin_rows(T, O, scene_small, prec):
    """Rows whose strip spans two adjacent azimuth bins (here most rows: an
    azimuth offset that changes by ~1/3 of a bin per strip) take the shared
    pass with the second bin summed after the range pass: against the FP64
    oracle, and a row subset bit for bit as the whole job."""
    S = scene_small
    az, rg = oracle_cpm(O, S, 1)
    az = np.array(az, np.float64)
    az[2] += 3e-3 * S.cfg.samples_per_burst / 4096.0
    kw = rs_inputs(S, 1, (az, rg), 0.0123)
    assert _two_bin_share(az, kw["mbox"], 0.0123) > 0.3
    mode = T.PREC_SPLIT if prec == "split" else T.PREC_FP64
    gpu = _resample_device(T, kw, mode)
    ref, _ = O.resample(**kw)
    err = rel_rms(gpu, ref)
    assert err < RS_TOL, err
    for r0, n in ((123, 54), (7, 1), (250, 13)):
        part = _resample_device(T, kw, mode, rows=(r0, n))
        bad = np.argwhere(part != gpu[r0:r0 + n])
        assert bad.size == 0, (r0, n, bad[:8].tolist(), bad.shape[0])


def test_resample_unaligned_buffers(T, O, scene_small):
    """Misaligned slave / output bases take the scalar-access paths."""
    S = scene_small
    cpm = oracle_cpm(O, S, 0)
    kw = rs_inputs(S, 0, cpm)
    ref, _ = O.resample(**kw)
    a = _resample_device(T, kw, T.PREC_SPLIT, out_offset=8, slave_offset=4)
    b = _resample_device(T, kw, T.PREC_SPLIT)
    assert rel_rms(a, ref) < RS_TOL
    assert rel_rms(a, b) < 1e-6


def test_resample_deterministic(T, O, scene_small):
    S = scene_small
    cpm = oracle_cpm(O, S, 1)
    kw = rs_inputs(S, 1, cpm, 0.01)
    a = T.deramp_demod_resample(**kw)
    b = T.deramp_demod_resample(**kw)
    assert np.array_equal(a, b)


def test_coherence_parity(T, O, scene_small):
    S = scene_small
    b = 1
    cpm = oracle_cpm(O, S, b)
    kw = rs_inputs(S, b, cpm)
    ref_rs, _ = O.resample(**kw)
    slave = c64(ref_rs)
    master = S.burst(0, b)
    for win_rg, win_az in [(10, 3), (24, 6), (5, 5)]:
        d = T.resample_first_burst(slave.view(np.complex64).reshape(slave.shape[:2]))
        gpu = T.coherence_est(master, d, win_rg, win_az)
        ref = O.coherence(master, slave, win_rg, win_az)
        err = np.abs(gpu - ref).max()
        assert err < COH_TOL, (win_rg, win_az, err)
    assert ref[5:-5, 12:-12].mean() > 0.9


def test_coherence_slave_equals_master(T, O, scene_small):
    S = scene_small
    m = S.burst(0, 0)
    s = m.astype(np.float32)
    d = T.resample_first_burst(s.view(np.complex64).reshape(s.shape[:2]))
    gpu = T.coherence_est(m, d, 10, 3, esd_variant=True)
    live = np.hypot(s[..., 0], s[..., 1]) >= 1e-3
    assert np.abs(gpu[live] - 1.0).max() < 1e-5
    assert np.all(gpu[~live] == 0)


@pytest.mark.parametrize("win_rg,win_az,crop", [(10, 3, None), (10, 6, None), (24, 6, None),
                                               (24, 3, None), (10, 3, (53, 40)),
                                               (24, 6, (53, 40))])
def test_coherence_tma_equals_generic(T, scene_small, win_rg, win_az, crop):
    """The TMA-staged coherence kernel (10- and 24-sample range windows,
    16-byte aligned rows) against the generic kernel (the slave placed 8 bytes off a
    16-byte boundary takes it): the same vertical sums, the horizontal
    sliding sum restarted every 4 instead of every 8 outputs, so the two
    agree to FP32 rounding of the window sums."""
    import ctypes as C
    import torch
    S = scene_small
    m = np.ascontiguousarray(S.burst(0, 1))
    s = np.ascontiguousarray(S.burst(1, 1)).astype(np.float32)
    if crop:   # a partial strip and a segment shorter than a chunk group
        m = np.ascontiguousarray(m[:crop[0], :crop[1]])
        s = np.ascontiguousarray(s[:crop[0], :crop[1]])
    L, W = m.shape[:2]
    dm = torch.from_numpy(m.view(np.int32).reshape(L, W)).cuda()
    ds = torch.from_numpy(s).cuda()
    big = torch.zeros(L * W * 2 + 2, dtype=torch.float32, device="cuda")
    ds_off = big[2:].view(L, W, 2)
    ds_off.copy_(ds)
    assert ds.data_ptr() % 16 == 0 and ds_off.data_ptr() % 16 == 8
    out = []
    for sl in (ds, ds_off):
        coh = torch.full((L, W), -1.0, dtype=torch.float32, device="cuda")
        job = T.CohJob(master=dm.data_ptr(), master_pitch=W * 4, slave=sl.data_ptr(),
                       slave_pitch=W * 8, coh=coh.data_ptr(), coh_pitch=W * 4, lines=L, pixels=W)
        torch.cuda.synchronize()
        T.check(T.lib.tops_coherence(C.byref(job), 1, win_rg, win_az, None), "tops_coherence")
        torch.cuda.synchronize()
        out.append(coh.cpu().numpy())
    assert np.abs(out[0] - out[1]).max() < 2e-6
    assert np.all(np.isfinite(out[0])) and out[0].min() >= 0.0 and out[0].max() <= 1.0 + 1e-6


def _esd_bands(O, S, shifts=None):
    nb, L, W = S.cfg.n_bursts, S.cfg.lines_per_burst, S.cfg.samples_per_burst
    m = S.swath[0]
    ov, tot, mx = O.overlap_size(np.array(m.burst_first_line_time[:nb]),
                                 np.array(m.burst_last_line_time[:nb]), m.dt)
    res = []
    for b in range(nb):
        cpm = oracle_cpm(O, S, b)
        r, _ = O.resample(**rs_inputs(S, b, cpm))
        res.append(r)
    mF = np.concatenate([S.slc[0][(i + 1) * L - ov[i]:(i + 1) * L] for i in range(nb - 1)])
    mB = np.concatenate([S.slc[0][(i + 1) * L:(i + 1) * L + ov[i]] for i in range(nb - 1)])
    sF = np.concatenate([res[i][L - ov[i]:] for i in range(nb - 1)])
    sB = np.concatenate([res[i + 1][:ov[i]] for i in range(nb - 1)])
    ss = O.spectral_sep(S.deramp[0]["kt"], L, m.dt)
    return mF, mB, c64(sF), c64(sB), ov, ss, m.dt


def test_esd_parity_and_known_answer(T, O, scene_esd):
    S = scene_esd
    mF, mB, sF, sB, ov, ss, dt = _esd_bands(O, S)
    ref, sums, used = O.esd(mF, mB, sF, sB, ov, 3, 10, 0.3, ss, dt)
    gpu = T.est_esd_shifts(mF, mB, sF.view(np.complex64)[..., 0], sB.view(np.complex64)[..., 0],
                           ov, 3, 10, 0.3, ss, dt)
    assert np.abs(gpu - ref).max() < ESD_TOL, (gpu, ref)
    # injected misregistration of 0.05 lines, seen through the reference's
    # spectral separation (L*dt instead of the true burst cycle)
    L, o = S.cfg.lines_per_burst, S.cfg.overlap_lines
    expect = -0.05 * (L - o - 1) / L
    assert np.all(np.abs(ref - expect) < 0.01), (ref, expect)


def test_esd_reference_window(T, O, scene_esd):
    """The reference's hard-coded 24 x 6 window (Func.cpp:2583-2585)."""
    S = scene_esd
    mF, mB, sF, sB, ov, ss, dt = _esd_bands(O, S)
    ref, _, _ = O.esd(mF, mB, sF, sB, ov, 6, 24, 0.3, ss, dt)
    gpu = T.est_esd_shifts(mF, mB, sF.view(np.complex64)[..., 0], sB.view(np.complex64)[..., 0],
                           ov, 6, 24, 0.3, ss, dt)
    assert np.abs(gpu - ref).max() < ESD_TOL


def _poly_grid(c, ymin, ymax, xmin, xmax):
    y = np.linspace(ymin, ymax, 31)
    x = np.linspace(xmin, xmax, 41)
    Y, X = np.meshgrid(y, x, indexing="ij")
    Lh = (Y - 0.5 * (ymin + ymax)) / (0.25 * (ymax - ymin))
    Ph = (X - 0.5 * (xmin + xmax)) / (0.25 * (xmax - xmin))
    return c[0] + c[1] * Lh + c[2] * Ph + c[3] * Lh * Lh + c[4] * Lh * Ph + c[5] * Ph * Ph


@pytest.mark.parametrize("b", [0, 1])
def test_geocoreg_parity(T, O, scene_small, b):
    S = scene_small
    g = S.geo_args(b)
    dem_int = np.rint(g["dem"]).astype(np.int32)
    az_o, rg_o, st, nv = O.geocoreg(dem_int.astype(np.float32), g["lat0"], g["lon0"], g["dlat"],
                                    g["dlon"], g["xmin"], g["xmax"], g["ymin"], g["ymax"], g["dt"],
                                    g["first_line_time"], g["slr_time"], g["range_spacing"],
                                    g["mid_time"], g["azi_init"], g["line_offset"], g["coefs"])
    m, s = S.swath
    L = S.cfg.lines_per_burst
    az_g, rg_g = T.geocoreg_warp(
        dem_int, g["lat0"], g["lon0"], g["dlat"], g["dlon"], g["xmin"], g["xmax"], g["ymin"],
        g["ymax"], b, b, L, g["dt"], g["first_line_time"], g["slr_time"], g["range_spacing"],
        (np.array(m.sv_t[:m.n_sv]), np.array(s.sv_t[:s.n_sv])), g["coefs"], g["azi_init"],
        S.cfg.samples_per_burst)
    box = (g["ymin"], g["ymax"], g["xmin"], g["xmax"])
    daz = np.abs(_poly_grid(az_g, *box) - _poly_grid(az_o, *box)).max()
    drg = np.abs(_poly_grid(rg_g, *box) - _poly_grid(rg_o, *box)).max()
    assert daz < OFF_TOL and drg < OFF_TOL, (daz, drg)


def test_geocoreg_not_positive_definite(T, scene_small):
    """All-nodata DEM: the normal matrix is singular -> TOPS_E_NOT_PD and the
    output coefficients are left untouched (as the reference)."""
    S = scene_small
    g = S.geo_args(0)
    dem_int = np.full(g["dem"].shape, -32768, np.int32)
    m, s = S.swath
    with pytest.raises(T.TopsError) as ei:
        T.geocoreg_warp(dem_int, g["lat0"], g["lon0"], g["dlat"], g["dlon"], g["xmin"], g["xmax"],
                        g["ymin"], g["ymax"], 0, 0, S.cfg.lines_per_burst, g["dt"],
                        g["first_line_time"], g["slr_time"], g["range_spacing"],
                        (np.array(m.sv_t[:m.n_sv]), np.array(s.sv_t[:s.n_sv])), g["coefs"],
                        g["azi_init"], S.cfg.samples_per_burst)
    assert ei.value.status == T.TOPS_E_NOT_PD


@pytest.mark.parametrize("prec", ["split", "fp64"])
def test_resample_row_subset_bit_exact(T, O, scene_esd, prec):
    """A job that produces a subset of the master rows (the overlap bands of
    the band-only dataflow, or any other range) gives those rows bit for bit
    as the job over the whole burst: the kernel's choices (ring window,
    phase reference column, work items) do not depend on the row range."""
    S = scene_esd
    cpm = oracle_cpm(O, S, 1)
    kw = rs_inputs(S, 1, cpm, 0.0123)
    mode = T.PREC_SPLIT if prec == "split" else T.PREC_FP64
    full = _resample_device(T, kw, mode)
    L, ov = S.cfg.lines_per_burst, S.cfg.overlap_lines
    for r0, n in ((L - ov, ov), (0, ov), (123, 54), (7, 1)):
        part = _resample_device(T, kw, mode, rows=(r0, n))
        bad = np.argwhere(part != full[r0:r0 + n])
        assert bad.size == 0, (r0, n, bad[:8].tolist(), bad.shape[0])


def test_fp64_peak_measurement(T):
    """tops_fp64_peak: the device's FP64 FMA rate under the current clocks,
    the denominator of the geometric coregistration's roofline.  A B200 runs
    FP64 FMAs at tens of TFLOP/s; two measurements agree to a few percent."""
    a = T.fp64_peak()
    b = T.fp64_peak()
    assert 5.0 < a < 200.0 and 5.0 < b < 200.0, (a, b)
    assert abs(a - b) / max(a, b) < 0.1, (a, b)
