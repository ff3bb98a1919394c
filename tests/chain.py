"""Shared helpers of the pipeline parity tests: the device plan run through
topsb200.Pair, the FP64 oracle chain the reference's drivers define
(geocoreg -> resample -> ESD -> shifted resample -> coherence), and the
LUT-bin rule that bounds where the two may differ beyond the coherence
tolerance.

The LUT-bin rule.  The resample takes the interpolation kernel of a pixel
from the bin int(frac(pos) * 2047 + 0.5) of its FP64 azimuth and range
positions (DerampAndResample.cu:108-112).  The bin is a step function of the
position: when the GPU's offset polynomial or ESD shift differs from the
oracle's by d px (1e-11..1e-10 here), a pixel whose position lies within
2047 * d bins of a step takes the neighbouring kernel, and its resampled
value moves by about 1e-3 of the amplitude -- within the SLC's relative RMS
tolerance, but enough to move the coherence of the boxes that contain it by
more than 1e-5.  Any implementation whose positions differ from the
reference's in the 11th digit does the same.  `bin_flip_mask` flags those
pixels from the oracle's positions and the measured position difference;
the tests require every larger-than-tolerance difference to lie on a flagged
pixel (ReSlaveESD) or in the box of one (coherence), and bound their count.
"""
import numpy as np

from conftest import c64

TOL_OFFSETS_PX = 1e-4
TOL_SLC_REL_RMS = 1e-4
TOL_ESD_PX = 1e-5
TOL_COH_ABS = 1e-5
# ReSlaveESD pixels whose kernel bin differs from the oracle's: at most this
# many per 1e7 output pixels (measured: about one)
MAX_FLIPS_PER_1E7 = 5
# a flipped pixel moves by ~1e-3 of the RMS amplitude; other pixels stay
# below ~2e-5 of it
FLIP_ERR_OVER_RMS = 1e-4


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


def oracle_chain(O, S, win_rg=10, win_az=3, thr=0.3, coherence=False):
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
    out = dict(cpm=np.array(cpm), reslave=np.concatenate(rs), reslave_esd=np.concatenate(re),
               shifts=shifts)
    if coherence:
        out["coh"] = np.concatenate(
            [O.coherence(S.burst(0, b), c64(re[b]), win_rg, win_az) for b in range(nb)])
    return out


def poly_grid(c, box):
    """An offset polynomial on a 31 x 41 grid over the burst box (y0..y1,
    x0..x1), with the reference's normalisation (cuConstants.cuh:53-65)."""
    ymin, ymax, xmin, xmax = box
    y = np.linspace(ymin, ymax, 31)
    x = np.linspace(xmin, xmax, 41)
    Y, X = np.meshgrid(y, x, indexing="ij")
    Lh = (Y - 0.5 * (ymin + ymax)) / (0.25 * (ymax - ymin))
    Ph = (X - 0.5 * (xmin + xmax)) / (0.25 * (xmax - xmin))
    return c[0] + c[1] * Lh + c[2] * Ph + c[3] * Lh * Lh + c[4] * Lh * Ph + c[5] * Ph * Ph


def positions(c, mbox, shift=0.0):
    """FP64 slave position of every output pixel of a burst's master box
    [x0, x1, y0, y1] (full-image lines): polynomial + shift."""
    x0, x1, y0, y1 = (float(v) for v in mbox)
    Lh = ((np.arange(int(y0), int(y1) + 1, dtype=np.float64) - 0.5 * (y0 + y1)) /
          (0.25 * (y1 - y0)))[:, None]
    Ph = ((np.arange(int(x0), int(x1) + 1, dtype=np.float64) - 0.5 * (x0 + x1)) /
          (0.25 * (x1 - x0)))[None, :]
    return c[0] + c[1] * Lh + c[2] * Ph + c[3] * Lh * Lh + c[4] * Lh * Ph + c[5] * Ph * Ph + shift


def bin_margin(pos):
    """Distance, in LUT bins, of each position to the nearest step of its
    kernel bin int(frac * 2047 + 0.5)."""
    u = (pos - np.trunc(pos)) * 2047.0 + 0.5
    return np.abs(u - np.rint(u))


def bin_flip_mask(ref_pos, gpu_pos):
    """Pixels whose bin may differ between the two positions: within the
    position difference (x 1.5, + 1e-12 px of evaluation-order rounding) of
    a bin step, in LUT-bin units."""
    d = 1.5 * 2047.0 * (np.abs(gpu_pos - ref_pos) + 1e-12)
    return bin_margin(ref_pos) <= d


def dilate(mask, rows, cols):
    """Every pixel within +-rows / +-cols of a set pixel."""
    def shift_or(m, k, axis):
        out = m.copy()
        n = m.shape[axis]
        for d in range(1, k + 1):
            if d >= n:
                break
            lo = [slice(None)] * 2
            hi = [slice(None)] * 2
            lo[axis], hi[axis] = slice(0, n - d), slice(d, n)
            out[tuple(lo)] |= m[tuple(hi)]
            out[tuple(hi)] |= m[tuple(lo)]
        return out
    return shift_or(shift_or(mask, rows, 0), cols, 1)


def check_burst_parity(S, gpu, ref, b, win_rg=10, win_az=3):
    """ReSlaveESD and coherence of burst b of a pair at the tolerances, with
    the LUT-bin rule for the pixels beyond them.  Returns a summary dict."""
    L = S.cfg.lines_per_burst
    sl = slice(b * L, (b + 1) * L)
    mb = S.boxes(b)[0]
    sh_r = 0.0 if b == 0 else float(ref["shifts"][b - 1])
    sh_g = 0.0 if b == 0 else float(gpu["shifts"][b - 1])
    flips = np.zeros((L, S.cfg.samples_per_burst), bool)
    for k in (0, 1):   # azimuth, range
        cr, cg = ref["cpm"][b, 6 * k:6 * k + 6], gpu["cpm"][b, 6 * k:6 * k + 6]
        pr = positions(cr, mb, sh_r if k == 0 else 0.0)
        pg = positions(cg, mb, sh_g if k == 0 else 0.0)
        flips |= bin_flip_mask(pr, pg)
    re_g, re_r = gpu["reslave_esd"][sl], ref["reslave_esd"][sl]
    rms = float(np.sqrt(np.mean(np.abs(re_r) ** 2)))
    err = np.abs(re_g - re_r) / rms
    big = err > FLIP_ERR_OVER_RMS
    assert not np.any(big & ~flips), ("ReSlaveESD differs off the bin steps", b,
                                      np.argwhere(big & ~flips)[:5], float(err.max()))
    n = err.size
    assert big.sum() <= max(1, int(np.ceil(MAX_FLIPS_PER_1E7 * n / 1e7))), (b, int(big.sum()))
    dc = np.abs(gpu["coh"][sl] - ref["coh"][sl])
    allowed = dilate(big, (win_az - 1) // 2 + 1, win_rg // 2 + 1)
    assert not np.any((dc > TOL_COH_ABS) & ~allowed), (
        "coherence differs outside the boxes of flipped pixels", b,
        np.argwhere((dc > TOL_COH_ABS) & ~allowed)[:5], float(dc.max()))
    return {"flipped": int(big.sum()), "coh_above_tol": int((dc > TOL_COH_ABS).sum()),
            "coh_max": float(dc.max()), "coh_max_off_flips": float(dc[~allowed].max()),
            "reslave_esd_max_err_over_rms": float(err.max())}
