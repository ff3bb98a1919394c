"""The oracle against the reference's own CUDA stages (pinning).

tests/golden/ref_stages.npz holds a seeded 3-burst scene (128 x 256 bursts,
24-line overlaps) and what the reference's GeoCoreg_warp_cuda,
DerampDemodResample(_ESD), EstESDShifts and CoherenceEst(_ESD) returned for
it on a B200, chained as the reference's stage drivers chain them
(tests/golden/make_golden.py).  Measured agreement (the bounds below leave
margin): geocoreg 2e-10 px; resample with the reference's FP32 phase storage
emulated 1e-7 relative RMS, FP64 phase 1.4e-6; ESD 2e-9 px; coherence 1.5e-6.
"""
import numpy as np
import pytest

from conftest import c64, rel_rms
from golden_io import load

G = load("ref_stages.npz")
H = load("ref_host.npz")
NB, L, W, _ = (int(v) for v in G["m_ints"])
WINDOWS = ((24, 6), (10, 3))


def poly_grid(c, b):
    y = np.linspace(b * L, (b + 1) * L - 1, 31)
    x = np.linspace(0, W - 1, 41)
    Y, X = np.meshgrid(y, x, indexing="ij")
    Lh = (Y - (b * L + 0.5 * (L - 1))) / (0.25 * (L - 1))
    Ph = (X - 0.5 * (W - 1)) / (0.25 * (W - 1))
    return c[0] + c[1] * Lh + c[2] * Ph + c[3] * Lh * Lh + c[4] * Lh * Ph + c[5] * Ph * Ph


def geo_args(b):
    lat0, lon0, dlat, dlon = G[f"dem_geo{b}"]
    mr, sr = G["m_reals"], G["s_reals"]
    mf, ml = G["m_burst_first"][b], G["m_burst_last"][b]
    sf, sl = G["s_burst_first"][b], G["s_burst_last"][b]
    mt, st = G["m_sv"][0], G["s_sv"][0]
    return dict(lat0=lat0, lon0=lon0, dlat=dlat, dlon=dlon, xmin=0, xmax=W - 1, ymin=b * L,
                ymax=(b + 1) * L - 1, dt=(mr[0], sr[0]), first_line_time=(mf, sf),
                slr_time=(mr[2], sr[2]), range_spacing=(mr[3], sr[3]),
                mid_time=(mt[len(mt) // 2], st[len(st) // 2]),
                azi_init=(0.5 * (mf + ml), 0.5 * (sf + sl)), line_offset=(b * L, b * L),
                coefs=[[H[f"{t}_c{a}"] for a in "xyz"] for t in ("m", "s")])


def rs_kwargs(b, shift, dt):
    box = np.array([0, W - 1, b * L, (b + 1) * L - 1], np.int32)
    return dict(slave=G["slave_slc"][b * L:(b + 1) * L], cpm_az=G["cpm_az"][b],
                cpm_rg=G["cpm_rg"][b], az_shift=float(shift), kaz=H["lut_kaz"],
                krg=H["lut_krg"], s_burst_idx=b, mbox=box, sbox=box.copy(), lines_per_burst=L,
                dt=float(dt), kt=H["s_kt"][0], tref=H["s_tref"][0], fdc=H["s_dc"][0])


def esd_bands(reslave):
    ov = H["m_ov"]
    ms = G["master_slc"]
    mF = np.concatenate([ms[(i + 1) * L - ov[i]:(i + 1) * L] for i in range(NB - 1)])
    mB = np.concatenate([ms[(i + 1) * L:(i + 1) * L + ov[i]] for i in range(NB - 1)])
    sF = np.concatenate([reslave[i][L - ov[i]:] for i in range(NB - 1)])
    sB = np.concatenate([reslave[i + 1][:ov[i]] for i in range(NB - 1)])
    return mF, mB, sF, sB, ov


def interior(wr, wa):
    """Pixels whose coherence box touches no pad (the reference's pads of
    CoherenceEst are uninitialised device memory, EstCoh.cu:793-797)."""
    dx, dy = (wr - 1) // 2, (wa - 1) // 2
    return slice(dy, L - (wa - 1 - dy)), slice(dx, W - (wr - 1 - dx))


@pytest.mark.parametrize("b", range(NB))
def test_oracle_geocoreg_matches_reference(O, b):
    a = geo_args(b)
    dem = G[f"dem{b}"].astype(np.float32)
    az, rg, st, nv = O.geocoreg(dem, **a)
    assert st == 0 and nv > 100
    daz = np.abs(poly_grid(az, b) - poly_grid(G["cpm_az"][b], b)).max()
    drg = np.abs(poly_grid(rg, b) - poly_grid(G["cpm_rg"][b], b)).max()
    assert daz < 1e-6 and drg < 1e-6, (daz, drg)


@pytest.mark.parametrize("b", range(NB))
def test_oracle_resample_matches_reference(O, b):
    """ReSlave (slave dt, no shift) and, after the first burst, ReSlaveESD
    (master dt, shift of the overlap before the burst)."""
    s_dt, m_dt = G["s_reals"][0], G["m_reals"][0]
    cases = [("reslave", 0.0, s_dt)]
    if b > 0:
        cases.append(("reslave_esd_24x6", G["esd_shift_24x6"][b - 1], m_dt))
    for key, shift, dt in cases:
        ref = G[key][b]
        kw = rs_kwargs(b, shift, dt)
        o32, cnt = O.resample(f32_phase=True, **kw)
        o64, _ = O.resample(**kw)
        assert cnt[0] > 0 and cnt[1] > 0 and cnt[2] > 0.8 * ref.size   # all three regions
        assert rel_rms(o32, ref) < 1e-6, (key, rel_rms(o32, ref))
        assert rel_rms(o64, ref) < 1e-4, (key, rel_rms(o64, ref))
        assert np.array_equal(ref == 0, o64 == 0)


@pytest.mark.parametrize("wr,wa", WINDOWS)
def test_oracle_esd_matches_reference(O, wr, wa):
    mF, mB, sF, sB, ov = esd_bands(G["reslave"])
    shift, _, used = O.esd(mF, mB, c64(sF), c64(sB), ov, wa, wr, 0.3, float(H["m_spec_sep"]),
                           float(G["m_reals"][0]))
    ref = G[f"esd_shift_{wr}x{wa}"]
    assert np.all(used > 0.9 * ov * W)
    assert np.abs(shift - ref).max() < 1e-6, (shift, ref)


@pytest.mark.parametrize("wr,wa", WINDOWS)
def test_oracle_coherence_matches_reference(O, wr, wa):
    inner = interior(wr, wa)
    for b in range(NB):
        ref = G[f"coh_{wr}x{wa}"][b]
        sl = G[f"reslave_esd_{wr}x{wa}"][b]
        oc = O.coherence(G["master_slc"][b * L:(b + 1) * L], c64(sl), wr, wa)
        err = np.abs(oc - ref)[inner].max()
        assert err < 1e-5, (b, err)
