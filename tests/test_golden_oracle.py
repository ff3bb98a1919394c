"""The oracle against the reference's own CUDA stages (pinning).

tests/golden/ref_stages{,2}.npz hold two seeded scenes (3 bursts of 128 x 256
with 24-line overlaps; 4 bursts of 160 x 300 with 30-line overlaps) and what
the reference's GeoCoreg_warp_cuda, DerampDemodResample(_ESD), EstESDShifts
and CoherenceEst(_ESD) returned for them on a B200, chained as the
reference's stage drivers chain them (tests/golden/make_golden.py).  Measured
agreement, worst over both scenes (the bounds below leave margin): geocoreg
1.5e-10 px; resample with the reference's FP32 phase storage emulated 9.4e-8
relative RMS, FP64 phase 2.1e-6; ESD 4.9e-9 px; coherence 1.5e-6.
"""
import numpy as np
import pytest

from conftest import c64, rel_rms
from golden_io import SCENES, WINDOWS, scene, scene_bursts


@pytest.mark.parametrize("sfx,b", scene_bursts())
def test_oracle_geocoreg_matches_reference(O, sfx, b):
    S = scene(sfx)
    a = S.geo_args(b)
    dem = S.G[f"dem{b}"].astype(np.float32)
    az, rg, st, nv = O.geocoreg(dem, **a)
    assert st == 0 and nv > 100
    daz = np.abs(S.poly_grid(az, b) - S.poly_grid(S.G["cpm_az"][b], b)).max()
    drg = np.abs(S.poly_grid(rg, b) - S.poly_grid(S.G["cpm_rg"][b], b)).max()
    assert daz < 1e-6 and drg < 1e-6, (daz, drg)


@pytest.mark.parametrize("sfx,b", scene_bursts())
def test_oracle_resample_matches_reference(O, sfx, b):
    S = scene(sfx)
    for key, shift, dt in S.resample_cases(b):
        ref = S.G[key][b]
        kw = S.rs_kwargs(b, shift, dt)
        o32, cnt = O.resample(f32_phase=True, **kw)
        o64, _ = O.resample(**kw)
        assert cnt[0] > 0 and cnt[1] > 0 and cnt[2] > 0.8 * ref.size   # all three regions
        assert rel_rms(o32, ref) < 1e-6, (key, rel_rms(o32, ref))
        assert rel_rms(o64, ref) < 1e-4, (key, rel_rms(o64, ref))
        assert np.array_equal(ref == 0, o64 == 0)


@pytest.mark.parametrize("sfx", SCENES)
@pytest.mark.parametrize("wr,wa", WINDOWS)
def test_oracle_esd_matches_reference(O, sfx, wr, wa):
    S = scene(sfx)
    mF, mB, sF, sB, ov = S.esd_bands(S.G["reslave"])
    shift, _, used = O.esd(mF, mB, c64(sF), c64(sB), ov, wa, wr, 0.3, float(S.H["m_spec_sep"]),
                           float(S.G["m_reals"][0]))
    ref = S.G[f"esd_shift_{wr}x{wa}"]
    assert np.all(used > 0.9 * ov * S.W)
    assert np.abs(shift - ref).max() < 1e-6, (shift, ref)


@pytest.mark.parametrize("sfx", SCENES)
@pytest.mark.parametrize("wr,wa", WINDOWS)
def test_oracle_coherence_matches_reference(O, sfx, wr, wa):
    S = scene(sfx)
    L = S.L
    inner = S.interior(wr, wa)
    for b in range(S.NB):
        ref = S.G[f"coh_{wr}x{wa}"][b]
        sl = S.G[f"reslave_esd_{wr}x{wa}"][b]
        oc = O.coherence(S.G["master_slc"][b * L:(b + 1) * L], c64(sl), wr, wa)
        err = np.abs(oc - ref)[inner].max()
        assert err < 1e-5, (b, err)
