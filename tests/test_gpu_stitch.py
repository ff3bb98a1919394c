"""Debursting row gather on the GPU (tops_stitch): dst row i = src row
map[i], byte for byte, for CInt16, float and complex64 rows with aligned
(16-byte vector) and unaligned (4-byte) bases and pitches, and on the
device-resident pipeline's coherence and ReSlaveESD."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _gather(T, src, dst, map_dev, height, row_bytes):
    T.check(T.lib.tops_stitch(C.c_void_p(src.data_ptr()), src.stride(0) * src.element_size(),
                              C.c_void_p(dst.data_ptr()), dst.stride(0) * dst.element_size(),
                              C.c_void_p(map_dev.data_ptr()), height, row_bytes, None),
            "tops_stitch")
    torch.cuda.synchronize()


@pytest.mark.parametrize("elem", [4, 8])          # CInt16 / float rows, complex64 rows
@pytest.mark.parametrize("aligned", [True, False])
def test_row_gather(T, elem, aligned):
    rng = np.random.default_rng(elem + 10 * aligned)
    rows, W = 700, 1000 if aligned else 997
    words = W * elem // 4
    base = torch.from_numpy(rng.integers(-2**31, 2**31 - 1, (rows, words + 8),
                                         dtype=np.int64).astype(np.int32)).cuda()
    off = 0 if aligned else 1
    src = base[:, off:off + words]                 # unaligned: base + 4 bytes, odd pitch
    m = np.sort(rng.choice(rows, 550, replace=False)).astype(np.int32)
    m_dev = torch.from_numpy(m).cuda()
    dst_base = torch.zeros((550, words + 8), dtype=torch.int32, device="cuda")
    dst = dst_base[:, off:off + words]
    _gather(T, src, dst, m_dev, len(m), words * 4)
    assert torch.equal(dst, src[m_dev.long()])
    # the columns beside the rows are untouched
    assert int(dst_base[:, :off].abs().sum()) == 0 and int(dst_base[:, off + words:].abs().sum()) == 0


def test_stitch_pipeline_outputs(T, scene_esd):
    S = scene_esd
    nb, L, W = S.cfg.n_bursts, S.cfg.lines_per_burst, S.cfg.samples_per_burst
    di = S.dem_info
    P = T.Pair(S.swath[0], S.swath[1], S.dem.shape, T.pair_opts())
    P.set_dem(S.dem, di.lat0, di.lon0, di.dlat, di.dlon, T.scene_windows(S))
    P.upload(S.slc[0], S.slc[1])
    P.run()
    out = P.download()
    fv, lv = np.full(nb, 7, np.int32), np.full(nb, L - 9, np.int32)
    m = T.stitch_line_map(S.swath[0], fv, lv, 0, nb - 1)
    # the reference truncates the first and last output line indices
    # separately (Func.cpp:2834-2835), so the last line may stop one short
    assert np.all(np.diff(m) > 0) and m[0] == fv[0]
    assert (nb - 1) * L + lv[-1] - 1 <= m[-1] <= (nb - 1) * L + lv[-1]
    m_dev = torch.from_numpy(m).cuda()
    B = P.buffers()
    for src_ptr, pitch, row_bytes, ref, dtype in (
            (B.coh, B.coh_pitch, W * 4, out["coh"], torch.float32),
            (B.reslave_esd, B.cplx_pitch, W * 8, out["reslave_esd"], torch.complex64)):
        dst = torch.empty((len(m), W), dtype=dtype, device="cuda")
        T.check(T.lib.tops_stitch(C.c_void_p(src_ptr), pitch, C.c_void_p(dst.data_ptr()),
                                  W * dst.element_size(), C.c_void_p(m_dev.data_ptr()), len(m),
                                  row_bytes, None), "tops_stitch")
        torch.cuda.synchronize()
        assert np.array_equal(dst.cpu().numpy(), ref[m])
    P.close()
