"""tops_esd_static: the ESD entry point that allocates no device memory.

Some callers cannot call cudaMalloc -- code that runs inside an HBM budget
it does not own, or loops where the allocator's implicit synchronisation is
not allowed.  tops_esd_static keeps its scratch in a static device array of
the library.  This checks it against tops_esd (caller-provided scratch) on
calls in a row with changing inputs, and that requests larger than the
static array are refused.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ESD_TOL = 1e-5   # pixels, as the other ESD parity tests


def _overlaps(T, S, torch):
    nb, L, W = S.cfg.n_bursts, S.cfg.lines_per_burst, S.cfg.samples_per_burst
    m = S.swath[0]
    ov, _, _ = T.overlap_size(np.array(m.burst_first_line_time[:nb]),
                              np.array(m.burst_last_line_time[:nb]), m.dt)
    master = torch.from_numpy(S.slc[0]).cuda()
    slave = torch.from_numpy(S.slc[1].astype(np.float32)).cuda()   # complex64 stand-in
    ss = T.spectral_sep(S.deramp[0]["kt"], L, m.dt)
    arr = (T.EsdOverlap * (nb - 1))()
    for i in range(nb - 1):
        f, b = (i + 1) * L - int(ov[i]), (i + 1) * L
        e = arr[i]
        e.mF = master.data_ptr() + f * W * 4
        e.mB = master.data_ptr() + b * W * 4
        e.m_pitch = W * 4
        e.sF = slave.data_ptr() + f * W * 8
        e.sB = slave.data_ptr() + b * W * 8
        e.s_pitch = W * 8
        e.lines, e.pixels = int(ov[i]), W
        e.spec_sep, e.dt = ss, m.dt
    return arr, nb - 1, (master, slave)


def _esd(T, torch, fn, arr, n, scratch=None, nbytes=0):
    """Shifts and (re, im) sums of one ESD call on the current stream."""
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
    sums = torch.full((2 * n,), float("nan"), dtype=torch.float64, device="cuda")
    if fn == "tops_esd":
        st = T.lib.tops_esd(arr, n, 3, 10, C.c_float(0.3), C.c_void_p(out.data_ptr()),
                            C.c_void_p(sums.data_ptr()), C.c_void_p(scratch.data_ptr()), nbytes,
                            C.c_void_p(stream))
    else:
        st = T.lib.tops_esd_static(arr, n, 3, 10, C.c_float(0.3), C.c_void_p(out.data_ptr()),
                                   C.c_void_p(sums.data_ptr()), C.c_void_p(stream))
    T.check(st, fn)
    torch.cuda.synchronize()
    return out.cpu().numpy(), sums.cpu().numpy()


def test_esd_static_matches_esd(T, scene_esd, scene_small):
    """Three calls in a row on two different inputs (A, B, A): each result
    is compared with tops_esd on its own input, so a result left over in the
    shared static array from the call before would be caught."""
    import torch
    inputs, refs = [], []
    for S in (scene_esd, scene_small):
        arr, n, keep = _overlaps(T, S, torch)
        nbytes = T.lib.tops_esd_scratch_bytes(arr, n)
        assert nbytes > 0
        scratch = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        refs.append(_esd(T, torch, "tops_esd", arr, n, scratch, nbytes))
        inputs.append((arr, n, keep))
    # the two inputs give different answers, so a stale result cannot pass
    assert refs[0][0].shape != refs[1][0].shape or np.any(refs[0][0] != refs[1][0])
    for call, k in enumerate((0, 1, 0)):
        arr, n, _ = inputs[k]
        a, sums = _esd(T, torch, "tops_esd_static", arr, n)
        r, r_sums = refs[k]
        assert np.all(np.isfinite(a)), (call, a)
        assert np.abs(a - r).max() <= ESD_TOL, (call, a, r)
        assert np.array_equal(sums, r_sums), call


def test_esd_static_rejects_oversized_request(T, scene_esd):
    import torch
    arr, n, keep = _overlaps(T, scene_esd, torch)
    big = (T.EsdOverlap * 1)()
    big[0] = arr[0]
    big[0].pixels = 224 * 200           # 200 strips
    big[0].lines = 32 * 200             # x 200 segments = 40000 partial sums
    big[0].m_pitch = big[0].pixels * 4
    big[0].s_pitch = big[0].pixels * 8
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = T.lib.tops_esd_static(big, 1, 3, 10, C.c_float(0.3), C.c_void_p(out.data_ptr()), None,
                               C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == T.TOPS_E_INVALID
