"""Drop-in at the link level: tests/dropin/ref_caller.cpp declares the stage
entry points exactly as the reference's host code does (Func.cpp:2163-2210,
2304-2324, 2422-2494: void returns, cuComplex* device pointers,
std::complex<short>/<float> arrays) and is linked against libtops_b200.so
with --no-undefined.  The CPU test proves every declaration resolves to the
library; the GPU test runs the reference driver's call sequence through
those declarations and compares the results with the FP64 oracle."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, PKG, c64, rel_rms

SRC = os.path.join(ROOT, "tests", "dropin", "ref_caller.cpp")
LIBDIR = os.path.join(PKG, "lib")


def build_caller(tmp_path):
    out = os.path.join(str(tmp_path), "libref_caller.so")
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", "-Werror",
           "-I/usr/local/cuda/include", SRC, "-L" + LIBDIR, "-ltops_b200",
           "-Wl,--no-undefined", "-Wl,-rpath," + LIBDIR, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


@pytest.fixture(scope="module")
def caller(tmp_path_factory, T):
    return build_caller(tmp_path_factory.mktemp("dropin"))


def test_reference_declarations_link(caller, T):
    """Every reference declaration resolves to libtops_b200.so."""
    r = subprocess.run(["nm", "-D", "--undefined-only", caller], capture_output=True, text=True)
    undef = {ln.split()[-1] for ln in r.stdout.splitlines() if ln.strip()}
    names = {"GeoCoreg_warp_cuda", "DerampDemodResample", "DerampDemodResample_ESD",
             "ResampleFirstBurst", "EstESDShifts", "CoherenceEst", "CoherenceEst_ESD"}
    assert names <= undef          # taken from outside the caller ...
    lib = C.CDLL(caller)           # ... and bound by the loader from the library
    for n in ("ref_caller_burst", "ref_caller_esd", "ref_caller_geocoreg"):
        assert hasattr(lib, n)
    for n in names:
        assert hasattr(T.lib, n)


def _grid(c, box):
    ymin, ymax, xmin, xmax = box
    y = np.linspace(ymin, ymax, 31)
    x = np.linspace(xmin, xmax, 41)
    Y, X = np.meshgrid(y, x, indexing="ij")
    Lh = (Y - 0.5 * (ymin + ymax)) / (0.25 * (ymax - ymin))
    Ph = (X - 0.5 * (xmin + xmax)) / (0.25 * (xmax - xmin))
    return c[0] + c[1] * Lh + c[2] * Ph + c[3] * Lh * Lh + c[4] * Lh * Ph + c[5] * Ph * Ph


@pytest.mark.gpu
def test_reference_call_sequence(caller, T, O, scene_small):
    """Geocoreg of both bursts, ReSlave, ESD of the overlap, the ESD-corrected
    resample kept on the device and its coherence -- all through the
    reference's declarations -- against the oracle at the parity tolerances."""
    S = scene_small
    lib = C.CDLL(caller)
    dp, fp, ip, vp = (C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int),
                      C.c_void_p)
    lib.ref_caller_burst.restype = C.c_int
    lib.ref_caller_burst.argtypes = [vp, vp, dp, dp, C.c_double, fp, fp, C.c_int, C.c_int,
                                     C.c_int, ip, ip, C.c_double, C.c_double, dp, dp, dp,
                                     C.c_int, C.c_int, C.c_int, vp, vp, fp]
    lib.ref_caller_esd.restype = None
    lib.ref_caller_esd.argtypes = [vp, vp, vp, vp, ip, dp, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_int, C.c_int, C.c_float, C.c_double, C.c_double]
    lib.ref_caller_geocoreg.restype = None
    lib.ref_caller_geocoreg.argtypes = ([C.c_int] * 6 + [C.c_double] * 2 + [C.c_int] * 2 +
                                        [dp, dp] + [C.c_double] * 7 + [C.c_int, dp, dp] +
                                        [C.c_int] * 3 + [C.c_double] * 4 + [ip] + [dp] * 6 +
                                        [C.c_double] * 2)
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))
    nb, L, W = S.cfg.n_bursts, S.cfg.lines_per_burst, S.cfg.samples_per_burst
    m, s = S.swath
    # ---- geocoreg of every burst (int DEM window, as the reference passes it)
    cpm = []
    for b in range(nb):
        g = S.geo_args(b)
        dem_int = np.ascontiguousarray(np.rint(g["dem"]).astype(np.int32))
        az_o, rg_o, st, _ = O.geocoreg(dem_int.astype(np.float32), g["lat0"], g["lon0"],
                                       g["dlat"], g["dlon"], g["xmin"], g["xmax"], g["ymin"],
                                       g["ymax"], g["dt"], g["first_line_time"], g["slr_time"],
                                       g["range_spacing"], g["mid_time"], g["azi_init"],
                                       g["line_offset"], g["coefs"])
        assert st == 0
        az, rg = np.full(6, np.nan), np.full(6, np.nan)
        mt = np.ascontiguousarray(m.sv_t[:m.n_sv], np.float64)
        stt = np.ascontiguousarray(s.sv_t[:s.n_sv], np.float64)
        (mx, my, mz), (sx, sy, sz) = [[np.ascontiguousarray(c, np.float64) for c in cc]
                                      for cc in g["coefs"]]
        assert len(mx) == len(sx)
        lib.ref_caller_geocoreg(b, b, g["xmin"], g["xmax"], g["ymin"], g["ymax"], g["dlat"],
                                g["dlon"], dem_int.shape[0], dem_int.shape[1], P(az, C.c_double),
                                P(rg, C.c_double), g["lat0"], g["lon0"], g["dt"][0], g["dt"][1],
                                float(L), g["first_line_time"][0], g["first_line_time"][1], W,
                                P(mt, C.c_double), P(stt, C.c_double), len(mt), len(stt),
                                len(mx), g["slr_time"][0], g["slr_time"][1],
                                g["range_spacing"][0], g["range_spacing"][1],
                                P(dem_int, C.c_int), P(mx, C.c_double), P(my, C.c_double),
                                P(mz, C.c_double), P(sx, C.c_double), P(sy, C.c_double),
                                P(sz, C.c_double), g["azi_init"][0], g["azi_init"][1])
        box = (g["ymin"], g["ymax"], g["xmin"], g["xmax"])
        assert np.abs(_grid(az, box) - _grid(az_o, box)).max() < 1e-4
        assert np.abs(_grid(rg, box) - _grid(rg_o, box)).max() < 1e-4
        cpm.append((az_o, rg_o))
    # ---- the oracle chain on the oracle's polynomials
    d = S.deramp[1]
    kw = lambda b, sh, dt: dict(slave=S.burst(1, b), cpm_az=cpm[b][0], cpm_rg=cpm[b][1],
                                az_shift=sh, kaz=S.kaz, krg=S.krg, s_burst_idx=b,
                                mbox=S.boxes(b)[0], sbox=S.boxes(b)[1], lines_per_burst=L, dt=dt,
                                kt=d["kt"][0], tref=d["tref"][0], fdc=d["dc"][0])
    rs = [O.resample(**kw(b, 0.0, s.dt))[0] for b in range(nb)]
    ov, _, _ = O.overlap_size(np.array(m.burst_first_line_time[:nb]),
                              np.array(m.burst_last_line_time[:nb]), m.dt)
    ov = np.ascontiguousarray(ov, np.int32)
    mF = np.ascontiguousarray(np.concatenate(
        [S.slc[0][(i + 1) * L - ov[i]:(i + 1) * L] for i in range(nb - 1)]))
    mB = np.ascontiguousarray(np.concatenate(
        [S.slc[0][(i + 1) * L:(i + 1) * L + ov[i]] for i in range(nb - 1)]))
    sF = np.ascontiguousarray(np.concatenate([rs[i][L - ov[i]:] for i in range(nb - 1)]),
                              np.complex64)
    sB = np.ascontiguousarray(np.concatenate([rs[i + 1][:ov[i]] for i in range(nb - 1)]),
                              np.complex64)
    spec = O.spectral_sep(S.deramp[0]["kt"], L, m.dt)
    shifts_o, _, _ = O.esd(mF, mB, c64(sF), c64(sB), ov, 3, 10, 0.3, spec, m.dt)
    # ---- ESD through the reference declaration
    shifts = np.full(nb - 1, np.nan)
    lib.ref_caller_esd(mF.ctypes.data, mB.ctypes.data, sF.ctypes.data, sB.ctypes.data,
                       P(ov, C.c_int), P(shifts, C.c_double), nb - 1, mF.shape[0], W, 3, 10,
                       int(ov.max()), 0.3, spec, m.dt)
    assert np.abs(shifts - shifts_o).max() < 1e-5, (shifts, shifts_o)
    # ---- per burst: ReSlave, ESD-corrected device copy, coherence
    kaz = np.ascontiguousarray(S.kaz, np.float32)
    krg = np.ascontiguousarray(S.krg, np.float32)
    kt, tref, fdc = (np.ascontiguousarray(d[k][0], np.float64) for k in ("kt", "tref", "dc"))
    for b in range(nb):
        first = int(b == 0)
        sh = 0.0 if first else float(shifts_o[b - 1])
        mb, sb = (np.ascontiguousarray(x, np.int32) for x in S.boxes(b))
        slave = np.ascontiguousarray(S.burst(1, b), np.int16)
        master = np.ascontiguousarray(S.burst(0, b), np.int16)
        az_c, rg_c = (np.ascontiguousarray(c, np.float64) for c in cpm[b])
        out_rs = np.zeros((L, W), np.complex64)
        out_re = np.zeros((L, W), np.complex64)
        coh = np.full((L, W), np.nan, np.float32)
        r = lib.ref_caller_burst(slave.ctypes.data, master.ctypes.data, P(az_c, C.c_double),
                                 P(rg_c, C.c_double), sh, P(kaz, C.c_float), P(krg, C.c_float),
                                 b, W, L, P(mb, C.c_int), P(sb, C.c_int), s.dt, m.dt,
                                 P(kt, C.c_double), P(tref, C.c_double), P(fdc, C.c_double), 10,
                                 3, first, out_rs.ctypes.data, out_re.ctypes.data,
                                 P(coh, C.c_float))
        assert r == 0
        re_o = rs[0] if first else O.resample(**kw(b, sh, m.dt))[0]
        assert rel_rms(out_rs, rs[b]) < 1e-4
        assert rel_rms(out_re, re_o) < 1e-4
        coh_o = O.coherence(master, c64(re_o), 10, 3)
        assert np.abs(coh - coh_o).max() < 1e-5
