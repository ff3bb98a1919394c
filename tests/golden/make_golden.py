#!/usr/bin/env python3
"""Golden fixtures from the reference's own code for the burst-pair path.

Test infrastructure.  The reference's host precomputes and its four CUDA
stages, built from the reference sources into oracle/_ref/ by
``make -C oracle/ref``, run on a small seeded synthetic scene; this script
stores every input they saw and what they returned:

    python tests/golden/make_golden.py host [--scene 2]   -> tests/golden/ref_host[2].npz
    python tests/golden/make_golden.py stitch          -> tests/golden/ref_stitch.npz
    python tests/golden/make_golden.py front           -> tests/golden/ref_front.npz
    python tests/golden/make_golden.py stages [--scene 2] [--out D]
                                                   -> D/ref_stages[2].npz (needs a GPU)
    python tests/golden/make_golden.py timing --scene subswath [--out D]
                                                   -> D/ref_timing_subswath.json (needs a GPU)

``timing`` is not a fixture: it times the reference's own CUDA stages, called
per burst as its drivers call them (each call copying its inputs to the device
and its outputs back), on the benchmark's full sub-swath pair, for context
beside the rebuild's numbers.

The scene comes from the product's seeded generator (tops_synth_*), but the
fixtures hold the generated arrays themselves, so the tests replay them
without regenerating anything.  The reference's entry points call
cudaDeviceReset and exit(0) on errors, so ``stages`` runs in its own process
and writes its file only after every call returned.

What each stage call gets mirrors the reference's stage drivers:
  * geocoreg: GeoCoreg_warp_cuda with the DEM window's own origin, burst gap 0
    and the whole int DEM uploaded (Func.cpp:2225-2278, Geocoreg_cuda.cu:788);
  * resample: DerampDemodResample with the slave's dt and the slave's burst-0
    deramp rows (Func.cpp:2326-2406);
  * ESD: EstESDShifts on the overlap bands (DataTypes.cpp:456-473), for the
    driver's 24 x 6 window and threshold 0.3 (Func.cpp:2583-2588) and for 10 x 3;
  * ESD resample and coherence: burst 0 through ResampleFirstBurst and
    CoherenceEst_ESD, later bursts through DerampDemodResample_ESD with the
    master's dt and the shift of the overlap before them, then CoherenceEst
    (Func.cpp:2640-2702).
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
sys.path.insert(0, os.path.join(ROOT, "insar-on-sentinel-1-tops-data_b200"))

# Scene 1: 3 bursts of 128 x 256 with 24-line overlaps.  Scene 2: 4 bursts of
# 160 x 300 with 30-line overlaps, the opposite misregistration, and a width
# that is no multiple of 16, 32 or the product's 112-column strips.  Widths
# like 300 stay inside the reference's buffers: its deramp kernel reads the
# per-column rows up to the next multiple of 16 (DerampAndResample.cu:138-140)
# and its prefix sums run over the whole row pitch (EstCoh.cu:502-521,
# EstESD.cu:1045-1056), both within the padded rows cudaMallocPitch returns,
# whose pitch the ESD driver checks to be a multiple of 32 complex samples
# (it returns no shifts otherwise; scene 2 got them).  The overlap line count
# is rounded up to a multiple of 8 before allocation (EstESD.cu:590, 950).
SCENES = {
    "1": dict(n_bursts=3, lines_per_burst=128, samples_per_burst=256, overlap_lines=24,
              dem_lines=128, dem_pixels=128, seed=23, az_shift_true=0.03),
    "2": dict(n_bursts=4, lines_per_burst=160, samples_per_burst=300, overlap_lines=30,
              dem_lines=160, dem_pixels=160, seed=29, az_shift_true=-0.04),
    # the benchmark's sub-swath pair (timing only)
    "subswath": dict(n_bursts=9, lines_per_burst=1500, samples_per_burst=21000,
                     overlap_lines=100, dem_lines=3600, dem_pixels=3600, seed=2),
}
SCENE = SCENES["1"]
DEM_MARGIN = 24
NODATA = -32768
ESD_THRESHOLD = 0.3
WINDOWS = ((24, 6), (10, 3))      # (range, azimuth): the driver's and the config's

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p


def _ptr(a, t):
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the reference must be contiguous"
    return a.ctypes.data_as(C.POINTER(t))


PAGE = 4096


def iso(a, dtype=None):
    """Copy of `a` in memory of its own: page-aligned, and no other buffer
    shares its last page.  The reference page-locks every host buffer it gets
    with cudaHostRegister and checks cudaGetLastError at the end of the call
    (exit(0) on any error), so two buffers on one page would end the process."""
    a = np.asarray(a, dtype=dtype)
    raw = np.empty(a.nbytes + 2 * PAGE, np.uint8)
    off = (-raw.ctypes.data) % PAGE
    v = raw[off:off + a.nbytes].view(a.dtype).reshape(a.shape)
    v[...] = a
    return v


def _lib(name):
    path = os.path.join(REF_DIR, name)
    if not os.path.exists(path):
        raise SystemExit(f"{path} missing: run `make -C oracle/ref` first")
    return C.CDLL(path)


# ------------------------------------------------------------------ scene
def swath_fields(info):
    """tops_swath_info -> plain arrays (what the reference reads from the annotation)."""
    nb = info.n_bursts
    return {
        "ints": np.array([nb, info.lines_per_burst, info.samples_per_burst,
                          info.first_valid_pixel], np.int64),
        "reals": np.array([info.dt, info.prf, info.slr_time, info.range_spacing, info.wavelength,
                           info.rsr, info.az_bandwidth, info.steering_rate_deg,
                           info.first_line_time, info.last_line_time], np.float64),
        "burst_first": np.array(info.burst_first_line_time[:nb], np.float64),
        "burst_last": np.array(info.burst_last_line_time[:nb], np.float64),
        "dc_list": np.array([[p.aztime, p.t0, p.c0, p.c1, p.c2] for p in info.dc_list[:info.n_dc]]),
        "fm_list": np.array([[p.aztime, p.t0, p.c0, p.c1, p.c2] for p in info.fm_list[:info.n_fm]]),
        "sv": np.array([info.sv_t[:info.n_sv], info.sv_x[:info.n_sv], info.sv_y[:info.n_sv],
                        info.sv_z[:info.n_sv]], np.float64),
    }


def make_scene():
    import topsb200 as T
    S = T.Scene(**SCENE)
    out = {}
    for w, tag in ((0, "m"), (1, "s")):
        for k, v in swath_fields(S.swath[w]).items():
            out[f"{tag}_{k}"] = v
    out["master_slc"] = np.ascontiguousarray(S.slc[0])
    out["slave_slc"] = np.ascontiguousarray(S.slc[1])
    di = S.dem_info
    for b in range(SCENE["n_bursts"]):
        r0, c0, nr, nc = S.dem_window(b, DEM_MARGIN)
        out[f"dem{b}"] = np.rint(S.dem[r0:r0 + nr, c0:c0 + nc]).astype(np.int32)
        out[f"dem_geo{b}"] = np.array([di.lat0 - r0 * di.dlat, di.lon0 + c0 * di.dlon,
                                       di.dlat, di.dlon])
    S.close()
    return out


# ------------------------------------------------------------ host part
def ref_host_outputs(F, tag, H):
    """Polyfit_Orbit, ComputeDerampPara, InKernelInit, EstOverlapSize and
    GetSpectralSep of one sub-swath, with the given DC list."""
    ints, reals = F[f"{tag}_ints"], F[f"{tag}_reals"]
    nb, L, W, fvp = (int(v) for v in ints)
    dt, prf, slr, rsp, lam, rsr, abw, steer, t_first, t_last = reals
    sv = np.ascontiguousarray(F[f"{tag}_sv"])
    t, x, y, z = (np.ascontiguousarray(v) for v in sv)
    cx, cy, cz = (np.zeros(8) for _ in range(3))
    n = H.ref_polyfit_orbit(len(t), _ptr(t, C.c_double), _ptr(x, C.c_double),
                            _ptr(y, C.c_double), _ptr(z, C.c_double), _ptr(cx, C.c_double),
                            _ptr(cy, C.c_double), _ptr(cz, C.c_double))
    cx, cy, cz = cx[:n].copy(), cy[:n].copy(), cz[:n].copy()
    res = {f"{tag}_cx": cx, f"{tag}_cy": cy, f"{tag}_cz": cz}
    for case, dcl in (("", F[f"{tag}_dc_list"]), ("_interp", F[f"{tag}_dc_list_interp"])):
        dcl = np.ascontiguousarray(dcl)
        fml = np.ascontiguousarray(F[f"{tag}_fm_list"])
        first = np.ascontiguousarray(F[f"{tag}_burst_first"])
        last = np.ascontiguousarray(F[f"{tag}_burst_last"])
        dc, fm, tref, kt = (np.zeros((nb, W)) for _ in range(4))
        st = H.ref_deramp_params(
            nb, L, W, fvp, slr, rsp, dt, t_first, t_last, steer, lam, _ptr(first, C.c_double),
            _ptr(last, C.c_double), _ptr(dcl, C.c_double), len(dcl), _ptr(fml, C.c_double),
            len(fml), _ptr(t, C.c_double), len(t), _ptr(cx, C.c_double), _ptr(cy, C.c_double),
            _ptr(cz, C.c_double), n, _ptr(dc, C.c_double), _ptr(fm, C.c_double),
            _ptr(tref, C.c_double), _ptr(kt, C.c_double))
        assert st == 0
        res.update({f"{tag}_dc{case}": dc, f"{tag}_fm{case}": fm, f"{tag}_tref{case}": tref,
                    f"{tag}_kt{case}": kt})
    first = np.ascontiguousarray(F[f"{tag}_burst_first"])
    last = np.ascontiguousarray(F[f"{tag}_burst_last"])
    ov = np.zeros(nb - 1, np.int32)
    tot, mx = C.c_int(), C.c_int()
    assert H.ref_overlap_size(nb, _ptr(first, C.c_double), _ptr(last, C.c_double), dt,
                              _ptr(ov, C.c_int), C.byref(tot), C.byref(mx)) == 0
    kt = np.ascontiguousarray(res[f"{tag}_kt"])
    res[f"{tag}_ov"] = ov
    res[f"{tag}_ov_total_max"] = np.array([tot.value, mx.value], np.int32)
    res[f"{tag}_spec_sep"] = np.array(H.ref_spectral_sep(nb, W, L, dt, _ptr(kt, C.c_double)))
    return res


# (prf, azimuth bandwidth, 2 x range sampling rate) of the extra LUT cases:
# the scene's own values are added in front
LUT_CASES = ((1717.128973878037, 327.0, 2 * 64.34523812571427e6),
             (486.486, 313.3, 2 * 64.345e6),
             (2000.0, 1000.0, 2 * 20.0e6))


def host(out_path):
    F = make_scene()
    H = _lib("libref_host.so")
    H.ref_polyfit_orbit.restype = C.c_int
    H.ref_deramp_params.restype = C.c_int
    H.ref_overlap_size.restype = C.c_int
    H.ref_spectral_sep.restype = C.c_double
    H.ref_spectral_sep.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, _dp]
    H.ref_lut.restype = C.c_int
    H.ref_lut.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, _fp, _fp]
    H.ref_deramp_params.argtypes = (
        [C.c_int] * 4 + [C.c_double] * 7 + [_dp, _dp, _dp, C.c_int, _dp, C.c_int, _dp, C.c_int,
                                            _dp, _dp, _dp, C.c_int, _dp, _dp, _dp, _dp])
    H.ref_overlap_size.argtypes = [C.c_int, _dp, _dp, C.c_double, _ip, _ip, _ip]
    H.ref_polyfit_orbit.argtypes = [C.c_int] + [_dp] * 7
    # a second DC list of exactly n_bursts estimates whose times bracket every
    # burst centre, so ComputeDerampPara interpolates (computeDC) instead of
    # copying per burst
    for tag in ("m", "s"):
        dcl = F[f"{tag}_dc_list"]
        reals = F[f"{tag}_reals"]
        nb = int(F[f"{tag}_ints"][0])
        times = np.linspace(reals[8] - 0.5, reals[9] + 0.5, nb)
        lst = np.array([dcl[k % len(dcl)] for k in range(nb)])
        lst[:, 0] = times
        lst[:, 2] += np.arange(nb) * 7.5
        F[f"{tag}_dc_list_interp"] = lst
    for tag in ("m", "s"):
        F.update(ref_host_outputs(F, tag, H))
    m_reals = F["m_reals"]
    cases = [(m_reals[1], m_reals[6], 2 * m_reals[5])] + list(LUT_CASES)
    kaz = np.zeros((len(cases), 2048, 12), np.float32)
    krg = np.zeros((len(cases), 2048, 12), np.float32)
    for i, (prf, abw, rsr2x) in enumerate(cases):
        a, r = np.zeros((2048, 12), np.float32), np.zeros((2048, 12), np.float32)
        assert H.ref_lut(12, prf, abw, rsr2x, _ptr(a, C.c_float), _ptr(r, C.c_float)) == 0
        kaz[i], krg[i] = a, r
    # the scene's tables in full (the resample fixtures use them), every case
    # as SHA-256 digests of the float32 bytes (bit-exact check)
    F["lut_params"] = np.array(cases)
    F["lut_kaz"], F["lut_krg"] = kaz[0], krg[0]
    F["lut_sha256"] = np.array([[hashlib.sha256(kaz[i].tobytes()).hexdigest(),
                                 hashlib.sha256(krg[i].tobytes()).hexdigest()]
                                for i in range(len(cases))])
    # the host fixture holds no SLC or DEM (the stage fixture does)
    keep = {k: v for k, v in F.items()
            if not (k.endswith("_slc") or k.startswith("dem"))}
    np.savez_compressed(out_path, **keep)
    print(f"wrote {out_path}: {len(keep)} arrays")


# ------------------------------------------------------------ front part
# Burst matching (ComputerBurstOverlap, Func.cpp:1610-1746) on sub-ranges of
# one synthetic 6-burst pair: (burst0, burstN) 1-based as in config.txt, and
# the scene bursts the master and the slave start at.  A slave that starts
# later than the master's burst0 takes the reference's second branch
# (Func.cpp:1685-1741).
FRONT_SCENE = dict(n_bursts=6, lines_per_burst=200, samples_per_burst=400, overlap_lines=20,
                   dem_lines=160, dem_pixels=160, seed=31)
FRONT_CASES = [(1, 6, 0, 0), (2, 5, 0, 0), (4, 6, 0, 0), (6, 6, 0, 0), (3, 6, 0, 2),
               (1, 4, 0, 2), (1, 6, 2, 0), (2, 3, 1, 3), (1, 6, 0, 3)]


class RefImage(C.Structure):
    _fields_ = [("n_bursts", C.c_int), ("lines_per_burst", C.c_int),
                ("samples_per_burst", C.c_int), ("dt", C.c_double), ("prf", C.c_double),
                ("rsr", C.c_double), ("slr_first", C.c_double), ("slr_last", C.c_double),
                ("first_line_time", C.c_double), ("last_line_time", C.c_double),
                ("burst_first_line_time", _dp), ("geo_lines", C.c_int), ("geo_points", C.c_int),
                ("az_time", _dp), ("slr_time", _dp), ("lat", _dp), ("lon", _dp),
                ("n_points", C.c_int), ("n_coef", C.c_int), ("orbit_t", _dp), ("cx", _dp),
                ("cy", _dp), ("cz", _dp)]


def sub_swath_info(info, k):
    """The sub-swath's bursts from k on (a copy; the state vectors stay)."""
    import topsb200 as T
    out = T.SwathInfo()
    C.memmove(C.byref(out), C.byref(info), C.sizeof(info))
    nb = info.n_bursts - k
    out.n_bursts = nb
    for b in range(nb):
        out.burst_first_line_time[b] = info.burst_first_line_time[b + k]
        out.burst_last_line_time[b] = info.burst_last_line_time[b + k]
    out.first_line_time = out.burst_first_line_time[0]
    out.last_line_time = out.burst_last_line_time[nb - 1]
    return out


def front(out_path):
    import topsb200 as T
    sys.path.insert(0, os.path.dirname(HERE))
    import s1_files
    H = _lib("libref_host.so")
    Fr = _lib("libref_front.so")
    H.ref_polyfit_orbit.restype = C.c_int
    H.ref_polyfit_orbit.argtypes = [C.c_int] + [_dp] * 7
    Fr.ref_burst_overlap.restype = None
    Fr.ref_burst_overlap.argtypes = [C.c_int, C.c_int, C.POINTER(RefImage), C.POINTER(RefImage),
                                     _ip]
    S = T.Scene(**FRONT_SCENE)
    out = {"cases": np.array(FRONT_CASES, np.int32)}
    keep = []

    def ref_image(info, grid):
        t, x, y, z = (np.ascontiguousarray(info_arr) for info_arr in
                      (info.sv_t[:info.n_sv], info.sv_x[:info.n_sv], info.sv_y[:info.n_sv],
                       info.sv_z[:info.n_sv]))
        cx, cy, cz = (np.zeros(8) for _ in range(3))
        n = H.ref_polyfit_orbit(len(t), _ptr(t, C.c_double), _ptr(x, C.c_double),
                                _ptr(y, C.c_double), _ptr(z, C.c_double), _ptr(cx, C.c_double),
                                _ptr(cy, C.c_double), _ptr(cz, C.c_double))
        bft = np.ascontiguousarray(info.burst_first_line_time[:info.n_bursts])
        g = {k: np.ascontiguousarray(grid[k], np.float64) for k in
             ("az_time", "slr_time", "lat", "lon")}
        keep.extend([t, cx, cy, cz, bft, *g.values()])
        slr_last = info.slr_time + (info.samples_per_burst - 1) * info.range_spacing / 299792458.0
        return RefImage(info.n_bursts, info.lines_per_burst, info.samples_per_burst, info.dt,
                        info.prf, info.rsr, info.slr_time, slr_last, info.first_line_time,
                        info.last_line_time, _ptr(bft, C.c_double), g["az_time"].shape[0],
                        g["az_time"].shape[1], _ptr(g["az_time"], C.c_double),
                        _ptr(g["slr_time"], C.c_double), _ptr(g["lat"], C.c_double),
                        _ptr(g["lon"], C.c_double), len(t), n, _ptr(t, C.c_double),
                        _ptr(cx, C.c_double), _ptr(cy, C.c_double), _ptr(cz, C.c_double))

    for i, (b0, bN, km, ks) in enumerate(FRONT_CASES):
        m = sub_swath_info(S.swath[0], km)
        sl = sub_swath_info(S.swath[1], ks)
        gm = s1_files.grid_from_scene(S, m, first_burst=km)
        gs = s1_files.grid_from_scene(S, sl, first_burst=ks)
        rm, rs = ref_image(m, gm), ref_image(sl, gs)
        res = np.full(4, -1, np.int32)
        Fr.ref_burst_overlap(b0, bN, C.byref(rm), C.byref(rs), _ptr(res, C.c_int))
        for tag, info, g in (("m", m, gm), ("s", sl, gs)):
            for k, v in swath_fields(info).items():
                out[f"c{i}_{tag}_{k}"] = v
            for k in ("az_time", "slr_time", "lat", "lon"):
                out[f"c{i}_{tag}_grid_{k}"] = g[k]
        out[f"c{i}_out"] = res
        print(f"case {i} burst {b0}..{bN} master from {km} slave from {ks}: {res.tolist()}")
    S.close()
    np.savez_compressed(out_path, **out)
    print(f"wrote {out_path}: {len(out)} arrays")


# ---------------------------------------------------------- stitch part
# Burst timings of the debursting cases: S1 IW-like (2.055 ms lines, 1500
# lines per burst, a 2.7585 s burst cycle, about 157 overlap lines), with
# per-burst valid-line margins and sub-ranges of bursts.
STITCH_CASES = [
    # n_bursts, dt, cycle, first valid, last valid, burst0, burstN, seed
    (9, 0.002055, 2.7585, 25, 1474, 0, 8, 1),
    (9, 0.002055, 2.7585, 25, 1474, 2, 5, 2),
    (9, 0.002055, 2.7585, 3, 1496, 0, 0, 3),
    (9, 0.002055, 2.7585, 60, 1440, 8, 8, 4),
    (4, 0.00205556, 2.7581, 40, 1460, 1, 3, 5),
    (3, 0.002055, 3.0824, 10, 1489, 0, 2, 6),   # bursts that just touch
]


def stitch(out_path):
    """Stitch_OneSubswath's line selection (Func.cpp:2822-2873) over the
    reference's own getLineIdxInMetaData (Func.cpp:2766-2820): yMin, yMax and
    the line times follow the reference's arithmetic (C int truncation of
    doubles); each line's row is getLineIdxInMetaData - burst0 * L."""
    H = _lib("libref_host.so")
    H.ref_line_idx.restype = C.c_int
    H.ref_line_idx.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_int, C.c_double,
                               C.c_int, C.c_int]
    out = {}
    L = 1500
    for ci, (nb, dt, cycle, fv, lv, b0, bN, seed) in enumerate(STITCH_CASES):
        rng = np.random.default_rng(seed)
        t0 = 51234.5 + rng.uniform(0, 1)
        first = t0 + cycle * np.arange(nb) + rng.uniform(-2e-4, 2e-4, nb)
        last = first + (L - 1) * dt
        fvs = np.full(nb, fv, np.int32) + rng.integers(0, 3, nb).astype(np.int32)
        lvs = np.full(nb, lv, np.int32) - rng.integers(0, 3, nb).astype(np.int32)
        first_line_time = first[0]
        t_first = first[b0] + int(fvs[b0]) * dt          # burstFirstValidLineTime (Func.cpp:401)
        t_last = first[bN] + int(lvs[bN]) * dt           # burstLastValidLineTime (Func.cpp:403)
        y_min = int((t_first - first_line_time) / dt)    # C truncation (Func.cpp:2834-2835)
        y_max = int((t_last - first_line_time) / dt)
        rows = []
        for y in range(y_min, y_max + 1):
            t = t_first + (y - y_min) * dt
            idx = H.ref_line_idx(nb, L, _ptr(first, C.c_double), _ptr(last, C.c_double), dt,
                                 nb * L, t, b0, bN)
            rows.append(idx - b0 * L if idx != -1 else -1)
        out[f"case{ci}_first"] = first
        out[f"case{ci}_last"] = last
        out[f"case{ci}_params"] = np.array([nb, L, b0, bN], np.int32)
        out[f"case{ci}_dt"] = np.array([dt, first_line_time])
        out[f"case{ci}_valid"] = np.stack([fvs, lvs])
        out[f"case{ci}_map"] = np.array(rows, np.int32)
    np.savez_compressed(out_path, **out)
    print(f"wrote {out_path}: {len(STITCH_CASES)} cases")


# ---------------------------------------------------------- stage part
def _stage_libs():
    R = _lib("libref_resample.so")
    RS_ARGS = [_vp, _dp, _dp, C.c_double, _vp, _fp, _fp, C.c_int, C.c_int, C.c_int, _ip, _ip,
               C.c_int, C.c_int, C.c_double, _dp, _dp, _dp, C.c_int]
    R.DerampDemodResample.restype = None
    R.DerampDemodResample.argtypes = RS_ARGS
    R.DerampDemodResample_ESD.restype = _vp
    R.DerampDemodResample_ESD.argtypes = RS_ARGS
    R.ResampleFirstBurst.restype = _vp
    R.ResampleFirstBurst.argtypes = [_vp, C.c_int, C.c_int]
    Co = _lib("libref_coherence.so")
    for f in (Co.CoherenceEst, Co.CoherenceEst_ESD):
        f.restype = None
        f.argtypes = [C.c_int] * 8 + [_vp, _vp, _fp]
    E = _lib("libref_esd.so")
    E.EstESDShifts.restype = None
    E.EstESDShifts.argtypes = [_vp, _vp, _vp, _vp, _ip, _dp, C.c_int, C.c_int, C.c_int, C.c_int,
                               C.c_int, C.c_int, C.c_float, C.c_double, C.c_double]
    G = _lib("libref_geocoreg.so")
    G.GeoCoreg_warp_cuda_full_dem.restype = None
    G.GeoCoreg_warp_cuda_full_dem.argtypes = [
        C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
        C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_int, C.c_double, C.c_double, C.c_double,
        C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp, C.c_int,
        C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_bool,
        C.c_bool, _ip, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double]
    return R, Co, E, G


def ref_geocoreg(G, F, H, b):
    """GeoCoreg_warp_cuda_full_dem for burst b with the arguments the stage
    driver builds (Func.cpp:2225-2278), DEM origin at the window's corner."""
    nb, L, W, _ = (int(v) for v in F["m_ints"])
    m_r, s_r = F["m_reals"], F["s_reals"]
    dem = iso(F[f"dem{b}"])
    lat0, lon0, dlat, dlon = F[f"dem_geo{b}"]
    mt = iso(F["m_sv"][0])
    st = iso(F["s_sv"][0])
    co = [iso(H[f"{t}_c{a}"]) for t in ("m", "s") for a in "xyz"]
    mf, ml = F["m_burst_first"][b], F["m_burst_last"][b]
    sf, sl = F["s_burst_first"][b], F["s_burst_last"][b]
    az, rg = iso(np.full(6, np.nan)), iso(np.full(6, np.nan))
    G.GeoCoreg_warp_cuda_full_dem(
        b, b, 0, W - 1, b * L, (b + 1) * L - 1, dlat, dlon, dem.shape[0], dem.shape[1],
        _ptr(az, C.c_double), _ptr(rg, C.c_double), lat0, lon0, NODATA, m_r[0], s_r[0], m_r[4],
        float(L), float(L), mf, sf, W, W, _ptr(mt, C.c_double), _ptr(st, C.c_double), len(mt),
        len(co[0]), len(st), len(co[3]), m_r[2], s_r[2], m_r[3], s_r[3], False, False,
        _ptr(dem, C.c_int), *(_ptr(c, C.c_double) for c in co), 0.5 * (mf + ml), 0.5 * (sf + sl))
    return np.array(az), np.array(rg)


def _rs_args(F, H, b, cpm_az, cpm_rg, shift, dt, out, kaz, krg):
    nb, L, W, _ = (int(v) for v in F["m_ints"])
    slave = iso(F["slave_slc"][b * L:(b + 1) * L])
    mbox = iso(np.array([0, W - 1, b * L, (b + 1) * L - 1], np.int32))
    sbox = iso(mbox)
    cpm_az, cpm_rg = iso(cpm_az), iso(cpm_rg)
    # the drivers pass the slave's burst-0 deramp rows for every burst (Func.cpp:2383)
    kt, tref, fdc = (iso(H[f"s_{k}"][0]) for k in ("kt", "tref", "dc"))
    keep = (slave, mbox, sbox, kt, tref, fdc, cpm_az, cpm_rg, out, kaz, krg)
    args = (slave.ctypes.data, _ptr(cpm_az, C.c_double), _ptr(cpm_rg, C.c_double), shift,
            out.ctypes.data, _ptr(kaz, C.c_float), _ptr(krg, C.c_float), b, W, L,
            _ptr(mbox, C.c_int), _ptr(sbox, C.c_int), L, W, dt, _ptr(kt, C.c_double),
            _ptr(tref, C.c_double), _ptr(fdc, C.c_double), 12)
    return args, keep


def _say(msg):
    print(msg, flush=True)


def _loaded_cudart():
    with open("/proc/self/maps") as f:
        return sorted({ln.split()[-1] for ln in f if "libcudart" in ln})


def stages(out_path, host_path):
    F = make_scene()
    H = dict(np.load(host_path))
    R, Co, E, G = _stage_libs()
    _say(f"CUDA runtime: {_loaded_cudart()}")
    nb, L, W, _ = (int(v) for v in F["m_ints"])
    kaz = iso(H["lut_kaz"])
    krg = iso(H["lut_krg"])
    res = dict(F)
    # geometric coregistration
    cpm = []
    for b in range(nb):
        cpm.append(ref_geocoreg(G, F, H, b))
        _say(f"geocoreg burst {b}: az {cpm[-1][0]} rg {cpm[-1][1]}")
    res["cpm_az"] = np.array([c[0] for c in cpm])
    res["cpm_rg"] = np.array([c[1] for c in cpm])
    assert np.all(np.isfinite(res["cpm_az"])) and np.all(np.isfinite(res["cpm_rg"]))
    # first resample pass (slave dt)
    s_dt, m_dt = F["s_reals"][0], F["m_reals"][0]
    reslave = np.zeros((nb, L, W), np.complex64)
    for b in range(nb):
        out = iso(np.zeros((L, W), np.complex64))
        args, keep = _rs_args(F, H, b, res["cpm_az"][b], res["cpm_rg"][b], 0.0,
                              s_dt, out, kaz, krg)
        R.DerampDemodResample(*args)
        reslave[b] = out
        _say(f"resample burst {b}: mean |out| {np.abs(out).mean():.3f}")
    res["reslave"] = reslave
    # ESD on the overlap bands
    ov = iso(H["m_ov"], np.int32)
    mslc = F["master_slc"]
    mF = iso(np.concatenate([mslc[(i + 1) * L - ov[i]:(i + 1) * L]
                                              for i in range(nb - 1)]))
    mB = iso(np.concatenate([mslc[(i + 1) * L:(i + 1) * L + ov[i]]
                                              for i in range(nb - 1)]))
    sF = iso(np.concatenate([reslave[i][L - ov[i]:] for i in range(nb - 1)]))
    sB = iso(np.concatenate([reslave[i + 1][:ov[i]] for i in range(nb - 1)]))
    spec = float(H["m_spec_sep"])
    for wr, wa in WINDOWS:
        shift = iso(np.full(nb - 1, np.nan))
        E.EstESDShifts(mF.ctypes.data, mB.ctypes.data, sF.ctypes.data, sB.ctypes.data,
                       _ptr(ov, C.c_int), _ptr(shift, C.c_double), nb - 1, mF.shape[0], W, wa, wr,
                       int(ov.max()), ESD_THRESHOLD, spec, m_dt)
        assert np.all(np.isfinite(shift)), shift
        res[f"esd_shift_{wr}x{wa}"] = np.array(shift)
        _say(f"ESD {wr}x{wa}: {shift}")
    # ESD resample + coherence, for each window
    for wr, wa in WINDOWS:
        shifts = res[f"esd_shift_{wr}x{wa}"].copy()
        shifts[np.abs(shifts) > 100] = 0.0       # Func.cpp:2612-2621
        reslave_esd = np.zeros((nb, L, W), np.complex64)
        coh = np.full((nb, L, W), np.nan, np.float32)
        for b in range(nb):
            master = iso(mslc[b * L:(b + 1) * L])
            c = iso(np.zeros((L, W), np.float32))
            if b == 0:
                first = iso(reslave[0])
                d = R.ResampleFirstBurst(first.ctypes.data, W, L)
                assert d
                reslave_esd[0] = first
                Co.CoherenceEst_ESD(0, 0, W, L, (wr - 1) // 2, (wa - 1) // 2, wr, wa,
                                    master.ctypes.data, d, _ptr(c, C.c_float))
            else:
                out = iso(np.zeros((L, W), np.complex64))
                args, keep = _rs_args(F, H, b, res["cpm_az"][b], res["cpm_rg"][b],
                                      float(shifts[b - 1]), m_dt, out, kaz, krg)
                d = R.DerampDemodResample_ESD(*args)
                assert d
                reslave_esd[b] = out
                Co.CoherenceEst(0, b * L, W, L, (wr - 1) // 2, (wa - 1) // 2, wr, wa,
                                master.ctypes.data, d, _ptr(c, C.c_float))
            coh[b] = c
            _say(f"ESD resample + coherence {wr}x{wa} burst {b}: mean coh {np.nanmean(c):.4f}")
        res[f"reslave_esd_{wr}x{wa}"] = reslave_esd
        res[f"coh_{wr}x{wa}"] = coh
    np.savez_compressed(out_path, **res)
    print(f"wrote {out_path}: {len(res)} arrays")


def timing(out_path, host_path, win=(10, 3), passes=2):
    """Wall time of the reference's stage calls on one sub-swath pair, per
    stage, in the order of its drivers (Func.cpp:2215-2763): geocoreg and
    resample per burst, ESD over the overlaps, then per burst the corrected
    resample kept on the device and its coherence.  The first pass warms the
    context; the last one is reported."""
    import json
    import time
    F = make_scene()
    H = dict(np.load(host_path))
    R, Co, E, G = _stage_libs()
    nb, L, W, _ = (int(v) for v in F["m_ints"])
    kaz, krg = iso(H["lut_kaz"]), iso(H["lut_krg"])
    s_dt, m_dt = F["s_reals"][0], F["m_reals"][0]
    wr, wa = win
    ov = iso(H["m_ov"], np.int32)
    mslc = F["master_slc"]
    spec = float(H["m_spec_sep"])
    for p in range(passes):
        t = dict(geocoreg=0.0, resample=0.0, esd=0.0, resample_esd=0.0, coherence=0.0)
        cpm = []
        for b in range(nb):
            t0 = time.perf_counter()
            cpm.append(ref_geocoreg(G, F, H, b))
            t["geocoreg"] += time.perf_counter() - t0
        reslave = np.zeros((nb, L, W), np.complex64)
        for b in range(nb):
            out = iso(np.zeros((L, W), np.complex64))
            args, keep = _rs_args(F, H, b, cpm[b][0], cpm[b][1], 0.0, s_dt, out, kaz, krg)
            t0 = time.perf_counter()
            R.DerampDemodResample(*args)
            t["resample"] += time.perf_counter() - t0
            reslave[b] = out
        mF = iso(np.concatenate([mslc[(i + 1) * L - ov[i]:(i + 1) * L] for i in range(nb - 1)]))
        mB = iso(np.concatenate([mslc[(i + 1) * L:(i + 1) * L + ov[i]] for i in range(nb - 1)]))
        sF = iso(np.concatenate([reslave[i][L - ov[i]:] for i in range(nb - 1)]))
        sB = iso(np.concatenate([reslave[i + 1][:ov[i]] for i in range(nb - 1)]))
        shift = iso(np.full(nb - 1, np.nan))
        t0 = time.perf_counter()
        E.EstESDShifts(mF.ctypes.data, mB.ctypes.data, sF.ctypes.data, sB.ctypes.data,
                       _ptr(ov, C.c_int), _ptr(shift, C.c_double), nb - 1, mF.shape[0], W, wa, wr,
                       int(ov.max()), ESD_THRESHOLD, spec, m_dt)
        t["esd"] += time.perf_counter() - t0
        shifts = np.array(shift)
        shifts[np.abs(shifts) > 100] = 0.0       # Func.cpp:2612-2621
        coh_mean = []
        for b in range(nb):
            master = iso(mslc[b * L:(b + 1) * L])
            c = iso(np.zeros((L, W), np.float32))
            if b == 0:
                first = iso(reslave[0])
                t0 = time.perf_counter()
                d = R.ResampleFirstBurst(first.ctypes.data, W, L)
                t1 = time.perf_counter()
                Co.CoherenceEst_ESD(0, 0, W, L, (wr - 1) // 2, (wa - 1) // 2, wr, wa,
                                    master.ctypes.data, d, _ptr(c, C.c_float))
            else:
                out = iso(np.zeros((L, W), np.complex64))
                args, keep = _rs_args(F, H, b, cpm[b][0], cpm[b][1], float(shifts[b - 1]), m_dt,
                                      out, kaz, krg)
                t0 = time.perf_counter()
                d = R.DerampDemodResample_ESD(*args)
                t1 = time.perf_counter()
                Co.CoherenceEst(0, b * L, W, L, (wr - 1) // 2, (wa - 1) // 2, wr, wa,
                                master.ctypes.data, d, _ptr(c, C.c_float))
            t2 = time.perf_counter()
            t["resample_esd"] += t1 - t0
            t["coherence"] += t2 - t1
            coh_mean.append(float(np.nanmean(c[20:-20, 20:-20])))
        total = sum(t.values())
        _say(f"pass {p}: {total:.3f} s, " + ", ".join(f"{k} {v:.3f} s" for k, v in t.items()))
    res = {"workload": f"{nb} burst pairs of {L}x{W} CInt16, DEM {SCENE['dem_lines']}x"
                       f"{SCENE['dem_pixels']}, window {wr}x{wa}",
           "form": "the reference's CUDA stages (oracle/_ref), per burst, host buffers",
           "seconds": total, "burst_pairs_per_s": nb / total,
           "stage_seconds": t, "esd_shifts": shifts.tolist(), "mean_coherence": coh_mean}
    with open(out_path, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps(res), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("part", choices=("host", "stitch", "stages", "front", "timing"))
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--scene", default="1", choices=sorted(SCENES))
    a = ap.parse_args()
    global SCENE
    SCENE = SCENES[a.scene]
    sfx = "" if a.scene == "1" else a.scene
    os.makedirs(a.out, exist_ok=True)
    if a.part == "host":
        host(os.path.join(a.out, f"ref_host{sfx}.npz"))
    elif a.part == "stitch":
        stitch(os.path.join(a.out, "ref_stitch.npz"))
    elif a.part == "front":
        front(os.path.join(a.out, "ref_front.npz"))
    elif a.part == "timing":
        hp = os.path.join(a.out, f"ref_host_{a.scene}.npz")
        if not os.path.exists(hp):
            host(hp)
        timing(os.path.join(a.out, f"ref_timing_{a.scene}.json"), hp)
    else:
        stages(os.path.join(a.out, f"ref_stages{sfx}.npz"), os.path.join(HERE, f"ref_host{sfx}.npz"))


if __name__ == "__main__":
    main()
