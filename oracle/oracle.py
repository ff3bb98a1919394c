"""ctypes bindings of the FP64 CPU oracle (oracle/_build/libtops_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only tests/,
__graft_entry__.smoke() and the cpu_baseline leg of bench.py may import this
module; the product never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libtops_oracle.so")


def build() -> None:
    subprocess.run(["make", "-s"], cwd=_HERE, check=True)


if not os.path.exists(LIB_PATH):
    build()
lib = C.CDLL(LIB_PATH)

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_long)
_sp = C.POINTER(C.c_int16)


class Poly(C.Structure):
    _fields_ = [("aztime", C.c_double), ("t0", C.c_double), ("c0", C.c_double),
                ("c1", C.c_double), ("c2", C.c_double)]


class DerampIn(C.Structure):
    _fields_ = [
        ("n_bursts", C.c_int), ("samples_per_burst", C.c_int), ("lines_per_burst", C.c_int),
        ("first_valid_pixel", C.c_int),
        ("slr_time_first_pixel", C.c_double), ("range_pixel_spacing", C.c_double),
        ("azimuth_time_interval", C.c_double), ("first_line_time", C.c_double),
        ("last_line_time", C.c_double), ("steering_rate_deg", C.c_double),
        ("wavelength", C.c_double),
        ("burst_first_line_time", _dp), ("burst_last_line_time", _dp),
        ("dc_list", C.POINTER(Poly)), ("n_dc", C.c_int),
        ("fm_list", C.POINTER(Poly)), ("n_fm", C.c_int),
        ("orb_cx", _dp), ("orb_cy", _dp), ("orb_cz", _dp), ("orb_ncoef", C.c_int),
        ("orb_mid_time", C.c_double),
    ]


class GeoIn(C.Structure):
    _fields_ = [
        ("dem_lines", C.c_int), ("dem_pixels", C.c_int),
        ("lat0", C.c_double), ("lon0", C.c_double), ("dlat", C.c_double), ("dlon", C.c_double),
        ("nodata", C.c_double),
        ("xmin", C.c_int), ("xmax", C.c_int), ("ymin", C.c_int), ("ymax", C.c_int),
        ("dt", C.c_double * 2), ("first_line_time", C.c_double * 2),
        ("slr_time", C.c_double * 2), ("range_spacing", C.c_double * 2),
        ("mid_time", C.c_double * 2), ("azi_init", C.c_double * 2),
        ("line_offset", C.c_int * 2),
        ("cx", _dp * 2), ("cy", _dp * 2), ("cz", _dp * 2),
        ("ncoef", C.c_int * 2),
    ]


class ResampleIn(C.Structure):
    _fields_ = [
        ("slave", _sp), ("slave_stride", C.c_long),
        ("mbox", C.c_int * 4), ("sbox", C.c_int * 4),
        ("cpm_az", C.c_double * 6), ("cpm_rg", C.c_double * 6), ("az_shift", C.c_double),
        ("kaz", _fp), ("krg", _fp), ("npoints", C.c_int),
        ("s_burst_idx", C.c_int), ("s_lines_per_burst", C.c_int),
        ("dt", C.c_double),
        ("kt", _dp), ("tref", _dp), ("fdc", _dp),
        ("f32_phase", C.c_int),
    ]


def _proto(name, restype, argtypes):
    f = getattr(lib, name)
    f.restype, f.argtypes = restype, argtypes


_proto("orc_lut", None, [C.c_int, C.c_double, C.c_double, C.c_double, _fp, _fp])
_proto("orc_polyfit_orbit", C.c_int, [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp])
_proto("orc_orbit_velocity", None, [C.c_double, _dp, _dp, _dp, C.c_int, _dp])
_proto("orc_compute_dc", None, [C.c_double, C.POINTER(Poly), C.c_int, C.POINTER(Poly)])
_proto("orc_deramp_params", None, [C.POINTER(DerampIn), _dp, _dp, _dp, _dp])
_proto("orc_overlap_size", None, [C.c_int, _dp, _dp, C.c_double, _ip, _ip, _ip])
_proto("orc_spectral_sep", C.c_double, [C.c_int, C.c_int, C.c_int, C.c_double, _dp])
_proto("orc_geocoreg", C.c_int, [C.POINTER(GeoIn), _fp, _dp, _dp, _dp, _lp])
_proto("orc_normalize_warp", C.c_double, [C.c_double, C.c_double, C.c_double])
_proto("orc_polyval", C.c_double, [C.c_double, C.c_double, _dp])
_proto("orc_resample", None, [C.POINTER(ResampleIn), _dp, _lp])
_proto("orc_resample_rows", None, [C.POINTER(ResampleIn), C.c_int, C.c_int, _dp])
_proto("orc_coherence", None, [_sp, _fp, C.c_int, C.c_int, C.c_int, C.c_int, _dp])
_proto("orc_esd", None, [_sp, _sp, _fp, _fp, _ip, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                         C.c_double, C.c_double, _dp, _dp, _lp])
_proto("orc_num_threads", C.c_int, [])
_proto("orc_set_num_threads", None, [C.c_int])


def _p(a, t):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(t))


def num_threads() -> int:
    return lib.orc_num_threads()


def set_num_threads(n: int) -> None:
    lib.orc_set_num_threads(n)


def lut(prf, abw, rsr2x, npoints=12):
    kaz = np.zeros((2048, npoints), np.float32)
    krg = np.zeros((2048, npoints), np.float32)
    lib.orc_lut(npoints, prf, abw, rsr2x, _p(kaz, C.c_float), _p(krg, C.c_float))
    return kaz, krg


def polyfit_orbit(t, x, y, z):
    t, x, y, z = (np.ascontiguousarray(v, np.float64) for v in (t, x, y, z))
    cx, cy, cz = (np.zeros(8) for _ in range(3))
    n = lib.orc_polyfit_orbit(len(t), _p(t, C.c_double), _p(x, C.c_double), _p(y, C.c_double),
                              _p(z, C.c_double), _p(cx, C.c_double), _p(cy, C.c_double),
                              _p(cz, C.c_double))
    return cx[:n].copy(), cy[:n].copy(), cz[:n].copy()


def deramp_params(info, coefs):
    """Deramp parameters from a SwathInfo-like object (fields of tops_swath_info)."""
    nb, W = info.n_bursts, info.samples_per_burst
    cx, cy, cz = (np.ascontiguousarray(c, np.float64) for c in coefs)
    first = np.array(info.burst_first_line_time[:nb], np.float64)
    last = np.array(info.burst_last_line_time[:nb], np.float64)
    dcl = (Poly * info.n_dc)(*[Poly(p.aztime, p.t0, p.c0, p.c1, p.c2)
                               for p in info.dc_list[:info.n_dc]])
    fml = (Poly * info.n_fm)(*[Poly(p.aztime, p.t0, p.c0, p.c1, p.c2)
                               for p in info.fm_list[:info.n_fm]])
    d = DerampIn()
    d.n_bursts, d.samples_per_burst, d.lines_per_burst = nb, W, info.lines_per_burst
    d.first_valid_pixel = info.first_valid_pixel
    d.slr_time_first_pixel, d.range_pixel_spacing = info.slr_time, info.range_spacing
    d.azimuth_time_interval = info.dt
    d.first_line_time, d.last_line_time = info.first_line_time, info.last_line_time
    d.steering_rate_deg, d.wavelength = info.steering_rate_deg, info.wavelength
    d.burst_first_line_time, d.burst_last_line_time = _p(first, C.c_double), _p(last, C.c_double)
    d.dc_list, d.n_dc = dcl, info.n_dc
    d.fm_list, d.n_fm = fml, info.n_fm
    d.orb_cx, d.orb_cy, d.orb_cz = _p(cx, C.c_double), _p(cy, C.c_double), _p(cz, C.c_double)
    d.orb_ncoef = len(cx)
    d.orb_mid_time = info.sv_t[info.n_sv // 2]
    dc, fm, tref, kt = (np.zeros((nb, W)) for _ in range(4))
    lib.orc_deramp_params(C.byref(d), _p(dc, C.c_double), _p(fm, C.c_double),
                          _p(tref, C.c_double), _p(kt, C.c_double))
    return {"dc": dc, "fmrate": fm, "tref": tref, "kt": kt}


def overlap_size(first, last, dt):
    first = np.ascontiguousarray(first, np.float64)
    last = np.ascontiguousarray(last, np.float64)
    n = len(first)
    ov = np.zeros(max(n - 1, 1), np.int32)
    tot, mx = C.c_int(), C.c_int()
    lib.orc_overlap_size(n, _p(first, C.c_double), _p(last, C.c_double), dt, _p(ov, C.c_int),
                         C.byref(tot), C.byref(mx))
    return ov[:n - 1], tot.value, mx.value


def spectral_sep(kt, L, dt):
    kt = np.ascontiguousarray(kt, np.float64)
    return lib.orc_spectral_sep(kt.shape[0], kt.shape[1], L, dt, _p(kt, C.c_double))


def geocoreg(dem, lat0, lon0, dlat, dlon, xmin, xmax, ymin, ymax, dt, first_line_time, slr_time,
             range_spacing, mid_time, azi_init, line_offset, coefs, nodata=-32768.0,
             want_pixels=False):
    """Returns (cpm_az[6], cpm_rg[6], status, n_valid[, pix[4][N]])."""
    dem = np.ascontiguousarray(dem, np.float32)
    g = GeoIn()
    g.dem_lines, g.dem_pixels = dem.shape
    g.lat0, g.lon0, g.dlat, g.dlon, g.nodata = lat0, lon0, dlat, dlon, nodata
    g.xmin, g.xmax, g.ymin, g.ymax = xmin, xmax, ymin, ymax
    for k in range(2):
        g.dt[k], g.first_line_time[k] = dt[k], first_line_time[k]
        g.slr_time[k], g.range_spacing[k] = slr_time[k], range_spacing[k]
        g.mid_time[k], g.azi_init[k], g.line_offset[k] = mid_time[k], azi_init[k], line_offset[k]
    keep = []
    for k in range(2):
        cx, cy, cz = (np.ascontiguousarray(c, np.float64) for c in coefs[k])
        keep += [cx, cy, cz]
        g.cx[k], g.cy[k], g.cz[k] = _p(cx, C.c_double), _p(cy, C.c_double), _p(cz, C.c_double)
        g.ncoef[k] = len(cx)
    az, rg = np.zeros(6), np.zeros(6)
    pix = np.zeros((4, dem.size)) if want_pixels else None
    nv = C.c_long()
    st = lib.orc_geocoreg(C.byref(g), _p(dem, C.c_float), _p(az, C.c_double), _p(rg, C.c_double),
                          _p(pix, C.c_double) if want_pixels else None, C.byref(nv))
    if want_pixels:
        return az, rg, st, nv.value, pix
    return az, rg, st, nv.value


def _rs_in(slave, cpm_az, cpm_rg, az_shift, kaz, krg, s_burst_idx, mbox, sbox, lines_per_burst, dt,
           kt, tref, fdc, f32_phase):
    slave = np.ascontiguousarray(slave, np.int16)
    r = ResampleIn()
    r.slave, r.slave_stride = _p(slave, C.c_int16), slave.shape[1]
    for i in range(4):
        r.mbox[i], r.sbox[i] = int(mbox[i]), int(sbox[i])
    for i in range(6):
        r.cpm_az[i], r.cpm_rg[i] = cpm_az[i], cpm_rg[i]
    r.az_shift = az_shift
    kaz = np.ascontiguousarray(kaz, np.float32)
    krg = np.ascontiguousarray(krg, np.float32)
    r.kaz, r.krg, r.npoints = _p(kaz, C.c_float), _p(krg, C.c_float), kaz.shape[1]
    r.s_burst_idx, r.s_lines_per_burst, r.dt = s_burst_idx, lines_per_burst, dt
    kt, tref, fdc = (np.ascontiguousarray(v, np.float64) for v in (kt, tref, fdc))
    r.kt, r.tref, r.fdc = _p(kt, C.c_double), _p(tref, C.c_double), _p(fdc, C.c_double)
    r.f32_phase = 1 if f32_phase else 0
    return r, (slave, kaz, krg, kt, tref, fdc)


def resample(slave, cpm_az, cpm_rg, az_shift, kaz, krg, s_burst_idx, mbox, sbox, lines_per_burst,
             dt, kt, tref, fdc, f32_phase=False, rows=None):
    """complex128 [mLines][mPixels] (or rows=(row0, nrows)) and region counts."""
    r, keep = _rs_in(slave, cpm_az, cpm_rg, az_shift, kaz, krg, s_burst_idx, mbox, sbox,
                     lines_per_burst, dt, kt, tref, fdc, f32_phase)
    mpix = mbox[1] - mbox[0] + 1
    mlin = mbox[3] - mbox[2] + 1
    if rows is not None:
        out = np.zeros((rows[1], mpix), np.complex128)
        lib.orc_resample_rows(C.byref(r), rows[0], rows[1], _p(out.view(np.float64), C.c_double))
        return out
    out = np.zeros((mlin, mpix), np.complex128)
    cnt = np.zeros(3, np.int64)
    lib.orc_resample(C.byref(r), _p(out.view(np.float64), C.c_double), _p(cnt, C.c_long))
    return out, cnt


_proto("orc_stitch_line_map", C.c_int, [C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_double, _ip,
                                        _ip, C.c_int, C.c_int, _ip, C.c_int])


def stitch_line_map(first_time, last_time, lines_per_burst, dt, first_line_time, first_valid,
                    last_valid, burst0, burstN):
    """Rows of the burst stack burst0..burstN copied by each output line
    (Stitch_OneSubswath, Func.cpp:2822-2933); None where the reference stops."""
    ft = np.ascontiguousarray(first_time, np.float64)
    lt = np.ascontiguousarray(last_time, np.float64)
    fv = np.ascontiguousarray(first_valid, np.int32)
    lv = np.ascontiguousarray(last_valid, np.int32)
    nb = len(ft)
    args = (nb, lines_per_burst, _p(ft, C.c_double), _p(lt, C.c_double), dt, first_line_time,
            _p(fv, C.c_int), _p(lv, C.c_int), burst0, burstN)
    h = lib.orc_stitch_line_map(*args, None, 0)
    if h <= 0:
        return None
    out = np.zeros(h, np.int32)
    if lib.orc_stitch_line_map(*args, _p(out, C.c_int), h) != h:
        return None
    return out


def coherence(master, slave, win_rg, win_az):
    master = np.ascontiguousarray(master, np.int16)
    slave = np.ascontiguousarray(slave, np.float32)
    lines, pixels = master.shape[0], master.shape[1]
    out = np.zeros((lines, pixels))
    lib.orc_coherence(_p(master, C.c_int16), _p(slave, C.c_float), lines, pixels, win_rg, win_az,
                      _p(out, C.c_double))
    return out


def esd(mF, mB, sF, sB, ov, win_az, win_rg, thr, spec_sep, dt):
    mF, mB = (np.ascontiguousarray(a, np.int16) for a in (mF, mB))
    sF, sB = (np.ascontiguousarray(a, np.float32) for a in (sF, sB))
    ov = np.ascontiguousarray(ov, np.int32)
    n = len(ov)
    W = mF.shape[1]
    shift, sums = np.zeros(n), np.zeros((n, 2))
    used = np.zeros(n, np.int64)
    lib.orc_esd(_p(mF, C.c_int16), _p(mB, C.c_int16), _p(sF, C.c_float), _p(sB, C.c_float),
                _p(ov, C.c_int), n, W, win_az, win_rg, thr, spec_sep, dt, _p(shift, C.c_double),
                _p(sums, C.c_double), _p(used, C.c_long))
    return shift, sums, used
