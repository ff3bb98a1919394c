"""ctypes bindings of libtops_b200.so (the B200 TOPS burst-pair processor).

Mirrors include/tops_b200.h and include/tops_synth.h.  The library must be
built (``make`` in this directory); importing this module raises if it is
missing -- there is no Python or CPU fallback for any GPU stage.

Device-side calls take raw device pointers; callers in this repository get
them from torch tensors (``tensor.data_ptr()``) and pass
``torch.cuda.current_stream().cuda_stream`` as the stream.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libtops_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"libtops_b200.so not built: run `make` in {_HERE}")
lib = C.CDLL(LIB_PATH)

TOPS_OK = 0
TOPS_E_INVALID = 1
TOPS_E_CUDA = 2
TOPS_E_NOMEM = 3
TOPS_E_NOT_PD = 4
TOPS_E_TIMEOUT = 5
TOPS_E_BUDGET = 6
TOPS_E_CONFIG = 7
TOPS_E_NODEVICE = 8
PREC_SPLIT = 0
PREC_FP64 = 1
LUT_BINS = 2048
NPOINTS = 12
MAX_BURSTS = 16

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


class TopsError(RuntimeError):
    def __init__(self, status: int, what: str):
        msg = lib.tops_status_string(status).decode()
        super().__init__(f"{what}: status {status} ({msg}), cuda error {lib.tops_last_cuda_error()}")
        self.status = status


def check(status: int, what: str) -> None:
    if status != TOPS_OK:
        raise TopsError(status, what)


# ------------------------------------------------------------------ structs
class Poly(C.Structure):
    _fields_ = [("aztime", C.c_double), ("t0", C.c_double), ("c0", C.c_double),
                ("c1", C.c_double), ("c2", C.c_double)]


class SynthCfg(C.Structure):
    _fields_ = [
        ("seed", C.c_long),
        ("n_bursts", C.c_int), ("lines_per_burst", C.c_int), ("samples_per_burst", C.c_int),
        ("overlap_lines", C.c_int),
        ("sigma_dn", C.c_double), ("wavelength", C.c_double), ("dt", C.c_double),
        ("rsr", C.c_double), ("steering_rate_deg", C.c_double), ("az_bandwidth", C.c_double),
        ("rg_bandwidth", C.c_double), ("altitude", C.c_double), ("inc_mid_deg", C.c_double),
        ("lat_center_deg", C.c_double),
        ("dem_lines", C.c_int), ("dem_pixels", C.c_int),
        ("hurst", C.c_double), ("h_min", C.c_double), ("h_max", C.c_double),
        ("dem_spacing_arcsec", C.c_double), ("bperp", C.c_double), ("bpar", C.c_double),
        ("along_track_s", C.c_double), ("az_shift_true", C.c_double),
        ("topo_phase", C.c_int), ("interp_taps", C.c_int), ("threads", C.c_int),
    ]


class SwathInfo(C.Structure):
    _fields_ = [
        ("n_bursts", C.c_int), ("lines_per_burst", C.c_int), ("samples_per_burst", C.c_int),
        ("first_valid_pixel", C.c_int),
        ("dt", C.c_double), ("prf", C.c_double), ("slr_time", C.c_double),
        ("range_spacing", C.c_double), ("wavelength", C.c_double), ("rsr", C.c_double),
        ("az_bandwidth", C.c_double), ("steering_rate_deg", C.c_double),
        ("first_line_time", C.c_double), ("last_line_time", C.c_double),
        ("burst_first_line_time", C.c_double * MAX_BURSTS),
        ("burst_last_line_time", C.c_double * MAX_BURSTS),
        ("n_dc", C.c_int), ("n_fm", C.c_int),
        ("dc_list", Poly * (MAX_BURSTS + 4)), ("fm_list", Poly * (MAX_BURSTS + 4)),
        ("n_sv", C.c_int),
        ("sv_t", C.c_double * 32), ("sv_x", C.c_double * 32), ("sv_y", C.c_double * 32),
        ("sv_z", C.c_double * 32),
    ]


class DemInfo(C.Structure):
    _fields_ = [("lines", C.c_int), ("pixels", C.c_int), ("lat0", C.c_double),
                ("lon0", C.c_double), ("dlat", C.c_double), ("dlon", C.c_double)]


class DerampDesc(C.Structure):
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


class ResampleJob(C.Structure):
    _fields_ = [
        ("slave", C.c_void_p), ("slave_pitch", C.c_size_t),
        ("out", C.c_void_p), ("out_pitch", C.c_size_t),
        ("kt", C.c_void_p), ("tref", C.c_void_p), ("fdc", C.c_void_p),
        ("mbox", C.c_int * 4), ("sbox", C.c_int * 4),
        ("cpm_az", C.c_double * 6), ("cpm_rg", C.c_double * 6),
        ("az_shift", C.c_double), ("az_shift_dev", C.c_void_p), ("cpm_dev", C.c_void_p),
        ("s_first_line", C.c_int), ("dt", C.c_double),
        ("out_row0", C.c_int), ("out_rows", C.c_int),
    ]


class CohJob(C.Structure):
    _fields_ = [("master", C.c_void_p), ("master_pitch", C.c_size_t),
                ("slave", C.c_void_p), ("slave_pitch", C.c_size_t),
                ("coh", C.c_void_p), ("coh_pitch", C.c_size_t),
                ("lines", C.c_int), ("pixels", C.c_int)]


class EsdOverlap(C.Structure):
    _fields_ = [("mF", C.c_void_p), ("mB", C.c_void_p), ("m_pitch", C.c_size_t),
                ("sF", C.c_void_p), ("sB", C.c_void_p), ("s_pitch", C.c_size_t),
                ("lines", C.c_int), ("pixels", C.c_int),
                ("spec_sep", C.c_double), ("dt", C.c_double)]


class GeoJob(C.Structure):
    _fields_ = [
        ("dem", C.c_void_p), ("dem_pitch", C.c_size_t),
        ("dem_lines", C.c_int), ("dem_pixels", C.c_int),
        ("lat0", C.c_double), ("lon0", C.c_double), ("dlat", C.c_double), ("dlon", C.c_double),
        ("nodata", C.c_double),
        ("xmin", C.c_int), ("xmax", C.c_int), ("ymin", C.c_int), ("ymax", C.c_int),
        ("dt", C.c_double * 2), ("first_line_time", C.c_double * 2),
        ("slr_time", C.c_double * 2), ("range_spacing", C.c_double * 2),
        ("mid_time", C.c_double * 2), ("azi_init", C.c_double * 2),
        ("line_offset", C.c_int * 2),
        ("coef", ((C.c_double * 8) * 3) * 2),
        ("ncoef", C.c_int * 2),
        ("cpm_dev", C.c_void_p), ("status_dev", C.c_void_p),
    ]


class Config(C.Structure):
    _fields_ = [
        ("process_dir", C.c_char * 512), ("masterpath", C.c_char * 512),
        ("slavepath", C.c_char * 512), ("polarisation", C.c_char * 64),
        ("preciseOrbitMaster", C.c_char * 512), ("preciseOrbitSlave", C.c_char * 512),
        ("SpecificDemPath", C.c_char * 512),
        ("firstsubswath", C.c_int), ("lastsubswath", C.c_int), ("multi_az", C.c_int),
        ("multi_rg", C.c_int), ("burst0", C.c_int), ("burstN", C.c_int),
        ("seed", C.c_long),
        ("n_bursts", C.c_int), ("lines_per_burst", C.c_int), ("samples_per_burst", C.c_int),
        ("overlap_lines", C.c_int), ("dem_lines", C.c_int), ("dem_pixels", C.c_int),
        ("sigma_dn", C.c_double), ("az_shift_true", C.c_double),
        ("coh_win_rg", C.c_int), ("coh_win_az", C.c_int), ("npoints", C.c_int),
        ("esd_coh_threshold", C.c_double),
        ("hbm_budget_gb", C.c_double), ("arrival_rate", C.c_double), ("n_jobs", C.c_int),
        ("stitch", C.c_int),
    ]


# --------------------------------------------------------------- prototypes
def _proto(name, restype, argtypes):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = argtypes
    return f


_vp = C.c_void_p
_proto("tops_status_string", C.c_char_p, [C.c_int])
_proto("tops_last_cuda_error", C.c_int, [])
_proto("tops_version", C.c_char_p, [])
_proto("tops_lut", C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, _fp, _fp])
_proto("tops_polyfit_orbit", C.c_int, [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _ip])
_proto("tops_deramp_params", C.c_int, [C.POINTER(DerampDesc), _dp, _dp, _dp, _dp])
_proto("tops_overlap_size", C.c_int, [C.c_int, _dp, _dp, C.c_double, _ip, _ip, _ip])
_proto("tops_spectral_sep", C.c_double, [C.c_int, C.c_int, C.c_int, C.c_double, _dp])
_proto("tops_config_defaults", C.c_int, [C.POINTER(Config)])
_proto("tops_config_read", C.c_int, [C.c_char_p, C.POINTER(Config), _ip])
_proto("tops_synth_defaults", C.c_int, [C.POINTER(SynthCfg)])
_proto("tops_synth_create", C.c_int, [C.POINTER(SynthCfg), C.POINTER(_vp)])
_proto("tops_synth_destroy", None, [_vp])
_proto("tops_synth_swath", C.c_int, [_vp, C.c_int, C.POINTER(SwathInfo)])
_proto("tops_synth_slc", C.POINTER(C.c_int16), [_vp, C.c_int])
_proto("tops_synth_dem", _fp, [_vp, C.POINTER(DemInfo)])
_proto("tops_synth_burst_dem_window", C.c_int, [_vp, C.c_int, C.c_int, _ip, _ip, _ip, _ip])
_proto("tops_synth_truth", C.c_int, [_vp, C.c_int, C.POINTER(C.c_long), C.POINTER(_dp)])
_proto("tops_synth_timing", C.c_int, [_vp, _dp])
# reference-compatible ABI (host buffers)
_proto("tops_fp64_peak", C.c_int, [_dp, _vp])
_proto("GeoCoreg_warp_cuda", C.c_int,
       [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
        C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_int, C.c_double, C.c_double, C.c_double,
        C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp, C.c_int,
        C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_bool,
        C.c_bool, _ip, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double])
_RS_ARGS = [_vp, _dp, _dp, C.c_double, _vp, _fp, _fp, C.c_int, C.c_int, C.c_int, _ip, _ip, C.c_int,
            C.c_int, C.c_double, _dp, _dp, _dp, C.c_int]
_proto("DerampDemodResample", C.c_int, _RS_ARGS)
_proto("DerampDemodResample_ESD", _vp, _RS_ARGS)
_proto("ResampleFirstBurst", _vp, [_vp, C.c_int, C.c_int])
_proto("EstESDShifts", C.c_int, [_vp, _vp, _vp, _vp, _ip, _dp, C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.c_int, C.c_int, C.c_float, C.c_double, C.c_double])
_COH_ARGS = [C.c_int] * 8 + [_vp, _vp, _fp]
_proto("CoherenceEst", C.c_int, _COH_ARGS)
_proto("CoherenceEst_ESD", C.c_int, _COH_ARGS)
_proto("tops_free_device", C.c_int, [_vp])
# device API
_proto("tops_lut_create", C.c_int, [_fp, _fp, C.POINTER(_vp)])
_proto("tops_lut_destroy", C.c_int, [_vp])
_proto("tops_resample", C.c_int, [_vp, C.POINTER(ResampleJob), C.c_int, _vp])
_proto("tops_resample_ex", C.c_int, [_vp, C.POINTER(ResampleJob), C.c_int, C.c_int, _vp])
_proto("tops_coherence", C.c_int, [C.POINTER(CohJob), C.c_int, C.c_int, C.c_int, _vp])
_proto("tops_esd_scratch_bytes", C.c_size_t, [C.POINTER(EsdOverlap), C.c_int])
_proto("tops_esd", C.c_int, [C.POINTER(EsdOverlap), C.c_int, C.c_int, C.c_int, C.c_float, _vp,
                             _vp, _vp, C.c_size_t, _vp])
_proto("tops_esd_static", C.c_int, [C.POINTER(EsdOverlap), C.c_int, C.c_int, C.c_int, C.c_float,
                                    _vp, _vp, _vp])
_proto("tops_geocoreg_scratch_bytes", C.c_size_t, [C.POINTER(GeoJob), C.c_int])
_proto("tops_geocoreg", C.c_int, [C.POINTER(GeoJob), C.c_int, _vp, C.c_size_t, _vp])


def fp64_peak(stream=0) -> float:
    """Measured FP64 FMA throughput of the device, TFLOP/s."""
    v = C.c_double(0.0)
    check(lib.tops_fp64_peak(C.byref(v), C.c_void_p(stream)), "tops_fp64_peak")
    return v.value


def ptr(a: np.ndarray, ctype):
    """ctypes pointer to a C-contiguous numpy array."""
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))


def vptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return C.c_void_p(a.ctypes.data)


# ------------------------------------------------------------ host helpers
def lut(prf: float, abw: float, rsr2x: float, npoints: int = NPOINTS):
    kaz = np.zeros((LUT_BINS, npoints), np.float32)
    krg = np.zeros((LUT_BINS, npoints), np.float32)
    check(lib.tops_lut(npoints, prf, abw, rsr2x, ptr(kaz, C.c_float), ptr(krg, C.c_float)),
          "tops_lut")
    return kaz, krg


def polyfit_orbit(t, x, y, z):
    t, x, y, z = (np.ascontiguousarray(v, np.float64) for v in (t, x, y, z))
    cx, cy, cz = (np.zeros(8) for _ in range(3))
    n = C.c_int(0)
    check(lib.tops_polyfit_orbit(len(t), ptr(t, C.c_double), ptr(x, C.c_double),
                                 ptr(y, C.c_double), ptr(z, C.c_double), ptr(cx, C.c_double),
                                 ptr(cy, C.c_double), ptr(cz, C.c_double), C.byref(n)),
          "tops_polyfit_orbit")
    return cx[:n.value].copy(), cy[:n.value].copy(), cz[:n.value].copy()


def overlap_size(first, last, dt):
    first = np.ascontiguousarray(first, np.float64)
    last = np.ascontiguousarray(last, np.float64)
    n = len(first)
    ov = np.zeros(max(n - 1, 1), np.int32)
    tot, mx = C.c_int(), C.c_int()
    check(lib.tops_overlap_size(n, ptr(first, C.c_double), ptr(last, C.c_double), dt,
                                ptr(ov, C.c_int), C.byref(tot), C.byref(mx)), "tops_overlap_size")
    return ov[:n - 1], tot.value, mx.value


def spectral_sep(kt: np.ndarray, L: int, dt: float) -> float:
    kt = np.ascontiguousarray(kt, np.float64)
    return lib.tops_spectral_sep(kt.shape[0], kt.shape[1], L, dt, ptr(kt, C.c_double))


def swath_deramp_params(info: SwathInfo, orbit_coefs, ncoef: int):
    """kt, tref, fdc (and FM rate) [n_bursts][W] for a swath."""
    nb, W = info.n_bursts, info.samples_per_burst
    cx, cy, cz = (np.ascontiguousarray(c, np.float64) for c in orbit_coefs)
    first = np.array(info.burst_first_line_time[:nb])
    last = np.array(info.burst_last_line_time[:nb])
    d = DerampDesc()
    d.n_bursts, d.samples_per_burst, d.lines_per_burst = nb, W, info.lines_per_burst
    d.first_valid_pixel = info.first_valid_pixel
    d.slr_time_first_pixel, d.range_pixel_spacing = info.slr_time, info.range_spacing
    d.azimuth_time_interval = info.dt
    d.first_line_time, d.last_line_time = info.first_line_time, info.last_line_time
    d.steering_rate_deg, d.wavelength = info.steering_rate_deg, info.wavelength
    d.burst_first_line_time, d.burst_last_line_time = ptr(first, C.c_double), ptr(last, C.c_double)
    d.dc_list = C.cast(info.dc_list, C.POINTER(Poly))
    d.n_dc = info.n_dc
    d.fm_list = C.cast(info.fm_list, C.POINTER(Poly))
    d.n_fm = info.n_fm
    d.orb_cx, d.orb_cy, d.orb_cz = ptr(cx, C.c_double), ptr(cy, C.c_double), ptr(cz, C.c_double)
    d.orb_ncoef = ncoef
    d.orb_mid_time = info.sv_t[info.n_sv // 2]
    dc, fm, tref, kt = (np.zeros((nb, W)) for _ in range(4))
    check(lib.tops_deramp_params(C.byref(d), ptr(dc, C.c_double), ptr(fm, C.c_double),
                                 ptr(tref, C.c_double), ptr(kt, C.c_double)), "tops_deramp_params")
    return {"dc": dc, "fmrate": fm, "tref": tref, "kt": kt}


class RunStats(C.Structure):
    _fields_ = [("subswaths", C.c_int), ("burst_pairs", C.c_int), ("seconds", C.c_double),
                ("shifts", C.c_double * MAX_BURSTS), ("load_seconds", C.c_double),
                ("process_seconds", C.c_double), ("write_seconds", C.c_double)]


_proto("tops_run_config", C.c_int, [C.c_char_p, C.POINTER(RunStats)])


def run_config(path: str) -> RunStats:
    """The config.txt-driven run (tops_run_config)."""
    st = RunStats()
    check(lib.tops_run_config(str(path).encode(), C.byref(st)), f"tops_run_config({path})")
    return st


def read_config(path: str) -> Config:
    cfg = Config()
    check(lib.tops_config_defaults(C.byref(cfg)), "tops_config_defaults")
    line = C.c_int(0)
    st = lib.tops_config_read(path.encode(), C.byref(cfg), C.byref(line))
    if st != TOPS_OK:
        raise TopsError(st, f"tops_config_read({path}) line {line.value}")
    return cfg


# ----------------------------------------------------------- synthetic scene
class Scene:
    """A seeded synthetic burst pair (tops_synth_create)."""

    def __init__(self, **overrides):
        cfg = SynthCfg()
        check(lib.tops_synth_defaults(C.byref(cfg)), "tops_synth_defaults")
        for k, v in overrides.items():
            if not hasattr(cfg, k):
                raise KeyError(k)
            setattr(cfg, k, v)
        self.cfg = cfg
        h = C.c_void_p()
        check(lib.tops_synth_create(C.byref(cfg), C.byref(h)), "tops_synth_create")
        self._h = h
        nb, L, W = cfg.n_bursts, cfg.lines_per_burst, cfg.samples_per_burst
        self.shape = (nb * L, W)
        self.swath = []
        for w in (0, 1):
            info = SwathInfo()
            check(lib.tops_synth_swath(h, w, C.byref(info)), "tops_synth_swath")
            self.swath.append(info)
        self.slc = []
        for w in (0, 1):
            p = lib.tops_synth_slc(h, w)
            a = np.ctypeslib.as_array(p, shape=(nb * L, W, 2))
            self.slc.append(a.copy())
        di = DemInfo()
        p = lib.tops_synth_dem(h, C.byref(di))
        self.dem_info = di
        self.dem = np.ctypeslib.as_array(p, shape=(di.lines, di.pixels)).copy()
        t = np.zeros(5)
        lib.tops_synth_timing(h, ptr(t, C.c_double))
        self.timing = t
        # orbit fits and deramp parameters (product host code)
        self.orbit = []
        self.deramp = []
        for w in (0, 1):
            info = self.swath[w]
            n = info.n_sv
            cx, cy, cz = polyfit_orbit(info.sv_t[:n], info.sv_x[:n], info.sv_y[:n], info.sv_z[:n])
            self.orbit.append((cx, cy, cz))
            self.deramp.append(swath_deramp_params(info, (cx, cy, cz), len(cx)))
        m = self.swath[0]
        self.kaz, self.krg = lut(m.prf, m.az_bandwidth, 2 * m.rsr)

    def dem_window(self, burst: int, margin: int = 24):
        r0, c0, nr, nc = (C.c_int() for _ in range(4))
        check(lib.tops_synth_burst_dem_window(self._h, burst, margin, C.byref(r0), C.byref(c0),
                                              C.byref(nr), C.byref(nc)), "dem window")
        return r0.value, c0.value, nr.value, nc.value

    def truth(self, burst: int) -> np.ndarray:
        n = C.c_long()
        p = _dp()
        check(lib.tops_synth_truth(self._h, burst, C.byref(n), C.byref(p)), "truth")
        return np.ctypeslib.as_array(p, shape=(n.value, 4)).copy()

    def close(self):
        if getattr(self, "_h", None):
            lib.tops_synth_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- per-burst views and stage inputs
    def burst(self, which: int, b: int) -> np.ndarray:
        L = self.cfg.lines_per_burst
        return np.ascontiguousarray(self.slc[which][b * L:(b + 1) * L])

    def boxes(self, b: int, burst_gap: int = 0):
        """MasterBox / SlaveBox of burst b (Func.cpp:2354-2371)."""
        L, W = self.cfg.lines_per_burst, self.cfg.samples_per_burst
        mb = np.array([0, W - 1, b * L, (b + 1) * L - 1], np.int32)
        sb = np.array([0, W - 1, (b + burst_gap) * L, (b + burst_gap + 1) * L - 1], np.int32)
        return mb, sb

    def geo_args(self, b: int, margin: int = 24):
        """Arguments of one burst's geometric coregistration (Func.cpp:2225-2278),
        with the DEM window's own origin (not the burst box corner)."""
        L, W = self.cfg.lines_per_burst, self.cfg.samples_per_burst
        m, s = self.swath
        r0, c0, nr, nc = self.dem_window(b, margin)
        di = self.dem_info
        return dict(
            dem=np.ascontiguousarray(self.dem[r0:r0 + nr, c0:c0 + nc]),
            lat0=di.lat0 - r0 * di.dlat, lon0=di.lon0 + c0 * di.dlon,
            dlat=di.dlat, dlon=di.dlon,
            xmin=0, xmax=W - 1, ymin=b * L, ymax=(b + 1) * L - 1,
            dt=(m.dt, s.dt),
            first_line_time=(m.burst_first_line_time[b], s.burst_first_line_time[b]),
            slr_time=(m.slr_time, s.slr_time), range_spacing=(m.range_spacing, s.range_spacing),
            mid_time=(m.sv_t[m.n_sv // 2], s.sv_t[s.n_sv // 2]),
            azi_init=(0.5 * (m.burst_first_line_time[b] + m.burst_last_line_time[b]),
                      0.5 * (s.burst_first_line_time[b] + s.burst_last_line_time[b])),
            line_offset=(b * L, b * L),
            coefs=(self.orbit[0], self.orbit[1]),
        )


# ------------------------------------------- reference-compatible ABI calls
def deramp_demod_resample(slave, cpm_az, cpm_rg, az_shift, kaz, krg, s_burst_idx, mbox, sbox,
                          lines_per_burst, dt, kt, tref, fdc, keep_device=False):
    """DerampDemodResample / DerampDemodResample_ESD on host arrays.

    slave: int16 [sLines][sPixels][2]; kt/tref/fdc: float64 [SamplesPerBurst].
    Returns complex64 [mLines][mPixels] (and the device pointer if keep_device)."""
    slave = np.ascontiguousarray(slave, np.int16)
    mbox = np.ascontiguousarray(mbox, np.int32)
    sbox = np.ascontiguousarray(sbox, np.int32)
    mlin, mpix = int(mbox[3] - mbox[2] + 1), int(mbox[1] - mbox[0] + 1)
    out = np.zeros((mlin, mpix), np.complex64)
    caz = np.ascontiguousarray(cpm_az, np.float64)
    crg = np.ascontiguousarray(cpm_rg, np.float64)
    kaz = np.ascontiguousarray(kaz, np.float32)
    krg = np.ascontiguousarray(krg, np.float32)
    kt, tref, fdc = (np.ascontiguousarray(v, np.float64) for v in (kt, tref, fdc))
    args = (vptr(slave), ptr(caz, C.c_double), ptr(crg, C.c_double), float(az_shift), vptr(out),
            ptr(kaz, C.c_float), ptr(krg, C.c_float), int(s_burst_idx), slave.shape[1],
            slave.shape[0], ptr(mbox, C.c_int), ptr(sbox, C.c_int), int(lines_per_burst),
            len(kt), float(dt), ptr(kt, C.c_double), ptr(tref, C.c_double),
            ptr(fdc, C.c_double), kaz.shape[1])
    if keep_device:
        d = lib.DerampDemodResample_ESD(*args)
        if not d:
            raise TopsError(TOPS_E_CUDA if lib.tops_last_cuda_error() else TOPS_E_INVALID,
                            "DerampDemodResample_ESD")
        return out, d
    check(lib.DerampDemodResample(*args), "DerampDemodResample")
    return out


def resample_first_burst(reslave: np.ndarray):
    a = np.ascontiguousarray(reslave, np.complex64)
    d = lib.ResampleFirstBurst(vptr(a), a.shape[1], a.shape[0])
    if not d:
        raise TopsError(TOPS_E_CUDA, "ResampleFirstBurst")
    return d


def coherence_est(master, d_slave, win_rg, win_az, esd_variant=False):
    """CoherenceEst(_ESD): master int16 [Dh][Dw][2] on the host, d_slave a device
    pointer from deramp_demod_resample(keep_device=True) / resample_first_burst
    (freed by the call, as in the reference).  Returns float32 [Dh][Dw]."""
    master = np.ascontiguousarray(master, np.int16)
    Dh, Dw = master.shape[0], master.shape[1]
    coh = np.zeros((Dh, Dw), np.float32)
    f = lib.CoherenceEst_ESD if esd_variant else lib.CoherenceEst
    check(f(0, 0, Dw, Dh, (win_rg - 1) // 2, (win_az - 1) // 2, win_rg, win_az, vptr(master),
            C.c_void_p(d_slave), ptr(coh, C.c_float)), "CoherenceEst")
    return coh


def est_esd_shifts(mF, mB, sF, sB, ov, win_az, win_rg, thr, spec_sep, dt):
    """EstESDShifts on the concatenated overlap bands (host arrays)."""
    mF, mB = (np.ascontiguousarray(a, np.int16) for a in (mF, mB))
    sF, sB = (np.ascontiguousarray(a, np.complex64) for a in (sF, sB))
    ov = np.ascontiguousarray(ov, np.int32)
    shift = np.zeros(len(ov))
    check(lib.EstESDShifts(vptr(mF), vptr(mB), vptr(sF), vptr(sB), ptr(ov, C.c_int),
                           ptr(shift, C.c_double), len(ov), mF.shape[0], mF.shape[1], win_az,
                           win_rg, int(ov.max()) if len(ov) else 0, float(thr), float(spec_sep),
                           float(dt)), "EstESDShifts")
    return shift


def geocoreg_warp(dem_int, lat0, lon0, dlat, dlon, xmin, xmax, ymin, ymax, m_burst, s_burst,
                  lines_per_burst, dt, first_line_time, slr_time, range_spacing, orbit_t,
                  coefs, azi_init, samples, wavelength=0.05547, nodata=-32768):
    """GeoCoreg_warp_cuda with its reference argument list (int DEM window).

    orbit_t: (master SV times, slave SV times); coefs: ((cx,cy,cz) master, slave)."""
    dem_int = np.ascontiguousarray(dem_int, np.int32)
    az, rg = np.zeros(6), np.zeros(6)
    mt, st_ = (np.ascontiguousarray(t, np.float64) for t in orbit_t)
    (mx, my, mz), (sx, sy, sz) = [[np.ascontiguousarray(c, np.float64) for c in cc] for cc in coefs]
    st = lib.GeoCoreg_warp_cuda(
        m_burst, s_burst, xmin, xmax, ymin, ymax, dlat, dlon, dem_int.shape[0], dem_int.shape[1],
        ptr(az, C.c_double), ptr(rg, C.c_double), lat0, lon0, nodata, dt[0], dt[1], wavelength,
        float(lines_per_burst), float(lines_per_burst), first_line_time[0], first_line_time[1],
        samples, samples, ptr(mt, C.c_double), ptr(st_, C.c_double), len(mt), len(mx), len(st_),
        len(sx), slr_time[0], slr_time[1], range_spacing[0], range_spacing[1], False, False,
        ptr(dem_int, C.c_int), ptr(mx, C.c_double), ptr(my, C.c_double), ptr(mz, C.c_double),
        ptr(sx, C.c_double), ptr(sy, C.c_double), ptr(sz, C.c_double), azi_init[0], azi_init[1])
    check(st, "GeoCoreg_warp_cuda")
    return az, rg


# ------------------------------------------------------- burst-pair pipeline
class PairOpts(C.Structure):
    _fields_ = [("win_rg", C.c_int), ("win_az", C.c_int), ("esd_threshold", C.c_float),
                ("reslave_full", C.c_int), ("burst0_deramp_rows", C.c_int),
                ("precision", C.c_int), ("compensated", C.c_int),
                ("coh_overlap", C.c_int)]


class DemWindow(C.Structure):
    _fields_ = [("row0", C.c_int), ("col0", C.c_int), ("rows", C.c_int), ("cols", C.c_int)]


class PairBuffers(C.Structure):
    _fields_ = [("master", C.c_void_p), ("slave", C.c_void_p), ("reslave", C.c_void_p),
                ("reslave_esd", C.c_void_p), ("coh", C.c_void_p), ("cpm", C.c_void_p),
                ("shifts", C.c_void_p), ("geo_status", C.c_void_p),
                ("slc_pitch", C.c_size_t), ("cplx_pitch", C.c_size_t), ("coh_pitch", C.c_size_t),
                ("n_bursts", C.c_int), ("lines", C.c_int), ("samples", C.c_int),
                ("n_launches", C.c_int)]


_proto("tops_pair_opts_default", C.c_int, [C.POINTER(PairOpts)])
_proto("tops_pair_footprint", C.c_size_t, [C.POINTER(SwathInfo), C.POINTER(PairOpts), C.c_int,
                                           C.c_int])
_proto("tops_pair_create", C.c_int, [C.POINTER(SwathInfo), C.POINTER(SwathInfo),
                                     C.POINTER(PairOpts), C.c_int, C.c_int, C.POINTER(_vp)])
_proto("tops_pair_destroy", C.c_int, [_vp])
_proto("tops_pair_set_dem", C.c_int, [_vp, _fp, C.c_double, C.c_double, C.c_double, C.c_double,
                                      C.POINTER(DemWindow), _vp])
_proto("tops_pair_upload", C.c_int, [_vp, _vp, _vp, _vp])
_proto("tops_pair_run", C.c_int, [_vp, _vp])
_proto("tops_pair_run_graph", C.c_int, [_vp, _vp])
_proto("tops_pair_download", C.c_int, [_vp, _vp, _vp, _fp, _dp, _dp, _vp])
_proto("tops_pair_buffers_get", C.c_int, [_vp, C.POINTER(PairBuffers)])
_proto("tops_plain_pair", C.c_int, [C.POINTER(SwathInfo), C.POINTER(SwathInfo), C.POINTER(PairOpts),
                                    _ip, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.POINTER(DemWindow), _vp, _vp, _vp, _vp, _fp, _dp,
                                    _dp])


class Tune(C.Structure):
    _fields_ = [("rs_seg_rows", C.c_int), ("rs_persistent", C.c_int),
                ("coh_seg_rows", C.c_int), ("coh_persistent", C.c_int)]


_proto("tops_pair_run_per_burst", C.c_int, [_vp, _vp])
_proto("tops_stream_synchronize", C.c_int, [_vp])
_proto("tops_tiff_write", C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _vp, C.c_size_t])
_proto("tops_tiff_read", C.c_int, [C.c_char_p, _ip, _ip, _ip, _vp, C.c_size_t])
_proto("tops_tiff_georef", C.c_int, [C.c_char_p, _dp])
_proto("tops_tiff_write_georef", C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, _vp,
                                           C.c_size_t, _dp])
TIFF_TYPES = {1: (np.int16, 2), 2: (np.float32, 1), 3: (np.complex64, 1), 4: (np.int16, 1)}


def _tiff_type(a: np.ndarray) -> int:
    if a.dtype == np.int16:
        return 1 if a.ndim == 3 else 4
    if a.dtype == np.float32:
        return 2
    if a.dtype == np.complex64:
        return 3
    raise TypeError(a.dtype)


def tiff_georef(path: str) -> np.ndarray:
    """GDAL-style geotransform of a GeoTIFF (tops_tiff_georef)."""
    gt = np.zeros(6)
    check(lib.tops_tiff_georef(str(path).encode(), ptr(gt, C.c_double)), "tops_tiff_georef")
    return gt


def tiff_write_georef(path: str, a: np.ndarray, gt) -> None:
    """tiff_write with a north-up geotransform (e.g. a DEM)."""
    a = np.ascontiguousarray(a)
    g = np.ascontiguousarray(gt, np.float64)
    check(lib.tops_tiff_write_georef(str(path).encode(), _tiff_type(a), a.shape[1], a.shape[0],
                                     C.c_void_p(a.ctypes.data), a.strides[0], ptr(g, C.c_double)),
          "tops_tiff_write_georef")


def tiff_write(path: str, a: np.ndarray) -> None:
    """CInt16 ([h][w][2] int16), int16, float32 or complex64 [h][w] raster."""
    if a.dtype == np.int16:
        t = 1 if a.ndim == 3 else 4
    elif a.dtype == np.float32:
        t = 2
    elif a.dtype == np.complex64:
        t = 3
    else:
        raise TypeError(a.dtype)
    a = np.ascontiguousarray(a)
    check(lib.tops_tiff_write(str(path).encode(), t, a.shape[1], a.shape[0],
                              C.c_void_p(a.ctypes.data), a.strides[0]), "tops_tiff_write")


def tiff_read(path: str) -> np.ndarray:
    t, w, h = C.c_int(), C.c_int(), C.c_int()
    check(lib.tops_tiff_read(str(path).encode(), C.byref(t), C.byref(w), C.byref(h), None, 0),
          "tops_tiff_read")
    dt, comps = TIFF_TYPES[t.value]
    out = np.zeros((h.value, w.value, comps) if comps > 1 else (h.value, w.value), dt)
    check(lib.tops_tiff_read(str(path).encode(), C.byref(t), C.byref(w), C.byref(h),
                             C.c_void_p(out.ctypes.data), out.nbytes), "tops_tiff_read")
    return out
_proto("tops_stitch_line_map", C.c_int, [C.POINTER(SwathInfo), _ip, _ip, C.c_int, C.c_int, _ip,
                                         C.c_int, _ip])
_proto("tops_stitch", C.c_int, [_vp, C.c_size_t, _vp, C.c_size_t, _vp, C.c_int, C.c_size_t, _vp])


def stitch_line_map(info: "SwathInfo", first_valid, last_valid, burst0: int, burstN: int):
    """Rows of the burst stack burst0..burstN that the debursted output lines
    copy (tops_stitch_line_map); raises TopsError where the reference stops."""
    fv = np.ascontiguousarray(first_valid, np.int32)
    lv = np.ascontiguousarray(last_valid, np.int32)
    h = C.c_int()
    check(lib.tops_stitch_line_map(C.byref(info), ptr(fv, C.c_int), ptr(lv, C.c_int), burst0,
                                   burstN, None, 0, C.byref(h)), "tops_stitch_line_map")
    out = np.zeros(h.value, np.int32)
    check(lib.tops_stitch_line_map(C.byref(info), ptr(fv, C.c_int), ptr(lv, C.c_int), burst0,
                                   burstN, ptr(out, C.c_int), h.value, C.byref(h)),
          "tops_stitch_line_map")
    return out
# ------------------------------------------------ Sentinel-1 front end (tops_s1.h)
class S1Annotation(C.Structure):
    _fields_ = [
        ("polarisation", C.c_char * 8), ("first_line_utc", C.c_char * 40),
        ("last_line_utc", C.c_char * 40), ("dc_method", C.c_char * 40),
        ("number_of_lines", C.c_int), ("number_of_samples", C.c_int),
        ("last_valid_pixel", C.c_int),
        ("azimuth_pixel_spacing", C.c_double), ("radar_frequency", C.c_double),
        ("heading", C.c_double), ("range_bandwidth", C.c_double),
        ("ascending_node_time", C.c_double), ("slr_time_last_pixel", C.c_double),
        ("first_valid_line", C.c_int * MAX_BURSTS), ("last_valid_line", C.c_int * MAX_BURSTS),
        ("burst_first_valid_time", C.c_double * MAX_BURSTS),
        ("burst_last_valid_time", C.c_double * MAX_BURSTS),
        ("burst_lat_min", C.c_double * MAX_BURSTS), ("burst_lat_max", C.c_double * MAX_BURSTS),
        ("burst_lon_min", C.c_double * MAX_BURSTS), ("burst_lon_max", C.c_double * MAX_BURSTS),
        ("geo_lines", C.c_int), ("geo_points_per_line", C.c_int),
    ]


class S1Geogrid(C.Structure):
    _fields_ = [("lines", C.c_int), ("points", C.c_int), ("az_time", _dp), ("slr_time", _dp),
                ("lat", _dp), ("lon", _dp)]


_proto("tops_s1_annotation_read", C.c_int, [C.c_char_p, C.POINTER(SwathInfo),
                                            C.POINTER(S1Annotation)])
_proto("tops_s1_geogrid_read", C.c_int, [C.c_char_p, C.c_int, _dp, _dp, _dp, _dp, _dp, _ip, _ip])
_proto("tops_s1_orbit_read", C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.POINTER(SwathInfo),
                                       _dp])
_proto("tops_s1_burst_overlap", C.c_int, [C.c_int, C.c_int, C.POINTER(SwathInfo),
                                          C.POINTER(S1Geogrid), C.POINTER(SwathInfo),
                                          C.POINTER(S1Geogrid), _ip, _ip, _ip, _ip])


def s1_annotation_read(path: str, info: "SwathInfo" = None):
    """(SwathInfo, S1Annotation) of one annotation file (tops_s1_annotation_read);
    the state vectors of a given info are kept."""
    info = info if info is not None else SwathInfo()
    ex = S1Annotation()
    check(lib.tops_s1_annotation_read(str(path).encode(), C.byref(info), C.byref(ex)),
          "tops_s1_annotation_read")
    return info, ex


def s1_geogrid_read(path: str) -> dict:
    """Geolocation grid arrays [lines][points] of an annotation file."""
    nl, npl = C.c_int(), C.c_int()
    check(lib.tops_s1_geogrid_read(str(path).encode(), 0, None, None, None, None, None,
                                   C.byref(nl), C.byref(npl)), "tops_s1_geogrid_read")
    n = nl.value * npl.value
    g = {k: np.zeros(n) for k in ("az_time", "slr_time", "lat", "lon", "incidence")}
    check(lib.tops_s1_geogrid_read(str(path).encode(), n, *(ptr(g[k], C.c_double) for k in
                                   ("az_time", "slr_time", "lat", "lon", "incidence")),
                                   C.byref(nl), C.byref(npl)), "tops_s1_geogrid_read")
    g = {k: v.reshape(nl.value, npl.value) for k, v in g.items()}
    return g


def s1_orbit_read(path: str, first_line_utc: str, last_line_utc: str, info: "SwathInfo"):
    """Fills info's state vectors from an EOF file (tops_s1_orbit_read);
    returns the [n][3] velocities."""
    vel = np.zeros((32, 3))
    check(lib.tops_s1_orbit_read(str(path).encode(), first_line_utc.encode(),
                                 last_line_utc.encode(), C.byref(info), ptr(vel, C.c_double)),
          "tops_s1_orbit_read")
    return vel[:info.n_sv].copy()


def _grid_struct(g: dict):
    keep = [np.ascontiguousarray(g[k], np.float64) for k in ("az_time", "slr_time", "lat", "lon")]
    lines, points = keep[0].shape
    return S1Geogrid(lines, points, *(ptr(a, C.c_double) for a in keep)), keep


def s1_burst_overlap(burst0: int, burstN: int, master: "SwathInfo", master_grid: dict,
                     slave: "SwathInfo", slave_grid: dict):
    """(m_burst0, m_burstN, s_burst0, s_burstN), 0-based (tops_s1_burst_overlap);
    burst0 / burstN are 1-based as in config.txt."""
    mg, k1 = _grid_struct(master_grid)
    sg, k2 = _grid_struct(slave_grid)
    out = [C.c_int(-1) for _ in range(4)]
    check(lib.tops_s1_burst_overlap(burst0, burstN, C.byref(master), C.byref(mg),
                                    C.byref(slave), C.byref(sg), *(C.byref(o) for o in out)),
          "tops_s1_burst_overlap")
    return tuple(o.value for o in out)


_proto("tops_pair_stage_times", C.c_int, [_vp, _vp, _fp])
_proto("tops_pair_process", C.c_int, [_vp, _vp, _vp, _vp, _vp, _fp, _dp, _dp, _vp])
_proto("tops_batch_create", C.c_int, [C.POINTER(_vp), C.c_int, C.POINTER(_vp)])
_proto("tops_batch_destroy", C.c_int, [_vp])
_proto("tops_batch_run", C.c_int, [_vp, _vp])
_proto("tops_batch_run_graph", C.c_int, [_vp, _vp])
_proto("tops_batch_launches", C.c_int, [_vp])
_proto("tops_batch_set_tune", C.c_int, [_vp, C.POINTER(Tune)])
_proto("tops_batch_get_tune", C.c_int, [_vp, C.POINTER(Tune)])
_proto("tops_batch_autotune", C.c_int, [_vp, _vp, C.POINTER(Tune), _dp])


def pair_opts(**kw) -> PairOpts:
    o = PairOpts()
    check(lib.tops_pair_opts_default(C.byref(o)), "tops_pair_opts_default")
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def scene_windows(scene: "Scene", margin: int = 24):
    nb = scene.cfg.n_bursts
    w = (DemWindow * nb)()
    for b in range(nb):
        r0, c0, nr, nc = scene.dem_window(b, margin)
        w[b] = DemWindow(r0, c0, nr, nc)
    return w


class Pair:
    """Device-resident burst-pair plan (tops_pair_*).  `stream` arguments are
    raw cudaStream_t values (0 = legacy default stream)."""

    def __init__(self, master: SwathInfo, slave: SwathInfo, dem_shape, opts: PairOpts = None):
        self.opts = opts or pair_opts()
        self.master, self.slave = master, slave
        self.nb, self.L, self.W = master.n_bursts, master.lines_per_burst, master.samples_per_burst
        self.dem_shape = dem_shape
        h = C.c_void_p()
        check(lib.tops_pair_create(C.byref(master), C.byref(slave), C.byref(self.opts),
                                   dem_shape[0], dem_shape[1], C.byref(h)), "tops_pair_create")
        self._h = h

    @staticmethod
    def footprint(master: SwathInfo, dem_shape, opts: PairOpts = None) -> int:
        opts = opts or pair_opts()
        return lib.tops_pair_footprint(C.byref(master), C.byref(opts), dem_shape[0], dem_shape[1])

    def set_dem(self, dem, lat0, lon0, dlat, dlon, windows, stream=0):
        dem = np.ascontiguousarray(dem, np.float32)
        assert dem.shape == tuple(self.dem_shape)
        self._dem_keep = dem
        check(lib.tops_pair_set_dem(self._h, ptr(dem, C.c_float), lat0, lon0, dlat, dlon, windows,
                                    C.c_void_p(stream)), "tops_pair_set_dem")

    def upload(self, master_slc, slave_slc, stream=0):
        check(lib.tops_pair_upload(self._h, C.c_void_p(master_slc.ctypes.data),
                                   C.c_void_p(slave_slc.ctypes.data), C.c_void_p(stream)),
              "tops_pair_upload")

    def run(self, stream=0, graph=False):
        f = lib.tops_pair_run_graph if graph else lib.tops_pair_run
        check(f(self._h, C.c_void_p(stream)), "tops_pair_run")

    def run_per_burst(self, stream=0):
        check(lib.tops_pair_run_per_burst(self._h, C.c_void_p(stream)), "tops_pair_run_per_burst")

    def download(self, reslave=True, stream=0):
        n = self.nb * self.L
        rs = np.zeros((n, self.W), np.complex64) if reslave else None
        re = np.zeros((n, self.W), np.complex64)
        coh = np.zeros((n, self.W), np.float32)
        cpm = np.zeros((self.nb, 12))
        sh = np.zeros(max(self.nb - 1, 1))
        check(lib.tops_pair_download(self._h, vptr(rs) if reslave else None, vptr(re),
                                     ptr(coh, C.c_float), ptr(cpm, C.c_double),
                                     ptr(sh, C.c_double), C.c_void_p(stream)), "tops_pair_download")
        return dict(reslave=rs, reslave_esd=re, coh=coh, cpm=cpm, shifts=sh[:self.nb - 1])

    def process(self, master_slc, slave_slc, out=None, reslave=True, stream=0):
        """Host to host in one pipelined call (tops_pair_process).  `out`:
        preallocated outputs (dict as download returns; pinned for
        overlapped copies), else fresh arrays.  Returns once enqueued when
        `out` is given; otherwise synchronises and returns the outputs."""
        fresh = out is None
        if fresh:
            n = self.nb * self.L
            out = dict(reslave=np.zeros((n, self.W), np.complex64) if reslave else None,
                       reslave_esd=np.zeros((n, self.W), np.complex64),
                       coh=np.zeros((n, self.W), np.float32), cpm=np.zeros((self.nb, 12)),
                       shifts=np.zeros(max(self.nb - 1, 1)))
        g = lambda k: out.get(k) if out.get(k) is not None else None
        check(lib.tops_pair_process(
            self._h, C.c_void_p(master_slc.ctypes.data), C.c_void_p(slave_slc.ctypes.data),
            vptr(g("reslave")) if g("reslave") is not None else None,
            vptr(g("reslave_esd")) if g("reslave_esd") is not None else None,
            ptr(g("coh"), C.c_float) if g("coh") is not None else None,
            ptr(g("cpm"), C.c_double) if g("cpm") is not None else None,
            ptr(g("shifts"), C.c_double) if g("shifts") is not None else None,
            C.c_void_p(stream)), "tops_pair_process")
        if fresh:
            check(lib.tops_stream_synchronize(C.c_void_p(stream)), "tops_stream_synchronize")
            out["shifts"] = out["shifts"][:self.nb - 1]
        return out

    def stage_times(self, stream=0):
        """ms of geocoreg, ReSlave resample, ESD, ReSlaveESD resample, coherence."""
        ms = np.zeros(5, np.float32)
        check(lib.tops_pair_stage_times(self._h, C.c_void_p(stream), ptr(ms, C.c_float)),
              "tops_pair_stage_times")
        return dict(zip(("geocoreg", "resample", "esd", "resample_esd", "coherence"),
                        map(float, ms)))

    def buffers(self) -> PairBuffers:
        b = PairBuffers()
        check(lib.tops_pair_buffers_get(self._h, C.byref(b)), "tops_pair_buffers_get")
        return b

    def close(self):
        if getattr(self, "_h", None):
            lib.tops_pair_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Several device-resident plans processed together (tops_batch_*): one
    launch per stage for all their bursts.  The plans stay owned by the
    caller and must outlive the batch."""

    def __init__(self, pairs):
        self.pairs = list(pairs)
        arr = (_vp * len(self.pairs))(*[p._h.value for p in self.pairs])
        h = _vp()
        check(lib.tops_batch_create(arr, len(self.pairs), C.byref(h)), "tops_batch_create")
        self._h = h

    def run(self, stream=0, graph=False):
        f = lib.tops_batch_run_graph if graph else lib.tops_batch_run
        check(f(self._h, C.c_void_p(stream)), "tops_batch_run")

    def launches(self) -> int:
        return lib.tops_batch_launches(self._h)

    def tune(self, t: "Tune" = None) -> "Tune":
        if t is not None:
            check(lib.tops_batch_set_tune(self._h, C.byref(t)), "tops_batch_set_tune")
        out = Tune()
        check(lib.tops_batch_get_tune(self._h, C.byref(out)), "tops_batch_get_tune")
        return out

    def autotune(self, stream=0):
        best = Tune()
        ms = np.zeros(2)
        check(lib.tops_batch_autotune(self._h, C.c_void_p(stream), C.byref(best),
                                      ptr(ms, C.c_double)), "tops_batch_autotune")
        return best, ms

    def close(self):
        if getattr(self, "_h", None):
            lib.tops_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------ serving loop
class ServerCfg(C.Structure):
    _fields_ = [("hbm_budget", C.c_size_t), ("slots", C.c_int)]


class JobDesc(C.Structure):
    _fields_ = [("master", SwathInfo), ("slave", SwathInfo), ("opts", PairOpts),
                ("dem_id", C.c_int), ("windows", DemWindow * MAX_BURSTS),
                ("master_slc", C.c_void_p), ("slave_slc", C.c_void_p),
                ("reslave", C.c_void_p), ("reslave_esd", C.c_void_p), ("coh", C.c_void_p),
                ("cpm", C.c_void_p), ("shifts", C.c_void_p)]


class JobDone(C.Structure):
    _fields_ = [("job_id", C.c_long), ("status", C.c_int), ("arrival_s", C.c_double),
                ("admit_s", C.c_double), ("done_s", C.c_double), ("footprint", C.c_size_t)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_long), ("admitted", C.c_long), ("completed", C.c_long),
                ("rejected", C.c_long), ("queued", C.c_long), ("running", C.c_long),
                ("hbm_in_use", C.c_size_t), ("hbm_peak", C.c_size_t)]


_proto("tops_server_create", C.c_int, [C.POINTER(ServerCfg), C.POINTER(_vp)])
_proto("tops_server_destroy", C.c_int, [_vp])
_proto("tops_server_add_dem", C.c_int, [_vp, _fp, C.c_int, C.c_int, C.c_double, C.c_double,
                                        C.c_double, C.c_double, _ip])
_proto("tops_server_submit", C.c_int, [_vp, C.POINTER(JobDesc), C.POINTER(C.c_long)])
_proto("tops_server_progress", C.c_int, [_vp])
_proto("tops_server_poll", C.c_int, [_vp, C.POINTER(JobDone), C.c_int, _ip])
_proto("tops_server_drain", C.c_int, [_vp])
_proto("tops_server_get_stats", C.c_int, [_vp, C.POINTER(ServerStats)])
_proto("tops_server_job_footprint", C.c_size_t, [C.POINTER(JobDesc)])
_proto("tops_arena_create", C.c_int, [C.c_size_t, C.c_size_t, C.POINTER(_vp)])
_proto("tops_arena_destroy", C.c_int, [_vp])
_proto("tops_arena_alloc", C.c_size_t, [_vp, C.c_size_t])
_proto("tops_arena_release", C.c_int, [_vp, C.c_size_t])
_proto("tops_arena_in_use", C.c_size_t, [_vp])
_proto("tops_arena_largest_free", C.c_size_t, [_vp])
_proto("tops_arena_free_ranges", C.c_int, [_vp])


def sub_swath(info: SwathInfo, b0: int, k: int) -> SwathInfo:
    """The description of bursts [b0, b0+k) of a sub-swath as a k-burst
    sub-swath: burst times, the per-burst FM-rate list and (when the
    annotation holds one estimate per burst) the DC list shift with it."""
    out = SwathInfo()
    C.memmove(C.byref(out), C.byref(info), C.sizeof(SwathInfo))
    out.n_bursts = k
    for i in range(k):
        out.burst_first_line_time[i] = info.burst_first_line_time[b0 + i]
        out.burst_last_line_time[i] = info.burst_last_line_time[b0 + i]
    for i in range(info.n_fm - b0):
        out.fm_list[i] = info.fm_list[b0 + i]
    out.n_fm = info.n_fm - b0
    if info.n_dc > info.n_bursts:
        for i in range(info.n_dc - b0):
            out.dc_list[i] = info.dc_list[b0 + i]
        out.n_dc = info.n_dc - b0
    return out


class Server:
    """tops_server_*: burst-pair jobs admitted by HBM footprint, one stream
    per slot.  Host buffers of a job must stay alive until it is done."""

    def __init__(self, hbm_budget: int, slots: int):
        cfg = ServerCfg(hbm_budget, slots)
        h = _vp()
        check(lib.tops_server_create(C.byref(cfg), C.byref(h)), "tops_server_create")
        self._h = h
        self._keep = {}

    def add_dem(self, dem, lat0, lon0, dlat, dlon) -> int:
        dem = np.ascontiguousarray(dem, np.float32)
        i = C.c_int()
        check(lib.tops_server_add_dem(self._h, ptr(dem, C.c_float), dem.shape[0], dem.shape[1],
                                      lat0, lon0, dlat, dlon, C.byref(i)), "tops_server_add_dem")
        return i.value

    def job(self, scene: "Scene", dem_id: int, b0: int = 0, k: int = None, opts=None,
            outputs=None, master_slc=None, slave_slc=None):
        """A job over bursts [b0, b0+k) of a scene; returns (desc, outputs)."""
        k = scene.cfg.n_bursts - b0 if k is None else k
        L, W = scene.cfg.lines_per_burst, scene.cfg.samples_per_burst
        d = JobDesc()
        d.master = sub_swath(scene.swath[0], b0, k)
        d.slave = sub_swath(scene.swath[1], b0, k)
        d.opts = opts or pair_opts()
        d.dem_id = dem_id
        for i in range(k):
            r0, c0, nr, nc = scene.dem_window(b0 + i)
            d.windows[i] = DemWindow(r0, c0, nr, nc)
        m = scene.slc[0] if master_slc is None else master_slc
        s = scene.slc[1] if slave_slc is None else slave_slc
        d.master_slc = m.ctypes.data + b0 * L * W * 4
        d.slave_slc = s.ctypes.data + b0 * L * W * 4
        if outputs is None:
            outputs = dict(reslave=np.zeros((k * L, W), np.complex64),
                           reslave_esd=np.zeros((k * L, W), np.complex64),
                           coh=np.zeros((k * L, W), np.float32), cpm=np.zeros((k, 12)),
                           shifts=np.zeros(max(k - 1, 1)))
        for f in ("reslave", "reslave_esd", "coh", "cpm", "shifts"):
            a = outputs.get(f)
            setattr(d, f, a.ctypes.data if a is not None else None)
        return d, outputs

    def submit(self, desc: JobDesc, keep=None) -> int:
        jid = C.c_long()
        check(lib.tops_server_submit(self._h, C.byref(desc), C.byref(jid)), "tops_server_submit")
        self._keep[jid.value] = (desc, keep)
        return jid.value

    def progress(self):
        check(lib.tops_server_progress(self._h), "tops_server_progress")

    def poll(self, max_n=256):
        arr = (JobDone * max_n)()
        n = C.c_int()
        check(lib.tops_server_poll(self._h, arr, max_n, C.byref(n)), "tops_server_poll")
        out = [arr[i] for i in range(n.value)]
        for d in out:
            self._keep.pop(d.job_id, None)
        return out

    def drain(self):
        check(lib.tops_server_drain(self._h), "tops_server_drain")

    def stats(self) -> ServerStats:
        st = ServerStats()
        check(lib.tops_server_get_stats(self._h, C.byref(st)), "tops_server_get_stats")
        return st

    def close(self):
        if getattr(self, "_h", None):
            lib.tops_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def plain_pair(scene: "Scene", opts: PairOpts = None, dem_int=None, windows=None):
    """Reference-shaped per-burst processing (tops_plain_pair) on host arrays."""
    opts = opts or pair_opts()
    S = scene
    n, W = S.shape
    di = S.dem_info
    dem_int = np.ascontiguousarray(np.rint(S.dem) if dem_int is None else dem_int, np.int32)
    windows = windows if windows is not None else scene_windows(S)
    rs = np.zeros((n, W), np.complex64)
    re = np.zeros((n, W), np.complex64)
    coh = np.zeros((n, W), np.float32)
    cpm = np.zeros((S.cfg.n_bursts, 12))
    sh = np.zeros(max(S.cfg.n_bursts - 1, 1))
    check(lib.tops_plain_pair(C.byref(S.swath[0]), C.byref(S.swath[1]), C.byref(opts),
                              ptr(dem_int, C.c_int), di.lines, di.pixels, di.lat0, di.lon0,
                              di.dlat, di.dlon, windows, vptr(S.slc[0]), vptr(S.slc[1]), vptr(rs),
                              vptr(re), ptr(coh, C.c_float), ptr(cpm, C.c_double),
                              ptr(sh, C.c_double)), "tops_plain_pair")
    return dict(reslave=rs, reslave_esd=re, coh=coh, cpm=cpm, shifts=sh[:S.cfg.n_bursts - 1])
