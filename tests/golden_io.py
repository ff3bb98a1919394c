"""Loading the golden fixtures made by tests/golden/make_golden.py.

ref_host.npz holds the reference's host precomputes (Polyfit_Orbit,
ComputeDerampPara, InKernelInit, EstOverlapSize, GetSpectralSep) on a seeded
synthetic sub-swath pair; ref_stages.npz holds the same scene's SLCs and DEM
windows with what the reference's four CUDA stages returned for them.
"""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    path = os.path.join(GOLDEN, name)
    with np.load(path) as d:
        return {k: d[k] for k in d.files}


def swath_info(T, F, tag, dc_key="dc_list"):
    """topsb200.SwathInfo rebuilt from a fixture's plain arrays."""
    info = T.SwathInfo()
    nb, L, W, fvp = (int(v) for v in F[f"{tag}_ints"])
    (info.dt, info.prf, info.slr_time, info.range_spacing, info.wavelength, info.rsr,
     info.az_bandwidth, info.steering_rate_deg, info.first_line_time,
     info.last_line_time) = (float(v) for v in F[f"{tag}_reals"])
    info.n_bursts, info.lines_per_burst, info.samples_per_burst = nb, L, W
    info.first_valid_pixel = fvp
    for b in range(nb):
        info.burst_first_line_time[b] = F[f"{tag}_burst_first"][b]
        info.burst_last_line_time[b] = F[f"{tag}_burst_last"][b]
    for name, key in (("dc", f"{tag}_{dc_key}"), ("fm", f"{tag}_fm_list")):
        lst = F[key]
        setattr(info, f"n_{name}", len(lst))
        arr = getattr(info, f"{name}_list")
        for k, row in enumerate(lst):
            arr[k] = T.Poly(*(float(v) for v in row))
    sv = F[f"{tag}_sv"]
    info.n_sv = sv.shape[1]
    for k in range(sv.shape[1]):
        info.sv_t[k], info.sv_x[k], info.sv_y[k], info.sv_z[k] = (float(v) for v in sv[:, k])
    return info


def burst_boxes(b, L, W):
    """MasterBox / SlaveBox of burst b with burst gap 0 (Func.cpp:2354-2371)."""
    box = np.array([0, W - 1, b * L, (b + 1) * L - 1], np.int32)
    return box, box.copy()
