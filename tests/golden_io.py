"""Loading the golden fixtures made by tests/golden/make_golden.py.

ref_host{sfx}.npz holds the reference's host precomputes (Polyfit_Orbit,
ComputeDerampPara, InKernelInit, EstOverlapSize, GetSpectralSep) on a seeded
synthetic sub-swath pair; ref_stages{sfx}.npz holds the same scene's SLCs and
DEM windows with what the reference's four CUDA stages returned for them.
Scene "" is 3 bursts of 128 x 256 with 24-line overlaps, scene "2" is 4
bursts of 160 x 300 with 30-line overlaps (other seed, other orbit draw).
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


SCENES = ("", "2")
WINDOWS = ((24, 6), (10, 3))


class Scene:
    """One golden scene: the stage fixture G, the host fixture H and the
    helpers that turn them into the arguments of each stage call."""

    def __init__(self, sfx):
        self.sfx = sfx
        self.G = load(f"ref_stages{sfx}.npz")
        self.H = load(f"ref_host{sfx}.npz")
        self.NB, self.L, self.W, _ = (int(v) for v in self.G["m_ints"])

    def __repr__(self):
        return f"scene{self.sfx or '1'}"

    def poly_grid(self, c, b):
        """The 6-term offset polynomial of burst b on a 31 x 41 grid of its
        pixels (normalised as the reference's warp polynomial)."""
        L, W = self.L, self.W
        y = np.linspace(b * L, (b + 1) * L - 1, 31)
        x = np.linspace(0, W - 1, 41)
        Y, X = np.meshgrid(y, x, indexing="ij")
        Lh = (Y - (b * L + 0.5 * (L - 1))) / (0.25 * (L - 1))
        Ph = (X - 0.5 * (W - 1)) / (0.25 * (W - 1))
        return c[0] + c[1] * Lh + c[2] * Ph + c[3] * Lh * Lh + c[4] * Lh * Ph + c[5] * Ph * Ph

    def geo_args(self, b):
        G, H, L, W = self.G, self.H, self.L, self.W
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

    def rs_kwargs(self, b, shift, dt):
        G, H, L = self.G, self.H, self.L
        box, sbox = burst_boxes(b, L, self.W)
        return dict(slave=G["slave_slc"][b * L:(b + 1) * L], cpm_az=G["cpm_az"][b],
                    cpm_rg=G["cpm_rg"][b], az_shift=float(shift), kaz=H["lut_kaz"],
                    krg=H["lut_krg"], s_burst_idx=b, mbox=box, sbox=sbox, lines_per_burst=L,
                    dt=float(dt), kt=H["s_kt"][0], tref=H["s_tref"][0], fdc=H["s_dc"][0])

    def resample_cases(self, b):
        """ReSlave (slave dt, no shift) and, after the first burst,
        ReSlaveESD (master dt, shift of the overlap before the burst)."""
        G = self.G
        cases = [("reslave", 0.0, G["s_reals"][0])]
        if b > 0:
            cases.append(("reslave_esd_24x6", G["esd_shift_24x6"][b - 1], G["m_reals"][0]))
        return cases

    def esd_bands(self, reslave):
        L, NB = self.L, self.NB
        ov = self.H["m_ov"]
        ms = self.G["master_slc"]
        mF = np.concatenate([ms[(i + 1) * L - ov[i]:(i + 1) * L] for i in range(NB - 1)])
        mB = np.concatenate([ms[(i + 1) * L:(i + 1) * L + ov[i]] for i in range(NB - 1)])
        sF = np.concatenate([reslave[i][L - ov[i]:] for i in range(NB - 1)])
        sB = np.concatenate([reslave[i + 1][:ov[i]] for i in range(NB - 1)])
        return mF, mB, sF, sB, ov

    def interior(self, wr, wa):
        """Pixels whose coherence box touches no pad (the reference's pads of
        CoherenceEst are uninitialised device memory, EstCoh.cu:793-797)."""
        dx, dy = (wr - 1) // 2, (wa - 1) // 2
        return slice(dy, self.L - (wa - 1 - dy)), slice(dx, self.W - (wr - 1 - dx))

    def dem_canvas(self):
        """The per-burst DEM windows of the fixture placed on one grid, with
        their offsets (the pipeline takes one DEM and a window per burst)."""
        G, NB = self.G, self.NB
        dlat, dlon = G["dem_geo0"][2], G["dem_geo0"][3]
        offs = []
        for b in range(NB):
            lat0, lon0 = G[f"dem_geo{b}"][:2]
            offs.append((int(round((G["dem_geo0"][0] - lat0) / dlat)),
                         int(round((lon0 - G["dem_geo0"][1]) / dlon))))
        r_min = min(r for r, _ in offs)
        c_min = min(c for _, c in offs)
        rows = max(r - r_min + G[f"dem{b}"].shape[0] for b, (r, _) in enumerate(offs))
        cols = max(c - c_min + G[f"dem{b}"].shape[1] for b, (_, c) in enumerate(offs))
        dem = np.full((rows, cols), -32768.0, np.float32)
        wins = []
        for b, (r, c) in enumerate(offs):
            d = G[f"dem{b}"]
            r0, c0 = r - r_min, c - c_min
            dem[r0:r0 + d.shape[0], c0:c0 + d.shape[1]] = d
            wins.append((r0, c0, d.shape[0], d.shape[1]))
        lat0 = G["dem_geo0"][0] - r_min * dlat
        lon0 = G["dem_geo0"][1] + c_min * dlon
        return dem, lat0, lon0, dlat, dlon, wins


_CACHE = {}


def scene(sfx):
    if sfx not in _CACHE:
        _CACHE[sfx] = Scene(sfx)
    return _CACHE[sfx]


def scene_bursts():
    """(scene, burst) pairs over every burst of every scene, for parametrize."""
    return [(s, b) for s in SCENES for b in range(scene(s).NB)]
