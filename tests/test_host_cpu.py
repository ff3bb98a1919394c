"""CPU tests: product host precomputes vs the oracle, config reader, C ABI
exports, and oracle known-answer checks.  No GPU calls."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import PKG, ROOT, c64, rel_rms


# ------------------------------------------------------------ C ABI exports
def _declared_functions():
    names = set()
    for h in sorted(f for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b([A-Za-z_]\w*)\s*\(", src, re.M):
            name = m.group(1)
            if name not in ("if", "for", "while", "return", "sizeof"):
                names.add(name)
    return sorted(names)


def test_library_exports_every_declared_symbol(T):
    names = _declared_functions()
    for n in ("DerampDemodResample", "GeoCoreg_warp_cuda", "tops_pair_process", "tops_batch_run",
              "tops_server_submit", "tops_stream_synchronize"):
        assert n in names, n
    missing = [n for n in names if not hasattr(T.lib, n)]
    assert not missing, missing


def test_reference_entry_points_present(T):
    for n in ["GeoCoreg_warp_cuda", "DerampDemodResample", "DerampDemodResample_ESD",
              "ResampleFirstBurst", "EstESDShifts", "CoherenceEst", "CoherenceEst_ESD"]:
        assert hasattr(T.lib, n)


def test_status_strings(T):
    assert T.lib.tops_status_string(0) == b"ok"
    assert b"positive definite" in T.lib.tops_status_string(T.TOPS_E_NOT_PD)


# ------------------------------------------------- host precomputes vs oracle
@pytest.mark.parametrize("prf,abw,rsr2x", [(486.4963503649635, 327.0, 2 * 64.345e6),
                                           (486.5, 313.0, 2 * 64.345e6)])
def test_lut_bit_identical_to_oracle(T, O, prf, abw, rsr2x):
    ka, kr = T.lut(prf, abw, rsr2x)
    oa, orr = O.lut(prf, abw, rsr2x)
    assert np.array_equal(ka, oa) and np.array_equal(kr, orr)
    # rows are normalised to ~1 (float rounding of each tap)
    assert np.abs(ka.astype(np.float64).sum(1) - 1).max() < 1e-6


def test_polyfit_orbit_matches_oracle(T, O, scene_small):
    m = scene_small.swath[0]
    n = m.n_sv
    a = T.polyfit_orbit(m.sv_t[:n], m.sv_x[:n], m.sv_y[:n], m.sv_z[:n])
    b = O.polyfit_orbit(m.sv_t[:n], m.sv_x[:n], m.sv_y[:n], m.sv_z[:n])
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    # the fit reproduces the state vectors to < 1 mm
    t = (np.array(m.sv_t[:n]) - m.sv_t[n // 2]) / 10.0
    x = np.polyval(a[0][::-1], t)
    assert np.abs(x - np.array(m.sv_x[:n])).max() < 1e-3


def test_deramp_params_match_oracle(O, scene_small):
    S = scene_small
    for w in (0, 1):
        o = O.deramp_params(S.swath[w], S.orbit[w])
        for k in ("dc", "fmrate", "tref", "kt"):
            assert np.array_equal(o[k], S.deramp[w][k]), k
    kt = S.deramp[0]["kt"]
    assert 1500 < kt.mean() < 2100   # ~1.76 kHz/s for S1 IW with 1.59 deg/s steering


def test_overlap_and_spectral_sep(T, O, scene_small):
    S = scene_small
    m = S.swath[0]
    nb = m.n_bursts
    first = np.array(m.burst_first_line_time[:nb])
    last = np.array(m.burst_last_line_time[:nb])
    a = T.overlap_size(first, last, m.dt)
    b = O.overlap_size(first, last, m.dt)
    assert np.array_equal(a[0], b[0]) and a[1:] == b[1:]
    assert np.all(a[0] == S.cfg.overlap_lines)
    ss_t = T.spectral_sep(S.deramp[0]["kt"], m.lines_per_burst, m.dt)
    ss_o = O.spectral_sep(S.deramp[0]["kt"], m.lines_per_burst, m.dt)
    assert ss_t == ss_o


# ------------------------------------------------------------- config file
def test_config_reference_keys(T, tmp_path):
    p = tmp_path / "config.txt"
    p.write_text("process_dir= /tmp/work\nmasterpath=/data/S1A_master.SAFE\n"
                 "slavepath=/data/S1B_slave.SAFE\npreciseOrbitMaster=/o/m.EOF\n"
                 "preciseOrbitSlave=/o/s.EOF\nSpecificDemPath=/dem/srtm.tif\n"
                 "firstsubswath=1\nburst0=2\nburstN=5\nlastsubswath=3\npolarisation=vh\n"
                 "unknown_key=whatever\n\n")
    c = T.read_config(str(p))
    assert c.process_dir == b"/tmp/work" and c.masterpath == b"/data/S1A_master.SAFE"
    assert (c.firstsubswath, c.lastsubswath, c.burst0, c.burstN) == (1, 3, 2, 5)
    assert c.polarisation == b"vh" and c.SpecificDemPath == b"/dem/srtm.tif"


def test_config_synthetic_keys_and_tabs(T, tmp_path):
    p = tmp_path / "config.txt"
    p.write_text("seed\t=\t42\nn_bursts=9\nlines_per_burst=1500\nsamples_per_burst=21000\n"
                 "coh_win_rg=10\ncoh_win_az=3\nhbm_budget_gb=150\narrival_rate=40\n")
    c = T.read_config(str(p))
    assert (c.seed, c.n_bursts, c.samples_per_burst) == (42, 9, 21000)
    assert c.hbm_budget_gb == 150.0 and c.arrival_rate == 40.0


@pytest.mark.parametrize("text", ["burst0=two\n", "n_bursts=\n", "coh_win_rg=10x\n",
                                  "burst0=5\nburstN=2\n", "npoints=6\n"])
def test_config_malformed(T, tmp_path, text):
    p = tmp_path / "config.txt"
    p.write_text(text)
    with pytest.raises(T.TopsError) as ei:
        T.read_config(str(p))
    assert ei.value.status == T.TOPS_E_CONFIG


def test_config_missing_file(T, tmp_path):
    with pytest.raises(T.TopsError):
        T.read_config(str(tmp_path / "nope.txt"))


# ------------------------------------------------- oracle known answers
def test_oracle_resample_identity(O, scene_small):
    """Identity polynomial, no deramp: the interior reproduces the input."""
    S = scene_small
    L, W = S.cfg.lines_per_burst, S.cfg.samples_per_burst
    mb, sb = S.boxes(0)
    # polyval(L^, P^) = y with L^ = (y - mid)/q  ->  c0 = mid, c1 = q
    caz = [0.5 * (mb[2] + mb[3]), 0.25 * (mb[3] - mb[2]), 0, 0, 0, 0]
    crg = [0.5 * (mb[0] + mb[1]), 0, 0.25 * (mb[1] - mb[0]), 0, 0, 0]
    z = np.zeros(W)
    out, cnt = O.resample(S.burst(1, 0), caz, crg, 0.0, S.kaz, S.krg, 0, mb, sb, L, S.swath[1].dt,
                          z, z, z)
    src = S.burst(1, 0)[..., 0] + 1j * S.burst(1, 0)[..., 1]
    # positions land on integer samples up to rounding: bin 0 or 2047
    assert rel_rms(out[10:-10, 10:-10], src[10:-10, 10:-10]) < 1e-6


def test_oracle_coherence_known_answers(O, scene_small):
    m = scene_small.burst(0, 0)
    s = m.astype(np.float32)
    coh = O.coherence(m, s, 10, 3)
    assert np.abs(coh[np.hypot(s[..., 0], s[..., 1]) >= 1e-3] - 1).max() < 1e-12
    # independent noise: coherence ~ bias level for 30 looks (~0.16)
    rng = np.random.default_rng(0)
    n = (rng.standard_normal(s.shape) * 700).astype(np.float32)
    coh = O.coherence(m, n, 10, 3)
    assert 0.1 < coh[5:-5, 5:-5].mean() < 0.25


def test_oracle_esd_known_phase(O):
    """dd with a constant phase p -> shift = p / (2 pi df dt)."""
    rng = np.random.default_rng(3)
    lines, W, p = 40, 256, 0.3
    a = (rng.standard_normal((lines, W, 2)) * 800).astype(np.int16)
    s = a.astype(np.float32)
    mF = a
    sF = s                                        # mF sF* real positive
    mB = a
    z = s[..., 0] + 1j * s[..., 1]
    sB = c64(z * np.exp(1j * p))                  # mB sB* ~ exp(-i p)
    shift, sums, used = O.esd(mF, mB, sF, sB, np.array([lines]), 3, 10, 0.3, 1500.0, 2e-3)
    assert used[0] > 0
    assert abs(shift[0] - p / (2 * np.pi * 1500.0 * 2e-3)) < 1e-9


def test_oracle_geocoreg_recovers_truth(O, scene_small):
    S = scene_small
    for b in range(S.cfg.n_bursts):
        g = S.geo_args(b)
        az, rg, st, nv = O.geocoreg(g["dem"], g["lat0"], g["lon0"], g["dlat"], g["dlon"],
                                    g["xmin"], g["xmax"], g["ymin"], g["ymax"], g["dt"],
                                    g["first_line_time"], g["slr_time"], g["range_spacing"],
                                    g["mid_time"], g["azi_init"], g["line_offset"], g["coefs"])
        assert st == 0
        tr = S.truth(b)
        Lh = (tr[:, 0] - 0.5 * (g["ymin"] + g["ymax"])) / (0.25 * (g["ymax"] - g["ymin"]))
        Ph = (tr[:, 1] - 0.5 * (g["xmin"] + g["xmax"])) / (0.25 * (g["xmax"] - g["xmin"]))
        A = np.stack([np.ones_like(Lh), Lh, Ph, Lh * Lh, Lh * Ph, Ph * Ph], 1)
        ins = ((tr[:, 0] >= g["ymin"]) & (tr[:, 0] <= g["ymax"]) & (tr[:, 1] >= g["xmin"]) &
               (tr[:, 1] <= g["xmax"]))
        # the quadratic fit leaves only the topographic residual (< 0.05 px)
        assert np.abs(A[ins] @ az - tr[ins, 2]).max() < 0.05
        assert np.abs(A[ins] @ rg - tr[ins, 3]).max() < 0.05
        # offsets of the synthetic geometry: <= 0.5 px azimuth, <= 3 px range
        assert np.abs(tr[ins, 2] - tr[ins, 0]).max() <= 0.5
        assert np.abs(tr[ins, 3] - tr[ins, 1]).max() <= 3.0


# ---------------------------------------------------------------- generator
def test_synth_deterministic(T):
    a = T.Scene(n_bursts=2, lines_per_burst=128, samples_per_burst=256, overlap_lines=16,
                dem_lines=96, dem_pixels=96, seed=9)
    b = T.Scene(n_bursts=2, lines_per_burst=128, samples_per_burst=256, overlap_lines=16,
                dem_lines=96, dem_pixels=96, seed=9, threads=1)
    assert np.array_equal(a.slc[0], b.slc[0]) and np.array_equal(a.slc[1], b.slc[1])
    assert np.array_equal(a.dem, b.dem)
    c = T.Scene(n_bursts=2, lines_per_burst=128, samples_per_burst=256, overlap_lines=16,
                dem_lines=96, dem_pixels=96, seed=10)
    assert not np.array_equal(a.slc[0], c.slc[0])


def test_synth_statistics(scene_small):
    S = scene_small
    z = S.slc[0].astype(np.float64)
    rms = np.sqrt((z ** 2).sum(-1).mean())
    assert 900 < rms < 1100                      # sigma = 1000 DN
    assert 0.0 <= S.dem.min() and S.dem.max() <= 1500.0 + 1e-3


def test_synth_invalid_config(T):
    with pytest.raises(T.TopsError):
        T.Scene(n_bursts=0)
    with pytest.raises(T.TopsError):
        T.Scene(overlap_lines=2000)


def test_device_slots_keep_devices_apart(tmp_path):
    """The reference-compatible wrappers' per-thread caches (workspace, LUT
    copy) hold one slot per device index, tagged with its device
    (csrc/device_slots.h): a call after a device change gets another slot,
    never the buffers of the previous device; indexes outside the table are
    refused."""
    import subprocess
    src = tmp_path / "slots.cpp"
    src.write_text(r"""
#include "device_slots.h"
#include <cstdio>
struct Cache { int dev = -1; int buffers = 0; };
int main() {
  static tops::DeviceSlots<Cache, 8> c;
  Cache *a = c.at(0);
  a->buffers = 7;                      // allocated on device 0
  Cache *b = c.at(1);                  // the thread switched to device 1
  if (b == a || b->dev != 1 || b->buffers != 0) return 1;
  if (c.at(0) != a || a->dev != 0 || a->buffers != 7) return 2;
  if (c.at(-1) || c.at(8)) return 3;
  std::puts("ok");
  return 0;
}
""")
    exe = tmp_path / "slots"
    inc = os.path.join(PKG, "csrc")
    r = subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I" + inc, str(src), "-o",
                        str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", (r.returncode, r.stdout)
