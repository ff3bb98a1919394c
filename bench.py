#!/usr/bin/env python3
"""Benchmark: burst-pairs/s of the TOPS burst-pair path on B200.

Workload (default): one full sub-swath pair -- 9 master and 9 slave bursts
of 1,500 x 21,000 CInt16, 100-line overlaps (8 ESD overlaps), DEM 3,600 x
3,600 float32 fBm -- synthetic and seeded.  A step is one pass of the whole
path over that pair: geometric coregistration of the 9 bursts, resampling
(ReSlave), ESD over the 8 overlaps, ESD-corrected resampling (ReSlaveESD) and
coherence.  One burst pair = one master burst with its slave burst, so a
step processes 9 burst pairs.

  value   device-resident batched form (inputs already in HBM), CUDA events
  e2e     same metric through the public C ABI with pinned host buffers:
          upload of both SLCs, the run, download of ReSlave, ReSlaveESD,
          coherence and shifts, all inside the timed region
  plain   the reference-shaped per-burst form (reference entry points, host
          buffers), for the batched-vs-plain ratio

Multi-GPU: one process per GPU (torchrun); each rank processes its own
sub-swath pair (replicas, no data exchange): weak scaling, timed as the max
over ranks.  `--impl reference` times the CPU FP64 port of the reference
path (the oracle) on the host cores, on bounded samples of the same work.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "insar-on-sentinel-1-tops-data_b200")
sys.path.insert(0, PKG)

import numpy as np  # noqa: E402

METRIC = "burst-pairs/s (coreg+resample+ESD+coh)"
UNIT = "burst-pairs/s"

CONFIGS = {
    # BASELINE config "Plain method, full subswath"
    "subswath": dict(n_bursts=9, lines_per_burst=1500, samples_per_burst=21000,
                     overlap_lines=100, dem_lines=3600, dem_pixels=3600, seed=2),
    # BASELINE config "Plain method, small" (parity-scale)
    "small": dict(n_bursts=2, lines_per_burst=1500, samples_per_burst=4096, overlap_lines=100,
                  dem_lines=512, dem_pixels=512, seed=1),
}
WIN_RG, WIN_AZ = 10, 3


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([v.strip() for v in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 5 + i and s[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def build_scene(T, cfg, rank):
    c = dict(cfg)
    c["seed"] = c["seed"] + 1000 * rank
    return T.Scene(**c)


def cpu_sample(scene_cfg, seconds_target=15.0):
    """FP64 oracle on a bounded sample of one burst pair; returns
    (burst-pairs/s, threads, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import topsb200 as T
    nthreads = os.cpu_count() or 1
    O.set_num_threads(nthreads)
    L, W = scene_cfg["lines_per_burst"], scene_cfg["samples_per_burst"]
    # a small scene with the same sampling and 2 bursts to take stage timings from
    S = T.Scene(n_bursts=2, lines_per_burst=L, samples_per_burst=min(W, 2048), overlap_lines=100,
                dem_lines=256, dem_pixels=256, seed=7)
    Ws = S.cfg.samples_per_burst
    b = 1
    g = S.geo_args(b)
    t0 = time.perf_counter()
    az, rg, st, nv = O.geocoreg(g["dem"], g["lat0"], g["lon0"], g["dlat"], g["dlon"], g["xmin"],
                                g["xmax"], g["ymin"], g["ymax"], g["dt"], g["first_line_time"],
                                g["slr_time"], g["range_spacing"], g["mid_time"], g["azi_init"],
                                g["line_offset"], g["coefs"])
    t_geo_px = (time.perf_counter() - t0) / g["dem"].size
    mb, sb = S.boxes(b)
    d = S.deramp[1]
    rows = 256
    t0 = time.perf_counter()
    out = O.resample(S.burst(1, b), az, rg, 0.0, S.kaz, S.krg, b, mb, sb, L, S.swath[1].dt,
                     d["kt"][0], d["tref"][0], d["dc"][0], rows=(600, rows))
    t_rs_px = (time.perf_counter() - t0) / (rows * Ws)
    sl = np.ascontiguousarray(out.astype(np.complex64)).view(np.float32).reshape(rows, Ws, 2)
    t0 = time.perf_counter()
    O.coherence(S.burst(0, b)[600:600 + rows], sl, WIN_RG, WIN_AZ)
    t_coh_px = (time.perf_counter() - t0) / (rows * Ws)
    ov = 100
    t0 = time.perf_counter()
    O.esd(S.burst(0, b)[:ov], S.burst(0, b)[ov:2 * ov], sl[:ov], sl[ov:2 * ov], np.array([ov]), WIN_AZ,
          WIN_RG, 0.3, 1500.0, 2.055e-3)
    t_esd_px = (time.perf_counter() - t0) / (ov * Ws)
    # per burst pair of the configured workload: 2 resamples + coherence of
    # L*W pixels, the ESD share of one overlap, and the burst's DEM window
    nb = scene_cfg["n_bursts"]
    dem_px = scene_cfg["dem_lines"] * scene_cfg["dem_pixels"] / nb
    per_pair = (2 * t_rs_px + t_coh_px) * L * W + t_esd_px * ov * W * (nb - 1) / nb + \
        t_geo_px * dem_px
    sample = (f"FP64 oracle, {nthreads} threads: geocoreg of a {g['dem'].shape[0]}x"
              f"{g['dem'].shape[1]} DEM window, resample + coherence of {rows} lines x {Ws}, ESD of "
              f"{ov} x {Ws}; per-pixel times scaled to one {L}x{W} burst pair")
    return 1.0 / per_pair, nthreads, sample


def run_reference(args, rank, world):
    if rank != 0:
        return
    cfg = CONFIGS[args.config]
    for _ in range(args.warmup):
        cpu_sample(cfg)
    vals = []
    for _ in range(args.steps):
        v, nthreads, sample = cpu_sample(cfg)
        vals.append(v)
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": args.config, **{k: v for k, v in cfg.items() if k != "seed"}},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="subswath", choices=sorted(CONFIGS))
    ap.add_argument("--e2e-steps", type=int, default=6)
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    import topsb200 as T
    assert torch.cuda.is_available(), "bench needs a CUDA device"
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    cfg = CONFIGS[args.config]
    t0 = time.time()
    S = build_scene(T, cfg, rank)
    gen_s = time.time() - t0
    nb, L, W = cfg["n_bursts"], cfg["lines_per_burst"], cfg["samples_per_burst"]
    di = S.dem_info
    opts = T.pair_opts(win_rg=WIN_RG, win_az=WIN_AZ)
    P = T.Pair(S.swath[0], S.swath[1], S.dem.shape, opts)
    windows = T.scene_windows(S)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    P.set_dem(S.dem, di.lat0, di.lon0, di.dlat, di.dlon, windows, sp)
    # pinned host buffers for the end-to-end form
    pin = lambda a: torch.from_numpy(a).pin_memory()
    h_m, h_s = pin(S.slc[0]), pin(S.slc[1])
    n = nb * L
    h_rs = torch.empty((n, W, 2), dtype=torch.float32).pin_memory()
    h_re = torch.empty((n, W, 2), dtype=torch.float32).pin_memory()
    h_coh = torch.empty((n, W), dtype=torch.float32).pin_memory()
    h_cpm = np.zeros((nb, 12))
    h_sh = np.zeros(max(nb - 1, 1))
    import ctypes as C
    upload = lambda: T.check(T.lib.tops_pair_upload(P._h, C.c_void_p(h_m.data_ptr()),
                                                    C.c_void_p(h_s.data_ptr()), C.c_void_p(sp)),
                             "upload")
    download = lambda: T.check(T.lib.tops_pair_download(
        P._h, C.c_void_p(h_rs.data_ptr()), C.c_void_p(h_re.data_ptr()),
        C.cast(C.c_void_p(h_coh.data_ptr()), C.POINTER(C.c_float)),
        T.ptr(h_cpm, C.c_double), T.ptr(h_sh, C.c_double), C.c_void_p(sp)), "download")
    with torch.cuda.stream(stream):
        upload()
    stream.synchronize()

    # ---- device-resident batched form
    B = P.buffers()

    def step():
        T.check(T.lib.tops_pair_run_graph(P._h, C.c_void_p(sp)), "run_graph")

    for _ in range(args.warmup):
        step()
    stream.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1) / args.steps
    ms_t = torch.tensor([ms], device="cuda")
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = world * nb * 1e3 / ms_max

    # ---- per-kernel timing of the dominant kernel (resample, ESD-corrected
    # pass: 9 bursts x 1500 x 21000 outputs per launch) on the launch stream
    rs_ms, rs_launches = kernel_times(T, P, S, opts, sp, torch, stream, args.steps)

    # ---- end-to-end through the C ABI with pinned host buffers
    e2e_ms = []
    for i in range(args.e2e_steps + 1):
        torch.cuda.synchronize()
        t = time.perf_counter()
        with torch.cuda.stream(stream):
            upload()
            step()
            download()
        stream.synchronize()
        if i > 0:
            e2e_ms.append((time.perf_counter() - t) * 1e3)
    e2e_step_ms = float(np.mean(e2e_ms))
    e2e_t = torch.tensor([e2e_step_ms], device="cuda")
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = world * nb * 1e3 / float(e2e_t.item())
    h2d = 2 * n * W * 4
    d2h = 2 * n * W * 8 + n * W * 4 + 8 * 12 * nb + 8 * (nb - 1)

    # ---- plain per-burst form (reference-shaped, host buffers)
    plain_ms = []
    if args.plain_steps > 0:
        dem_int = np.rint(S.dem).astype(np.int32)
        for i in range(args.plain_steps + 1):
            t = time.perf_counter()
            T.plain_pair(S, opts, dem_int=dem_int, windows=windows)
            if i > 0:
                plain_ms.append((time.perf_counter() - t) * 1e3)
    plain_value = nb * 1e3 / float(np.mean(plain_ms)) if plain_ms else None

    peak, peak_kind = peaks()
    npx = n * W
    rs_bytes = 12.0 * npx
    achieved = rs_bytes / (rs_ms * 1e-3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "resample_traffic.json")
    if os.path.exists(tf):
        t_info = json.load(open(tf))
        traffic = t_info.get("bytes_per_output_px", 0.0) * npx or None

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 geometry)",
        "data": "synthetic (seeded); inputs > L2, no flush needed",
        "config": {"workload": f"{args.config}: {nb} burst pairs of {L}x{W} CInt16, "
                               f"{cfg['overlap_lines']}-line overlaps, DEM "
                               f"{cfg['dem_lines']}x{cfg['dem_pixels']}",
                   "window": f"{WIN_RG}x{WIN_AZ}", "form": "device-resident batched, CUDA graph",
                   "l2": "inputs larger than L2 (no flush)"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_step_ms,
                "latency_ms": {"p50": float(np.percentile(e2e_ms, 50)),
                               "p99": float(np.percentile(e2e_ms, 99))}},
        "plain": {"value": plain_value, "unit": UNIT,
                  "ms_per_step": float(np.mean(plain_ms)) if plain_ms else None,
                  "batched_over_plain_device": (value / world / plain_value) if plain_value else None,
                  "e2e_over_plain": (e2e_value / world / plain_value) if plain_value else None},
        "gpu_launches": args.steps * B.n_launches if B.n_launches else None,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": "resample_kernel",
                     "algorithmic_bytes_per_launch": rs_bytes, "launch_ms": rs_ms,
                     "peak_kind": peak_kind},
        "stages_ms": rs_launches,
        "clocks": clk.summary(),
        "scene_gen_s": gen_s,
    }
    if not args.no_cpu and rank == 0:
        v, nthreads, sample = cpu_sample(cfg)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
                                "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    P.close()
    if world > 1:
        dist.destroy_process_group()


def kernel_times(T, P, S, opts, sp, torch, stream, steps):
    """Average duration of each stage's launches over `steps` eager runs,
    measured with CUDA events on the launch stream."""
    import ctypes as C
    nb, L, W = S.cfg.n_bursts, S.cfg.lines_per_burst, S.cfg.samples_per_burst
    B = P.buffers()
    # Rebuild the stage launches of tops_pair_run through the device API so
    # events can bracket each stage.
    lut = C.c_void_p()
    T.check(T.lib.tops_lut_create(T.ptr(S.kaz, C.c_float), T.ptr(S.krg, C.c_float), C.byref(lut)),
            "lut")
    d = S.deramp[1]
    kt = torch.from_numpy(d["kt"][0].copy()).cuda()
    tref = torch.from_numpy(d["tref"][0].copy()).cuda()
    fdc = torch.from_numpy(d["dc"][0].copy()).cuda()
    jobs = (T.ResampleJob * nb)()
    for b in range(nb):
        j = jobs[b]
        j.slave = B.slave + b * L * B.slc_pitch
        j.slave_pitch = B.slc_pitch
        j.out = B.reslave_esd + b * L * B.cplx_pitch
        j.out_pitch = B.cplx_pitch
        j.kt, j.tref, j.fdc = kt.data_ptr(), tref.data_ptr(), fdc.data_ptr()
        mb, sb = S.boxes(b)
        for i in range(4):
            j.mbox[i] = int(mb[i])
            j.sbox[i] = int(sb[i])
        j.cpm_dev = B.cpm + 12 * b * 8
        j.az_shift_dev = (B.shifts + (b - 1) * 8) if b > 0 else None
        j.s_first_line = b * L
        j.dt = S.swath[0].dt
        j.out_row0 = 0
        j.out_rows = -1
    cj = (T.CohJob * nb)()
    for b in range(nb):
        c = cj[b]
        c.master = B.master + b * L * B.slc_pitch
        c.master_pitch = B.slc_pitch
        c.slave = B.reslave_esd + b * L * B.cplx_pitch
        c.slave_pitch = B.cplx_pitch
        c.coh = B.coh + b * L * B.coh_pitch
        c.coh_pitch = B.coh_pitch
        c.lines, c.pixels = L, W
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    t_rs, t_coh = [], []
    for i in range(steps + 2):
        ev[0].record(stream)
        T.check(T.lib.tops_resample(lut, jobs, nb, C.c_void_p(sp)), "resample")
        ev[1].record(stream)
        T.check(T.lib.tops_coherence(cj, nb, WIN_RG, WIN_AZ, C.c_void_p(sp)), "coherence")
        ev[2].record(stream)
        stream.synchronize()
        if i >= 2:
            t_rs.append(ev[0].elapsed_time(ev[1]))
            t_coh.append(ev[1].elapsed_time(ev[2]))
    T.lib.tops_lut_destroy(lut)
    # restore the pipeline's own outputs
    T.check(T.lib.tops_pair_run(P._h, C.c_void_p(sp)), "run")
    stream.synchronize()
    rs = float(np.mean(t_rs))
    coh = float(np.mean(t_coh))
    npx = nb * L * W
    return rs, {"resample_esd_ms": rs, "resample_gbs": 12.0 * npx / rs / 1e6,
                "coherence_ms": coh, "coherence_gbs": 16.0 * npx / coh / 1e6}


if __name__ == "__main__":
    main()
