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
path (the oracle) on the host cores, one burst pair of the workload per step;
the `cpu_baseline` object of the default run is the same path on a sample of
about 12 s.
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
    # one full sub-swath pair
    "subswath": dict(n_bursts=9, lines_per_burst=1500, samples_per_burst=21000,
                     overlap_lines=100, dem_lines=3600, dem_pixels=3600, seed=2),
    # three bursts of the full width: a profiling case whose inputs exceed L2
    # but whose device footprint stays near 3 GB
    "subswath3": dict(n_bursts=3, lines_per_burst=1500, samples_per_burst=21000,
                      overlap_lines=100, dem_lines=3600, dem_pixels=3600, seed=2),
    # two bursts of a narrow swath (parity scale)
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


def rank_config(cfg, rank):
    """The scene of one rank: replicas only -- every rank processes its own
    sub-swath pair (same sizes, seed + 1000 rank); nothing is exchanged."""
    c = dict(cfg)
    c["seed"] = c["seed"] + 1000 * rank
    return c


def build_scene(T, cfg, rank):
    return T.Scene(**rank_config(cfg, rank))


def max_over_ranks(v, dist, world, device):
    """The slowest rank's value (all ranks take this collective step)."""
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(world, pairs_per_rank, ms_max):
    """Burst pairs of all ranks per second of the slowest rank."""
    return world * pairs_per_rank * 1e3 / ms_max


class CpuPath:
    """The FP64 oracle (OpenMP over rows, all host threads) run burst pair by
    burst pair over a scene of the workload, in the order of the reference's
    stage drivers: geocoreg of the burst's DEM window, the resample, ESD of the
    overlap with the previous burst, the ESD-corrected resample and the
    coherence.  Used only for the CPU baseline."""

    def __init__(self, S):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        self.O, self.S = O, S
        self.threads = os.cpu_count() or 1
        O.set_num_threads(self.threads)
        m = S.swath[0]
        nb = S.cfg.n_bursts
        self.ov, _, _ = O.overlap_size(np.array(m.burst_first_line_time[:nb]),
                                       np.array(m.burst_last_line_time[:nb]), m.dt)
        self.spec = O.spectral_sep(S.deramp[0]["kt"], S.cfg.lines_per_burst, m.dt)
        self.prev = None
        self.next_burst = 0

    def pair(self):
        """Process the next burst pair; returns its wall time in seconds."""
        O, S = self.O, self.S
        nb, L = S.cfg.n_bursts, S.cfg.lines_per_burst
        b = self.next_burst
        self.next_burst = (b + 1) % nb
        t0 = time.perf_counter()
        g = S.geo_args(b)
        az, rg, st, nv = O.geocoreg(g["dem"], g["lat0"], g["lon0"], g["dlat"], g["dlon"],
                                    g["xmin"], g["xmax"], g["ymin"], g["ymax"], g["dt"],
                                    g["first_line_time"], g["slr_time"], g["range_spacing"],
                                    g["mid_time"], g["azi_init"], g["line_offset"], g["coefs"])
        mb, sb = S.boxes(b)
        d = S.deramp[1]
        kw = dict(slave=S.burst(1, b), cpm_az=az, cpm_rg=rg, kaz=S.kaz, krg=S.krg,
                  s_burst_idx=b, mbox=mb, sbox=sb, lines_per_burst=L, kt=d["kt"][0],
                  tref=d["tref"][0], fdc=d["dc"][0])
        rs, _ = O.resample(az_shift=0.0, dt=S.swath[1].dt, **kw)
        rs = rs.astype(np.complex64)
        master = S.burst(0, b)
        if b == 0 or self.prev is None:
            rse = rs
        else:
            o = int(self.ov[b - 1])
            band = lambda a: np.ascontiguousarray(a).view(np.float32).reshape(a.shape[0], -1, 2)
            mF = S.burst(0, b - 1)[L - o:]
            mB = master[:o]
            shift, _, _ = O.esd(mF, mB, band(self.prev[L - o:]), band(rs[:o]), np.array([o]),
                                WIN_AZ, WIN_RG, 0.3, self.spec, S.swath[0].dt)
            sh = float(shift[0]) if abs(shift[0]) <= 100 else 0.0
            rse, _ = O.resample(az_shift=sh, dt=S.swath[0].dt, **kw)
            rse = rse.astype(np.complex64)
        O.coherence(master, np.ascontiguousarray(rse).view(np.float32).reshape(L, -1, 2),
                    WIN_RG, WIN_AZ)
        self.prev = rs
        return time.perf_counter() - t0

    def describe(self, pairs):
        S = self.S
        return (f"FP64 oracle (C, OpenMP, {self.threads} threads) on {pairs} burst pairs of the "
                f"workload ({S.cfg.lines_per_burst}x{S.cfg.samples_per_burst} each, in burst "
                f"order): geocoreg of the burst's DEM window, resample, ESD of the overlap with "
                f"the previous burst, ESD-corrected resample, coherence {WIN_RG}x{WIN_AZ}")


def cpu_baseline(S, seconds=12.0):
    """Burst pairs/s of the CPU path on a bounded sample: bursts in order
    until `seconds` have passed (at least two, at most all of them)."""
    cp = CpuPath(S)
    times = []
    while len(times) < S.cfg.n_bursts and (len(times) < 2 or sum(times) < seconds):
        times.append(cp.pair())
    return len(times) / sum(times), cp.threads, cp.describe(len(times))


def run_reference(args, rank, world):
    """The reference arm: the CPU path (the FP64 oracle port of the reference's
    algorithm) on the host cores, one burst pair of the workload per step."""
    if rank != 0:
        return
    import topsb200 as T
    cfg = CONFIGS[args.config]
    S = build_scene(T, cfg, 0)
    cp = CpuPath(S)
    for _ in range(args.warmup):
        cp.pair()
    times = [cp.pair() for _ in range(args.steps)]
    value = len(times) / sum(times)
    nb, L, W = cfg["n_bursts"], cfg["lines_per_burst"], cfg["samples_per_burst"]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": workload_name(args.config, cfg),
                       "window": f"{WIN_RG}x{WIN_AZ}"},
            "form": "CPU FP64 port, one burst pair per step",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cp.threads, "kind": "port",
                             "sample": cp.describe(len(times))},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# Three sub-swaths of 9 bursts with uneven sizes (seeded): lines drawn from
# 1450-1550 and samples from 18000-25500 per sub-swath.
BATCH_SEED = 4


def batch_shapes():
    rng = np.random.default_rng(BATCH_SEED)
    return [dict(n_bursts=9, lines_per_burst=int(rng.integers(1450, 1551)),
                 samples_per_burst=int(rng.integers(18000, 25501)), overlap_lines=100,
                 dem_lines=3600, dem_pixels=3600, seed=40 + k) for k in range(3)]


def batch_scenes(T):
    t0 = time.time()
    scenes = [T.Scene(**sh) for sh in batch_shapes()]
    return scenes, time.time() - t0


def batch_result(T, torch, scenes, steps, warmup, world=1):
    """Batched uneven bursts: the 3 sub-swath pairs as one batch (one launch
    per stage, autotuned tiles, one CUDA graph) against the per-burst launch
    loop on the same device-resident data."""
    shapes = batch_shapes()
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    opts = T.pair_opts(win_rg=WIN_RG, win_az=WIN_AZ)
    plans = []
    for S in scenes:
        P = T.Pair(S.swath[0], S.swath[1], S.dem.shape, opts)
        di = S.dem_info
        P.set_dem(S.dem, di.lat0, di.lon0, di.dlat, di.dlon, T.scene_windows(S), sp)
        P.upload(S.slc[0], S.slc[1], sp)
        plans.append(P)
    stream.synchronize()
    B = T.Batch(plans)
    tune, stage_ms = B.autotune(sp)
    n_pairs = sum(sh["n_bursts"] for sh in shapes)
    npx = sum(sh["n_bursts"] * sh["lines_per_burst"] * sh["samples_per_burst"] for sh in shapes)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        stream.synchronize()
        return e0.elapsed_time(e1) / steps

    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        ms_batch = timed(lambda: B.run(sp, graph=True), steps, warmup)
    launches_batch = B.launches()

    def loop():
        for P in plans:
            P.run_per_burst(sp)
    ms_loop = timed(loop, max(2, steps // 4), 1)
    launches_loop = sum(P.buffers().n_launches for P in plans)
    value = world * n_pairs * 1e3 / ms_batch
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
        "warmup": warmup, "ms_per_step": ms_batch, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 geometry)",
        "data": "synthetic (seeded); inputs > L2, no flush needed",
        "config": {"workload": "batch: 3 sub-swath pairs x 9 bursts, uneven sizes " +
                               ", ".join(f"{sh['lines_per_burst']}x{sh['samples_per_burst']}"
                                         for sh in shapes),
                   "window": f"{WIN_RG}x{WIN_AZ}",
                   "form": "one batch: one launch per stage for all 27 bursts, CUDA graph"},
        "tune": {"rs_seg_rows": tune.rs_seg_rows, "rs_persistent": tune.rs_persistent,
                 "coh_seg_rows": tune.coh_seg_rows, "coh_persistent": tune.coh_persistent,
                 "resample_esd_ms": float(stage_ms[0]), "coherence_ms": float(stage_ms[1])},
        "gpu_launches": steps * launches_batch, "gpu_launches_per_step": launches_batch,
        "per_burst_loop": {"value": n_pairs * 1e3 / ms_loop, "unit": UNIT, "ms_per_step": ms_loop,
                           "launches_per_step": launches_loop,
                           "batched_over_loop": ms_loop / ms_batch},
        "resample_roofline": {"achieved_gbs": 12.0 * npx / (float(stage_ms[0]) * 1e6),
                              "peak_gbs": peaks()[0],
                              "frac": 12.0 * npx / (float(stage_ms[0]) * 1e6) / peaks()[0]},
        "clocks": clk.summary(),
    }
    B.close()
    for P in plans:
        P.close()
    return line


def run_batch(args, rank, world):
    import torch
    import topsb200 as T
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    scenes, gen_s = batch_scenes(T)
    line = batch_result(T, torch, scenes, args.steps, args.warmup, world)
    line["scene_gen_s"] = gen_s
    print(json.dumps(line), flush=True)


SERVE_RATE = 40.0          # jobs/s (Poisson)
SERVE_BUDGET = 150 << 30   # bytes of HBM the jobs may hold at once
SERVE_SLOTS = 8


def serve_jobs(n, shapes):
    """Seeded job stream: arrival time, sub-swath, first burst, bursts (1-9)."""
    rng = np.random.default_rng(SERVE_SEED)
    t = np.cumsum(rng.exponential(1.0 / SERVE_RATE, n))
    jobs = []
    for i in range(n):
        s = int(rng.integers(len(shapes)))
        k = int(rng.integers(1, shapes[s]["n_bursts"] + 1))
        b0 = int(rng.integers(0, shapes[s]["n_bursts"] - k + 1))
        jobs.append((float(t[i]), s, b0, k))
    return jobs


SERVE_SEED = 7


def serve_result(T, torch, scenes, n_jobs, world=1):
    """Serving: a seeded Poisson stream of burst-pair jobs (1-9 bursts of the
    three uneven sub-swaths) through the serving loop -- admission by HBM
    footprint under a 150 GB budget, one stream per slot, DEM tiles resident.
    Reports latency percentiles and sustained throughput, then a closed-loop
    pass (all jobs at once) for the saturation throughput.  Jobs produce the
    final products (ReSlaveESD, coherence, offsets, shifts); the first-pass
    resample covers only the overlap bands ESD needs."""
    shapes = batch_shapes()
    pin = [(torch.from_numpy(S.slc[0]).pin_memory(), torch.from_numpy(S.slc[1]).pin_memory())
           for S in scenes]
    slc = [(a.numpy(), b.numpy()) for a, b in pin]
    # one pinned sink for every job's outputs (timing only; results are
    # checked by the tests)
    mx = max(sh["n_bursts"] * sh["lines_per_burst"] * sh["samples_per_burst"] for sh in shapes)
    sink_c = torch.empty(mx * 2, dtype=torch.float32).pin_memory().numpy().view(np.complex64)
    sink_f = torch.empty(mx, dtype=torch.float32).pin_memory().numpy()
    sink = dict(reslave=None, reslave_esd=sink_c, coh=sink_f, cpm=np.zeros((9, 12)),
                shifts=np.zeros(8))
    opts = T.pair_opts(win_rg=WIN_RG, win_az=WIN_AZ, reslave_full=0)

    def one_pass(jobs, closed_loop):
        srv = T.Server(SERVE_BUDGET, SERVE_SLOTS)
        dems = [srv.add_dem(S.dem, S.dem_info.lat0, S.dem_info.lon0, S.dem_info.dlat,
                            S.dem_info.dlon) for S in scenes]
        descs = [srv.job(scenes[s], dems[s], b0, k, opts=opts, outputs=sink,
                         master_slc=slc[s][0], slave_slc=slc[s][1])[0] for _, s, b0, k in jobs]
        torch.cuda.synchronize()
        start = time.perf_counter()
        for (ta, s, b0, k), d in zip(jobs, descs):
            if not closed_loop:
                while time.perf_counter() - start < ta:
                    srv.progress()
            srv.submit(d)
        srv.drain()
        done = srv.poll(4096)
        st = srv.stats()
        srv.close()
        assert all(x.status == T.TOPS_OK for x in done), [x.status for x in done]
        lat = np.array([x.done_s - x.arrival_s for x in done]) * 1e3
        queue = np.array([x.admit_s - x.arrival_s for x in done]) * 1e3
        span = max(x.done_s for x in done) - min(x.arrival_s for x in done)
        pairs = sum(k for _, _, _, k in jobs)
        return dict(pairs_per_s=pairs / span, jobs=len(done), pairs=pairs, span_s=span,
                    latency_ms={"p50": float(np.percentile(lat, 50)),
                                "p99": float(np.percentile(lat, 99)),
                                "max": float(lat.max())},
                    queue_ms={"p50": float(np.percentile(queue, 50)),
                              "p99": float(np.percentile(queue, 99))},
                    hbm_peak_gb=st.hbm_peak / 1e9)

    jobs = serve_jobs(n_jobs, shapes)
    one_pass(jobs[:4], True)                        # warm-up: LUTs, kernel attributes
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        open_loop = one_pass(jobs, False)
    closed = one_pass(jobs, True)
    # plain per-burst form on one 3-burst job for the comparison
    S = scenes[0]
    t = time.perf_counter()
    T.plain_pair(S, T.pair_opts(win_rg=WIN_RG, win_az=WIN_AZ))
    plain = S.cfg.n_bursts / (time.perf_counter() - t)
    line = {
        "metric": METRIC, "value": closed["pairs_per_s"], "unit": UNIT, "n_gpus": world,
        "steps": 1, "warmup": 1, "ms_per_step": closed["span_s"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (f64 geometry)", "data": "synthetic (seeded)",
        "config": {"workload": f"serve: {n_jobs} Poisson jobs ({SERVE_RATE:.0f}/s), 1-9 bursts "
                               "of 3 uneven sub-swaths",
                   "budget_gb": SERVE_BUDGET / 2**30, "slots": SERVE_SLOTS,
                   "window": f"{WIN_RG}x{WIN_AZ}"},
        "open_loop": open_loop, "closed_loop": closed,
        "plain": {"value": plain, "unit": UNIT, "job": f"{S.cfg.n_bursts} bursts of "
                  f"{S.cfg.lines_per_burst}x{S.cfg.samples_per_burst}"},
        "served_over_plain": closed["pairs_per_s"] / plain,
        "clocks": clk.summary(),
    }
    return line


def run_serve(args, rank, world):
    import torch
    import topsb200 as T
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    scenes, gen_s = batch_scenes(T)
    line = serve_result(T, torch, scenes, args.jobs, world)
    line["scene_gen_s"] = gen_s
    print(json.dumps(line), flush=True)


def precision_result(T, torch, steps, warmup, world=1):
    """Precision variant on the small workload's inputs (2 bursts of 1500 x
    4096): the pipeline with the split-precision deramp (default), with the
    all-FP64 deramp, and with the split deramp plus compensated ESD and
    coherence sums, each timed on the device and each output compared with
    the FP64 host oracle run on the same inputs."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cfg = CONFIGS["small"]
    S = build_scene(T, cfg, 0)
    nb, L, W = cfg["n_bursts"], cfg["lines_per_burst"], cfg["samples_per_burst"]
    O.set_num_threads(os.cpu_count() or 1)
    # ---- oracle chain (FP64), as the pipeline chains the stages
    m, s = S.swath
    ov, _, _ = O.overlap_size(np.array(m.burst_first_line_time[:nb]),
                              np.array(m.burst_last_line_time[:nb]), m.dt)
    spec = O.spectral_sep(S.deramp[0]["kt"], L, m.dt)
    d = S.deramp[1]
    cpm, rs1, rse, coh = [], [], [], []
    for b in range(nb):
        g = S.geo_args(b)
        az, rg, st, _ = O.geocoreg(np.rint(g["dem"]).astype(np.float32), g["lat0"], g["lon0"],
                                   g["dlat"], g["dlon"], g["xmin"], g["xmax"], g["ymin"],
                                   g["ymax"], g["dt"], g["first_line_time"], g["slr_time"],
                                   g["range_spacing"], g["mid_time"], g["azi_init"],
                                   g["line_offset"], g["coefs"])
        cpm.append((az, rg))
    kw = lambda b, sh, dt: dict(slave=S.burst(1, b), cpm_az=cpm[b][0], cpm_rg=cpm[b][1],
                                az_shift=sh, kaz=S.kaz, krg=S.krg, s_burst_idx=b,
                                mbox=S.boxes(b)[0], sbox=S.boxes(b)[1], lines_per_burst=L, dt=dt,
                                kt=d["kt"][0], tref=d["tref"][0], fdc=d["dc"][0])
    for b in range(nb):
        rs1.append(O.resample(**kw(b, 0.0, s.dt))[0])
    c64 = lambda a: np.ascontiguousarray(a.astype(np.complex64)).view(np.float32).reshape(
        a.shape[0], a.shape[1], 2)
    mF = np.concatenate([S.slc[0][(i + 1) * L - ov[i]:(i + 1) * L] for i in range(nb - 1)])
    mB = np.concatenate([S.slc[0][(i + 1) * L:(i + 1) * L + ov[i]] for i in range(nb - 1)])
    sF = np.concatenate([rs1[i][L - ov[i]:] for i in range(nb - 1)])
    sB = np.concatenate([rs1[i + 1][:ov[i]] for i in range(nb - 1)])
    shifts, _, _ = O.esd(mF, mB, c64(sF), c64(sB), ov, WIN_AZ, WIN_RG, 0.3, spec, m.dt)
    for b in range(nb):
        sh = shifts[b - 1] if b > 0 else 0.0
        rse.append(O.resample(**kw(b, sh, m.dt))[0])
        coh.append(O.coherence(S.burst(0, b), c64(rse[b]), WIN_RG, WIN_AZ))

    def grid(c, b):
        y = np.linspace(b * L, (b + 1) * L - 1, 31)
        x = np.linspace(0, W - 1, 41)
        Y, X = np.meshgrid(y, x, indexing="ij")
        Lh = (Y - (b * L + 0.5 * (L - 1))) / (0.25 * (L - 1))
        Ph = (X - 0.5 * (W - 1)) / (0.25 * (W - 1))
        return c[0] + c[1] * Lh + c[2] * Ph + c[3] * Lh * Lh + c[4] * Lh * Ph + c[5] * Ph * Ph

    rel = lambda a, r: float(np.sqrt(np.sum(np.abs(a - r) ** 2) / np.sum(np.abs(r) ** 2)))
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    modes = {}
    di = S.dem_info
    for name, prec, comp in (("split", T.PREC_SPLIT, 0), ("fp64", T.PREC_FP64, 0),
                             ("split_compensated", T.PREC_SPLIT, 1)):
        P = T.Pair(S.swath[0], S.swath[1], S.dem.shape,
                   T.pair_opts(win_rg=WIN_RG, win_az=WIN_AZ, precision=prec, compensated=comp))
        P.set_dem(np.rint(S.dem), di.lat0, di.lon0, di.dlat, di.dlon, T.scene_windows(S), sp)
        P.upload(S.slc[0], S.slc[1], sp)
        for _ in range(warmup):
            P.run(sp, graph=True)
        stream.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            P.run(sp, graph=True)
        e1.record(stream)
        stream.synchronize()
        ms = e0.elapsed_time(e1) / steps
        stage = P.stage_times(sp)
        out = P.download(stream=sp)
        stream.synchronize()
        P.close()
        err = {
            "offsets_px": max(float(np.abs(grid(out["cpm"][b, :6], b) - grid(cpm[b][0], b)).max())
                              for b in range(nb)),
            "offsets_rg_px": max(float(np.abs(grid(out["cpm"][b, 6:], b) -
                                              grid(cpm[b][1], b)).max()) for b in range(nb)),
            "reslave_rel_rms": max(rel(out["reslave"][b * L:(b + 1) * L], rs1[b])
                                   for b in range(nb)),
            "reslave_esd_rel_rms": max(rel(out["reslave_esd"][b * L:(b + 1) * L], rse[b])
                                       for b in range(nb)),
            "esd_shift_px": float(np.abs(out["shifts"] - shifts).max()),
            "coherence_max_abs": max(float(np.abs(out["coh"][b * L:(b + 1) * L] - coh[b]).max())
                                     for b in range(nb)),
        }
        # where the largest differences sit: per-pixel error of ReSlaveESD
        # against the burst's RMS amplitude, and the coherence error map
        dc = np.concatenate([np.abs(out["coh"][b * L:(b + 1) * L] - coh[b]) for b in range(nb)])
        ds = np.concatenate([np.abs(out["reslave_esd"][b * L:(b + 1) * L] - rse[b]) /
                             np.sqrt(np.mean(np.abs(rse[b]) ** 2)) for b in range(nb)])
        at = np.unravel_index(int(np.argmax(dc)), dc.shape)
        err["coherence_max_at"] = {"line": int(at[0]), "sample": int(at[1]),
                                   "coh": float(np.concatenate(coh)[at])}
        err["coherence_p99_99_abs"] = float(np.percentile(dc, 99.99))
        err["coherence_px_above_1e-5"] = int((dc > 1e-5).sum())
        ats = np.unravel_index(int(np.argmax(ds)), ds.shape)
        err["reslave_esd_max_abs_over_rms"] = float(ds.max())
        err["reslave_esd_max_at"] = {"line": int(ats[0]), "sample": int(ats[1])}
        modes[name] = {"ms_per_step": ms, "pairs_per_s": nb * 1e3 / ms,
                       "esd_ms": stage["esd"], "coherence_ms": stage["coherence"],
                       "error_vs_fp64_oracle": err}
    line = {
        "metric": METRIC, "value": modes["split"]["pairs_per_s"], "unit": UNIT, "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": modes["split"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 split / f64", "data": "synthetic (seeded)",
        "config": {"workload": workload_name("precision (small inputs)", cfg),
                   "window": f"{WIN_RG}x{WIN_AZ}"},
        "modes": modes,
        "tolerances": {"offsets_px": 1e-4, "reslave_rel_rms": 1e-4, "esd_shift_px": 1e-5,
                       "coherence_max_abs": 1e-5},
    }
    return line


def run_precision(args, rank, world):
    import torch
    import topsb200 as T
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    print(json.dumps(precision_result(T, torch, args.steps, args.warmup, world)), flush=True)


def run_product(args, rank, world):
    """The config.txt-driven run (tops_run_config) over 3 synthetic sub-swaths
    of 3 bursts of 1500 x 21000, writing ReSlave, ReSlaveESD and Coh TIFFs:
    its wall time against the summed load (synthetic generation), pair-run
    and write times, which the run overlaps across sub-swaths."""
    import shutil
    import tempfile
    import topsb200 as T
    if rank != 0:
        return
    d = tempfile.mkdtemp(prefix="tops_run_")
    try:
        keys = dict(process_dir=os.path.join(d, "out"), masterpath="(synthetic)",
                    slavepath="(synthetic)", firstsubswath=1, lastsubswath=3, burst0=1, burstN=3,
                    stitch=0, **CONFIGS["subswath3"])
        cfg = os.path.join(d, "config.txt")
        with open(cfg, "w") as f:
            f.write("".join(f"{k}={v}\n" for k, v in keys.items()))
        st = T.run_config(cfg)
        written = sum(os.path.getsize(os.path.join(d, "out", n)) for n in os.listdir(os.path.join(d, "out")))
    finally:
        shutil.rmtree(d, ignore_errors=True)
    serial = st.load_seconds + st.process_seconds + st.write_seconds
    print(json.dumps({
        "metric": "burst-pairs/s (config run: synthetic inputs, TIFF outputs)",
        "value": st.burst_pairs / st.seconds, "unit": UNIT, "n_gpus": 1,
        "higher_is_better": True,
        "config": {"workload": "3 sub-swaths x 3 bursts of 1500x21000, DEM 3600x3600",
                   "window": f"{WIN_RG}x{WIN_AZ}"},
        "seconds": st.seconds, "load_seconds": st.load_seconds,
        "process_seconds": st.process_seconds, "write_seconds": st.write_seconds,
        "serial_sum_seconds": serial, "overlap_saved_seconds": serial - st.seconds,
        "bytes_written": written}), flush=True)


def workload_name(name, cfg):
    return (f"{name}: {cfg['n_bursts']} burst pairs of {cfg['lines_per_burst']}x"
            f"{cfg['samples_per_burst']} CInt16, {cfg['overlap_lines']}-line overlaps, DEM "
            f"{cfg['dem_lines']}x{cfg['dem_pixels']}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="subswath",
                    choices=sorted(CONFIGS) + ["batch", "serve", "precision", "product"])
    ap.add_argument("--jobs", type=int, default=40, help="serve: number of arriving jobs")
    ap.add_argument("--e2e-steps", type=int, default=6)
    ap.add_argument("--plain-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="default run: skip the precision, batch and serving measurements")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.config == "batch":
        return run_batch(args, rank, world)
    if args.config == "serve":
        return run_serve(args, rank, world)
    if args.config == "precision":
        return run_precision(args, rank, world)
    if args.config == "product":
        return run_product(args, rank, world)

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
    h_cpm = torch.zeros((nb, 12), dtype=torch.float64).pin_memory().numpy()
    h_sh = torch.zeros(max(nb - 1, 1), dtype=torch.float64).pin_memory().numpy()
    import ctypes as C
    upload = lambda: T.check(T.lib.tops_pair_upload(P._h, C.c_void_p(h_m.data_ptr()),
                                                    C.c_void_p(h_s.data_ptr()), C.c_void_p(sp)),
                             "upload")
    download = lambda: T.check(T.lib.tops_pair_download(
        P._h, C.c_void_p(h_rs.data_ptr()), C.c_void_p(h_re.data_ptr()),
        C.cast(C.c_void_p(h_coh.data_ptr()), C.POINTER(C.c_float)),
        T.ptr(h_cpm, C.c_double), T.ptr(h_sh, C.c_double), C.c_void_p(sp)), "download")
    process = lambda: T.check(T.lib.tops_pair_process(
        P._h, C.c_void_p(h_m.data_ptr()), C.c_void_p(h_s.data_ptr()),
        C.c_void_p(h_rs.data_ptr()), C.c_void_p(h_re.data_ptr()),
        C.cast(C.c_void_p(h_coh.data_ptr()), C.POINTER(C.c_float)),
        T.ptr(h_cpm, C.c_double), T.ptr(h_sh, C.c_double), C.c_void_p(sp)), "process")
    with torch.cuda.stream(stream):
        upload()
    stream.synchronize()

    # ---- device-resident batched form
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
    launches_per_step = P.buffers().n_launches   # counted by the runs above
    overlap = overlap_report(T, torch, S, windows, stream, h_m, h_s, args.steps, args.warmup,
                             dist, world, nb)
    ms_max = max_over_ranks(ms, dist, world, "cuda")
    value = whole_job_value(world, nb, ms_max)

    # ---- per-stage timing (CUDA events between the stages of one eager run,
    # on the launch stream), averaged over `steps` runs
    stages = stage_report(T, P, S, windows, sp, args.steps)
    stages.update(stitch_report(T, P, S, torch, stream, args.steps))
    # the roofline kernel: the ReSlave resample, one launch over every burst
    # (the ReSlaveESD stage also holds the first burst's copy)
    rs_ms = stages["resample"]["ms"]

    # ---- end-to-end through the C ABI with pinned host buffers: the
    # pipelined host-to-host call (copies of one burst beside the kernels of
    # the others), and for comparison upload + graph run + download in series
    def timed(fn, steps):
        out = []
        for i in range(steps + 1):
            torch.cuda.synchronize()
            t = time.perf_counter()
            fn()
            stream.synchronize()
            if i > 0:
                out.append((time.perf_counter() - t) * 1e3)
        return out

    def serial():
        upload()
        step()
        download()

    e2e_ms = timed(process, args.e2e_steps)
    serial_ms = timed(serial, max(1, args.e2e_steps // 2))
    # the same call without the ReSlave download (the reference writes ReSlave
    # only as an intermediate raster): ReSlaveESD, coherence, offsets, shifts
    process_no_rs = lambda: T.check(T.lib.tops_pair_process(
        P._h, C.c_void_p(h_m.data_ptr()), C.c_void_p(h_s.data_ptr()), None,
        C.c_void_p(h_re.data_ptr()), C.cast(C.c_void_p(h_coh.data_ptr()), C.POINTER(C.c_float)),
        T.ptr(h_cpm, C.c_double), T.ptr(h_sh, C.c_double), C.c_void_p(sp)), "process")
    no_rs_ms = timed(process_no_rs, max(1, args.e2e_steps // 2))
    e2e_step_ms = float(np.mean(e2e_ms))
    e2e_value = whole_job_value(world, nb, max_over_ranks(e2e_step_ms, dist, world, "cuda"))
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
    # HBM ceilings of a pair (stage-boundary bytes at the measured copy
    # bandwidth): the plain dataflow (two resamples, coherence, ESD) and a
    # fused one that only reads the SLCs and writes ReSlaveESD and coherence
    ov_px = stages["esd"]["bytes"] / 24.0
    plain_bytes = 40.0 * npx + 24.0 * ov_px
    fused_bytes = 20.0 * npx
    ceilings = {"plain_dataflow_pairs_per_s": nb * peak * 1e9 / plain_bytes,
                "fused_pairs_per_s": nb * peak * 1e9 / fused_bytes,
                "bytes_per_pair_plain": plain_bytes / nb, "bytes_per_pair_fused": fused_bytes / nb}
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
        "config": {"workload": workload_name(args.config, cfg),
                   "window": f"{WIN_RG}x{WIN_AZ}"},
        "form": "device-resident batched, CUDA graph",
        "l2": "inputs larger than L2 (no flush)",
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_step_ms,
                "form": "tops_pair_process (per-burst copy/compute pipeline)",
                "serial_ms_per_step": float(np.mean(serial_ms)),
                "without_reslave_download": {
                    "value": whole_job_value(world, nb, max_over_ranks(float(np.mean(no_rs_ms)),
                                                                       dist, world, "cuda")),
                    "ms_per_step": float(np.mean(no_rs_ms)),
                    "d2h_bytes_per_step": d2h - n * W * 8},
                "latency_ms": {"p50": float(np.percentile(e2e_ms, 50)),
                               "p99": float(np.percentile(e2e_ms, 99))}},
        "plain": {"value": plain_value, "unit": UNIT,
                  "ms_per_step": float(np.mean(plain_ms)) if plain_ms else None,
                  "batched_over_plain_device": (value / world / plain_value) if plain_value else None,
                  "e2e_over_plain": (e2e_value / world / plain_value) if plain_value else None},
        "gpu_launches": args.steps * launches_per_step,
        "gpu_launches_per_step": launches_per_step,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": "resample_kernel",
                     "algorithmic_bytes_per_launch": rs_bytes, "launch_ms": rs_ms,
                     "peak_kind": peak_kind},
        "stages": stages,
        "coh_overlap": overlap,
        "hbm_ceilings": ceilings,
        "clocks": clk.summary(),
        "scene_gen_s": gen_s,
    }
    if not args.no_cpu and rank == 0 and world == 1:
        v, nthreads, sample = cpu_baseline(S)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": nthreads, "kind": "port",
                                "sample": sample}
    P.close()
    if not args.no_extras and rank == 0 and world == 1 and args.config == "subswath":
        # the other workloads, measured in the same run: precision variant
        # (small inputs against the FP64 oracle), batched uneven sub-swaths
        # and the serving loop (the 150 GB serving budget last: the other
        # plans are released by then)
        t0 = time.time()
        line["precision"] = compact_precision(
            precision_result(T, torch, max(3, args.steps // 2), 3))
        scenes, _ = batch_scenes(T)
        line["batch"] = compact_batch(batch_result(T, torch, scenes, max(3, args.steps // 2), 3))
        line["serve"] = compact_serve(serve_result(T, torch, scenes, args.jobs))
        line["extras_s"] = time.time() - t0
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def compact_precision(p):
    return {"workload": p["config"]["workload"], "tolerances": p["tolerances"],
            "modes": {k: {"pairs_per_s": v["pairs_per_s"], "ms_per_step": v["ms_per_step"],
                          "esd_ms": v["esd_ms"], "coherence_ms": v["coherence_ms"],
                          "error_vs_fp64_oracle": {
                              e: v["error_vs_fp64_oracle"][e]
                              for e in ("offsets_px", "offsets_rg_px", "reslave_rel_rms",
                                        "reslave_esd_rel_rms", "esd_shift_px",
                                        "coherence_max_abs", "coherence_p99_99_abs",
                                        "coherence_px_above_1e-5")}}
                      for k, v in p["modes"].items()}}


def compact_batch(b):
    return {"workload": b["config"]["workload"], "value": b["value"], "unit": b["unit"],
            "ms_per_step": b["ms_per_step"], "per_burst_loop": b["per_burst_loop"],
            "tune": b["tune"], "resample_roofline": b["resample_roofline"],
            "gpu_launches_per_step": b["gpu_launches_per_step"], "clocks": b["clocks"]}


def compact_serve(v):
    return {"workload": v["config"]["workload"], "budget_gb": v["config"]["budget_gb"],
            "slots": v["config"]["slots"], "closed_loop": v["closed_loop"],
            "open_loop": v["open_loop"], "plain": v["plain"],
            "served_over_plain": v["served_over_plain"], "clocks": v["clocks"]}


STITCH_MARGIN = 20   # invalid lines at each burst edge of the synthetic bursts


def stitch_report(T, P, S, torch, stream, steps):
    """Debursting of the pair's coherence and ReSlaveESD (tops_stitch over
    the line map of bursts 0..n-1, STITCH_MARGIN invalid lines at each burst
    edge): device time per gather with CUDA events, bytes read + written."""
    import ctypes as C
    nb, L, W = S.cfg.n_bursts, S.cfg.lines_per_burst, S.cfg.samples_per_burst
    fv = np.full(nb, STITCH_MARGIN, np.int32)
    lv = np.full(nb, L - 1 - STITCH_MARGIN, np.int32)
    m = T.stitch_line_map(S.swath[0], fv, lv, 0, nb - 1)
    m_dev = torch.from_numpy(m).cuda()
    B = P.buffers()
    peak, _ = peaks()
    out = {}
    for name, src, pitch, eb in (("stitch_coh", B.coh, B.coh_pitch, 4),
                                 ("stitch_reslave_esd", B.reslave_esd, B.cplx_pitch, 8)):
        dst = torch.empty((len(m), W * eb // 4), dtype=torch.int32, device="cuda")
        run = lambda: T.check(T.lib.tops_stitch(
            C.c_void_p(src), pitch, C.c_void_p(dst.data_ptr()), W * eb, C.c_void_p(m_dev.data_ptr()),
            len(m), W * eb, C.c_void_p(stream.cuda_stream)), "tops_stitch")
        for _ in range(3):
            run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(max(steps, 1)):
            run()
        e1.record(stream)
        stream.synchronize()
        ms = e0.elapsed_time(e1) / max(steps, 1)
        nbytes = 2.0 * len(m) * W * eb
        gbs = nbytes / (ms * 1e-3) / 1e9
        out[name] = {"ms": ms, "bytes": nbytes, "gbs": gbs, "frac_hbm": gbs / peak,
                     "lines": int(len(m))}
    return out


def overlap_report(T, torch, S, windows, stream, h_m, h_s, steps, warmup, dist, world, nb):
    """The same graph step with tops_pair_opts.coh_overlap = 1: each chunk's
    coherence on a second stream right after its ReSlaveESD resample."""
    import ctypes as C
    sp = stream.cuda_stream
    di = S.dem_info
    Q = T.Pair(S.swath[0], S.swath[1], S.dem.shape,
               T.pair_opts(win_rg=WIN_RG, win_az=WIN_AZ, coh_overlap=1))
    Q.set_dem(S.dem, di.lat0, di.lon0, di.dlat, di.dlon, windows, sp)
    T.check(T.lib.tops_pair_upload(Q._h, C.c_void_p(h_m.data_ptr()), C.c_void_p(h_s.data_ptr()),
                                   C.c_void_p(sp)), "upload")
    step = lambda: T.check(T.lib.tops_pair_run_graph(Q._h, C.c_void_p(sp)), "run_graph")
    for _ in range(warmup):
        step()
    stream.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    stream.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / steps, dist, world, "cuda")
    launches = Q.buffers().n_launches
    Q.close()
    return {"value": whole_job_value(world, nb, ms), "ms_per_step": ms,
            "launches_per_step": launches,
            "form": "graph step, ReSlaveESD in up to 3 chunks of bursts, each chunk's coherence "
                    "on a second stream after its resample (same outputs bit for bit)"}


def stage_report(T, P, S, windows, sp, steps):
    """Per-stage device time of the pair (tops_pair_stage_times, averaged
    over `steps` eager runs), with each stage's algorithmic bytes, achieved
    GB/s and fraction of the measured HBM copy bandwidth; geocoreg, which is
    FP64-compute-bound, also as DEM pixels/s."""
    nb, L, W = S.cfg.n_bursts, S.cfg.lines_per_burst, S.cfg.samples_per_burst
    runs = [P.stage_times(sp) for _ in range(max(steps, 1))]
    ms = {k: float(np.mean([r[k] for r in runs])) for k in runs[0]}
    peak, _ = peaks()
    npx = nb * L * W
    m = S.swath[0]
    T_first = np.array(m.burst_first_line_time[:nb])
    T_last = np.array(m.burst_last_line_time[:nb])
    ov = np.floor((T_last[:-1] - T_first[1:]) / m.dt).astype(np.int64) if nb > 1 else []
    dem_px = sum(int(windows[b].rows) * int(windows[b].cols) for b in range(nb))
    nbytes = {"geocoreg": 4.0 * dem_px + 96.0 * nb, "resample": 12.0 * npx,
              "esd": 24.0 * float(np.sum(ov)) * W, "resample_esd": 12.0 * npx,
              "coherence": 16.0 * npx}
    out = {}
    for k, t in ms.items():
        gbs = nbytes[k] / (t * 1e-3) / 1e9 if t > 0 else None
        out[k] = {"ms": t, "bytes": nbytes[k], "gbs": gbs,
                  "frac_hbm": (gbs / peak) if gbs else None}
    out["geocoreg"]["dem_px"] = dem_px
    out["geocoreg"]["dem_mpx_per_s"] = dem_px / (ms["geocoreg"] * 1e-3) / 1e6
    out["geocoreg"]["bound"] = "fp64"
    # FP64 roofline: FP64 operations per DEM pixel from an ncu count of the
    # kernel on this workload (DFMA counted twice), over the FP64 FMA rate
    # measured on this device now
    gf = os.path.join(ROOT, "profiles", "geocoreg_fp64.json")
    if os.path.exists(gf):
        per_px = json.load(open(gf)).get("fp64_flops_per_dem_px")
        if per_px:
            pk = T.fp64_peak(sp)
            tf = per_px * dem_px / (ms["geocoreg"] * 1e-3) / 1e12
            out["geocoreg"].update({"fp64_tflops": tf, "fp64_peak_tflops": pk,
                                    "frac_fp64": tf / pk if pk > 0 else None,
                                    "fp64_flops_per_dem_px": per_px,
                                    "fp64_peak_kind": "measured (tops_fp64_peak)"})
    return out


if __name__ == "__main__":
    main()
