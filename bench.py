"""Benchmark of the Cahn-Hilliard step (3-D 256^3, dt 0.005, M 1, kappa 1,
periodic, c0 = 0 + U[-0.05, 0.05] from seed 42).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  `value` is FP64 (the drop-in precision, the same
arithmetic as the reference build) in GLUPS = lattice-site updates per
second, summed over ranks; the FP32 path (FP32 field, FP64 reductions, mass
feedback) is reported beside it under "fp32".  Each timed step is one fused
kernel launch; an L2 flush (a 512 MB write, then a 256 MB read) runs between timed steps and is
outside the timed events.  Multi-GPU: one independent replica per rank
(the simulation does not shard; no inter-GPU traffic), time = max over ranks.

--impl reference times the reference CPU build (oracle/_ref/chref_bench: the
reference's own SfieldFD/PFApp step loop with the CHBasic model) on the
host's cores, one MPI-shim rank per core, on a bounded number of steps.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 256
DT, KAP, M = 0.005, 1.0, 1.0
CO, AMP, SEED = 0.0, 0.1, 42
CONFIG = {"workload": "3-D Cahn-Hilliard 256^3 explicit step, dt 0.005, M 1, kappa 1, periodic, "
                      "c0 = 0 + U[-0.05,0.05] seed 42",
          "grid": [N, N, N], "dt": DT, "kappa": KAP, "M": M,
          "l2": "flushed between timed steps, untimed: a 512 MB write, then a 256 MB read of another buffer "
                "so that no dirty line of the flush is left to write back inside the timed step",
          "parallelism": "replicas (one independent simulation per GPU)"}
METRIC = "GLUPS & % HBM roofline (FP32 vs FP64)"
# DRAM traffic per launch is read from the committed ncu summaries (one
# capture of the same kernel and tiling), not measured inside this run
TRAFFIC_SOURCE = {"fp64": "ncu capture in profiles/ncu_ch_march_fp64_256.md (same kernel and tiling)",
                  "fp32": "ncu capture in profiles/ncu_ch_march2_fp32_256.md (same kernel and tiling)"}
TRAFFIC_FILE = {"fp64": "ncu_ch_march_fp64_256.md", "fp32": "ncu_ch_march2_fp32_256.md"}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(dtype):
    """DRAM bytes per launch of the step kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", TRAFFIC_FILE[dtype])
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1])
            except ValueError:
                return None
    return None


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML every `period_s`
    while a timed region runs (start()/stop() around each region; samples
    accumulate).  Falls back to nvidia-smi when NVML is unavailable."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, device, period_s=0.002):
        self.device, self.period = device, period_s
        self.sm, self.reasons, self.smax = [], set(), None
        self._thread, self._stop = None, None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.nv = None

    def _sample_nvml(self):
        nv = self.nv
        self.sm.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
        mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        for name, const in self.REASONS:
            if mask & getattr(nv, const):
                self.reasons.add(name)

    def _sample_smi(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        r = subprocess.run(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-i",
                            str(self.device)], capture_output=True, text=True, timeout=10)
        parts = [x.strip() for x in r.stdout.strip().split(",")]
        if len(parts) >= 6:
            self.sm.append(float(parts[0]))
            self.smax = float(parts[1])
            for (name, _), v in zip(self.REASONS, parts[2:6]):
                if v.lower() == "active":
                    self.reasons.add(name)

    def start(self):
        import threading
        self._stop = threading.Event()

        def run():
            while not self._stop.is_set():
                try:
                    self._sample_nvml() if self.nv else self._sample_smi()
                except Exception:
                    pass
                self._stop.wait(self.period if self.nv else 0.2)

        self._thread = threading.Thread(target=run, daemon=True)
        self._thread.start()

    def stop(self):
        if self._thread:
            self._stop.set()
            self._thread.join()
            self._thread = None

    def summary(self):
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.smax,
                "reasons": sorted(self.reasons), "samples": len(self.sm),
                "source": "NVML, every 2 ms inside the timed regions" if self.nv else "nvidia-smi"}


# ------------------------------------------------------------------ our arm
C4_EDGES = (64, 96, 128, 160, 192)
C5_EDGES_2D = (128, 256, 512, 1024)
C5_EDGES_3D = (64, 96, 128, 160, 192, 224, 256)


def batch_jobs(mb, njobs=64, seed=7):
    """Batched sweep: njobs cubic grids, edges uniform from C4_EDGES, c0 ~ U[-0.4,0.4],
    kappa ~ U[0.5,2], uniform noise of amplitude 0.05, per-job IC seed 1000+j."""
    import numpy as np
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(njobs):
        e = int(rng.choice(C4_EDGES))
        c0, kap = float(rng.uniform(-0.4, 0.4)), float(rng.uniform(0.5, 2.0))
        jobs.append(((e, e, e), c0, kap, 1000 + j))
    return jobs


# variable-mobility models at 256^3: parameters that keep the mobility off its
# clamps, each model's own initial field (co + 0.1*(r - 0.5)) and its
# reference default noise strength 0.1
MODEL_LEG = (
    ("TIPSphil", dict(alpha=150.0, beta=0.1, N=50.0, Tinit=300.0, Tbath=280.0, Tcrystal=200.0, gamma=1.0, D0=1.0,
                      Mweight=0.5, Mvolume=1.0), 0.3),
    ("TIPSbathPHIL", dict(alpha=150.0, beta=0.1, N=50.0, Tinit=320.0, Tbath=260.0, Tcrystal=200.0, gamma=1.0,
                          D0=1.0, Mweight=0.5, Mvolume=1.0), 0.3),
    ("SIPS", dict(Mweight=1.0, Mvolume=1.0, gamma=1.0), 0.1),
    ("SIPSternary", dict(Kpp=1.0, Knn=1.0, Mpp=1.0, Mnn=1.0), 0.2),
)


def run_models(mb, torch, dev, steps, warmup, flush, sampler, peak):
    """The variable-mobility steps at 256^3 (FP64, the default two passes:
    mu and 1/mob of every site; then div(mob grad mu), the update and the
    noise term), CUDA events around each step, L2 flushed between steps.
    GLUPS counts field site updates (SIPSternary: two fields).  `achieved`
    is the algorithmic 16 B per site update (read c, write c'); the two
    passes move 56 B (pass 1: read c, write mu and 1/mob; pass 2: read c,
    mu, 1/mob, write c')."""
    n = N
    sites = float(n) ** 3
    out = {}
    for name, kw, co in MODEL_LEG:
        base = mb.ic_generate((n, n, n), 0.0, 0.1, False, SEED)
        bc = (1, 1, 1) if name == "TIPSphil" else (0, 1, 1)
        p = mb.make_params(n, n, n, 0.01, bc=bc, noise=0.1, noise_seed=SEED)
        if name == "SIPSternary":
            sim = mb.Ternary(p, dev, **kw)
            sim.set_fields(co + base, 0.1 - base)
            fields = 2
        else:
            if name == "SIPS":
                sim = mb.CHSim(p, dev, sips=mb.make_sips_params(**kw))
            else:
                sim = mb.CHSim(p, dev, fh=mb.make_fh_params(10 ** 6, bath=name == "TIPSbathPHIL", **kw))
            sim.set_field(co + base)
            fields = 1
        del base
        ext = torch.cuda.ExternalStream(sim.stream, device=f"cuda:{dev}")
        for _ in range(warmup):
            sim.step(1)
        sim.sync()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        torch.cuda.synchronize()
        sampler.start()
        for e0, e1 in evs:
            with torch.cuda.stream(ext):
                flush.fill_(1)
            e0.record(ext)
            sim.step(1)
            e1.record(ext)
        sim.sync()
        torch.cuda.synchronize()
        sampler.stop()
        ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in evs)
        sim.close()
        upd = fields * sites
        out[name] = {"value": upd / (ms * 1e-3) / 1e9, "unit": "GLUPS", "ms_per_step": ms,
                     "achieved_gbs": upd * 16 / (ms * 1e-3) / 1e9, "frac": upd * 16 / (ms * 1e-3) / 1e9 / peak,
                     "design_gbs": upd * 56 / (ms * 1e-3) / 1e9, "fields": fields}
    out["workload"] = (f"{n}^3 FP64 per field, dt 0.01, noise 0.1, {steps} timed steps after {warmup} warm-up, "
                       "L2 flushed between steps; TIPSphil periodic, the others no-flux x")
    out["bytes"] = "achieved: 16 B per site update (algorithmic); design_gbs: 56 B per site update (two passes)"
    return out


def run_batch(mb, torch, dev, steps, sampler):
    import numpy as np
    jobs = batch_jobs(mb)
    params = [mb.make_params(*d, DT, kappa=k, precision="fp32") for d, _, k, _ in jobs]
    b = mb.Batch(params, dev)
    try:
        for j, (d, c0, _, seed) in enumerate(jobs):
            b.set_field(j, mb.ic_generate(d, c0, 0.05, False, seed))
        # tiles chosen by the autotuner for this batch (times scratch copies,
        # keeps the fields)
        tuned = b.autotune(trials=5)
        # warm-up (and graph capture): 4 steps, a multiple of the feedback
        # cadence, so that the mass is read after steps at which the FP32
        # feedback has just measured and corrected it
        b.step(4)
        b.sync()
        r0 = [b.reduce(j) for j in range(len(jobs))]
        m0 = [r["mass"] for r in r0]
        ext = torch.cuda.ExternalStream(b.stream, device=f"cuda:{dev}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        sampler.start()
        e0.record(ext)
        b.step(steps)
        e1.record(ext)
        b.sync()
        torch.cuda.synchronize()
        sampler.stop()
        ms = e0.elapsed_time(e1)
        info = b.info()
        sites_j = [d[0] * d[1] * d[2] for d, _, _, _ in jobs]
        # mass drift relative to the mass scale sum|c| ~ N*|c0|+noise: per site
        m1 = [b.reduce(j)["mass"] for j in range(len(jobs))]
        drift = max(abs(m1[j] - m0[j]) / sites_j[j] for j in range(len(jobs)))
        drift_rel = max(abs(m1[j] - m0[j]) / r0[j]["abs_mass"] for j in range(len(jobs)))
    finally:
        b.close()
    sites = float(sum(d[0] * d[1] * d[2] for d, _, _, _ in jobs))
    return {"jobs": len(jobs), "sites": sites, "steps": steps, "ms": ms,
            "value": sites * steps / (ms * 1e-3) / 1e9, "unit": "GLUPS", "precision": f"fp32 (mass feedback every {mb.MASS_EVERY} step(s))",
            "launches_per_step": info["launches_per_step"], "persistent_ctas": info["ctas"],
            "tiles": f"autotuned: CTAs of ~{tuned['threads']} threads, z-chunks of ~{tuned['planes']} planes",
            "max_mass_drift_per_site": drift, "max_mass_drift_rel": drift_rel,
            "mass_drift_note": f"max over jobs of |M({4 + steps}) - M(4)| / sites, FP64 sums of the stored fields; the "
                               f"feedback measures and corrects the mass after every {mb.MASS_EVERY} step(s)",
            "workload": "64 cubic jobs, edges uniform from {64,96,128,160,192}, c0 U[-0.4,0.4], kappa U[0.5,2], "
                        "noise amplitude 0.05, seeds 1000+j (draws seed 7), dt 0.005",
            "l2": "fields (about 1.5 GB) larger than L2"}


def run_precision(mb, dev, steps, n=512, seed=42, every=250):
    """Precision study (C3): the off-critical quench at n^3, c0 = 0.3 plus
    Gaussian noise sigma 0.02, dt 0.005, M 1, kappa 1.5, stepped in FP32
    (FP64 reductions, mass feedback) and in FP64 -- the drop-in path, which
    is bit-identical to the reference build and so serves as the FP64 oracle
    at a size the CPU build cannot run in minutes.  Reports the FP32 max-norm
    error at step 100, the mass drift of both, the free energy of both every
    `every` steps, and the structure-factor peak wavenumber of both at the
    end."""
    import numpy as np
    ic = mb.ic_generate((n, n, n), 0.3, 0.02, True, seed)
    kw = dict(kappa=1.5, M=1.0)
    t0 = time.perf_counter()
    sims = {prec: mb.CHSim(mb.make_params(n, n, n, DT, precision=prec, **kw), dev) for prec in ("fp64", "fp32")}
    out = {"workload": f"{n}^3, c0 = 0.3 + N(0, 0.02^2) seed {seed}, dt 0.005, M 1, kappa 1.5, {steps} steps; "
                       f"FP32 = FP32 field, FP64 reductions, mass feedback every {mb.MASS_EVERY} step(s); FP64 = the drop-in path"}
    try:
        for sim in sims.values():
            sim.set_field(ic)
        del ic
        r0 = {p: s.reduce() for p, s in sims.items()}
        curve = {p: [(0, r0[p]["energy"])] for p in sims}
        done = 0
        marks = sorted(set([min(100, steps)] + list(range(every, steps + 1, every)) + [steps]))
        for m in marks:
            for s in sims.values():
                s.step(m - done)
            done = m
            r = {p: s.reduce() for p, s in sims.items()}
            for p in sims:
                curve[p].append((m, r[p]["energy"]))
            if m == min(100, steps):
                a = sims["fp64"].get_field()
                b = sims["fp32"].get_field()
                out["maxnorm_fp32_vs_fp64_at_step"] = m
                out["maxnorm_fp32_vs_fp64"] = float(np.max(np.abs(a - b)))
                del a, b
        r1 = {p: s.reduce() for p, s in sims.items()}
        for p in sims:
            out[f"mass_drift_rel_{p}"] = abs(r1[p]["mass"] - r0[p]["mass"]) / abs(r0[p]["mass"])
        out["mass_fp32_minus_fp64_rel"] = abs(r1["fp32"]["mass"] - r1["fp64"]["mass"]) / abs(r1["fp64"]["mass"])
        out["energy"] = {p: [[m, e] for m, e in curve[p]] for p in sims}
        out["energy_rel_diff_max"] = max(abs(e32 - e64) / abs(e64) for (_, e32), (_, e64)
                                         in zip(curve["fp32"], curve["fp64"]))
        out["energy_decays"] = {p: all(b[1] <= a[1] for a, b in zip(curve[p], curve[p][1:])) for p in sims}
        k1 = {p: s.structure_factor(64)[2] for p, s in sims.items()}
        out["sk_peak_k1"] = k1
        out["sk_peak_rel_diff"] = abs(k1["fp32"] - k1["fp64"]) / abs(k1["fp64"])
        out["wall_s"] = time.perf_counter() - t0
    finally:
        for s in sims.values():
            s.close()
    return out


def batch_same_mix(mb, torch, dev, arrivals, noise, steps=100, warmup=10):
    """The served burst's jobs (same shapes, precisions, parameters and
    fields) stepped together as one batch, `steps` steps timed by CUDA
    events on the batch's stream: what the batch path gives on the served
    mix, against which the served throughput is compared."""
    params = [mb.make_params(*dims, dt, kappa=kap, precision=prec) for (_, dims, dt, prec, _, kap, _, _) in arrivals]
    b = mb.Batch(params, dev)
    try:
        for j, (_, dims, _, _, c0, _, _, _) in enumerate(arrivals):
            b.set_field(j, noise[dims] + c0)
        b.step(warmup)
        b.sync()
        ext = torch.cuda.ExternalStream(b.stream, device=f"cuda:{dev}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(ext)
        b.step(steps)
        e1.record(ext)
        b.sync()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        launches = b.info()["launches_per_step"]
    finally:
        b.close()
    sites = float(sum(d[0] * d[1] * d[2] for (_, d, *_r) in arrivals))
    return {"glups": sites * steps / (ms * 1e-3) / 1e9, "steps": steps, "launches_per_step": launches}


def run_serve(mb, dev, window_s, seed=11, rate=20.0, burst=0, torch=None, slots=256):
    """Served stream: Poisson arrivals at `rate` jobs/s for `window_s` seconds, then drain.
    burst > 0: that many jobs of the same mix submitted at once into a server
    of `slots` job slots, so that jobs wait in its queue for most of the run
    (the server's saturated throughput is measured over the ticks that begin
    with a backlog); with `torch` the first `slots` of those jobs, as many as
    the server runs at once, are then stepped as one batch for comparison."""
    import numpy as np
    rng = np.random.default_rng(seed)
    arrivals, t = [], 0.0
    while True:
        if burst:
            if len(arrivals) >= burst:
                break
        else:
            t += rng.exponential(1.0 / rate)
            if t > window_s:
                break
        if rng.random() < 0.5:
            e = int(rng.choice(C5_EDGES_2D))
            dims, dt = (e, e, 1), 0.01
        else:
            e = int(rng.choice(C5_EDGES_3D))
            dims, dt = (e, e, e), DT
        prec = "fp32" if rng.random() < 0.5 else "fp64"
        arrivals.append((t, dims, dt, prec, float(rng.uniform(-0.4, 0.4)), float(rng.uniform(0.5, 2.0)),
                         int(rng.integers(500, 5001)), int(rng.integers(1, 1 << 30))))
    # one seeded noise field per grid shape, made before the clock starts (a
    # client generating 16.7 M-site fields inline could not keep up with the
    # arrival rate); each job adds its own mean c0
    noise = {}
    for (_, dims, *_rest) in arrivals:
        if dims not in noise:
            noise[dims] = mb.ic_generate(dims, 0.0, 0.05, False, seed + len(noise))
    # every job's field and parameters are made before the clock starts, so
    # that submitting is only the server's own copy of the field (building
    # the few GB of fields inline took the client seconds, during which the
    # server ran short of work)
    ics = [noise[dims] + c0 for (_, dims, _, _, c0, *_r) in arrivals]
    params = [mb.make_params(*dims, dt, kappa=kap, precision=prec) for (_, dims, dt, prec, _, kap, _, _) in arrivals]
    srv = mb.Server(dev, hbm_budget_gb=150.0, max_jobs=slots, steps_per_tick=100)
    ids = []
    try:
        t0 = time.perf_counter()
        for i, ((ta, dims, dt, prec, c0, kap, nsteps, s), p) in enumerate(zip(arrivals, params)):
            lag = ta - (time.perf_counter() - t0)
            if lag > 0:
                time.sleep(lag)
            ids.append((srv.submit(p, ics[i], nsteps), p))
            ics[i] = None  # the server holds its own copy
        submit_s = time.perf_counter() - t0
        for jid, p in ids:
            srv.result(jid, p, timeout_us=600_000_000, want_field=False)
        wall = time.perf_counter() - t0
        st = srv.stats()
    finally:
        srv.close()
    same_mix = (batch_same_mix(mb, torch, dev, arrivals[:slots], noise) if (burst and torch is not None)
                else None)
    upd = sum(d[0] * d[1] * d[2] * n for (_, d, _, _, _, _, n, _) in arrivals)
    upd_bytes = sum(d[0] * d[1] * d[2] * n * (8 if pr == "fp32" else 16) for (_, d, _, pr, _, _, n, _) in arrivals)
    return {"sims_per_hour": st["sims_per_hour"], "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
            "gbs": st["site_updates_per_s"] * upd_bytes / upd / 1e9,
            "mean_ms": st["mean_ms"], "completed": st["completed"], "failed": st["failed"],
            "worker_s": {k: st[k] for k in ("step_s", "admit_s", "retire_s")},
            "ticks": st["ticks"], "rebuilds": st["rebuilds"], "refreshes": st["refreshes"],
            "glups": st["site_updates_per_s"] / 1e9, "hbm_peak_gb": st["hbm_peak_gb"], "wall_s": wall,
            "sat_glups": st["sat_site_updates_per_s"] / 1e9, "sat_ticks": st["sat_ticks"], "slots": slots,
            "gpu_busy": st["gpu_s"] / wall if wall > 0 else None,
            "submitted": len(arrivals), "batch_same_mix": same_mix, "submit_s": submit_s,
            "arrivals": arrivals, "noise": noise,
            "workload": (f"{burst} jobs submitted at once into {slots} slots (seed {seed})" if burst else
                         f"Poisson arrivals {rate:g}/s for {window_s:g} s (seed {seed})") + ": 50% 2-D edge "
                        "{128,256,512,1024} dt 0.01, 50% 3-D edge {64..256 step 32} dt 0.005, 50/50 fp32/fp64, "
                        "steps U[500,5000], c0 U[-0.4,0.4] plus uniform noise of amplitude 0.05 (one seeded "
                        "field per shape), kappa U[0.5,2], budget 150 GB, ticks of 100 steps"}


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import mesobasic_b200 as mb

    torch.cuda.set_device(local_rank)
    dev = local_rank
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", dev))

    ic = mb.ic_generate((N, N, N), CO, AMP, False, SEED)
    flush_w = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    flush_r = torch.ones(64 << 20, dtype=torch.float32, device=f"cuda:{dev}")  # 256 MB

    class _Flush:
        """L2 flush between timed steps: a write larger than L2, then a read
        of another buffer larger than L2, which writes back and evicts the
        dirty lines of the first."""
        @staticmethod
        def fill_(v):
            flush_w.fill_(v)
            flush_r.sum()

    flush = _Flush()
    sampler = ClockSampler(dev)
    results = {}

    def timed_steps(sim, K, W):
        ext = torch.cuda.ExternalStream(sim.stream, device=f"cuda:{dev}")
        for _ in range(W):
            sim.step(1)
        sim.sync()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        sampler.start()
        for e0, e1 in evs:
            with torch.cuda.stream(ext):
                flush.fill_(1)
            e0.record(ext)
            sim.step(1)
            e1.record(ext)
        sim.sync()
        torch.cuda.synchronize()
        sampler.stop()
        if dist:
            dist.barrier()
        ms = [e0.elapsed_time(e1) for e0, e1 in evs]
        return sum(ms), ms

    def e2e(params, K):
        """Through the C ABI with pinned host buffers: upload of the initial
        field, K steps, download of the final field, all inside the region."""
        host_in = torch.from_numpy(ic.reshape(-1)).pin_memory()
        host_out = torch.empty(N * N * N, dtype=torch.float64).pin_memory()
        with mb.CHSim(params, dev) as sim:
            sim.set_field_ptr(host_in.data_ptr())  # warm-up of the same path
            sim.step(2)
            sim.get_field_ptr(host_out.data_ptr())
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            t0 = time.perf_counter()
            sim.set_field_ptr(host_in.data_ptr())
            sim.step(K)
            sim.get_field_ptr(host_out.data_ptr())
            t = time.perf_counter() - t0
            if dist:
                tt = torch.tensor([t], device=f"cuda:{dev}", dtype=torch.float64)
                dist.all_reduce(tt, op=dist.ReduceOp.MAX)
                t = float(tt.item())
        return t

    peak, peak_kind = load_peaks()
    for prec in ("fp64", "fp32"):
        params = mb.make_params(N, N, N, DT, kappa=KAP, M=M, precision=prec)
        with mb.CHSim(params, dev) as sim:
            sim.set_field(ic)
            tot_ms, ms = timed_steps(sim, args.steps, args.warmup)
            tiling = sim.tiling.as_tuple()
        if dist:
            tt = torch.tensor([tot_ms], device=f"cuda:{dev}", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            tot_ms = float(tt.item())
        results[prec] = dict(ms_total=tot_ms, ms=ms, tiling=tiling)
    e2e_t = {prec: e2e(mb.make_params(N, N, N, DT, kappa=KAP, M=M, precision=prec), args.steps)
             for prec in ("fp64", "fp32")}
    models = (run_models(mb, torch, dev, min(args.steps, 20), max(args.warmup, 3), flush, sampler, load_peaks()[0])
              if args.model_steps else None)
    batch = run_batch(mb, torch, dev, args.batch_steps, sampler) if args.batch_steps > 0 else None
    precision = run_precision(mb, dev, args.precision_steps) if args.precision_steps > 0 else None
    clocks = sampler.summary()
    serve = None
    if args.serve_seconds > 0:
        # the served stream's latencies vary from run to run (arrivals are
        # timed by the wall clock, so the job mix of each tick changes): run
        # it several times and report the median run by sims/hour
        runs = [run_serve(mb, dev, args.serve_seconds) for _ in range(max(1, args.serve_runs))]
        for r in runs:  # the inputs of a run are not part of its record
            r.pop("arrivals")
            r.pop("noise")
        runs.sort(key=lambda r: r["sims_per_hour"])
        serve = dict(runs[len(runs) // 2])
        serve["runs"] = [{k: r[k] for k in ("sims_per_hour", "p50_ms", "p99_ms", "glups")} for r in runs]
        serve["reported"] = f"median of {len(runs)} runs by sims_per_hour"
        if args.serve_burst > 0:
            # saturated: a burst of the same mix into fewer slots than jobs,
            # so that the queue holds jobs for most of the run
            # (its throughput spreads by +-20 % from run to run: the median of
            # serve_runs runs by whole-run GLUPS, the same jobs as one batch once)
            sats = [run_serve(mb, dev, args.serve_seconds, burst=args.serve_burst, slots=args.serve_slots)
                    for _ in range(max(1, args.serve_runs))]
            sats.sort(key=lambda r: r["glups"])
            sat = sats[len(sats) // 2]
            sat["batch_same_mix"] = batch_same_mix(mb, torch, dev, sat["arrivals"][:args.serve_slots], sat["noise"])
            for r in sats:
                r.pop("arrivals")
                r.pop("noise")
            serve["saturated"] = {k: sat[k] for k in ("glups", "sat_glups", "sat_ticks", "slots", "gpu_busy", "sims_per_hour",
                                                      "p50_ms", "p99_ms", "completed", "ticks", "rebuilds",
                                                      "refreshes", "wall_s", "submit_s")}
            serve["saturated_worker_s"] = sat["worker_s"]
            serve["saturated"]["runs_glups"] = [round(r["glups"], 1) for r in sats]
            # the fraction uses the mix's algorithmic bytes (8 B per FP32
            # site update, 16 B per FP64)
            serve["saturated"]["roofline_frac"] = sat["gbs"] / peak
            serve["saturated"]["vs_batch"] = sat["glups"] / batch["value"] if batch else None
            # against the batch path on jobs of the same mix (mixed
            # precisions, 2-D and 3-D), as many at once as the server's slots:
            # the server's own overhead (ticks, admission, retiring) without
            # the difference in workload.  sat_glups counts the ticks that
            # began with a backlog; glups the whole run, the final drain
            # (the last long jobs running alone) included
            bm = sat["batch_same_mix"]
            serve["saturated"]["batch_same_mix_glups"] = bm["glups"]
            serve["saturated"]["vs_batch_same_mix"] = sat["sat_glups"] / bm["glups"]
            serve["saturated"]["vs_batch_same_mix_whole_run"] = sat["glups"] / bm["glups"]
            serve["saturated"]["workload"] = sat["workload"]
    if batch and dist:
        tt = torch.tensor([batch["ms"]], device=f"cuda:{dev}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        batch["ms"] = float(tt.item())
        batch["value"] = world * batch["sites"] * batch["steps"] / (batch["ms"] * 1e-3) / 1e9

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    sites = float(N) ** 3
    out = {}
    for prec, es in (("fp64", 8), ("fp32", 4)):
        r = results[prec]
        ms_step = r["ms_total"] / args.steps
        glups = world * sites / (ms_step * 1e-3) / 1e9
        achieved = sites * 2 * es / (statistics.mean(r["ms"]) * 1e-3) / 1e9  # GB/s, algorithmic bytes
        traffic = load_traffic(prec)
        e2e_glups = world * sites * args.steps / e2e_t[prec] / 1e9
        out[prec] = {
            "value": glups, "ms_per_step": ms_step,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs, burst)",
                         "algorithmic_bytes_per_launch": sites * 2 * es},
            "e2e": {"value": e2e_glups, "unit": "GLUPS", "h2d_bytes_per_step": sites * 8 / args.steps,
                    "d2h_bytes_per_step": sites * 8 / args.steps,
                    "region": f"upload of the FP64 initial field from pinned memory, {args.steps} steps, download "
                              "of the final field, through mg_ch_set_field / mg_ch_step / mg_ch_get_field; "
                              "bytes per step = one field each way / steps"},
            "tiling": {"ty": r["tiling"][0], "nchunk": r["tiling"][1], "nbuf": r["tiling"][2]},
            "ms_per_step_min": min(r["ms"]), "ms_per_step_max": max(r["ms"]),
        }
    if batch:
        batch["roofline_frac"] = batch["value"] * 8 / peak  # GB/s of algorithmic bytes / peak
    cpu = cpu_baseline_sample()
    detail = {"fp64": out["fp64"], "fp32": out["fp32"], "batch": batch, "serve": serve, "precision": precision,
              "models": models, "cpu_baseline": cpu, "clocks": clocks}
    if args.detail:
        with open(args.detail, "w") as f:
            json.dump(detail, f, indent=1)
    r64, r32 = out["fp64"]["roofline"], out["fp32"]["roofline"]
    line = {
        "metric": METRIC, "value": out["fp64"]["value"], "unit": "GLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": out["fp64"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(CONFIG, precision="fp64 drop-in (bit-identical to the reference build)"),
        "roofline": {k: r64[k] for k in ("bound", "achieved", "peak", "unit", "frac", "traffic")}
                    | {"traffic_source": TRAFFIC_SOURCE["fp64"], "peak_kind": r64["peak_kind"]},
        "e2e": {k: out["fp64"]["e2e"][k] for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step")},
        "fp32": {"value": out["fp32"]["value"], "ms_per_step": out["fp32"]["ms_per_step"],
                 "frac": r32["frac"], "achieved_gbs": r32["achieved"], "traffic": r32["traffic"],
                 "speedup_vs_fp64": out["fp32"]["value"] / out["fp64"]["value"],
                 "e2e": out["fp32"]["e2e"]["value"],
                 "mass_correct": mb.MASS_EVERY},
        "batch": None if not batch else {
            "value": batch["value"], "roofline_frac": batch["roofline_frac"], "jobs": batch["jobs"],
            "steps": batch["steps"], "launches_per_step": batch["launches_per_step"], "tiles": batch["tiles"],
            "max_mass_drift_per_site": batch["max_mass_drift_per_site"],
            "max_mass_drift_rel": batch["max_mass_drift_rel"]},
        "serve": None if not serve else {
            "sims_per_hour": serve["sims_per_hour"], "p50_ms": serve["p50_ms"], "p99_ms": serve["p99_ms"],
            "glups": serve["glups"], "runs": len(serve["runs"]), "reported": serve["reported"],
            "saturated": None if not serve.get("saturated") else
            {k: v for k, v in serve["saturated"].items() if k != "workload"}
            | {"workload": f"burst of {args.serve_burst} jobs of the same mix into {args.serve_slots} "
                            "slots (detail file)"}},
        "precision": None if not precision else {
            k: precision.get(k) for k in ("maxnorm_fp32_vs_fp64", "mass_drift_rel_fp32", "mass_drift_rel_fp64",
                                          "sk_peak_rel_diff", "energy_rel_diff_max")},
        "models": None if not models else {k: round(v["value"], 2) for k, v in models.items() if isinstance(v, dict)},
        "cpu_baseline": cpu,
        "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "gpu_launches": args.steps,
        "notes": "fp64 = headline (one fused step launch per timed step, L2 flushed between steps); fp32 = FP32 "
                 "field with FP64 mass feedback; batch = C4 64 jobs; serve = C5 stream, median run; "
                 "per-leg detail in the --detail file",
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


# ------------------------------------------------------- reference CPU arm
def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference_build(steps, ranks, n=N, timeout=600):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not os.path.exists(oracle.REF_BENCH):
        raise FileNotFoundError(oracle.REF_BENCH)
    # the slab split needs nx divisible by the rank count
    while ranks > 1 and n % ranks:
        ranks -= 1
    env = dict(os.environ, MB_SHIM_NP=str(ranks), MB_SHIM_SLOT_MB="16")
    args = [oracle.REF_BENCH, f"Domain/nx={n}", f"Domain/ny={n}", f"Domain/nz={n}", f"Time/dt={DT}",
            f"Time/nstep={steps}", f"PFApp/kap={KAP}", f"PFApp/M={M}", f"PFApp/co={CO}", f"PFApp/noise_amp={AMP}",
            f"PFApp/seed={SEED}", "PFApp/vtk=0", "PFApp/init_output=0"]
    r = subprocess.run(args, env=env, capture_output=True, text=True, timeout=timeout, cwd="/tmp")
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-500:])
    return json.loads(r.stdout.strip().splitlines()[-1]), ranks


def cpu_baseline_sample():
    """Reference CPU build on all host cores, a bounded sample (3 steps of 256^3)."""
    try:
        d, ranks = run_reference_build(3, host_cores())
        return {"value": d["site_updates_per_s"] / 1e9, "unit": "GLUPS", "cores": ranks, "kind": "reference",
                "sample": f"3 steps of the 256^3 workload, {ranks} MPI-shim ranks (one per core), step loop only"}
    except Exception as e:  # the reference build is test infrastructure; report why it is missing
        return {"value": None, "unit": "GLUPS", "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    cores = host_cores()
    budget_s = 120.0
    # warm-up run (also sizes the sample): W steps, then as many of the K
    # timed steps as fit the budget
    probe, ranks = run_reference_build(args.warmup, cores)
    per_step = probe["seconds"] / max(args.warmup, 1)
    total = args.steps + args.warmup
    steps = max(1, min(args.steps, int(budget_s / max(per_step, 1e-6))))
    d, ranks = run_reference_build(steps, cores)
    glups = d["site_updates_per_s"] / 1e9
    line = {
        "metric": METRIC, "value": glups, "unit": "GLUPS", "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": d["seconds"] / steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "warmup_note": f"{args.warmup} warm-up steps in a separate run of the same build (it also sizes the sample)",
        "config": dict(CONFIG, precision="fp64", l2="n/a (CPU)"),
        "cpu_baseline": {"value": glups, "unit": "GLUPS", "cores": ranks, "kind": "reference",
                         "sample": f"{steps} of the requested {total} steps of the 256^3 workload on {ranks} "
                                   f"MPI-shim ranks (one per host core), step loop wall time"},
        "e2e": {"value": glups, "unit": "GLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--batch-steps", type=int, default=1000, help="steps of the batched sweep (0: skip)")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="arrival window of the served stream (0: skip)")
    ap.add_argument("--serve-runs", type=int, default=3, help="runs of the served stream (the median is reported)")
    ap.add_argument("--serve-burst", type=int, default=160, help="jobs of the saturated served leg (0: skip)")
    ap.add_argument("--serve-slots", type=int, default=40, help="job slots of the saturated served leg's server")
    ap.add_argument("--precision-steps", type=int, default=2000,
                    help="steps of the 512^3 FP32-vs-FP64 precision study (0: skip)")
    ap.add_argument("--model-steps", type=int, default=1, help="time the variable-mobility models (0: skip)")
    ap.add_argument("--detail", default=None, help="write every leg's full record to this JSON file")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
