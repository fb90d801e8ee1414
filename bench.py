"""Benchmark of the Cahn-Hilliard step (3-D 256^3, dt 0.005, M 1, kappa 1,
periodic, c0 = 0 + U[-0.05, 0.05] from seed 42).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  `value` is FP64 (the drop-in precision, the same
arithmetic as the reference build) in GLUPS = lattice-site updates per
second, summed over ranks; the FP32 path (FP32 field, FP64 reductions, mass
feedback) is reported beside it under "fp32".  Each timed step is one fused
kernel launch; an L2 flush (a 512 MB write) runs between timed steps and is
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
          "l2": "flushed between timed steps (512 MB write, untimed)",
          "parallelism": "replicas (one independent simulation per GPU)"}
METRIC = "GLUPS & % HBM roofline (FP32 vs FP64)"


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(dtype):
    """DRAM bytes per launch of the step kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", f"ncu_ch_step_{dtype}_256.md")
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
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            parts = [x.strip() for x in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ our arm
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
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    results = {}

    def timed_steps(sim, K, W, sampler=None):
        ext = torch.cuda.ExternalStream(sim.stream, device=f"cuda:{dev}")
        for _ in range(W):
            sim.step(1)
        sim.sync()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for e0, e1 in evs:
            with torch.cuda.stream(ext):
                flush.fill_(1)
            e0.record(ext)
            sim.step(1)
            e1.record(ext)
        sim.sync()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        wall = time.perf_counter() - t0
        ms = [e0.elapsed_time(e1) for e0, e1 in evs]
        return sum(ms), ms, wall

    def e2e(params, K):
        """Through the C ABI with pinned host buffers; copies inside the region."""
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
    sampler = ClockSampler(dev)
    with sampler:
        for prec in ("fp64", "fp32"):
            params = mb.make_params(N, N, N, DT, kappa=KAP, M=M, precision=prec)
            with mb.CHSim(params, dev) as sim:
                sim.set_field(ic)
                tot_ms, ms, wall = timed_steps(sim, args.steps, args.warmup)
                tiling = sim.tiling.as_tuple()
            if dist:
                tt = torch.tensor([tot_ms], device=f"cuda:{dev}", dtype=torch.float64)
                dist.all_reduce(tt, op=dist.ReduceOp.MAX)
                tot_ms = float(tt.item())
            results[prec] = dict(ms_total=tot_ms, ms=ms, wall=wall, tiling=tiling)
    clocks = sampler.summary()
    e2e_t = {prec: e2e(mb.make_params(N, N, N, DT, kappa=KAP, M=M, precision=prec), args.steps)
             for prec in ("fp64", "fp32")}

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
                    "d2h_bytes_per_step": sites * 8 / args.steps},
            "tiling": {"ty": r["tiling"][0], "nchunk": r["tiling"][1], "nbuf": r["tiling"][2]},
            "ms_per_step_min": min(r["ms"]), "ms_per_step_max": max(r["ms"]),
        }
    cpu = cpu_baseline_sample()
    line = {
        "metric": METRIC, "value": out["fp64"]["value"], "unit": "GLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": out["fp64"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(CONFIG, precision="fp64 drop-in (bit-identical to the reference build)"),
        "roofline": out["fp64"]["roofline"],
        "e2e": out["fp64"]["e2e"],
        "fp32": {k: out["fp32"][k] for k in ("value", "ms_per_step", "roofline", "e2e", "tiling")}
                | {"dtype": "f32 field, f64 reductions, mass feedback",
                   "speedup_vs_fp64": out["fp32"]["value"] / out["fp64"]["value"]},
        "tiling": out["fp64"]["tiling"],
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": args.steps,
        "gpu_launches_note": "one fused ch_step_kernel launch per timed step (fp64 region); fp32 region likewise",
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
    # size the sample: one probe step, then as many steps as fit the budget
    probe, ranks = run_reference_build(1, cores)
    per_step = probe["seconds"]
    total = args.steps + args.warmup
    steps = max(1, min(args.steps, int(budget_s / max(per_step, 1e-6))))
    d, ranks = run_reference_build(steps, cores)
    glups = d["site_updates_per_s"] / 1e9
    line = {
        "metric": METRIC, "value": glups, "unit": "GLUPS", "n_gpus": world, "steps": steps, "warmup": 0,
        "ms_per_step": d["seconds"] / steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
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
