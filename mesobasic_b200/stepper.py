"""Command-line stepper: runs one simulation through the C ABI and reports
GLUPS.  Used for quick measurements, tiling sweeps and profiler captures.

    python -m mesobasic_b200.stepper --n 256 --precision fp32 --steps 20
    python -m mesobasic_b200.stepper --n 256 --tiling 8,8,6 --steps 20
    python -m mesobasic_b200.stepper --n 256 --autotune
    python -m mesobasic_b200.stepper --n 256 --sweep   # every valid tiling, sorted
    python -m mesobasic_b200.stepper --n 256 --model tipsphil --steps 4

--model tipsphil runs the variable-mobility TIPSphil step (FP64, periodic,
dt 0.01, noise 0.1, c = 0.3 + U[-0.05, 0.05]) with the quench of the
models leg of the benchmark.
"""
from __future__ import annotations

import argparse
import itertools
import json
import time

import numpy as np

import mesobasic_b200 as mb


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=256, help="cube edge (overridden by --dims)")
    ap.add_argument("--dims", type=str, default=None, help="nx,ny,nz")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--mass-correct", type=int, default=None)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--dt", type=float, default=0.005)
    ap.add_argument("--kappa", type=float, default=1.0)
    ap.add_argument("--tiling", type=str, default=None, help="ty,nchunk,nbuf")
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--sweep", action="store_true")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--model", choices=["ch", "tipsphil"], default="ch")
    return ap.parse_args()


# TIPSphil quench of the benchmark's models leg
TIPSPHIL = dict(alpha=150.0, beta=0.1, N=50.0, Tinit=300.0, Tbath=280.0, Tcrystal=200.0, gamma=1.0, D0=1.0,
                Mweight=0.5, Mvolume=1.0)


def time_steps(sim, steps, warmup):
    sim.step(warmup)
    sim.sync()
    t0 = time.perf_counter()
    sim.step(steps)
    sim.sync()
    return (time.perf_counter() - t0) / steps


def main():
    a = parse()
    dims = tuple(int(v) for v in a.dims.split(",")) if a.dims else (a.n, a.n, a.n)
    p = mb.make_params(*dims, a.dt, kappa=a.kappa, precision=a.precision, mass_correct=a.mass_correct)
    sites = float(np.prod(dims))
    bytes_site = 16 if a.precision == "fp64" else 8
    ic = mb.ic_generate(dims, 0.0, 0.1, False, 42)
    if a.model == "tipsphil":
        p = mb.make_params(*dims, 0.01, noise=0.1, noise_seed=42)
        with mb.CHSim(p, a.device, fh=mb.make_fh_params(10 ** 6, **TIPSPHIL)) as sim:
            sim.set_field(0.3 + ic)
            s = time_steps(sim, a.steps, a.warmup)
            print(json.dumps({"dims": dims, "model": "TIPSphil", "tiling": sim.tiling.as_tuple(),
                              "ms_per_step": s * 1e3, "glups": sites / s * 1e-9}))
        return
    if a.autotune:
        t, ms = mb.autotune(p, a.device, trials=max(5, a.steps))
        print(json.dumps({"autotune": t.as_tuple(), "ms": ms, "glups": sites / ms * 1e-6}))
        return
    with mb.CHSim(p, a.device) as sim:
        sim.set_field(ic)
        if a.tiling:
            ty, nc, nb = (int(v) for v in a.tiling.split(","))
            sim.tiling = (ty, nc, nb, 0)
        if a.sweep:
            res = []
            tys = [1] if (dims[2] == 1 or dims[1] == 1) else list(range(1, 31))
            for ty, nc, nb in itertools.product(tys, (1, 2, 4, 6, 8, 10, 12, 16, 24, 32, 48, 64), (3, 4, 6, 8)):
                try:
                    sim.tiling = (ty, nc, nb, 0)
                except mb.MGError:
                    continue
                s = time_steps(sim, a.steps, a.warmup)
                res.append((s, ty, nc, nb))
            res.sort()
            for s, ty, nc, nb in res[:15]:
                print(json.dumps({"tiling": [ty, nc, nb], "ms": s * 1e3, "glups": sites / s * 1e-9,
                                  "gbs": sites * bytes_site / s * 1e-9}))
            return
        s = time_steps(sim, a.steps, a.warmup)
        t = sim.tiling
        print(json.dumps({"dims": dims, "precision": a.precision, "tiling": t.as_tuple(), "ms_per_step": s * 1e3,
                          "glups": sites / s * 1e-9, "gbs": sites * bytes_site / s * 1e-9}))


if __name__ == "__main__":
    main()
