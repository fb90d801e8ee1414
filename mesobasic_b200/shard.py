"""Independent simulation jobs spread over several GPUs, one process per GPU.

A single simulation never spans GPUs (one process drives one GPU, no domain
decomposition), so a multi-GPU run is a set of independent jobs: each rank
takes a share of the job list, steps it on its own GPU with the batch API,
and rank 0 gathers the results.  The only collectives are host-side
gathers of results and statistics after the work; nothing crosses between
GPUs while jobs run.

    import torch.distributed as dist
    dist.init_process_group("nccl")            # torchrun, one rank per GPU
    out = run_jobs(specs, steps=1000)          # rank 0: every job's result

`assign` is deterministic (the same list gives the same split on every
rank), so ranks agree on the split without exchanging it.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Sequence


@dataclass(frozen=True)
class JobSpec:
    """One job: grid, time step, coefficients, precision and initial condition
    (mean c0, uniform noise amplitude, MT19937 seed, as mg_ic_generate)."""
    dims: tuple
    dt: float
    kappa: float = 1.0
    M: float = 1.0
    precision: str = "fp32"
    c0: float = 0.0
    noise: float = 0.05
    seed: int = 42
    steps: int = 1000

    @property
    def sites(self) -> int:
        return int(self.dims[0]) * int(self.dims[1]) * int(self.dims[2])

    @property
    def cost(self) -> float:
        # site-updates, FP64 counted twice (twice the bytes per site)
        return self.sites * self.steps * (2.0 if self.precision == "fp64" else 1.0)


def assign(specs: Sequence[JobSpec], world: int) -> list[int]:
    """Rank of each job: largest jobs first, each to the least-loaded rank
    (ties to the lower rank, equal jobs in list order)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(specs)), key=lambda i: (-specs[i].cost, i))
    load = [0.0] * world
    rank_of = [0] * len(specs)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        rank_of[i] = r
        load[r] += specs[i].cost
    return rank_of


def gpu_runner(device: int) -> Callable[[list[JobSpec]], list[dict]]:
    """Steps a rank's jobs together on `device` (one batch; jobs with the
    same step count advance in lockstep, the rest in later batches)."""
    import mesobasic_b200 as mb

    def run(specs: list[JobSpec]) -> list[dict]:
        out = [None] * len(specs)
        by_steps: dict[int, list[int]] = {}
        for i, s in enumerate(specs):
            by_steps.setdefault(s.steps, []).append(i)
        for steps, idx in sorted(by_steps.items()):
            params = [mb.make_params(*specs[i].dims, specs[i].dt, kappa=specs[i].kappa, M=specs[i].M,
                                     precision=specs[i].precision) for i in idx]
            b = mb.Batch(params, device)
            try:
                for k, i in enumerate(idx):
                    s = specs[i]
                    b.set_field(k, mb.ic_generate(s.dims, s.c0, s.noise, False, s.seed))
                b.step(steps)
                b.sync()
                for k, i in enumerate(idx):
                    out[i] = {"field": b.get_field(k), "stats": b.reduce(k)}
            finally:
                b.close()
        return out

    return run


def run_jobs(specs: Sequence[JobSpec], runner: Callable[[list[JobSpec]], list[dict]] | None = None,
             group=None) -> list[dict] | None:
    """Runs this rank's share of `specs` with `runner` (default: the GPU of
    this rank's LOCAL_RANK) and gathers every result on rank 0, in list
    order; other ranks get None.  Without an initialised process group the
    whole list runs here."""
    import torch.distributed as dist

    specs = list(specs)
    if not (dist.is_available() and dist.is_initialized()):
        if runner is None:
            runner = gpu_runner(0)
        return runner(specs)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    if runner is None:
        import os
        runner = gpu_runner(int(os.environ.get("LOCAL_RANK", rank)))
    mine = [i for i, r in enumerate(assign(specs, world)) if r == rank]
    results = runner([specs[i] for i in mine]) if mine else []
    payload = list(zip(mine, results))
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(payload, gathered, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * len(specs)
    for part in gathered:
        for i, res in part:
            out[i] = res
    missing = [i for i, r in enumerate(out) if r is None]
    if missing:
        raise RuntimeError(f"jobs {missing} returned no result")
    return out
