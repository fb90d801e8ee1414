"""Job sharding over ranks (mesobasic_b200/shard.py) on CPU: the split is
deterministic and balanced, and a world_size-2 gloo run gathers every job's
result exactly once on rank 0.  The runner is a CPU stand-in (the oracle's
C step), so no GPU is needed."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from mesobasic_b200.shard import JobSpec, assign  # noqa: E402


def specs():
    dims = [(16, 12, 8), (8, 8, 8), (24, 8, 4), (16, 16, 1), (8, 12, 6), (12, 12, 12), (32, 8, 1)]
    return [JobSpec(dims=d, dt=0.005, kappa=0.5 + 0.25 * i, c0=0.05 * i, noise=0.1, seed=100 + i, steps=3 + i,
                    precision="fp64" if i % 3 == 0 else "fp32") for i, d in enumerate(dims)]


def test_assign_is_deterministic_and_balanced():
    s = specs()
    a = assign(s, 2)
    assert a == assign(list(s), 2)
    load = [sum(x.cost for x, r in zip(s, a) if r == k) for k in range(2)]
    assert max(load) - min(load) <= max(x.cost for x in s)
    assert assign(s, 1) == [0] * len(s)
    assert sorted(set(assign(s, 4))) == [0, 1, 2, 3]
    with pytest.raises(ValueError):
        assign(s, 0)


def oracle_runner(batch):
    import oracle
    out = []
    for s in batch:
        ic = oracle.ic(s.dims, s.c0, s.noise, False, s.seed)
        f = oracle.run(ic, s.dims, (1.0, 1.0, 1.0), s.dt, s.M, s.kappa, s.steps)
        out.append({"field": f, "rank": int(os.environ["RANK"])})
    return out


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from mesobasic_b200.shard import run_jobs
        out = run_jobs(specs(), runner=oracle_runner)
        if rank == 0:
            q.put([(r["rank"], r["field"]) for r in out])
        else:
            q.put(out)
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_gloo_run_gathers_every_job_once():
    import oracle
    oracle.build()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rank0 = [g for g in got if g is not None]
    assert len(rank0) == 1 and got.count(None) == 1
    res = rank0[0]
    s = specs()
    a = assign(s, 2)
    assert [r for r, _ in res] == a  # each job ran on its assigned rank
    for spec, (_, field) in zip(s, res):
        ic = oracle.ic(spec.dims, spec.c0, spec.noise, False, spec.seed)
        want = oracle.run(ic, spec.dims, (1.0, 1.0, 1.0), spec.dt, spec.M, spec.kappa, spec.steps)
        assert np.array_equal(field, want)


@pytest.mark.gpu
def test_gpu_runner_equals_standalone_runs():
    """Without a process group the whole list runs on this GPU in batches
    grouped by step count; each result equals the job run alone."""
    import mesobasic_b200 as mb
    from mesobasic_b200.shard import run_jobs
    s = [JobSpec(dims=(64, 32, 16), dt=0.005, seed=1, steps=20), JobSpec(dims=(32, 32, 1), dt=0.01, seed=2, steps=20),
         JobSpec(dims=(64, 64, 8), dt=0.005, precision="fp64", seed=3, steps=7)]
    out = run_jobs(s)
    for spec, r in zip(s, out):
        p = mb.make_params(*spec.dims, spec.dt, kappa=spec.kappa, M=spec.M, precision=spec.precision)
        with mb.CHSim(p) as sim:
            sim.set_field(mb.ic_generate(spec.dims, spec.c0, spec.noise, False, spec.seed))
            sim.step(spec.steps)
            want = sim.get_field()
        assert np.array_equal(r["field"], want)
