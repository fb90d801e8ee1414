"""Batched persistent launches and the continuous-batching server: every
job's result is the same, bit for bit, alone and in the mix."""
import time

import numpy as np
import pytest

import mesobasic_b200 as mb

pytestmark = pytest.mark.gpu


def job_set(seed=7, n=10):
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(n):
        if j % 3 == 2:
            e = int(rng.choice([64, 128, 256]))
            p = mb.make_params(e, e, 1, 0.01, kappa=float(rng.uniform(0.5, 2.0)),
                               precision="fp32" if j % 2 else "fp64")
        else:
            e = int(rng.choice([32, 64, 96]))
            p = mb.make_params(e, e, e, 0.005, kappa=float(rng.uniform(0.5, 2.0)),
                               precision="fp32" if j % 2 else "fp64")
        ic = mb.ic_generate((p.nx, p.ny, p.nz), float(rng.uniform(-0.4, 0.4)), 0.05, False, 1000 + j)
        jobs.append((p, ic))
    return jobs


def alone(p, ic, nsteps):
    with mb.CHSim(p) as sim:
        sim.set_field(ic)
        sim.step(nsteps)
        return sim.get_field(), sim.reduce()


def test_batch_equals_standalone_bitwise():
    jobs = job_set()
    b = mb.Batch([p for p, _ in jobs])
    try:
        for i, (_, ic) in enumerate(jobs):
            b.set_field(i, ic)
        b.step(60)
        info = b.info()
        # one launch per class: precision, 2-D or 3-D, row width (compile-time widths)
        classes = {(p.precision, p.nz == 1, p.nx) for p, _ in jobs}
        assert info["items"] >= len(jobs) and info["launches_per_step"] <= len(classes)
        for i, (p, ic) in enumerate(jobs):
            want, _ = alone(p, ic, 60)
            assert np.array_equal(b.get_field(i), want), i
    finally:
        b.close()


def test_c4_style_batch_autotune_keeps_results():
    """FP32 cubic jobs of mixed march widths (64..192): one launch per width
    class and step, the classes side by side in one captured graph; re-tiling
    the batch by the autotuner between steps leaves every job bit-identical
    to its standalone run."""
    rng = np.random.default_rng(3)
    jobs = []
    for j, e in enumerate((64, 96, 128, 160, 192, 64, 128)):
        p = mb.make_params(e, e, e, 0.005, kappa=float(rng.uniform(0.5, 2.0)), precision="fp32")
        jobs.append((p, mb.ic_generate((e, e, e), float(rng.uniform(-0.4, 0.4)), 0.05, False, 2000 + j)))
    widths = len({p.nx for p, _ in jobs})
    b = mb.Batch([p for p, _ in jobs])
    try:
        for i, (_, ic) in enumerate(jobs):
            b.set_field(i, ic)
        b.step(12)
        assert b.info()["launches_per_step"] == widths
        tuned = b.autotune(trials=2)
        assert tuned["threads"] > 0 and tuned["planes"] > 0 and tuned["ms_per_step"] > 0
        b.step(13)
        assert b.info()["launches_per_step"] <= widths
        for i, (p, ic) in enumerate(jobs):
            want, st = alone(p, ic, 25)
            assert np.array_equal(b.get_field(i), want), i
            assert b.reduce(i)["step"] == 25
    finally:
        b.close()


def test_batch_fp64_job_matches_oracle(oracle):
    p = mb.make_params(64, 32, 24, 0.005, kappa=1.3)
    q = mb.make_params(96, 96, 1, 0.01)
    ic0 = oracle.ic((64, 32, 24), 0.1, 0.2, False, 1)
    ic1 = oracle.ic((96, 96, 1), -0.2, 0.2, False, 2)
    b = mb.Batch([p, q])
    try:
        b.set_field(0, ic0)
        b.set_field(1, ic1)
        b.step(25)
        assert np.array_equal(b.get_field(0), oracle.run(ic0, (64, 32, 24), (1, 1, 1), 0.005, 1.0, 1.3, 25))
        assert np.array_equal(b.get_field(1), oracle.run(ic1, (96, 96, 1), (1, 1, 1), 0.01, 1.0, 1.0, 25))
    finally:
        b.close()


def test_server_results_identical_alone_and_mixed():
    jobs = job_set(seed=11, n=12)
    steps = [40 + 17 * i for i in range(len(jobs))]
    srv = mb.Server(hbm_budget_gb=4.0, max_jobs=64, steps_per_tick=25)
    try:
        ids = []
        for (p, ic), n in zip(jobs, steps):
            ids.append(srv.submit(p, ic, n))
            time.sleep(0.002)  # arrivals while others are on the GPU
        for (p, ic), n, jid in zip(jobs, steps, ids):
            got, st = srv.result(jid, p, timeout_us=120_000_000)
            want, wst = alone(p, ic, n)
            assert np.array_equal(got, want), jid
            assert st["step"] == n
        s = srv.stats()
        assert s["completed"] == len(jobs) and s["failed"] == 0
        assert s["p99_ms"] >= s["p50_ms"] > 0
    finally:
        srv.close()


def test_server_absorbs_job_set_changes_without_recapture():
    """A stream of 3-D FP32 jobs of march widths: after the first ticks set
    up the launch lanes, admissions and retirements rewrite the lanes'
    device tables instead of recapturing the step graph, and every result
    is still bit-identical to its standalone run."""
    rng = np.random.default_rng(5)
    jobs = []
    for j in range(14):
        e = int(rng.choice([64, 96, 128]))
        p = mb.make_params(e, e, e, 0.005, kappa=float(rng.uniform(0.5, 2.0)), precision="fp32")
        jobs.append((p, mb.ic_generate((e, e, e), float(rng.uniform(-0.4, 0.4)), 0.05, False, 3000 + j),
                     int(rng.integers(30, 90))))
    srv = mb.Server(hbm_budget_gb=8.0, max_jobs=64, steps_per_tick=10)
    try:
        ids = []
        for p, ic, n in jobs:
            ids.append(srv.submit(p, ic, n))
            time.sleep(0.003)
        for (p, ic, n), jid in zip(jobs, ids):
            got, st = srv.result(jid, p, timeout_us=120_000_000)
            want, _ = alone(p, ic, n)
            assert np.array_equal(got, want), jid
        s = srv.stats()
        assert s["completed"] == len(jobs) and s["failed"] == 0
        assert s["refreshes"] > 0
        assert s["rebuilds"] < s["ticks"]
    finally:
        srv.close()


def test_server_with_few_slots_recycles_them_and_keeps_results():
    """More jobs than slots, submitted at once: jobs wait in the queue, each
    tick admits the next ones beside the running steps, and a retired job's
    slot is reused only after the next rebuild.  Every result is still
    bit-identical to its standalone run, and the saturated rate and the
    device time of the ticks are reported."""
    jobs = job_set(seed=23, n=10)
    steps = [30 + 11 * i for i in range(len(jobs))]
    srv = mb.Server(hbm_budget_gb=4.0, max_jobs=3, steps_per_tick=20)
    try:
        ids = [srv.submit(p, ic, n) for (p, ic), n in zip(jobs, steps)]
        for (p, ic), n, jid in zip(jobs, steps, ids):
            got, st = srv.result(jid, p, timeout_us=120_000_000)
            want, _ = alone(p, ic, n)
            assert np.array_equal(got, want), jid
            assert st["step"] == n
        s = srv.stats()
        assert s["completed"] == len(jobs) and s["failed"] == 0
        assert s["sat_ticks"] > 0 and s["sat_site_updates_per_s"] > 0
        assert 0 < s["gpu_s"] <= s["step_s"] + 1e-3
    finally:
        srv.close()


def test_server_admission_respects_budget():
    # budget fits two 128^3 FP64 jobs (2 x 2 x 16.8 MB) but not three
    p = mb.make_params(128, 128, 128, 0.005)
    ic = mb.ic_generate((128, 128, 128), 0.0, 0.1, False, 3)
    srv = mb.Server(hbm_budget_gb=0.075, max_jobs=8, steps_per_tick=10)
    try:
        ids = [srv.submit(p, ic, 200) for _ in range(4)]
        peak_running = 0
        t0 = time.time()
        while time.time() - t0 < 60:
            st = srv.stats()
            peak_running = max(peak_running, st["running"])
            if st["completed"] == 4:
                break
            time.sleep(0.001)
        for jid in ids:
            srv.result(jid, p, timeout_us=60_000_000, want_field=False)
        st = srv.stats()
        assert st["hbm_peak_gb"] <= 0.075
        assert peak_running <= 2
    finally:
        srv.close()


def test_server_rejects_job_over_budget():
    srv = mb.Server(hbm_budget_gb=0.01, max_jobs=4)
    try:
        p = mb.make_params(256, 256, 256, 0.005)
        with pytest.raises(mb.MGError) as e:
            srv.submit(p, np.zeros((256, 256, 256)), 10)
        assert e.value.code == mb._lib.MG_ENOMEM
    finally:
        srv.close()
