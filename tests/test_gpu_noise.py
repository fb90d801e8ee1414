"""The per-step noise term (TIPSphil.cpp:200-209 with a counter-based
generator): exact against the oracle's restatement, the right distribution,
and the same result alone, batched and served."""
import numpy as np
import pytest

import mesobasic_b200 as mb

pytestmark = pytest.mark.gpu

SEED = 0x1234_5678_9ABC


def test_first_step_noise_exact(oracle):
    dims, c0, dt, noise = (21, 5, 3), 0.2, 0.01, 0.7  # 315 sites: a partial last draw
    n = int(np.prod(dims))
    for prec in ("fp64", "fp32"):
        with mb.CHSim(mb.make_params(*dims, dt, precision=prec, mass_correct=0, noise=noise, noise_seed=SEED)) as sim:
            sim.set_field(np.full(dims[::-1], c0))
            sim.step(1)  # a constant field does not change: only the noise
            got = sim.get_field().reshape(-1)
        inc = oracle.noise_increments(n, 1, SEED, noise, dt)
        if prec == "fp64":
            assert np.array_equal(got, c0 + inc)
        else:
            want = (np.float32(c0) + inc.astype(np.float32)).astype(np.float64)
            assert np.array_equal(got, want)


def test_fp64_steps_with_noise_bit_identical(oracle):
    dims, dt, noise = (24, 20, 16), 0.005, 0.3
    n = int(np.prod(dims))
    ic = oracle.ic(dims, 0.0, 0.2, False, 4)
    want = ic.copy()
    for s in range(1, 4):
        want = oracle.run(want, dims, (1.0, 1.0, 1.0), dt, 1.0, 1.0, 1)
        want = want + oracle.noise_increments(n, s, SEED, noise, dt).reshape(want.shape)
    with mb.CHSim(mb.make_params(*dims, dt, noise=noise, noise_seed=SEED)) as sim:
        sim.set_field(ic)
        sim.step(3)
        got = sim.get_field()
    assert np.array_equal(got, want), np.abs(got - want).max()


def test_noise_distribution():
    dims, c0, dt, noise = (256, 64, 64), -0.1, 0.01, 2.0
    with mb.CHSim(mb.make_params(*dims, dt, noise=noise, noise_seed=7)) as sim:
        sim.set_field(np.full(dims[::-1], c0))
        sim.step(1)
        r = (sim.get_field().reshape(-1) - c0) / (dt * noise)
    n = r.size
    assert r.min() > -0.5 and r.max() < 0.5
    assert abs(r.mean()) < 5 / np.sqrt(12 * n)
    assert abs(r.var() - 1 / 12) < 0.002
    hist, _ = np.histogram(r, bins=16, range=(-0.5, 0.5))
    assert np.all(np.abs(hist / (n / 16) - 1) < 0.02)


def jobs():
    out = []
    for k, (dims, prec) in enumerate([((64, 32, 16), "fp32"), ((32, 32, 1), "fp64"), ((48, 24, 20), "fp64")]):
        p = mb.make_params(*dims, 0.005, precision=prec, noise=0.5, noise_seed=100 + k)
        out.append((p, dims, mb.ic_generate(dims, 0.1 * k, 0.2, False, 9 + k)))
    return out


def alone(p, ic, nsteps):
    with mb.CHSim(p) as sim:
        sim.set_field(ic)
        sim.step(nsteps)
        return sim.get_field()


def test_batch_with_noise_equals_standalone():
    js = jobs()
    b = mb.Batch([p for p, _, _ in js])
    try:
        for i, (_, _, ic) in enumerate(js):
            b.set_field(i, ic)
        b.step(12)
        for i, (p, _, ic) in enumerate(js):
            assert np.array_equal(b.get_field(i), alone(p, ic, 12)), i
    finally:
        b.close()


def test_server_with_noise_equals_standalone():
    """Jobs end inside a tick: their later, skipped steps add no noise."""
    js = jobs()
    with_steps = [7, 23, 41]
    srv = mb.Server(0, hbm_budget_gb=10.0, max_jobs=8, steps_per_tick=16)
    try:
        ids = [srv.submit(p, ic, n) for (p, _, ic), n in zip(js, with_steps)]
        for jid, (p, _, ic), n in zip(ids, js, with_steps):
            got, _ = srv.result(jid, p, timeout_us=120_000_000)
            assert np.array_equal(got, alone(p, ic, n)), n
    finally:
        srv.close()
