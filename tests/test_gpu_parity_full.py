"""FP64 parity at the benchmark sizes, against the reference CPU build itself
(oracle/_ref/chref_bench: the reference's own PFApp step loop and SfieldFD
operators with the CHBasic model, one MPI-shim rank per host core).

* 3-D 256^3, dt 0.005, M 1, kappa 1, periodic, c0 = 0 + U[-0.05, 0.05] from
  seed 42, 100 steps: the drop-in configuration the headline is quoted on.
* 3-D 512^3, c0 = 0.3 + N(0, 0.02^2) from seed 42, kappa 1.5, dt 0.005,
  10 steps: the start of the precision study, whose FP64 path is the FP64
  reference for the FP32 field there.

Both must be bit-identical (which is within the 1e-12 relative max-norm the
drop-in is held to)."""
import os
import tempfile

import numpy as np
import pytest

import mesobasic_b200 as mb


def host_ranks(nx):
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    r = max(1, min(cores, 32))
    while nx % r:
        r -= 1
    return r


def compare(oracle, dims, dt, kap, co, amp, gaussian, seed, nsteps):
    if not oracle.ref_available() or not os.path.exists(oracle.REF_BENCH):
        pytest.skip("reference CPU build not present (make -C oracle ref)")
    with tempfile.TemporaryDirectory() as work:
        want, rec = oracle.ref_bench_field(dims, dt, 1.0, kap, co, amp, gaussian, seed, nsteps,
                                           host_ranks(dims[0]), work)
    ic = mb.ic_generate(dims, co, amp, gaussian, seed)
    with mb.CHSim(mb.make_params(*dims, dt, kappa=kap, M=1.0), 0) as sim:
        assert sim.tiling.path == 0, "tiled kernel not selected"
        sim.set_field(ic)
        del ic
        sim.step(nsteps)
        got = sim.get_field()
    err = float(np.max(np.abs(got - want))) / float(np.max(np.abs(want)))
    assert err <= 1e-12, f"relative max-norm {err:.3e} after {nsteps} steps"
    assert np.array_equal(got, want), f"not bit-identical (relative max-norm {err:.3e})"
    return rec


@pytest.mark.gpu
def test_c2_256_fp64_100_steps_bit_identical_to_reference_build(oracle):
    compare(oracle, (256, 256, 256), 0.005, 1.0, 0.0, 0.1, False, 42, 100)


@pytest.mark.gpu
def test_c3_512_fp64_start_bit_identical_to_reference_build(oracle):
    compare(oracle, (512, 512, 512), 0.005, 1.5, 0.3, 0.02, True, 42, 10)
