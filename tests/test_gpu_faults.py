"""Failure detection on the GPU without a GPU fault: a bounded device wait
is made to run out (its barrier expects bytes that never arrive) and the
kernel reports the error status that the host reads; the context stays
usable."""
import numpy as np
import pytest

import mesobasic_b200 as mb

pytestmark = pytest.mark.gpu


def test_bounded_tma_wait_reports_error_and_context_survives(monkeypatch, oracle):
    dims = (64, 16, 8)
    ic = oracle.ic(dims, 0.0, 0.2, False, 1)
    monkeypatch.setenv("MG_SPIN_LIMIT", "20000")
    monkeypatch.setenv("MG_FAULT_TX_EXTRA", "16")
    with mb.CHSim(mb.make_params(*dims, 0.005)) as sim:
        sim.set_field(ic)
        sim.step(1)
        with pytest.raises(mb.MGError) as e:
            sim.sync(timeout_us=60_000_000)
        assert e.value.code == mb._lib.MG_EDEVICE
        assert sim.steps == 0  # the step did not complete
        # copies may have been in flight when the kernel gave up: the handle
        # refuses further steps instead of stepping untrusted state
        with pytest.raises(mb.MGError) as e2:
            sim.step(1)
        assert e2.value.code == mb._lib.MG_EDEVICE
    monkeypatch.delenv("MG_FAULT_TX_EXTRA")
    monkeypatch.delenv("MG_SPIN_LIMIT")
    # same process, same device: a fresh handle works and is exact
    with mb.CHSim(mb.make_params(*dims, 0.005)) as sim:
        sim.set_field(ic)
        sim.step(5)
        assert np.array_equal(sim.get_field(), oracle.run(ic, dims, (1, 1, 1), 0.005, 1.0, 1.0, 5))
