"""Shared test setup: the `gpu` marker, paths, and fixtures that load the
golden vectors and the oracles (oracle/)."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    if not os.path.exists(O.ORACLE_SO):
        O.build(reference=False)
    return O


def golden_cases():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        idx = json.load(f)
    return sorted(k for k in idx if k.startswith("ch"))


def load_golden(name):
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    meta = json.loads(str(d["meta"]))
    return meta, {k: d[k] for k in d.files if k != "meta"}
