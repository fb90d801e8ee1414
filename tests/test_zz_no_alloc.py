"""mg_field_stats_noalloc (the diagnostics reduction with static device
scratch, no allocation) against mg_ch_reduce, through the C ABI.

Collected last on purpose: it must give the same answers in a fresh process
and after every other GPU test has run in the same process."""
import ctypes

import numpy as np
import pytest

import mesobasic_b200 as mb
from mesobasic_b200 import _lib

pytestmark = pytest.mark.gpu

TIMEOUT_US = 30_000_000


def noalloc_stats(L, field_dev, params, stream):
    st = _lib.Stats()
    rc = L.mg_field_stats_noalloc(field_dev, ctypes.byref(params), 0, stream, TIMEOUT_US, ctypes.byref(st))
    return rc, st.as_dict()


def handle_stats(L, h):
    st = _lib.Stats()
    _lib.check(L.mg_ch_reduce(h, ctypes.byref(st)))
    return st.as_dict()


def assert_close(got, want):
    scale = max(want["abs_mass"], 1.0)
    assert abs(got["mass"] - want["mass"]) <= 1e-12 * scale, (got, want)
    assert abs(got["abs_mass"] - want["abs_mass"]) <= 1e-12 * scale, (got, want)
    assert abs(got["energy"] - want["energy"]) <= 1e-12 * max(abs(want["energy"]), 1.0), (got, want)
    assert got["max_abs"] == want["max_abs"]
    assert got["nonfinite"] == want["nonfinite"] == 0


CASES = [
    ((64, 48, 40), "fp64", (1, 1, 1), (1.0, 1.0, 1.0)),
    ((96, 64, 32), "fp32", (1, 1, 1), (1.0, 1.0, 1.0)),
    ((128, 96, 1), "fp64", (1, 1, 1), (1.0, 1.0, 1.0)),
    ((40, 24, 16), "fp64", (0, 0, 0), (1.0, 0.5, 2.0)),
    ((64, 40, 1), "fp32", (0, 1, 1), (0.5, 0.5, 1.0)),
]


@pytest.mark.parametrize("dims,prec,bc,sp", CASES)
def test_noalloc_matches_reduce(dims, prec, bc, sp):
    L = _lib.load()
    p = mb.make_params(*dims, 0.001, kappa=1.3, dx=sp[0], dy=sp[1], dz=sp[2], bc=bc, precision=prec)
    ic = mb.ic_generate(dims, 0.1, 0.4, False, 7)
    h = ctypes.c_void_p()
    _lib.check(L.mg_ch_create(ctypes.byref(p), 0, ctypes.byref(h)))
    try:
        _lib.check(L.mg_ch_set_field(h, ic.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        _lib.check(L.mg_ch_step(h, 20))
        want = handle_stats(L, h)  # also waits for the steps
        dev, stream = L.mg_ch_field_device(h), L.mg_ch_stream(h)
        rc1, first = noalloc_stats(L, dev, p, stream)
        rc2, second = noalloc_stats(L, dev, p, stream)
        assert rc1 == rc2 == _lib.MG_OK, L.mg_last_error()
        assert first["step"] == second["step"] == -1
        assert_close(first, want)
        assert first == second  # fixed reduction order: identical on repeat
    finally:
        L.mg_ch_destroy(h)


def test_noalloc_rejects_too_many_planes():
    """The size check runs on the host before any device work."""
    L = _lib.load()
    dims = (32, 16, 8)
    p = mb.make_params(*dims, 0.001)
    h = ctypes.c_void_p()
    _lib.check(L.mg_ch_create(ctypes.byref(p), 0, ctypes.byref(h)))
    try:
        big = mb.make_params(8, 8, 5000, 0.001)
        rc, _ = noalloc_stats(L, L.mg_ch_field_device(h), big, L.mg_ch_stream(h))
        assert rc == _lib.MG_EINVAL
        assert b"at most 4096" in L.mg_last_error()
        # a valid call on the same thread still works afterwards
        ic = np.zeros(int(np.prod(dims)))
        _lib.check(L.mg_ch_set_field(h, ic.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        _lib.check(L.mg_ch_sync(h, TIMEOUT_US))
        rc, st = noalloc_stats(L, L.mg_ch_field_device(h), p, L.mg_ch_stream(h))
        assert rc == _lib.MG_OK and st["mass"] == 0.0 and st["max_abs"] == 0.0
    finally:
        L.mg_ch_destroy(h)


def test_noalloc_counts_nonfinite_sites_like_reduce():
    """NaN and Inf sites: both calls return MG_ENONFINITE with the same count."""
    L = _lib.load()
    dims = (24, 16, 8)
    p = mb.make_params(*dims, 0.001)
    ic = mb.ic_generate(dims, 0.0, 0.2, False, 3).reshape(-1).copy()
    ic[[5, 77, 1000]] = np.nan
    ic[2000] = np.inf
    ic[2001] = -np.inf
    h = ctypes.c_void_p()
    _lib.check(L.mg_ch_create(ctypes.byref(p), 0, ctypes.byref(h)))
    try:
        _lib.check(L.mg_ch_set_field(h, ic.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        st = _lib.Stats()
        assert L.mg_ch_reduce(h, ctypes.byref(st)) == _lib.MG_ENONFINITE
        want = st.as_dict()
        for _ in range(2):
            rc, got = noalloc_stats(L, L.mg_ch_field_device(h), p, L.mg_ch_stream(h))
            assert rc == _lib.MG_ENONFINITE, L.mg_last_error()
            assert got["nonfinite"] == want["nonfinite"] == 5
    finally:
        L.mg_ch_destroy(h)
