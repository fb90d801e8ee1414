"""The C-ABI boundary without a GPU: the library loads, exports every
function include/*.h declares, rejects bad arguments before touching a
device, and its host-side helpers (seeded IC, VTK writer) match the
reference."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

import mesobasic_b200 as mb
from mesobasic_b200 import _lib


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(mg_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_function():
    lib = mb.load()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the whole header too
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


@pytest.mark.parametrize("bad", [
    dict(nx=0), dict(dx=0.0), dict(dt=float("nan")), dict(bx=2), dict(precision=5),
    dict(precision=0, mass_correct=1),
])
def test_create_rejects_bad_params_before_device_work(bad):
    kw = dict(nx=8, ny=8, nz=8, dx=1.0, dy=1.0, dz=1.0, dt=0.01, M=1.0, kappa=1.0, bx=1, by=1, bz=1,
              precision=0, mass_correct=0)
    kw.update(bad)
    p = _lib.Params(**kw)
    h = ctypes.c_void_p()
    rc = mb.load().mg_ch_create(ctypes.byref(p), 0, ctypes.byref(h))
    assert rc == _lib.MG_EINVAL
    assert mb.load().mg_last_error()
    assert not h.value


@pytest.mark.parametrize("bad", [dict(chiPN=0.034), dict(N=float("nan")), dict(Mvolume=0.0), dict(prec="fp32"),
                                 dict(nx=0)])
def test_sips_create_rejects_bad_params_before_device_work(bad):
    bad = dict(bad)
    p = mb.make_params(bad.pop("nx", 8), 8, 8, 0.01, precision=bad.pop("prec", "fp64"))
    sp = mb.make_sips_params(**bad)
    h = ctypes.c_void_p()
    assert mb.load().mg_sips_create(ctypes.byref(p), ctypes.byref(sp), 0, ctypes.byref(h)) == _lib.MG_EINVAL
    assert not h.value


@pytest.mark.parametrize("bad", [dict(Kpp=float("inf")), dict(Mnn=float("nan")), dict(prec="fp32"), dict(nx=-1)])
def test_ternary_create_rejects_bad_params_before_device_work(bad):
    bad = dict(bad)
    p = mb.make_params(bad.pop("nx", 8), 8, 8, 0.01, precision=bad.pop("prec", "fp64"))
    v = dict(mb.TERNARY_DEFAULTS, **bad)
    tp = _lib.TernaryParams(*(v[k] for k in mb.TERNARY_DEFAULTS))
    h = ctypes.c_void_p()
    assert mb.load().mg_ternary_create(ctypes.byref(p), ctypes.byref(tp), 0, ctypes.byref(h)) == _lib.MG_EINVAL
    assert not h.value
    with pytest.raises(ValueError):
        mb.make_sips_params(chi=1.0)


def test_batch_rejects_bad_job():
    good = mb.make_params(8, 8, 8, 0.01)
    bad = mb.make_params(8, 0, 8, 0.01)
    arr = (_lib.Params * 2)(good, bad)
    h = ctypes.c_void_p()
    rc = mb.load().mg_batch_create(arr, 2, 0, ctypes.byref(h))
    assert rc == _lib.MG_EINVAL and b"job 1" in mb.load().mg_last_error()


def test_ic_generate_matches_oracle_and_reference(oracle):
    from conftest import load_golden
    for name in ("ch3d_24x20x16", "ch3d_gauss_32x16x8", "ch2d_64x48"):
        meta, arr = load_golden(name)
        ic = mb.ic_generate(tuple(meta["dims"]), meta["co"], meta["amp"], meta["gaussian"], meta["seed"])
        assert np.array_equal(ic, arr["ic"])
    dims = (33, 7, 5)
    assert np.array_equal(mb.ic_generate(dims, 0.3, 0.02, True, 123), oracle.ic(dims, 0.3, 0.02, True, 123))


def test_vtk_writer_byte_identical_to_reference(tmp_path, oracle):
    dims = (8, 6, 4)
    ic = mb.ic_generate(dims, 0.1, 0.2, False, 5)
    c2 = oracle.run(ic, dims, (1, 1, 1), 0.01, 1.0, 1.0, 2)
    for name, field, reps in (("c_0.vtk", ic, 2), ("c_2.vtk", c2, 1)):
        p = tmp_path / name
        for _ in range(reps):
            mb.vtk_write(p, "c", field, dims, 2, 1, 1)
        assert p.read_bytes() == (GOLDEN and open(os.path.join(GOLDEN, "vtk_ref", name), "rb").read())


def test_vtk_writer_skips_and_negative_zero(tmp_path, oracle):
    dims = (9, 7, 5)
    c = oracle.ic(dims, 0.0, 0.002, False, 3)  # many values round to -0.000 / 0.000
    p = tmp_path / "v.vtk"
    mb.vtk_write(p, "phi", c, dims, 3, 2, 2)
    assert p.read_text() == oracle.vtk_text(c, dims, "phi", 3, 2, 2)


def test_noalloc_rejects_tall_2d_field_on_the_host():
    """A 2-D field (nz == 1) with more than 4096 rows is refused before any
    device work, and the message names the ny limit (no GPU needed: the
    pointer is never touched)."""
    import ctypes
    import mesobasic_b200 as mb
    from mesobasic_b200 import _lib
    L = _lib.load()
    p = mb.make_params(64, 5000, 1, 0.01)
    st = _lib.Stats()
    rc = L.mg_field_stats_noalloc(ctypes.c_void_p(256), ctypes.byref(p), 0, None, 1000, ctypes.byref(st))
    assert rc == _lib.MG_EINVAL
    msg = L.mg_last_error()
    assert b"5000 planes" in msg and b"ny of a 2-D field" in msg and b"at most 4096" in msg


def test_create_returns_a_status_without_crashing():
    """mg_ch_create / mg_batch_create build an engine on the host before any
    device call: on a machine without a GPU they return MG_ECUDA or MG_EINVAL
    (with a GPU, MG_OK), never crash.  Guards against objects built against
    different layouts of the engine's classes."""
    import ctypes
    import mesobasic_b200 as mb
    from mesobasic_b200 import _lib
    L = _lib.load()
    p = mb.make_params(32, 16, 8, 0.005)
    h = ctypes.c_void_p()
    rc = L.mg_ch_create(ctypes.byref(p), 0, ctypes.byref(h))
    assert rc in (_lib.MG_OK, _lib.MG_ECUDA, _lib.MG_EINVAL), rc
    if rc == _lib.MG_OK:
        L.mg_ch_destroy(h)
    arr = (_lib.Params * 2)(p, mb.make_params(64, 64, 64, 0.005, precision="fp32"))
    b = ctypes.c_void_p()
    rc = L.mg_batch_create(arr, 2, 0, ctypes.byref(b))
    assert rc in (_lib.MG_OK, _lib.MG_ECUDA, _lib.MG_EINVAL), rc
    if rc == _lib.MG_OK:
        L.mg_batch_destroy(b)
