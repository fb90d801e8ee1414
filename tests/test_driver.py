"""The C++ driver meso_b200 (reference input file -> CHBasicGPU plugin ->
VTK output).  CPU tests cover the input-file rules and the error exits that
happen before any device work; GPU tests compare its VTK output byte for
byte with files the reference driver wrote (tests/golden/vtk_ref) and its raw
dumps bit for bit with the oracle."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "mesobasic_b200", "meso_b200")


def driver():
    if not os.path.exists(DRIVER):
        from mesobasic_b200 import build
        build.build()
    assert os.path.exists(DRIVER), "meso_b200 was not built"
    return DRIVER


def params(tmp_path, text, *args):
    (tmp_path / "input.dat").write_text(text)
    r = subprocess.run([driver(), "--print-params", *args], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout)


def test_input_file_rules(tmp_path):
    text = """# leading comment
[Domain]
    nx = 32      # trailing comment
    ny=16
    nz =8
    dx= 0.5
    nx = 64      # redefined: the later value wins
[./Sub]
    key = 'two words'
[../]
    dz = 2.0e0
[]
[Time]
    nstep = 2.0e1
    dt = 1e-3
[]
[PFApp]
    app = true
    kap = notanumber
[]
"""
    d = params(tmp_path, text, "Time/dt=0.002")
    v, r = d["variables"], d["resolved"]
    assert d["sections"] == ["Domain/", "Domain/Sub/", "Time/", "PFApp/"]
    assert v["Domain/nx"] == "64" and r["nx"] == 64
    assert r["ny"] == 16 and r["nz"] == 8 and r["dx"] == 0.5 and r["dz"] == 2.0
    assert v["Domain/Sub/key"] == "two words"
    assert r["nstep"] == 20  # ints are read through a double
    assert r["dt"] == 0.002  # command line overrides the file
    assert r["kap"] == 1.0   # unreadable number: the default
    assert r["type"] == "CHBasic" and r["precision"] == "fp64"


def run_driver(tmp_path, text, *args, timeout=300):
    (tmp_path / "input.dat").write_text(text)
    return subprocess.run([driver(), *args], cwd=tmp_path, capture_output=True, text=True, timeout=timeout)


def test_unknown_model_type_fails_loudly(tmp_path):
    # CHTernary: a type the reference's factory has commented out
    r = run_driver(tmp_path, "[Domain]\nnx=8\n[]\n[PFApp]\napp = true\ntype = CHTernary\n[]\n")
    assert r.returncode == 1 and "CHTernary" in r.stderr and "SIPSternary" in r.stderr


def test_more_outputs_than_steps_is_an_error(tmp_path):
    r = run_driver(tmp_path, "[Time]\nnstep=2\n[]\n[Output]\nnumOutputs=5\n[]\n[PFApp]\napp=true\n[]\n")
    assert r.returncode == 1 and "numOutputs" in r.stderr


@pytest.mark.gpu
def test_vtk_output_byte_identical_to_reference_driver(tmp_path):
    src = os.path.join(GOLDEN, "vtk_ref")
    (tmp_path / "vtkoutput").mkdir()
    (tmp_path / "vtkoutput" / "stale.vtk").write_text("old")
    r = run_driver(tmp_path, open(os.path.join(src, "input.dat")).read())
    assert r.returncode == 0, r.stderr
    got = sorted(os.listdir(tmp_path / "vtkoutput"))
    assert got == ["c_0.vtk", "c_2.vtk", "c_4.vtk"]  # stale file removed
    for name in got:
        assert (tmp_path / "vtkoutput" / name).read_bytes() == open(os.path.join(src, name), "rb").read(), name


def read_dump(path):
    raw = open(path, "rb").read()
    hdr = np.frombuffer(raw[:20], dtype=np.int32)
    nx, ny, nz = (int(v) for v in hdr[1:4])
    return hdr, np.frombuffer(raw[20:], dtype=np.float64).reshape(nz, ny, nx)


@pytest.mark.gpu
@pytest.mark.parametrize("dims,bc", [((24, 20, 16), (1, 1, 1)), ((32, 24, 1), (1, 0, 1))])
def test_raw_dump_bit_identical_to_oracle(tmp_path, oracle, dims, bc):
    nx, ny, nz = dims
    text = f"""[Domain]
nx = {nx}
ny = {ny}
nz = {nz}
[]
[Time]
nstep = 30
dt = 0.005
[]
[Output]
numOutputs = 3
[]
[PFApp]
app = true
type = CHBasicGPU
co = 0.05
noise_amp = 0.3
seed = 9
bx = {bc[0]}
by = {bc[1]}
bz = {bc[2]}
vtk = 0
dump_prefix = dump
[]
"""
    r = run_driver(tmp_path, text)
    assert r.returncode == 0, r.stderr
    ic = oracle.ic(dims, 0.05, 0.3, False, 9)
    for step in (0, 10, 20, 30):
        hdr, got = read_dump(tmp_path / f"dump_{step}.rank0")
        assert list(hdr) == [0, nx, ny, nz, step]
        want = ic if step == 0 else oracle.run(ic, dims, (1.0, 1.0, 1.0), 0.005, 1.0, 1.0, step, bc=bc)
        assert np.array_equal(got, want), (step, np.abs(got - want).max())


@pytest.mark.gpu
def test_fp32_run_writes_output_within_tolerance(tmp_path, oracle):
    dims = (64, 32, 16)
    text = """[Domain]
nx = 64
ny = 32
nz = 16
[]
[Time]
nstep = 100
dt = 0.005
[]
[Output]
numOutputs = 1
[]
[PFApp]
app = true
precision = fp32
noise_amp = 0.2
vtk = 0
dump_prefix = d
[]
"""
    r = run_driver(tmp_path, text, "--timing")
    assert r.returncode == 0, r.stderr
    t = json.loads(r.stdout.strip().splitlines()[-1])
    assert t["steps"] == 100 and t["site_updates_per_s"] > 0
    ic = oracle.ic(dims, 0.0, 0.2, False, 42)
    want = oracle.run(ic, dims, (1.0, 1.0, 1.0), 0.005, 1.0, 1.0, 100)
    _, got = read_dump(tmp_path / "d_100.rank0")
    assert np.abs(got - want).max() <= 1e-4
