"""The drop-in plugin run by the reference's own driver.

oracle/_ref/meso_ref_gpu is the reference's main -> MesoExecute -> PFApp
(src/base/main.cpp, src/base/MesoExecute.cpp:107-152,
src/phase_field/PFApp.cpp:10-121) with mesobasic_b200/plugin/CHBasicGPU.hpp
registered in PFBaseClass::PFFactory as a maintainer would add it, linked
against libmesogpu.so.  With PFApp/type = CHBasicGPU the reference driver
steps on the GPU; its vtkoutput/ must be byte-identical to the same driver's
CPU run with the CHBasic oracle model (oracle/_ref/meso_ref)."""
import os
import subprocess

import pytest

INPUT = """[Domain]
nx = {nx}
ny = {ny}
nz = {nz}
dx = 1.0
dy = 1.0
dz = 1.0
[]
[Time]
nstep = {nstep}
dt = {dt}
[]
[Output]
numOutputs = {nout}
[]
[PFApp]
app = true
type = {type}
co = 0.05
M = 1.0
kap = 1.0
noise_amp = 0.2
seed = 7
bx = {bx}
[]
"""


def run(binary, cwd, text):
    (cwd / "input.dat").write_text(text)
    r = subprocess.run([binary], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-1500:] + r.stderr[-1500:]
    out = cwd / "vtkoutput"
    return {n: (out / n).read_bytes() for n in sorted(os.listdir(out))}


@pytest.mark.gpu
@pytest.mark.parametrize("dims,bx", [((32, 24, 16), 1), ((48, 40, 1), 1), ((24, 20, 12), 0)])
def test_reference_driver_steps_on_gpu_byte_identical(tmp_path, oracle, dims, bx):
    if not os.path.exists(oracle.REF_MESO) or not os.path.exists(oracle.REF_MESO_GPU):
        pytest.skip("reference driver builds not present (make -C oracle ref ref-gpu)")
    nx, ny, nz = dims
    kw = dict(nx=nx, ny=ny, nz=nz, nstep=40, dt=0.005 if nz > 1 else 0.01, nout=4, bx=bx)
    (tmp_path / "cpu").mkdir()
    (tmp_path / "gpu").mkdir()
    want = run(oracle.REF_MESO, tmp_path / "cpu", INPUT.format(type="CHBasic", **kw))
    got = run(oracle.REF_MESO_GPU, tmp_path / "gpu", INPUT.format(type="CHBasicGPU", **kw))
    assert list(got) == list(want) == [f"c_{s}.vtk" for s in sorted((0, 10, 20, 30, 40), key=str)]
    for name in want:
        assert got[name] == want[name], name
