"""The variable-mobility (TIPSphil) step against the reference's own
TIPSphil::updatePhaseField run on the same field (oracle.fh_ref_run, noise
off).  FP64; log, exp and pow differ from the host's libm by an ulp or two,
so the bar is a relative max-norm of 1e-12 rather than bit identity."""
import os
import subprocess

import numpy as np
import pytest

import mesobasic_b200 as mb

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# a quench that phase-separates: chi = alpha/T + beta crosses the spinodal
QUENCH = dict(alpha=150.0, beta=0.1, N=50.0, A=1.0, Tinit=300.0, Tbath=280.0, Tcrystal=200.0, nu=1.0,
              gamma=1.0, D0=1.0, Mweight=0.5, Mvolume=1.0)


def gpu_run(dims, fh, nstep_total, ic, nsteps, dt=0.01, kap=1.0, spacing=(1.0, 1.0, 1.0), bc=(1, 1, 1)):
    p = mb.make_params(*dims, dt, kappa=kap, dx=spacing[0], dy=spacing[1], dz=spacing[2], bc=bc)
    with mb.CHSim(p, fh=mb.make_fh_params(nstep_total, **fh)) as sim:
        sim.set_field(ic)
        sim.step(nsteps)
        return sim.get_field(), sim.mobility()


def rel_err(got, want):
    return np.abs(got - want).max() / np.abs(want).max()


CASES = [
    ("3d periodic", (24, 20, 16), QUENCH, (1.0, 1.0, 1.0), (1, 1, 1), 0.3, 0.1),
    ("3d no-flux, unequal spacing", (20, 12, 10), QUENCH, (1.0, 1.25, 1.5), (0, 0, 1), 0.35, 0.1),
    ("2d mixed boundaries", (48, 36, 1), QUENCH, (1.0, 1.0, 1.0), (1, 0, 1), 0.3, 0.1),
    # values below 0 (the sqrt branch of mu, the lower-limit mobility), the
    # crystallisation factor (T <= Tcrystal) and the D0 clamps
    ("branches", (16, 16, 8), dict(QUENCH, Tcrystal=290.0, D0=0.5), (1.0, 1.0, 1.0), (1, 1, 1), 0.02, 0.1),
]


@pytest.mark.parametrize("name,dims,fh,spacing,bc,co,amp", CASES, ids=[c[0] for c in CASES])
def test_matches_reference_tipsphil(oracle, name, dims, fh, spacing, bc, co, amp):
    ic = oracle.ic(dims, co, amp, False, 21)
    want = oracle.fh_ref_run(ic, dims, dict(fh, kap=1.0), 50, 1, 10, spacing=spacing, dt=0.01, bc=bc)
    got, mob = gpu_run(dims, fh, 50, ic, 10, spacing=spacing, bc=bc)
    assert rel_err(got, want) <= 1e-12, rel_err(got, want)
    assert np.all(mob > 0) and np.all(mob <= fh["D0"])
    assert np.abs(got - ic).max() > 1e-4  # the model moved the field


def test_reference_defaults_run(oracle):
    """The reference's defaults (D0 = 1e-7: the mobility sits at its clamps)."""
    dims = (16, 12, 8)
    ic = oracle.ic(dims, 0.5, 0.1, False, 2)
    want = oracle.fh_ref_run(ic, dims, {}, 20, 1, 5)
    got, mob = gpu_run(dims, {}, 20, ic, 5)
    assert rel_err(got, want) <= 1e-12
    assert np.allclose(mob, 1e-7 * 0.001, rtol=0, atol=1e-20) or np.allclose(mob, 1e-7, rtol=1e-15)


def test_rejects_fp32_and_bad_parameters():
    with pytest.raises(mb.MGError):
        mb.CHSim(mb.make_params(16, 8, 8, 0.01, precision="fp32"), fh=mb.make_fh_params(10))
    with pytest.raises(mb.MGError):
        mb.CHSim(mb.make_params(16, 8, 8, 0.01), fh=mb.make_fh_params(0))


def test_driver_runs_tipsphil(tmp_path):
    text = """[Domain]
nx = 32
ny = 24
nz = 16
[]
[Time]
nstep = 40
dt = 0.01
[]
[Output]
numOutputs = 2
[]
[PFApp]
app = true
type = TIPSphil
co = 0.3
alpha = 150
beta = 0.1
N = 50
Tinit = 300
Tbath = 280
Tcrystal = 200
gamma = 1
D0 = 1
Mweight = 0.5
Mvolume = 1
mobStep = 10
noiseStr = 0.05
[]
"""
    (tmp_path / "input.dat").write_text(text)
    r = subprocess.run([os.path.join(ROOT, "mesobasic_b200", "meso_b200")], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    names = sorted(os.listdir(tmp_path / "vtkoutput"))
    assert names == ["c_0.vtk", "c_20.vtk", "c_40.vtk", "mob_10.vtk"], names
    body = (tmp_path / "vtkoutput" / "mob_10.vtk").read_text().splitlines()
    assert body[10] == "SCALARS mob float" and len(body) == 12 + 32 * 24 * 16


@pytest.mark.parametrize("thermCond,dims", [(1.0, (32, 12, 8)), (4.0, (40, 24, 1))])
def test_bath_matches_reference_tipsbathphil(oracle, thermCond, dims):
    """TIPSbathPHIL: the temperature follows the 1-D bath profile along x."""
    fh = dict(QUENCH, Tinit=320.0, Tbath=260.0)
    ic = oracle.ic(dims, 0.3, 0.1, False, 8)
    want = oracle.fh_ref_run(ic, dims, dict(fh, kap=1.0), 50, 1, 10, bc=(0, 1, 1), bath=True, thermCond=thermCond)
    p = mb.make_params(*dims, 0.01, bc=(0, 1, 1))
    with mb.CHSim(p, fh=mb.make_fh_params(50, bath=True, thermCond=thermCond, **fh)) as sim:
        sim.set_field(ic)
        sim.step(10)
        got = sim.get_field()
    assert rel_err(got, want) <= 1e-12, rel_err(got, want)
    # and not the uniform ramp
    ramp = oracle.fh_ref_run(ic, dims, dict(fh, kap=1.0), 50, 1, 10, bc=(0, 1, 1))
    assert np.abs(got - ramp).max() > 1e-6


def test_driver_runs_tipsbathphil(tmp_path):
    text = """[Domain]
nx = 32
ny = 16
nz = 8
[]
[Time]
nstep = 20
dt = 0.01
[]
[Output]
numOutputs = 1
[]
[PFApp]
app = true
type = TIPSbathPHIL
co = 0.3
alpha = 150
beta = 0.1
N = 50
Tinit = 320
Tbath = 260
Tcrystal = 200
gamma = 1
D0 = 1
Mweight = 0.5
Mvolume = 1
thermCond = 2
noiseStr = 0
[]
"""
    (tmp_path / "input.dat").write_text(text)
    r = subprocess.run([os.path.join(ROOT, "mesobasic_b200", "meso_b200")], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    names = sorted(os.listdir(tmp_path / "vtkoutput"))
    assert names == ["polymer_0.vtk", "polymer_20.vtk", "temp_0.vtk", "temp_20.vtk"], names
    t0 = (tmp_path / "vtkoutput" / "temp_0.vtk").read_text().splitlines()
    assert t0[12] == "460.000"
    t20 = [float(v) for v in (tmp_path / "vtkoutput" / "temp_20.vtk").read_text().splitlines()[12:12 + 32]]
    assert 260.0 < t20[0] < t20[-1] <= 320.0  # warmer away from the bath at x = 0


@pytest.mark.parametrize("dims,bc,sips", [((32, 20, 16), (1, 1, 1), False), ((32, 12, 10), (0, 0, 1), False),
                                          ((48, 36, 1), (1, 0, 1), False), ((32, 16, 12), (0, 1, 1), True)])
def test_fused_kernel_matches_two_pass(oracle, dims, bc, sips):
    """The fused z-marching variable-mobility kernel (fh_march_kernel, tiling
    path 0) and the two-pass kernels (the default) take the same operations
    in the same order, noise included.  The compiler may contract the FP64
    log and exp inlined into each kernel differently, which moves a result
    by an ulp now and then (5 sites of 10,240 after one step, measured):
    most sites agree bit for bit and the rest to within an ulp or two."""
    ic = oracle.ic(dims, 0.3, 0.1, False, 5)
    p = mb.make_params(*dims, 0.01, bc=bc, noise=0.1, noise_seed=9)
    kw = dict(sips=mb.make_sips_params(Mweight=1.0, Mvolume=1.0, gamma=1.0)) if sips else \
        dict(fh=mb.make_fh_params(50, **QUENCH))
    out = []
    for fused in (False, True):
        with mb.CHSim(p, **kw) as sim:
            if fused:
                sim.tiling = (0, 0, 3, 0)  # path 0, ty 0: the fused kernel's own tiling
                assert sim.tiling.path == 0 and sim.tiling.ty >= 1
            sim.set_field(ic)
            sim.step(12)
            out.append(sim.get_field())
    assert rel_err(out[1], out[0]) <= 1e-14, rel_err(out[1], out[0])
    assert np.mean(out[0] == out[1]) >= 0.9
    assert np.abs(out[1] - ic).max() > 1e-4
