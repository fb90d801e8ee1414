"""The SIPS and SIPSternary steps against the reference's own
SIPS::updatePhaseField and SIPSternary::updatePhaseField run on the same
fields (oracle.sips_ref_run, oracle.ternary_ref_run; noise off), the noise
rules of both models, and the driver.

SIPS takes log, exp, pow, erf and sqrt, which differ from the host's libm by
an ulp or two: the bar is a relative max-norm of 1e-12.  The SIPSternary step
is additions, multiplications and divisions only: bit-identical."""
import os
import subprocess

import numpy as np
import pytest

import mesobasic_b200 as mb

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SEED = 0x5151_0042

# a mobility that is not pinned at its clamps (the reference's defaults give
# exp(-10 * 300) = 0, so every site sits at the 1e-5 floor)
MOVE = dict(Mweight=1.0, Mvolume=1.0, gamma=1.0)


def rel_err(got, want):
    return np.abs(got - want).max() / np.abs(want).max()


def sips_gpu(dims, sp, ic, nsteps, NSdepth=0, dt=0.01, kap=1.0, spacing=(1.0, 1.0, 1.0), bc=(0, 1, 1), noise=0.0):
    p = mb.make_params(*dims, dt, kappa=kap, dx=spacing[0], dy=spacing[1], dz=spacing[2], bc=bc, noise=noise,
                       noise_seed=SEED)
    with mb.CHSim(p, sips=mb.make_sips_params(NSdepth, **sp)) as sim:
        sim.set_field(ic)
        sim.step(nsteps)
        return sim.get_field(), sim.mobility()


def with_bath(ic, depth, value=0.0):
    out = ic.copy()
    out[:, :, :depth] = value
    return out


SIPS_CASES = [
    ("3d no-flux x", (24, 16, 12), MOVE, 0, 0.1, 0.1, (1.0, 1.0, 1.0), (0, 1, 1), 0.01),
    ("bath planes", (32, 12, 8), dict(MOVE, chiCond=0.5), 6, 0.15, 0.1, (1.0, 1.0, 1.0), (0, 1, 1), 0.01),
    ("2d", (40, 24, 1), MOVE, 3, 0.2, 0.1, (1.0, 1.0, 1.0), (0, 1, 1), 0.01),
    ("periodic, unequal spacing", (20, 12, 10), dict(MOVE, chiPS=0.6, chiPN=1.8), 0, 0.3, 0.2, (1.0, 1.25, 1.5),
     (1, 1, 1), 0.01),
    # values below 0 and above 1 (the clamped Flory-Huggins argument, the sqrt
    # branch, the mobility clamps), the reference's default mobility law
    ("branches", (16, 16, 8), {}, 2, 0.5, 1.4, (1.0, 1.0, 1.0), (0, 1, 1), 0.001),
]


@pytest.mark.parametrize("name,dims,sp,depth,co,amp,spacing,bc,dt", SIPS_CASES, ids=[c[0] for c in SIPS_CASES])
def test_sips_matches_reference(oracle, name, dims, sp, depth, co, amp, spacing, bc, dt):
    ic = with_bath(oracle.ic(dims, co, amp, False, 31), depth)
    want = oracle.sips_ref_run(ic, dims, sp, 1, 10, NSdepth=depth, spacing=spacing, dt=dt, bc=bc)
    got, mob = sips_gpu(dims, sp, ic, 10, NSdepth=depth, dt=dt, spacing=spacing, bc=bc)
    assert rel_err(got, want) <= 1e-12, rel_err(got, want)
    assert np.all(np.isfinite(mob)) and np.all(mob > 0)
    assert np.abs(got - ic).max() > 1e-7  # the model moved the field


def test_sips_later_steps_match_reference(oracle):
    """The erf front depends on the step number: steps 41..45."""
    dims = (24, 8, 8)
    ic = oracle.ic(dims, 0.1, 0.1, False, 5)
    warm = oracle.sips_ref_run(ic, dims, MOVE, 1, 40)
    want = oracle.sips_ref_run(warm, dims, MOVE, 41, 5)
    p = mb.make_params(*dims, 0.01, bc=(0, 1, 1))
    with mb.CHSim(p, sips=mb.make_sips_params(**MOVE)) as sim:
        sim.set_field(ic)
        sim.step(45)
        got = sim.get_field()
    assert rel_err(got, want) <= 1e-12, rel_err(got, want)


def test_sips_noise_skips_sites_at_or_above_cutoff(oracle):
    """One step with noise: the noise-free step plus the Philox increments,
    except where the stepped value is >= phiCutoff (SIPS.cpp:239-240)."""
    dims, dt, noise, cut = (20, 12, 6), 0.01, 0.5, 0.45
    ic = oracle.ic(dims, 0.45, 0.2, False, 9)
    sp = dict(MOVE, phiCutoff=cut)
    clean, _ = sips_gpu(dims, sp, ic, 1, dt=dt)
    noisy, _ = sips_gpu(dims, sp, ic, 1, dt=dt, noise=noise)
    inc = oracle.noise_increments(int(np.prod(dims)), 1, SEED, noise, dt).reshape(clean.shape)
    gated = clean >= cut
    assert 0.2 < gated.mean() < 0.8
    want = np.where(gated, clean + dt * 0.0, clean + inc)
    assert np.array_equal(noisy, want)


def test_sips_rejections():
    with pytest.raises(mb.MGError):
        mb.CHSim(mb.make_params(16, 8, 8, 0.01, precision="fp32"), sips=mb.make_sips_params())
    with pytest.raises(mb.MGError):
        mb.CHSim(mb.make_params(16, 8, 8, 0.01), sips=mb.make_sips_params(chiPS=1.0, chiPN=1.0))


# ---------------------------------------------------------------- SIPSternary
TERNARY_CASES = [
    ("3d no-flux x", (20, 16, 12), dict(Kpp=1.5, Knn=0.7, Mpp=1.0, Mnn=2.0), (1.0, 1.0, 1.0), (0, 1, 1), 0),
    ("2d periodic, unequal spacing", (32, 24, 1), dict(Kpp=1.0, Knn=2.0, Mpp=0.3, Mnn=0.7), (1.0, 1.5, 1.0),
     (1, 1, 1), 0),
    ("bath planes", (24, 10, 8), dict(Kpp=1.0, Knn=1.0, Mpp=1.0, Mnn=1.0), (1.0, 1.0, 1.0), (0, 1, 0), 4),
]


def ternary_ics(oracle, dims, depth, seed=17):
    d = oracle.ic(dims, 0.0, 0.1, False, seed)  # 0.0 + 0.1*(r - 0.5), one r per site
    c, n = 0.2 + d, 0.1 - d
    return with_bath(c, depth, 0.0), with_bath(n, depth, 1.0)


@pytest.mark.parametrize("name,dims,kw,spacing,bc,depth", TERNARY_CASES, ids=[c[0] for c in TERNARY_CASES])
def test_ternary_bit_identical_to_reference(oracle, name, dims, kw, spacing, bc, depth):
    c0, n0 = ternary_ics(oracle, dims, depth)
    wc, wn = oracle.ternary_ref_run(c0, n0, dims, 1, 12, spacing=spacing, dt=0.01, bc=bc, **kw)
    p = mb.make_params(*dims, 0.01, dx=spacing[0], dy=spacing[1], dz=spacing[2], bc=bc)
    with mb.Ternary(p, **kw) as t:
        t.set_fields(c0, n0)
        t.step(12)
        gc, gn = t.get_fields()
    assert np.array_equal(gc, wc), np.abs(gc - wc).max()
    assert np.array_equal(gn, wn), np.abs(gn - wn).max()
    assert np.abs(gc - c0).max() > 1e-6 and np.abs(gn - n0).max() > 1e-6


def test_ternary_noise_is_negated_on_n(oracle):
    """With K = 0 a step leaves both fields as they are (mu = 0.0 - 0*lap),
    so one step adds exactly the noise: +inc on c, -inc on n
    (SIPSternary.cpp:263-274)."""
    dims, dt, noise = (17, 6, 5), 0.01, 0.8  # 510 sites: a partial last draw
    c0, n0 = ternary_ics(oracle, dims, 0)
    p = mb.make_params(*dims, dt, noise=noise, noise_seed=SEED)
    with mb.Ternary(p, Kpp=0.0, Knn=0.0) as t:
        t.set_fields(c0, n0)
        t.step(1)
        gc, gn = t.get_fields()
    inc = oracle.noise_increments(int(np.prod(dims)), 1, SEED, noise, dt).reshape(c0.shape)
    assert np.array_equal(gc, c0 + inc)
    assert np.array_equal(gn, n0 + (-inc))


def test_ternary_rejects_fp32():
    with pytest.raises(mb.MGError):
        mb.Ternary(mb.make_params(16, 8, 8, 0.01, precision="fp32"))


def test_ternary_batch_vtk_matches_host_writer(tmp_path, oracle):
    dims = (24, 10, 6)
    c0, n0 = ternary_ics(oracle, dims, 3)
    with mb.Ternary(mb.make_params(*dims, 0.01, bc=(0, 1, 1))) as t:
        t.set_fields(c0, n0)
        t.step(3)
        t.write_vtk(1, tmp_path / "dev.vtk", "n", 2, 1, 1)
        mb.vtk_write(tmp_path / "host.vtk", "n", t.get_field(1), dims, 2, 1, 1)
    assert (tmp_path / "dev.vtk").read_bytes() == (tmp_path / "host.vtk").read_bytes()


# -------------------------------------------------------------------- driver
def run_driver(tmp_path, text):
    (tmp_path / "input.dat").write_text(text)
    r = subprocess.run([os.path.join(ROOT, "mesobasic_b200", "meso_b200")], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return sorted(os.listdir(tmp_path / "vtkoutput"))


def values(path, nx, count):
    return [float(v) for v in path.read_text().splitlines()[12:12 + count]]


def test_driver_runs_sips(tmp_path):
    names = run_driver(tmp_path, """[Domain]
nx = 32
ny = 16
nz = 8
[]
[Time]
nstep = 20
dt = 0.01
[]
[Output]
numOutputs = 2
[]
[PFApp]
app = true
type = SIPS
co = 0.2
NSdepth = 4
Mweight = 1
Mvolume = 1
gamma = 1
noiseStr = 0.05
[]
""")
    assert names == ["c_0.vtk", "c_10.vtk", "c_20.vtk"], names
    row = values(tmp_path / "vtkoutput" / "c_0.vtk", 32, 32)
    assert row[:4] == [0.0] * 4 and all(0.14 < v < 0.26 for v in row[4:])


def test_driver_runs_sipsternary(tmp_path):
    names = run_driver(tmp_path, """[Domain]
nx = 24
ny = 12
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
type = SIPSternary
NSdepth = 3
Kpp = 1.5
noiseStr = 0.1
[]
""")
    assert names == ["c_0.vtk", "c_20.vtk", "n_0.vtk", "n_20.vtk"], names
    c = values(tmp_path / "vtkoutput" / "c_0.vtk", 24, 24)
    n = values(tmp_path / "vtkoutput" / "n_0.vtk", 24, 24)
    assert c[:3] == [0.0] * 3 and n[:3] == [1.0] * 3
    # c + n = co + no wherever the film is (one r per site), up to the %.3f rounding
    assert all(abs(a + b - 0.3) <= 0.0011 for a, b in zip(c[3:], n[3:]))
