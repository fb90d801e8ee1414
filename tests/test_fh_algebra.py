"""The one-division forms of the variable-mobility passes against the
reference's arithmetic, in numpy (no GPU).

The update passes take the mobility of a site inside the Flory-Huggins range
(0 < c < 1) as one quotient, 1/mob = f''/Dp = kT (u + N c) / (2 N c u D e)
with u = 1 - c and e = exp(-gamma phi^nu), the reference's clamps on Mc
becoming bounds on that quotient (fh_site_r in csrc/ch_device.cuh); and the
divergence div(mob grad mu) as the three axes over one common denominator
(fh_axis_frac, fh_div_frac).  These tests restate both forms and the
reference's own chains (TIPSphil.cpp:151-176, SIPS.cpp:190-204 with
philliesDiffusion and secondDerFH at SIPS.cpp:267-285, SfieldFD.cpp:333-355)
and check that they agree to a few ulp over the clamp and crystallisation
branches.  The kernels themselves are checked against the reference classes
on the GPU (tests/test_gpu_fh.py, tests/test_gpu_sips.py)."""
import numpy as np
import pytest

import mesobasic_b200 as mb

# c = 1e-300 drives f'' and the quotient towards overflow: the clamp branch
pytestmark = pytest.mark.filterwarnings("ignore:overflow encountered:RuntimeWarning")

RNG = np.random.default_rng(7)
CC = np.concatenate([RNG.uniform(1e-9, 1 - 1e-9, 200_000), np.array([1e-300, 0.5, 1 - 2.0 ** -53])])


def ref_rmob_tipsphil(cc, T, p):
    """1/Mc of TIPSphil.cpp:151-176 for 0 < cc < 1, every step as written."""
    kT = T / 273.0
    D = min(p["D0"] * (T / p["Tinit"]), p["D0"])
    cc_phil = cc * p["Mweight"] / p["Mvolume"]
    ddf = 0.5 * (1.0 / (p["N"] * cc) + 1.0 / (1.0 - cc))
    ddf = ddf * kT
    Dp = D * np.exp(-p["gamma"] * cc_phil ** p["nu"])
    Mc = Dp / ddf
    Mc = np.where(Mc < 0.000001, 0.000001, Mc)
    Mc = np.where(Mc > p["D0"], p["D0"], Mc)
    if T <= p["Tcrystal"]:
        Mc = Mc * 0.001
    return 1.0 / Mc


def quotient_rmob(cc, kT, N, Dm, conv, gamma, nu, qlo, qhi, rlo, rhi, fac):
    """fh_site_r's reciprocal mobility from the column constants."""
    u = 1.0 - cc
    e = np.exp(-gamma * (cc * conv) ** nu)
    q = (kT * (N * cc + u)) / (2.0 * (N * cc) * u * (Dm * e))
    return np.where(q > qlo, rlo, np.where(q < qhi, rhi, q * fac))


def tipsphil_column(T, p):
    """fh_column's clamp constants for TIPSphil / TIPSbathPHIL."""
    D = min(p["D0"] * (T / p["Tinit"]), p["D0"])
    cryst = T <= p["Tcrystal"]
    mlo = p["D0"] if 0.000001 > p["D0"] else 0.000001
    return dict(kT=T / 273.0, N=p["N"], Dm=D, conv=p["Mweight"] / p["Mvolume"], gamma=p["gamma"], nu=p["nu"],
                qlo=1000000.0, qhi=1.0 / p["D0"], rlo=1.0 / (mlo * 0.001 if cryst else mlo),
                rhi=1.0 / (p["D0"] * 0.001 if cryst else p["D0"]), fac=1000.0 if cryst else 1.0)


QUENCH = dict(mb.FH_DEFAULTS, alpha=150.0, beta=0.1, N=50.0, Tinit=300.0, Tbath=280.0, Tcrystal=200.0, gamma=1.0,
              D0=1.0, Mweight=0.5, Mvolume=1.0)


@pytest.mark.parametrize("name,p,T", [
    ("benchmark quench", QUENCH, 290.0),
    ("reference defaults (every site on a clamp, crystallised)", dict(mb.FH_DEFAULTS), 273.0),
    ("crystallised, D0 clamp", dict(QUENCH, Tcrystal=295.0, D0=0.5), 290.0),
    ("N = 1, steep Phillies term", dict(QUENCH, N=1.0, gamma=3.0, Mweight=30.0, Mvolume=1.1), 300.0),
    ("D0 below the lower clamp", dict(QUENCH, D0=1e-7), 290.0),
])
def test_tipsphil_mobility_quotient_matches_reference_chain(name, p, T):
    want = ref_rmob_tipsphil(CC, T, p)
    got = quotient_rmob(CC, **tipsphil_column(T, p))
    rel = np.abs(got - want) / np.abs(want)
    assert rel.max() <= 1e-14, (name, rel.max())
    # clamped sites take exactly the reference's clamped value
    lo = ref_rmob_tipsphil(np.array([1e-300]), T, p)[0]
    assert np.all(got[want == lo] == lo)


def ref_rmob_sips(cc, scale, p):
    """1/(Mc * mobScale) of SIPS.cpp:190-204 for 0 < cc < 1."""
    kT = p["Tinit"] / 273.0
    cc_phil = cc * p["Mweight"] / p["Mvolume"]
    ddf = 0.5 * (1.0 / (p["N"] * cc) + 1.0 / (1.0 - cc)) * kT
    Dp = p["D0"] * np.exp(-p["gamma"] * cc_phil ** p["nu"])
    Mc = Dp / ddf
    Mc = np.where(Mc > 1.0, 1.0, np.where(Mc < 0.00001, 0.00001, Mc))
    return 1.0 / (Mc * scale)


@pytest.mark.parametrize("scale", [1.2, 0.7, 0.0023])
@pytest.mark.parametrize("p", [dict(mb.SIPS_DEFAULTS), dict(mb.SIPS_DEFAULTS, N=5.0, gamma=1.0, Mweight=1.0, Mvolume=1.0)])
def test_sips_mobility_quotient_matches_reference_chain(scale, p):
    col = dict(kT=p["Tinit"] / 273.0, N=p["N"], Dm=p["D0"], conv=p["Mweight"] / p["Mvolume"], gamma=p["gamma"],
               nu=p["nu"], qlo=100000.0, qhi=1.0, rlo=1.0 / (0.00001 * scale), rhi=1.0 / (1.0 * scale),
               fac=1.0 / scale)
    want = ref_rmob_sips(CC, scale, p)
    got = quotient_rmob(CC, **col)
    rel = np.abs(got - want) / np.abs(want)
    assert rel.max() <= 1e-14, rel.max()


def test_divergence_over_one_denominator_matches_per_axis_form():
    """SfieldFD::Laplacian(const SfieldFD&) (SfieldFD.cpp:333-355), per axis
    with harmonic-mean faces, against 2 (nx qy qz + ny qx qz + nz qx qy) /
    (qx qy qz), reciprocal mobilities spanning the models' clamps (1 to
    1e9), unequal spacings divided as the reference divides."""
    n = 200_000
    a0 = RNG.normal(0.0, 3.0, n)
    r0 = 10.0 ** RNG.uniform(0.0, 9.0, n)
    d2 = (1.0, 1.5625, 2.25)
    want = np.zeros(n)
    scale = np.zeros(n)
    fr = []
    for ax in range(3):
        am, ap = a0 + RNG.normal(0.0, 1e-2, n), a0 + RNG.normal(0.0, 1e-2, n)
        rm, rp = 10.0 ** RNG.uniform(0.0, 9.0, n), 10.0 ** RNG.uniform(0.0, 9.0, n)
        if ax == 2:  # a no-flux border: the neighbour is the site itself
            am[: n // 4], rm[: n // 4] = a0[: n // 4], r0[: n // 4]
        b1, b2 = 2.0 / (rm + r0), 2.0 / (rp + r0)  # faces from the stored reciprocals, as the update pass reads them
        want = want + (am * b1 + ap * b2 - (b1 + b2) * a0) / d2[ax]
        scale = scale + (np.abs(am * b1) + np.abs(ap * b2) + np.abs((b1 + b2) * a0)) / d2[ax]
        s1, s2 = rm + r0, rp + r0
        fr.append(((am - a0) * s2 + (ap - a0) * s1, s1 * s2 * d2[ax]))
    (nx, qx), (ny, qy), (nz, qz) = fr
    qxy = qx * qy
    got = 2.0 * ((nx * qy + ny * qx) * qz + nz * qxy) / (qxy * qz)
    assert np.all(np.isfinite(got))
    assert (np.abs(got - want) / scale).max() <= 1e-14
