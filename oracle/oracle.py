"""TEST INFRASTRUCTURE ONLY: Python access to the oracles.

* ``libchoracle.so``: the plain-C restatement of the reference's CH step
  (ch_oracle.c), built by ``make -C oracle``.
* ``_ref/libchref.so`` and ``_ref/chref_bench``: the reference CPU build
  (the reference's own SfieldFD/Rand/PFApp sources plus the CHBasic model),
  built by ``make -C oracle ref`` where the reference sources are present.
* numpy restatements of the quantities the reference does not compute:
  structure factor and its peak wavenumber, the linear-stability growth
  factor, and the legacy-VTK text of ``SfieldFD::writeVTKFile``.

Only tests, the smoke check and the benchmark's CPU-baseline leg import this
module; the product never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_bin", "libchoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libchref.so")
REF_BENCH = os.path.join(HERE, "_ref", "chref_bench")
REF_MESO = os.path.join(HERE, "_ref", "meso_ref")
REF_MESO_GPU = os.path.join(HERE, "_ref", "meso_ref_gpu")


def reference_src() -> str | None:
    """The reference checkout the recipe compiles: $MESO_REFERENCE, else a
    checkout named ``reference`` beside this repository; None when neither
    holds the reference's ``src`` tree."""
    cands = [os.environ.get("MESO_REFERENCE", ""),
             os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")]
    for c in cands:
        if c and os.path.isdir(os.path.join(c, "src", "phase_field")):
            return os.path.abspath(c)
    return None

_i3 = ctypes.c_int * 3
_d3 = ctypes.c_double * 3
_d6 = ctypes.c_double * 6
_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)


def build(reference: bool | None = None) -> None:
    """Compile the C restatement, and the reference build when its sources
    exist (reference_src()).  The reference driver with the GPU plugin
    (meso_ref_gpu) is linked too when libmesogpu.so has been built."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    src = reference_src()
    if reference is None:
        reference = src is not None
    if reference:
        if src is None:
            raise FileNotFoundError("reference sources not found: set MESO_REFERENCE")
        targets = ["ref"]
        if os.path.exists(os.path.join(os.path.dirname(HERE), "mesobasic_b200", "libmesogpu.so")):
            targets.append("ref-gpu")
        subprocess.run(["make", "-s", "-C", HERE, *targets, f"REF={src}", f"-j{os.cpu_count() or 4}"], check=True)


def _lib(path):
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (make -C oracle [ref])")
    return ctypes.CDLL(path)


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        _oracle = _lib(ORACLE_SO)
        L = _oracle
        L.cho_ic.argtypes = [_i3, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_uint32, _dp]
        L.cho_step.argtypes = [_i3, _d3, ctypes.c_double, ctypes.c_double, ctypes.c_double, _i3, _dp, _dp, _dp]
        L.cho_run.argtypes = [_i3, _d3, ctypes.c_double, ctypes.c_double, ctypes.c_double, _i3, _dp, ctypes.c_int]
        L.cho_run.restype = ctypes.c_int
        L.cho_reduce.argtypes = [_i3, _d3, ctypes.c_double, _i3, _dp, _d6]
        L.cho_reduce_f32.argtypes = [_i3, _d3, ctypes.c_double, _i3, _fp, _d6]
        L.cho_rand_init.argtypes = [ctypes.c_void_p, ctypes.c_uint32]
        L.cho_rand_u32.argtypes = [ctypes.c_void_p]
        L.cho_rand_u32.restype = ctypes.c_uint32
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        _ref = _lib(REF_SO)
        _ref.chref_run.argtypes = [_i3, _d3, ctypes.c_double, ctypes.c_double, ctypes.c_double, _i3, _dp,
                                   ctypes.c_int, _dp]
        _ref.chref_run.restype = ctypes.c_int
        _ref.chref_ic.argtypes = [_i3, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_uint32, _dp]
        _ref.chref_ic.restype = ctypes.c_int
        _ref.fhref_run.argtypes = [_i3, _d3, ctypes.c_double, _i3, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_int, _dp, ctypes.c_int, _dp]
        _ref.fhref_run.restype = ctypes.c_int
        _ref.sipsref_run.argtypes = [_i3, _d3, ctypes.c_double, _i3, _dp, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int,
                                     _dp]
        _ref.sipsref_run.restype = ctypes.c_int
        _ref.ternref_run.argtypes = [_i3, _d3, ctypes.c_double, _i3, _dp, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp,
                                     _dp]
        _ref.ternref_run.restype = ctypes.c_int
    return _ref


def _as_field(c, dims):
    nx, ny, nz = dims
    a = np.ascontiguousarray(c, dtype=np.float64).reshape(nz, ny, nx)
    return a


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


# ----------------------------------------------------------------- restatement
def mt_u32(seed: int, count: int) -> np.ndarray:
    """First `count` outputs of the MT19937 restatement (rand.cpp:24-78)."""
    L = oracle_lib()
    state = ctypes.create_string_buffer(625 * 4)
    L.cho_rand_init(state, seed)
    return np.array([L.cho_rand_u32(state) for _ in range(count)], dtype=np.uint32)


def ic(dims, co, amp, gaussian=False, seed=42) -> np.ndarray:
    """Seeded initial condition, shape (nz, ny, nx), float64."""
    nx, ny, nz = dims
    out = np.empty((nz, ny, nx), dtype=np.float64)
    oracle_lib().cho_ic(_i3(*dims), co, amp, int(bool(gaussian)), seed, _ptr(out))
    return out


def run(c, dims, spacing=(1.0, 1.0, 1.0), dt=0.01, M=1.0, kap=1.0, nsteps=1, bc=(1, 1, 1)) -> np.ndarray:
    """nsteps CH steps of the C restatement; returns a new (nz, ny, nx) array."""
    a = _as_field(c, dims).copy()
    rc = oracle_lib().cho_run(_i3(*dims), _d3(*spacing), dt, M, kap, _i3(*bc), _ptr(a), nsteps)
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    return a


def reduce(c, dims, spacing=(1.0, 1.0, 1.0), kap=1.0, bc=(1, 1, 1)) -> dict:
    """Mass / energy diagnostics (ch_oracle.h), float64 or float32 input."""
    nx, ny, nz = dims
    out = _d6()
    if np.asarray(c).dtype == np.float32:
        a = np.ascontiguousarray(c, dtype=np.float32).reshape(nz, ny, nx)
        oracle_lib().cho_reduce_f32(_i3(*dims), _d3(*spacing), kap, _i3(*bc), _ptr(a, _fp), out)
    else:
        a = _as_field(c, dims)
        oracle_lib().cho_reduce(_i3(*dims), _d3(*spacing), kap, _i3(*bc), _ptr(a), out)
    keys = ["mass", "mass_plain", "energy", "abs_mass", "max_abs", "nonfinite"]
    return dict(zip(keys, list(out)))


# ------------------------------------------------------------ reference build
def ref_run(c, dims, spacing=(1.0, 1.0, 1.0), dt=0.01, M=1.0, kap=1.0, nsteps=1, bc=(1, 1, 1)) -> np.ndarray:
    """nsteps steps of the reference CPU build (SfieldFD + CHBasic)."""
    a = _as_field(c, dims)
    out = np.empty_like(a)
    ref_lib().chref_run(_i3(*dims), _d3(*spacing), dt, M, kap, _i3(*bc), _ptr(a), nsteps, _ptr(out))
    return out


# TIPSphil's parameters in the order fhref_run takes them, with the
# reference constructor's defaults (TIPSphil.cpp:41-59)
FH_KEYS = ("alpha", "beta", "N", "A", "Tinit", "Tbath", "Tcrystal", "nu", "gamma", "D0", "Mweight", "Mvolume", "kap")
FH_DEFAULTS = dict(alpha=1.0, beta=1.0, N=100.0, A=1.0, Tinit=273.0, Tbath=273.0, Tcrystal=273.0, nu=1.0,
                   gamma=10.0, D0=1e-7, Mweight=100.0, Mvolume=0.1, kap=1.0)


def fh_ref_run(c, dims, fh, nstep_total, first, nsteps, spacing=(1.0, 1.0, 1.0), dt=0.01, bc=(1, 1, 1), bath=False,
               thermCond=1.0):
    """Steps first..first+nsteps-1 of the reference's own TIPSphil update
    (or TIPSbathPHIL's with bath=True: Flory-Huggins mu, Phillies mobility,
    variable-mobility Laplacian) on c, noise off; fh maps FH_KEYS to values
    (missing keys: FH_DEFAULTS)."""
    a = _as_field(c, dims)
    out = np.empty_like(a)
    prm = np.array([fh.get(k, FH_DEFAULTS[k]) for k in FH_KEYS], dtype=np.float64)
    ref_lib().fhref_run(_i3(*dims), _d3(*spacing), dt, _i3(*bc), _ptr(prm), int(bool(bath)), float(thermCond),
                        nstep_total, first, _ptr(a), nsteps, _ptr(out))
    return out


# SIPS's parameters in the order sipsref_run takes them, with the reference
# constructor's defaults (SIPS.cpp:22-59)
SIPS_KEYS = ("N", "A", "Tinit", "chiPS", "chiPN", "chiCond", "phiCutoff", "nu", "gamma", "D0", "Mweight", "Mvolume",
             "kap")
SIPS_DEFAULTS = dict(N=100.0, A=1.0, Tinit=273.15, chiPS=0.034, chiPN=2.5, chiCond=1.0, phiCutoff=0.5, nu=1.0,
                     gamma=10.0, D0=1.0, Mweight=100.0, Mvolume=0.1, kap=1.0)


def sips_ref_run(c, dims, sp, first, nsteps, NSdepth=0, spacing=(1.0, 1.0, 1.0), dt=0.01, bc=(0, 1, 1)):
    """Steps first..first+nsteps-1 of the reference's own SIPS update
    (SIPS.cpp:130-249) on c, noise off; sp maps SIPS_KEYS to values."""
    a = _as_field(c, dims)
    out = np.empty_like(a)
    prm = np.array([sp.get(k, SIPS_DEFAULTS[k]) for k in SIPS_KEYS], dtype=np.float64)
    ref_lib().sipsref_run(_i3(*dims), _d3(*spacing), dt, _i3(*bc), _ptr(prm), int(NSdepth), first, _ptr(a), nsteps,
                          _ptr(out))
    return out


def ternary_ref_run(c, n, dims, first, nsteps, Kpp=1.0, Knn=1.0, Mpp=1.0, Mnn=1.0, spacing=(1.0, 1.0, 1.0), dt=0.01,
                    bc=(0, 1, 1)):
    """Steps first..first+nsteps-1 of the reference's own SIPSternary update
    (SIPSternary.cpp:132-278) on the fields c and n, noise off."""
    a = _as_field(c, dims)
    b = _as_field(n, dims)
    oc, on = np.empty_like(a), np.empty_like(b)
    prm = np.array([Kpp, Knn, Mpp, Mnn], dtype=np.float64)
    ref_lib().ternref_run(_i3(*dims), _d3(*spacing), dt, _i3(*bc), _ptr(prm), first, _ptr(a), _ptr(b), nsteps,
                          _ptr(oc), _ptr(on))
    return oc, on


def ref_bench_field(dims, dt, M, kap, co, amp, gaussian, seed, nsteps, ranks, workdir, timeout=900):
    """Runs the reference CPU build's own step loop (chref_bench: PFApp ->
    CHBasic on SfieldFD, MPI-shim ranks as forked processes) for nsteps
    from its seeded initial condition and returns the final field, shape
    (nz, ny, nx), assembled from the ranks' x-slab dumps.  ranks must divide
    nx.  Also returns the run's JSON record (wall time of the step loop)."""
    import json
    nx, ny, nz = dims
    if nx % ranks:
        raise ValueError(f"{ranks} ranks do not divide nx = {nx}")
    prefix = os.path.join(workdir, "refdump")
    env = dict(os.environ, MB_SHIM_NP=str(ranks), MB_SHIM_SLOT_MB=str(max(16, (ny + 2) * (nz + 2) * 8 // (1 << 20) + 2)))
    args = [REF_BENCH, f"Domain/nx={nx}", f"Domain/ny={ny}", f"Domain/nz={nz}", f"Time/dt={dt!r}",
            f"Time/nstep={nsteps}", f"PFApp/M={M!r}", f"PFApp/kap={kap!r}", f"PFApp/co={co!r}",
            f"PFApp/noise_amp={amp!r}", f"PFApp/noise_type={'gaussian' if gaussian else 'uniform'}",
            f"PFApp/seed={seed}", "PFApp/vtk=0", "PFApp/init_output=0", f"PFApp/dump_prefix={prefix}"]
    r = subprocess.run(args, env=env, capture_output=True, text=True, timeout=timeout, cwd=workdir)
    if r.returncode != 0:
        raise RuntimeError(f"chref_bench failed ({r.returncode}): {r.stderr[-800:]}")
    rec = json.loads(r.stdout.strip().splitlines()[-1])
    out = np.empty((nz, ny, nx), dtype=np.float64)
    for rk in range(ranks):
        path = f"{prefix}_{nsteps}.rank{rk}"
        with open(path, "rb") as f:
            hdr = np.frombuffer(f.read(20), dtype=np.int32)
            xoff, lnx, lny, lnz, step = (int(v) for v in hdr)
            if (lny, lnz, step) != (ny, nz, nsteps):
                raise RuntimeError(f"dump {path}: header {hdr.tolist()} does not match the run")
            slab = np.fromfile(f, dtype=np.float64, count=lnx * lny * lnz).reshape(lnz, lny, lnx)
        out[:, :, xoff:xoff + lnx] = slab
        os.remove(path)
    return out, rec


def ref_ic(dims, co, amp, gaussian=False, seed=42) -> np.ndarray:
    nx, ny, nz = dims
    out = np.empty((nz, ny, nx), dtype=np.float64)
    ref_lib().chref_ic(_i3(*dims), co, amp, int(bool(gaussian)), seed, _ptr(out))
    return out


# ------------------------------------------------- quantities with no reference
def structure_factor(c, dims, spacing=(1.0, 1.0, 1.0), nbins=None):
    """Radially binned S(k) = |FFT(c - <c>)|^2 / N and its first-moment
    wavenumber k1 = sum(|k| S) / sum(S) over every mode in the bins.

    Bin b holds |k| in [b*dk, (b+1)*dk) with dk = 2*pi/max(L); the k = 0
    mode is excluded.  k_centres[b] is the mean |k| and S_binned[b] the mean
    S of the modes in bin b.  Returns (k_centres, S_binned, counts, k1)."""
    nx, ny, nz = dims
    a = np.asarray(c, dtype=np.float64).reshape(nz, ny, nx)
    f = np.fft.fftn(a - a.mean())
    s = (f.real ** 2 + f.imag ** 2) / a.size
    L = max(nx * spacing[0], ny * spacing[1], nz * spacing[2])
    dk = 2 * np.pi / L
    # |k|/dk = sqrt(sum (m_d L/L_d)^2), exact integers on equal box lengths
    mx = np.fft.fftfreq(nx, d=1.0 / nx) * (L / (nx * spacing[0]))
    my = np.fft.fftfreq(ny, d=1.0 / ny) * (L / (ny * spacing[1]))
    mz = np.fft.fftfreq(nz, d=1.0 / nz) * (L / (nz * spacing[2]))
    q = np.sqrt(mz[:, None, None] ** 2 + my[None, :, None] ** 2 + mx[None, None, :] ** 2)
    kk = q * dk
    if nbins is None:
        nbins = int(np.floor(q.max() + 1e-9)) + 1
    b = np.floor(q + 1e-9).astype(np.int64)
    mask = (kk > 0) & (b < nbins)
    sb = np.bincount(b[mask], weights=s[mask], minlength=nbins)
    cnt = np.bincount(b[mask], minlength=nbins)
    ksum = np.bincount(b[mask], weights=kk[mask], minlength=nbins)
    kc = np.where(cnt > 0, ksum / np.maximum(cnt, 1), (np.arange(nbins) + 0.5) * dk)
    sbar = np.where(cnt > 0, sb / np.maximum(cnt, 1), 0.0)
    ks = (kk[mask] * s[mask]).sum()
    k1 = float(ks / sb.sum()) if sb.sum() > 0 else 0.0
    return kc, sbar, cnt, k1


def growth_factor(k_vec, dims_active, c0, kap, dt, M=1.0, spacing=(1.0, 1.0, 1.0)):
    """Per-step amplification of a small Fourier mode about a uniform c0:
    1 + dt*M*lam*(3*c0^2 - 1 - kap*lam), lam = -sum_d 4/dx_d^2 sin^2(k_d dx_d/2)."""
    lam = 0.0
    for kd, dd, on in zip(k_vec, spacing, dims_active):
        if on:
            lam -= 4.0 / dd ** 2 * np.sin(kd * dd / 2.0) ** 2
    return 1.0 + dt * M * lam * (3 * c0 ** 2 - 1 - kap * lam)


def vtk_text(c, dims, tag, iskip=1, jskip=1, kskip=1) -> str:
    """Text of SfieldFD::writeVTKFile (SfieldFD.cpp:363-430) for one rank:
    header, then one `%.3f` value per line, x fastest, with the skip rules
    of :407-413 (x uses the global index test ig%iskip == 0 on 1-based ig;
    y and z step by jskip/kskip from 1)."""
    nx, ny, nz = dims
    a = np.asarray(c, dtype=np.float64).reshape(nz, ny, nx)
    d = "   "

    def num(v):  # ostream default formatting of 1.0*skip
        return f"{v:g}"

    lines = ["# vtk DataFile Version 3.1", "VTK file containing grid data", "ASCII", " ",
             "DATASET STRUCTURED_POINTS",
             f"DIMENSIONS{d}{nx // iskip}{d}{ny // jskip}{d}{nz // kskip}",
             f"ORIGIN {d}0{d}0{d}0",
             f"SPACING{d}{num(1.0 * iskip)}{d}{num(1.0 * jskip)}{d}{num(1.0 * kskip)}",
             " ",
             f"POINT_DATA {(nx // iskip) * (ny // jskip) * (nz // kskip)}",
             f"SCALARS {tag} float",
             "LOOKUP_TABLE default"]
    xs = [i for i in range(1, nx + 1) if i % iskip == 0]
    for k in range(1, nz + 1, kskip):
        for j in range(1, ny + 1, jskip):
            row = a[k - 1, j - 1]
            lines.extend(f"{row[i - 1]:.3f}" for i in xs)
    return "\n".join(lines) + "\n"


# --------------------------------------------------------------- noise term
PHILOX_M = (0xD2511F53, 0xCD9E8D57)
PHILOX_W = (0x9E3779B9, 0xBB67AE85)


def philox4x32_10(ctr, key):
    """Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011) on Python ints:
    counter of four 32-bit words, key of two; returns four 32-bit words."""
    c, k = list(ctr), list(key)
    for r in range(10):
        if r:
            k = [(k[0] + PHILOX_W[0]) & 0xFFFFFFFF, (k[1] + PHILOX_W[1]) & 0xFFFFFFFF]
        p0, p1 = PHILOX_M[0] * c[0], PHILOX_M[1] * c[2]
        c = [(p1 >> 32) ^ c[1] ^ k[0], p1 & 0xFFFFFFFF, (p0 >> 32) ^ c[3] ^ k[1], p0 & 0xFFFFFFFF]
    return c


def noise_increments(n, step, seed, noise, dt):
    """dt * (noise * (r - 0.5)) per site, r = (word + 0.5) * 2^-32 with the
    word for site s from philox4x32_10((s//4, 0, step, 0) split into 32-bit
    halves, seed) -- the per-step fluctuation term of TIPSphil.cpp:200-209
    with a counter-based generator in place of rand()."""
    key = (seed & 0xFFFFFFFF, seed >> 32)
    words = np.empty(4 * ((n + 3) // 4), dtype=np.float64)
    for g in range(len(words) // 4):
        words[4 * g:4 * g + 4] = philox4x32_10((g & 0xFFFFFFFF, g >> 32, step & 0xFFFFFFFF, step >> 32), key)
    r = words[:n] * 2.3283064365386963e-10 + 1.1641532182693481e-10
    return dt * (noise * (r - 0.5))
