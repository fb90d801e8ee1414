"""mesobasic_b200: the Cahn-Hilliard step of mesoBasic's phase-field app on
B200 GPUs, behind the C ABI of libmesogpu.so (include/mesogpu.h).

Python objects here are thin owners of C-ABI handles:

* :class:`CHSim`  -- one simulation (the GPU body of a PFBaseClass model)
* :class:`Batch`  -- many simulations stepped by shared persistent launches
* :class:`Server` -- continuous batching of jobs under an HBM budget

Fields are numpy float64 arrays of shape (nz, ny, nx) (x fastest).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import (MG_FP32, MG_FP64, MG_JOB_DONE, MG_JOB_FAILED, MG_JOB_QUEUED, MG_JOB_RUNNING, MGError,
                   FhParams, Params, ServerStats, SipsParams, Stats, TernaryParams, Tiling, check, load)

__all__ = ["CHSim", "Batch", "Ternary", "Server", "Params", "Stats", "Tiling", "MGError", "MG_FP32", "MG_FP64",
           "make_params", "make_fh_params", "make_sips_params", "ic_generate", "vtk_write", "autotune", "load"]


# FP32 mass feedback cadence: the stored field is summed and corrected after
# every step, so the total mass meets the 1e-10 relative bound at every step
# (every K-th step with mass_correct=K: on target at the measured steps,
# predicted in between)
MASS_EVERY = 1


def make_params(nx, ny, nz, dt, kappa=1.0, M=1.0, dx=1.0, dy=1.0, dz=1.0, bc=(1, 1, 1),
                precision="fp64", mass_correct=None, noise=0.0, noise_seed=0) -> Params:
    prec = MG_FP32 if precision in ("fp32", MG_FP32) else MG_FP64
    if mass_correct is None:
        mass_correct = MASS_EVERY if prec == MG_FP32 else 0
    return Params(nx, ny, nz, dx, dy, dz, dt, M, kappa, bc[0], bc[1], bc[2], prec, int(mass_correct), float(noise),
                  int(noise_seed))


def _dims(p: Params):
    return (p.nz, p.ny, p.nx)


def _f64(a, shape):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.size != int(np.prod(shape)):
        raise ValueError(f"field has {a.size} values, expected {int(np.prod(shape))}")
    return a


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


# the reference TIPSphil constructor's defaults (TIPSphil.cpp:41-59)
FH_DEFAULTS = dict(alpha=1.0, beta=1.0, N=100.0, A=1.0, Tinit=273.0, Tbath=273.0, Tcrystal=273.0, nu=1.0,
                   gamma=10.0, D0=1e-7, Mweight=100.0, Mvolume=0.1)


def make_fh_params(nstep, bath=False, thermCond=1.0, **kw) -> FhParams:
    """Variable-mobility parameters: TIPSphil's uniform quench, or with
    bath=True TIPSbathPHIL's 1-D bath profile; unnamed ones take the
    reference's defaults."""
    unknown = set(kw) - set(FH_DEFAULTS)
    if unknown:
        raise ValueError(f"unknown variable-mobility parameters {sorted(unknown)}")
    v = dict(FH_DEFAULTS, **kw)
    return FhParams(*(float(v[k]) for k in FH_DEFAULTS), int(nstep), int(bool(bath)), float(thermCond))


# SIPS.cpp:22-59 (NSdepth is separate: an integer)
SIPS_DEFAULTS = dict(N=100.0, A=1.0, Tinit=273.15, chiPS=0.034, chiPN=2.5, chiCond=1.0, phiCutoff=0.5, nu=1.0,
                     gamma=10.0, D0=1.0, Mweight=100.0, Mvolume=0.1)


def make_sips_params(NSdepth=0, **kw) -> SipsParams:
    """SIPS parameters; unnamed ones take the reference's defaults."""
    unknown = set(kw) - set(SIPS_DEFAULTS)
    if unknown:
        raise ValueError(f"unknown SIPS parameters {sorted(unknown)}")
    v = dict(SIPS_DEFAULTS, **kw)
    return SipsParams(*(float(v[k]) for k in SIPS_DEFAULTS), int(NSdepth))


# SIPSternary.cpp:21-63
TERNARY_DEFAULTS = dict(Kpp=1.0, Knn=1.0, Mpp=1.0, Mnn=1.0)


class CHSim:
    """One simulation on one GPU: the Cahn-Hilliard step; with `fh`
    (make_fh_params) the variable-mobility TIPSphil step; with `sips`
    (make_sips_params) the SIPS step."""

    def __init__(self, params: Params, device: int = 0, fh: FhParams = None, sips: SipsParams = None):
        self._L = load()
        self.params = params
        h = ctypes.c_void_p()
        if fh is not None and sips is not None:
            raise ValueError("give fh or sips, not both")
        if fh is not None:
            check(self._L.mg_fh_create(ctypes.byref(params), ctypes.byref(fh), device, ctypes.byref(h)))
        elif sips is not None:
            check(self._L.mg_sips_create(ctypes.byref(params), ctypes.byref(sips), device, ctypes.byref(h)))
        else:
            check(self._L.mg_ch_create(ctypes.byref(params), device, ctypes.byref(h)))
        self._h = h

    def mobility(self) -> np.ndarray:
        """Mobility field of the last step (variable-mobility jobs)."""
        out = np.empty(self.shape, dtype=np.float64)
        check(self._L.mg_fh_mobility(self._h, _dptr(out)))
        return out

    def close(self):
        if getattr(self, "_h", None):
            self._L.mg_ch_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def shape(self):
        return _dims(self.params)

    def set_field(self, c):
        a = _f64(c, self.shape)
        check(self._L.mg_ch_set_field(self._h, _dptr(a)))

    def set_field_ptr(self, host_ptr: int):
        """Upload from a raw host pointer (e.g. pinned memory) of nx*ny*nz doubles."""
        check(self._L.mg_ch_set_field(self._h, ctypes.cast(host_ptr, ctypes.POINTER(ctypes.c_double))))

    def step(self, nsteps: int = 1):
        check(self._L.mg_ch_step(self._h, int(nsteps)))

    def sync(self, timeout_us: int = -1):
        check(self._L.mg_ch_sync(self._h, int(timeout_us)))

    def get_field(self, out=None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape, dtype=np.float64)
        check(self._L.mg_ch_get_field(self._h, _dptr(out)))
        return out

    def get_field_ptr(self, host_ptr: int):
        check(self._L.mg_ch_get_field(self._h, ctypes.cast(host_ptr, ctypes.POINTER(ctypes.c_double))))

    def write_vtk(self, path, tag="c", iskip=1, jskip=1, kskip=1):
        """Appends the current field as legacy VTK, formatted on the GPU."""
        check(self._L.mg_ch_write_vtk(self._h, str(path).encode(), tag.encode(), iskip, jskip, kskip))

    def reduce(self, allow_nonfinite: bool = False) -> dict:
        st = Stats()
        rc = self._L.mg_ch_reduce(self._h, ctypes.byref(st))
        if not (allow_nonfinite and rc == _lib.MG_ENONFINITE):
            check(rc)
        return st.as_dict()

    def structure_factor(self, nbins: int):
        k = np.zeros(nbins)
        s = np.zeros(nbins)
        k1 = ctypes.c_double()
        check(self._L.mg_ch_structure_factor(self._h, nbins, _dptr(k), _dptr(s), ctypes.byref(k1)))
        return k, s, k1.value

    @property
    def stream(self) -> int:
        return self._L.mg_ch_stream(self._h) or 0

    @property
    def steps(self) -> int:
        return self._L.mg_ch_steps(self._h)

    @property
    def tiling(self) -> Tiling:
        t = Tiling()
        check(self._L.mg_ch_get_tiling(self._h, ctypes.byref(t)))
        return t

    @tiling.setter
    def tiling(self, t):
        if not isinstance(t, Tiling):
            t = Tiling(*t)
        check(self._L.mg_ch_set_tiling(self._h, ctypes.byref(t)))


class Batch:
    """Independent simulations stepped together."""

    def __init__(self, params_list, device: int = 0):
        self._L = load()
        self.params = list(params_list)
        arr = (Params * len(self.params))(*self.params)
        h = ctypes.c_void_p()
        check(self._L.mg_batch_create(arr, len(self.params), device, ctypes.byref(h)))
        self._h = h

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def write_vtk(self, job: int, path, tag="c", iskip=1, jskip=1, kskip=1):
        """Appends job's field to `path` as legacy VTK formatted on the GPU."""
        check(self._L.mg_batch_write_vtk(self._h, job, str(path).encode(), tag.encode(), iskip, jskip, kskip))

    def close(self):
        if getattr(self, "_h", None):
            self._L.mg_batch_destroy(self._h)
            self._h = None

    __del__ = close

    def __len__(self):
        return len(self.params)

    def set_field(self, job: int, c):
        a = _f64(c, _dims(self.params[job]))
        check(self._L.mg_batch_set_field(self._h, job, _dptr(a)))

    def step(self, nsteps: int = 1):
        check(self._L.mg_batch_step(self._h, int(nsteps)))

    def sync(self, timeout_us: int = -1):
        check(self._L.mg_batch_sync(self._h, int(timeout_us)))

    def get_field(self, job: int) -> np.ndarray:
        out = np.empty(_dims(self.params[job]), dtype=np.float64)
        check(self._L.mg_batch_get_field(self._h, job, _dptr(out)))
        return out

    def autotune(self, trials: int = 5) -> dict:
        """Chooses the batch's tile targets by timing a scratch copy of the
        batch (mg_batch_autotune) and re-tiles it; the fields are kept."""
        t, p, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check(self._L.mg_batch_autotune(self._h, int(trials), ctypes.byref(t), ctypes.byref(p), ctypes.byref(ms)))
        return {"threads": t.value, "planes": p.value, "ms_per_step": ms.value}

    def reduce(self, job: int) -> dict:
        st = Stats()
        check(self._L.mg_batch_reduce(self._h, job, ctypes.byref(st)))
        return st.as_dict()

    @property
    def stream(self) -> int:
        return self._L.mg_batch_stream(self._h) or 0

    def info(self) -> dict:
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(self._L.mg_batch_info(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return {"items": a.value, "ctas": b.value, "launches_per_step": c.value}


class Ternary(Batch):
    """SIPSternary's two fields, polymer c (job 0) and non-solvent n (job 1),
    stepped as the reference's update computes them (mg_ternary_create);
    `kw` takes Kpp, Knn, Mpp, Mnn (TERNARY_DEFAULTS)."""

    def __init__(self, params: Params, device: int = 0, **kw):
        unknown = set(kw) - set(TERNARY_DEFAULTS)
        if unknown:
            raise ValueError(f"unknown SIPSternary parameters {sorted(unknown)}")
        v = dict(TERNARY_DEFAULTS, **kw)
        self._L = load()
        self.params = [params, params]
        tp = TernaryParams(*(float(v[k]) for k in TERNARY_DEFAULTS))
        h = ctypes.c_void_p()
        check(self._L.mg_ternary_create(ctypes.byref(params), ctypes.byref(tp), device, ctypes.byref(h)))
        self._h = h

    def set_fields(self, c, n):
        self.set_field(0, c)
        self.set_field(1, n)

    def get_fields(self):
        return self.get_field(0), self.get_field(1)


class Server:
    """Continuous-batching server (background thread inside the library)."""

    def __init__(self, device: int = 0, hbm_budget_gb: float = 150.0, max_jobs: int = 256,
                 steps_per_tick: int = 100):
        self._L = load()
        h = ctypes.c_void_p()
        check(self._L.mg_server_create(device, hbm_budget_gb, max_jobs, steps_per_tick, ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._L.mg_server_destroy(self._h)
            self._h = None

    __del__ = close

    def submit(self, params: Params, ic, nsteps: int) -> int:
        a = _f64(ic, _dims(params))
        jid = ctypes.c_longlong()
        check(self._L.mg_server_submit(self._h, ctypes.byref(params), _dptr(a), int(nsteps), ctypes.byref(jid)))
        return jid.value

    def poll(self, job_id: int) -> int:
        s = ctypes.c_int()
        check(self._L.mg_server_poll(self._h, job_id, ctypes.byref(s)))
        return s.value

    def result(self, job_id: int, params: Params, timeout_us: int = -1, want_field: bool = True):
        out = np.empty(_dims(params), dtype=np.float64) if want_field else None
        st = Stats()
        check(self._L.mg_server_result(self._h, job_id, int(timeout_us), _dptr(out) if want_field else None,
                                       ctypes.byref(st)))
        return out, st.as_dict()

    def stats(self) -> dict:
        st = ServerStats()
        check(self._L.mg_server_stats_get(self._h, ctypes.byref(st)))
        return st.as_dict()


def ic_generate(dims, co, amp, gaussian=False, seed=42) -> np.ndarray:
    """Seeded initial condition (reference loop order, MT19937), shape (nz, ny, nx)."""
    nx, ny, nz = dims
    out = np.empty((nz, ny, nx), dtype=np.float64)
    check(load().mg_ic_generate((ctypes.c_int * 3)(*dims), co, amp, int(bool(gaussian)), seed, _dptr(out)))
    return out


def vtk_write(path, tag, field, dims, iskip=1, jskip=1, kskip=1):
    nx, ny, nz = dims
    a = _f64(field, (nz, ny, nx))
    check(load().mg_vtk_write(str(path).encode(), tag.encode(), _dptr(a), (ctypes.c_int * 3)(*dims), iskip, jskip,
                              kskip))


def autotune(params: Params, device: int = 0, trials: int = 10):
    t = Tiling()
    ms = ctypes.c_double()
    check(load().mg_autotune(ctypes.byref(params), device, trials, ctypes.byref(t), ctypes.byref(ms)))
    return t, ms.value
