"""ctypes binding of libmesogpu.so (the C ABI declared in include/mesogpu.h).

This is the binding a Python caller of the reference's phase-field plugin
would write; it adds no computation of its own.  Loading fails loudly when
the library has not been built: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmesogpu.so")

MG_OK = 0
MG_EINVAL = -1
MG_ENOMEM = -2
MG_ECUDA = -3
MG_ETIMEOUT = -4
MG_ENONFINITE = -5
MG_EDEVICE = -6
MG_ENOTFOUND = -7

MG_FP64 = 0
MG_FP32 = 1

MG_JOB_QUEUED, MG_JOB_RUNNING, MG_JOB_DONE, MG_JOB_FAILED = 0, 1, 2, 3

ERROR_NAMES = {MG_EINVAL: "MG_EINVAL", MG_ENOMEM: "MG_ENOMEM", MG_ECUDA: "MG_ECUDA",
               MG_ETIMEOUT: "MG_ETIMEOUT", MG_ENONFINITE: "MG_ENONFINITE", MG_EDEVICE: "MG_EDEVICE",
               MG_ENOTFOUND: "MG_ENOTFOUND"}


class Params(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("dt", ctypes.c_double), ("M", ctypes.c_double), ("kappa", ctypes.c_double),
                ("bx", ctypes.c_int), ("by", ctypes.c_int), ("bz", ctypes.c_int),
                ("precision", ctypes.c_int), ("mass_correct", ctypes.c_int),
                ("noise", ctypes.c_double), ("noise_seed", ctypes.c_ulonglong)]


class FhParams(ctypes.Structure):
    _fields_ = [("alpha", ctypes.c_double), ("beta", ctypes.c_double), ("N", ctypes.c_double), ("A", ctypes.c_double),
                ("Tinit", ctypes.c_double), ("Tbath", ctypes.c_double), ("Tcrystal", ctypes.c_double),
                ("nu", ctypes.c_double), ("gamma", ctypes.c_double), ("D0", ctypes.c_double),
                ("Mweight", ctypes.c_double), ("Mvolume", ctypes.c_double), ("nstep", ctypes.c_longlong),
                ("bath", ctypes.c_int), ("thermCond", ctypes.c_double)]


class SipsParams(ctypes.Structure):
    _fields_ = [("N", ctypes.c_double), ("A", ctypes.c_double), ("Tinit", ctypes.c_double),
                ("chiPS", ctypes.c_double), ("chiPN", ctypes.c_double), ("chiCond", ctypes.c_double),
                ("phiCutoff", ctypes.c_double), ("nu", ctypes.c_double), ("gamma", ctypes.c_double),
                ("D0", ctypes.c_double), ("Mweight", ctypes.c_double), ("Mvolume", ctypes.c_double),
                ("NSdepth", ctypes.c_int)]


class TernaryParams(ctypes.Structure):
    _fields_ = [("Kpp", ctypes.c_double), ("Knn", ctypes.c_double), ("Mpp", ctypes.c_double),
                ("Mnn", ctypes.c_double)]


class Stats(ctypes.Structure):
    _fields_ = [("mass", ctypes.c_double), ("energy", ctypes.c_double), ("abs_mass", ctypes.c_double),
                ("max_abs", ctypes.c_double), ("nonfinite", ctypes.c_longlong), ("step", ctypes.c_longlong)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tiling(ctypes.Structure):
    _fields_ = [("ty", ctypes.c_int), ("nchunk", ctypes.c_int), ("nbuf", ctypes.c_int), ("path", ctypes.c_int)]

    def as_tuple(self):
        return (self.ty, self.nchunk, self.nbuf, self.path)


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("failed", ctypes.c_longlong), ("running", ctypes.c_longlong), ("queued", ctypes.c_longlong),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("sims_per_hour", ctypes.c_double), ("site_updates_per_s", ctypes.c_double),
                ("hbm_in_use_gb", ctypes.c_double), ("hbm_peak_gb", ctypes.c_double),
                ("step_s", ctypes.c_double), ("admit_s", ctypes.c_double), ("retire_s", ctypes.c_double),
                ("ticks", ctypes.c_longlong), ("rebuilds", ctypes.c_longlong), ("refreshes", ctypes.c_longlong),
                ("sat_site_updates_per_s", ctypes.c_double), ("sat_ticks", ctypes.c_longlong),
                ("gpu_s", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_P = ctypes.POINTER
_vp = ctypes.c_void_p
_dp = _P(ctypes.c_double)
_i3 = ctypes.c_int * 3

# name: (restype, argtypes)
SIGNATURES = {
    "mg_last_error": (ctypes.c_char_p, []),
    "mg_ch_create": (ctypes.c_int, [_P(Params), ctypes.c_int, _P(_vp)]),
    "mg_ch_set_field": (ctypes.c_int, [_vp, _dp]),
    "mg_ch_step": (ctypes.c_int, [_vp, ctypes.c_int]),
    "mg_ch_sync": (ctypes.c_int, [_vp, ctypes.c_longlong]),
    "mg_ch_get_field": (ctypes.c_int, [_vp, _dp]),
    "mg_ch_reduce": (ctypes.c_int, [_vp, _P(Stats)]),
    "mg_ch_write_vtk": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "mg_ch_structure_factor": (ctypes.c_int, [_vp, ctypes.c_int, _dp, _dp, _dp]),
    "mg_ch_stream": (_vp, [_vp]),
    "mg_ch_field_device": (_vp, [_vp]),
    "mg_ch_steps": (ctypes.c_longlong, [_vp]),
    "mg_ch_get_tiling": (ctypes.c_int, [_vp, _P(Tiling)]),
    "mg_ch_set_tiling": (ctypes.c_int, [_vp, _P(Tiling)]),
    "mg_ch_destroy": (None, [_vp]),
    "mg_fh_create": (ctypes.c_int, [_P(Params), _P(FhParams), ctypes.c_int, _P(_vp)]),
    "mg_fh_mobility": (ctypes.c_int, [_vp, _dp]),
    "mg_sips_create": (ctypes.c_int, [_P(Params), _P(SipsParams), ctypes.c_int, _P(_vp)]),
    "mg_ternary_create": (ctypes.c_int, [_P(Params), _P(TernaryParams), ctypes.c_int, _P(_vp)]),
    "mg_autotune": (ctypes.c_int, [_P(Params), ctypes.c_int, ctypes.c_int, _P(Tiling), _dp]),
    "mg_ic_generate": (ctypes.c_int, [_i3, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_uint, _dp]),
    "mg_vtk_write": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, _dp, _i3, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int]),
    "mg_batch_create": (ctypes.c_int, [_P(Params), ctypes.c_int, ctypes.c_int, _P(_vp)]),
    "mg_batch_set_field": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "mg_batch_step": (ctypes.c_int, [_vp, ctypes.c_int]),
    "mg_batch_sync": (ctypes.c_int, [_vp, ctypes.c_longlong]),
    "mg_batch_get_field": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "mg_batch_reduce": (ctypes.c_int, [_vp, ctypes.c_int, _P(Stats)]),
    "mg_batch_write_vtk": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int]),
    "mg_batch_stream": (_vp, [_vp]),
    "mg_batch_info": (ctypes.c_int, [_vp, _P(ctypes.c_int), _P(ctypes.c_int), _P(ctypes.c_int)]),
    "mg_batch_destroy": (None, [_vp]),
    "mg_batch_autotune": (ctypes.c_int, [_vp, ctypes.c_int, _P(ctypes.c_int), _P(ctypes.c_int), _P(ctypes.c_double)]),
    "mg_server_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, _P(_vp)]),
    "mg_server_submit": (ctypes.c_int, [_vp, _P(Params), _dp, ctypes.c_longlong, _P(ctypes.c_longlong)]),
    "mg_server_poll": (ctypes.c_int, [_vp, ctypes.c_longlong, _P(ctypes.c_int)]),
    "mg_server_result": (ctypes.c_int, [_vp, ctypes.c_longlong, ctypes.c_longlong, _dp, _P(Stats)]),
    "mg_server_stats_get": (ctypes.c_int, [_vp, _P(ServerStats)]),
    "mg_server_destroy": (None, [_vp]),
    "mg_field_stats_noalloc": (ctypes.c_int, [_vp, _P(Params), ctypes.c_int, _vp, ctypes.c_longlong, _P(Stats)]),
}


class MGError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {message}")
        self.code = code


_lib = None


def load() -> ctypes.CDLL:
    """Loads libmesogpu.so; raises if it is missing (build it first)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built: run `python -m mesobasic_b200.build` "
                          "(the GPU path has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> int:
    if rc != MG_OK:
        msg = load().mg_last_error()
        raise MGError(rc, msg.decode() if msg else "")
    return rc
