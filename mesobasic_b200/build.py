"""Builds libmesogpu.so (sm_100a) and the meso_b200 driver in-tree.

    python -m mesobasic_b200.build            # library + driver
    python -m mesobasic_b200.build --verbose  # also prints ptxas register/smem usage

nvcc cross-compiles for sm_100a without a GPU.  Objects go to _build/ at the
repository root; the shared library and driver land next to this file so they
travel with the package.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libmesogpu.so")
DRIVER = os.path.join(PKG, "meso_b200")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["engine.cu", "march_f32.cu", "march_f64.cu", "capi.cu", "server.cu", "noalloc.cu", "vtk_device.cu"]
CPP_SOURCES = ["host_io.cpp"]
HEADERS = ["ch_device.cuh", "ch_kernels.cuh", "ch_lean.cuh", "ch_march.cuh", "ch_march2.cuh", "fh_march.cuh", "ch_types.h", "mg_device.cuh", "engine.h"]
DRIVER_SOURCES = ["input_file.cpp", "pf_model.cpp", "chbasic_gpu.cpp", "tipsphil_gpu.cpp", "sips_gpu.cpp", "meso_b200.cpp"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str], verbose: bool) -> str:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    return r.stdout + r.stderr


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "mesogpu.h")]
    objs = []
    jobs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + headers):
            flags = [NVCC, *ARCH, "-Xptxas=-v", "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                     f"-I{INCLUDE}", f"-I{CSRC}", "-c", s, "-o", o]
            jobs.append((src, flags))

    def compile_one(job):
        src, flags = job
        import time
        t0 = time.time()
        out = _run(flags, verbose)
        # stamp the object with the time its compile started: a source or
        # header edited while it compiled stays newer, so it is rebuilt
        os.utime(flags[flags.index("-o") + 1], (t0, t0))
        with open(os.path.join(BUILD, src + ".ptxas.txt"), "w") as f:  # registers / spills per kernel
            f.write(out)
        return out

    # the translation units compile independently: run them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for out in ex.map(compile_one, jobs):
            if verbose and out:
                print(out)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + headers):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", f"-I{INCLUDE}",
                  "-c", s, "-o", o], verbose)
    if force or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, f"-L{CUDA_HOME}/lib64", "-lcufft",
              f"-Xlinker=-rpath,{CUDA_HOME}/lib64"], verbose)
    # host driver (reference input file -> GPU plugin -> VTK output)
    dsrcs = [os.path.join(HOST, s) for s in DRIVER_SOURCES]
    if all(os.path.exists(s) for s in dsrcs):
        dhdrs = [os.path.join(HOST, h) for h in os.listdir(HOST) if h.endswith(".hpp")]
        if force or _newer(DRIVER, dsrcs + dhdrs + [LIB, os.path.join(INCLUDE, "mesogpu.h")]):
            _run(["g++", "-O2", "-std=c++17", "-Wall", "-ffp-contract=off", f"-I{INCLUDE}", f"-I{HOST}",
                  *dsrcs, "-o", DRIVER, f"-L{PKG}", "-lmesogpu", "-Wl,-rpath,$ORIGIN", "-lpthread"], verbose)
    return LIB


def clean() -> None:
    shutil.rmtree(BUILD, ignore_errors=True)
    for p in (LIB, DRIVER):
        if os.path.exists(p):
            os.remove(p)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--clean", action="store_true")
    args = ap.parse_args()
    if args.clean:
        clean()
    print(build(verbose=args.verbose, force=args.force))
