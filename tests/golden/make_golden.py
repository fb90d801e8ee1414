"""Generates the golden fixtures in this directory from the REFERENCE CPU
build (oracle/_ref: the reference's own SfieldFD, Rand, PFApp and
MesoExecute sources compiled with the CHBasic model).

    make -C oracle ref && python tests/golden/make_golden.py

Needs the reference sources; the fixtures it writes are committed, so the
tests never need them.  Every case records its parameters beside the arrays.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

# name, dims, spacing, dt, M, kap, bc, co, amp, gaussian, seed, steps to record
CASES = [
    ("ch3d_24x20x16", (24, 20, 16), (1.0, 1.0, 1.0), 0.005, 1.0, 1.0, (1, 1, 1), 0.0, 0.1, False, 42, (1, 10, 100)),
    ("ch2d_64x48", (64, 48, 1), (1.0, 1.0, 1.0), 0.01, 1.0, 1.0, (1, 1, 1), 0.0, 0.2, False, 42, (1, 100)),
    ("ch3d_odd_5x7x3", (5, 7, 3), (0.9, 1.1, 1.3), 0.001, 1.3, 1.5, (1, 1, 1), 0.1, 0.2, False, 7, (1, 60)),
    ("ch3d_noflux_12x10x6", (12, 10, 6), (1.0, 1.0, 1.0), 0.004, 1.0, 1.0, (1, 0, 0), 0.0, 0.2, False, 3, (1, 40)),
    ("ch3d_gauss_32x16x8", (32, 16, 8), (1.0, 1.0, 1.0), 0.005, 1.0, 1.5, (1, 1, 1), 0.3, 0.02, True, 42, (1, 100)),
    ("ch2d_noflux_32x20", (32, 20, 1), (0.5, 0.5, 1.0), 0.0004, 1.0, 0.8, (0, 1, 1), -0.1, 0.3, False, 11, (1, 50)),
]

VTK_INPUT = """[Domain]
    nx = 8
    ny = 6
    nz = 4
    dx = 1
    dy = 1
    dz = 1
[]

[Time]
    nstep = 4
    dt = 0.01
[]

[Output]
    numOutputs = 2
    iskip = 2
    jskip = 1
    kskip = 1
[]

[PFApp]
    app = true
    type = CHBasic
    co = 0.1
    M = 1.0
    kap = 1.0
    noise_amp = 0.2
    seed = 5
[]
"""


def main() -> None:
    if not O.ref_available():
        O.build(reference=True)
    index = {}
    for (name, dims, sp, dt, M, kap, bc, co, amp, gauss, seed, rec) in CASES:
        ic = O.ref_ic(dims, co, amp, gauss, seed)
        arrays = {"ic": ic}
        prev, c = 0, ic
        for s in rec:
            c = O.ref_run(c, dims, sp, dt, M, kap, s - prev, bc)
            arrays[f"step{s}"] = c
            prev = s
        meta = dict(dims=dims, spacing=sp, dt=dt, M=M, kap=kap, bc=bc, co=co, amp=amp, gaussian=gauss, seed=seed,
                    steps=list(rec))
        np.savez(os.path.join(HERE, f"{name}.npz"), meta=json.dumps(meta), **arrays)
        index[name] = meta
    # MT19937 outputs of the reference Rand class, read back through the
    # reference IC with co = 0.5, amp = 1 (c = u up to one rounding of u - 0.5,
    # far below the 1/4294967295 spacing): u32 = round(c * 4294967295)
    mt = {}
    for seed in (42, 5489):
        u = O.ref_ic((16, 1, 1), 0.5, 1.0, False, seed).ravel()
        mt[str(seed)] = [int(round(v * 4294967295.0)) for v in u]
    index["mt19937_first16"] = mt
    index["mt19937_5489_10000th"] = 4123659995  # the C++ standard's known answer for std::mt19937
    # legacy VTK written by the reference driver (MesoExecute + PFApp + SfieldFD::writeVTKFile)
    tmp = tempfile.mkdtemp()
    try:
        with open(os.path.join(tmp, "input.dat"), "w") as f:
            f.write(VTK_INPUT)
        subprocess.run([O.REF_MESO], cwd=tmp, check=True, capture_output=True)
        out = os.path.join(HERE, "vtk_ref")
        shutil.rmtree(out, ignore_errors=True)
        shutil.copytree(os.path.join(tmp, "vtkoutput"), out)
        with open(os.path.join(out, "input.dat"), "w") as f:
            f.write(VTK_INPUT)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
