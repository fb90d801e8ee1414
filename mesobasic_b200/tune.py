"""Builds the tiling cache shipped beside libmesogpu.so (tune_cache.json),
which mg_ch_create consults for every job whose shape and precision it
holds.  Each entry is the fastest decomposition mg_autotune measured on this
GPU for that shape.

    python -m mesobasic_b200.tune                      # every preset shape
    python -m mesobasic_b200.tune --shapes 256x256x256 --precisions fp32
    python -m mesobasic_b200.tune --out /tmp/cache.json --trials 20

Preset shapes: the grids of the benchmark workloads -- 2-D 128^2..1024^2
(the 2-D runs and the served stream), 3-D 64^3..256^3 in steps of 32 (the
batched sweep and the served stream) and 512^3 (FP32 precision study).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "tune_cache.json")

PRESET_2D = [128, 256, 512, 1024]
PRESET_3D = [64, 96, 128, 160, 192, 224, 256]


def preset(precisions):
    shapes = []
    for prec in precisions:
        shapes += [((n, n, 1), prec) for n in PRESET_2D]
        shapes += [((n, n, n), prec) for n in PRESET_3D]
        if prec == "fp32":
            shapes.append(((512, 512, 512), prec))
    return shapes


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--shapes", default=None, help="comma-separated NXxNYxNZ (default: the preset list)")
    ap.add_argument("--precisions", default="fp32,fp64")
    ap.add_argument("--trials", type=int, default=10)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--fresh", action="store_true", help="start from an empty cache file")
    a = ap.parse_args(argv)
    precs = [p for p in a.precisions.split(",") if p]
    if a.shapes:
        shapes = [(tuple(int(v) for v in s.split("x")), p) for s in a.shapes.split(",") for p in precs]
    else:
        shapes = preset(precs)
    if a.fresh and os.path.exists(a.out):
        os.remove(a.out)
    # mg_autotune writes its results into the file MG_TUNE_CACHE names
    os.environ["MG_TUNE_CACHE"] = os.path.abspath(a.out)
    import mesobasic_b200 as mb

    for dims, prec in shapes:
        p = mb.make_params(*dims, 0.005, precision=prec)
        t0 = time.perf_counter()
        t, ms = mb.autotune(p, a.device, trials=a.trials)
        sites = dims[0] * dims[1] * dims[2]
        print(json.dumps({"dims": dims, "precision": prec, "tiling": t.as_tuple(), "ms": ms,
                          "glups": sites / ms * 1e-6 if ms > 0 else None,
                          "tune_s": round(time.perf_counter() - t0, 1)}), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
