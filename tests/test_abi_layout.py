"""The ctypes mirrors of the C ABI's structs (mesobasic_b200/_lib.py) have the
layout include/mesogpu.h gives them: a small C program compiled against the
header prints each struct's size and each field's offset, and every ctypes
field must sit at the same offset.  A field added on one side only would
otherwise make the library write past (or short of) the caller's struct."""
import ctypes
import os
import shutil
import subprocess

import pytest

from mesobasic_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "mg_ch_params": _lib.Params,
    "mg_ch_stats": _lib.Stats,
    "mg_tiling": _lib.Tiling,
    "mg_fh_params": _lib.FhParams,
    "mg_sips_params": _lib.SipsParams,
    "mg_ternary_params": _lib.TernaryParams,
    "mg_server_stats": _lib.ServerStats,
}


def c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "mesogpu.h"', "int main(void) {"]
    for cname, cls in STRUCTS.items():
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'    printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", f"-I{os.path.join(ROOT, 'include')}", str(src), "-o", str(exe)], check=True,
                   capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        name, key, val = line.split()
        got[(name, key)] = int(val)
    return got


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not found")
def test_ctypes_structs_match_the_header(tmp_path):
    got = c_layout(tmp_path)
    for cname, cls in STRUCTS.items():
        assert ctypes.sizeof(cls) == got[(cname, "size")], f"{cname}: size"
        for field, _ in cls._fields_:
            assert getattr(cls, field).offset == got[(cname, field)], f"{cname}.{field}: offset"
