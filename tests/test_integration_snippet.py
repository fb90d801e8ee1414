"""The reference-side plugin shown in INTEGRATION.md compiles against the
reference's own headers (PFBaseClass.hpp, CommonParams.h, GetPot) and this
repository's include/mesogpu.h, and links against libmesogpu.so.  CPU only;
skipped where the reference sources are not present."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE_SRC = "/root/reference/src"


def snippet():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, re.S)
    code = [b for b in blocks if "class CHBasicGPU" in b]
    assert len(code) == 1
    return code[0]


@pytest.mark.skipif(not os.path.isdir(REFERENCE_SRC), reason="reference sources not present")
def test_plugin_snippet_compiles_against_reference_headers(tmp_path):
    from mesobasic_b200 import build
    lib = build.build()
    hdr = tmp_path / "CHBasicGPU.hpp"
    hdr.write_text(snippet())
    main = tmp_path / "use.cpp"
    main.write_text('#include "CHBasicGPU.hpp"\n'
                    "PFBaseClass* make(const CommonParams& p, const GetPot& in) { return new CHBasicGPU(p, in); }\n"
                    "int main() { return 0; }\n")
    pftypes = os.path.join(REFERENCE_SRC, "phase_field", "PFTypes")
    cmd = ["g++", "-std=c++17", "-w", f"-I{tmp_path}", f"-I{os.path.join(ROOT, 'include')}",
           f"-I{os.path.join(ROOT, 'oracle', 'shim')}", f"-I{pftypes}", str(main), "-o", str(tmp_path / "use"),
           f"-L{os.path.dirname(lib)}", "-lmesogpu", f"-Wl,-rpath,{os.path.dirname(lib)}"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
