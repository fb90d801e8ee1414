"""The drop-in plugin header (mesobasic_b200/plugin/CHBasicGPU.hpp) compiles
against the reference's own headers (PFBaseClass.hpp, CommonParams.h, GetPot)
and this repository's include/mesogpu.h, and links against libmesogpu.so.
CPU only; skipped where the reference checkout is not found ($MESO_REFERENCE,
or a checkout named `reference` beside this repository).  The GPU test
tests/test_gpu_reference_driver.py runs the same header inside the
reference's driver."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PLUGIN = os.path.join(ROOT, "mesobasic_b200", "plugin")


def reference_src():
    import oracle
    return oracle.reference_src()


def test_plugin_header_compiles_against_reference_headers(tmp_path):
    ref = reference_src()
    if ref is None:
        pytest.skip("reference checkout not found (set MESO_REFERENCE)")
    from mesobasic_b200 import build
    lib = build.build()
    main = tmp_path / "use.cpp"
    main.write_text('#include "CHBasicGPU.hpp"\n'
                    "PFBaseClass* make(const CommonParams& p, const GetPot& in) { return new CHBasicGPU(p, in); }\n"
                    "int main() { return 0; }\n")
    pftypes = os.path.join(ref, "src", "phase_field", "PFTypes")
    cmd = ["g++", "-std=c++17", "-w", f"-I{PLUGIN}", f"-I{os.path.join(ROOT, 'include')}",
           f"-I{os.path.join(ROOT, 'oracle', 'shim')}", f"-I{pftypes}", str(main), "-o", str(tmp_path / "use"),
           f"-L{os.path.dirname(lib)}", "-lmesogpu", f"-Wl,-rpath,{os.path.dirname(lib)}"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]


def test_reference_driver_with_plugin_is_built():
    """The oracle recipe links the reference driver with the plugin
    registered (oracle/_ref/meso_ref_gpu) wherever the reference is built."""
    import oracle
    if not os.path.exists(oracle.REF_MESO):
        pytest.skip("reference build not present (make -C oracle ref)")
    assert os.path.exists(oracle.REF_MESO_GPU), "make -C oracle ref-gpu did not run"
    out = subprocess.run(["nm", "-C", oracle.REF_MESO_GPU], capture_output=True, text=True).stdout
    assert "CHBasicGPU" in out and "mg_ch_create" in out
