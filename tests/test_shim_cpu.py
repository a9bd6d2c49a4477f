"""The Neumann() drop-in shims (doi_b200/shim/) compile against the reference packages' own headers and the
library header, as a maintainer would build them in place of neumann.cu.  Compiled as host C++ with the
same host-emulation headers oracle/build.sh uses for the reference sources; skipped where the reference
tree is absent.  (The GPU test tests/test_gpu_cli.py::test_reference_main_with_library_neumann runs the
reference's forward main linked with the FisherInfo_IO shim.)"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("RTE_REFERENCE_DIR", os.path.join(os.path.dirname(ROOT), "reference"))


@pytest.mark.parametrize("shim,package", [("neumann_b200.cu", "FisherInfo_IO/src"),
                                          ("neumann_b200_gpu_package.cu", "GPU package/src")])
def test_shim_compiles_against_reference_headers(shim, package):
    inc = os.path.join(REF, package)
    if not os.path.isdir(inc):
        pytest.skip("reference tree not present")
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no g++")
    cmd = [cxx, "-fsyntax-only", "-std=c++17", "-fopenmp", "-Wall", "-Wno-unknown-pragmas", "-x", "c++",
           "-D__CUDACC__", "-include", os.path.join(ROOT, "oracle", "ref", "fim_emu.h"),
           "-I", os.path.join(ROOT, "oracle", "ref", "include"), "-I", inc, "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "doi_b200", "shim", shim)]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    assert r.returncode == 0, r.stdout[-3000:]
    # warnings from the shim itself (not from the reference headers it includes) would show its own file
    own = [ln for ln in r.stdout.splitlines() if shim in ln and "warning" in ln]
    assert not own, own
