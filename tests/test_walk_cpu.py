"""The exact path walks of the pair kernels (doi_b200/csrc/rte_walk.cuh), built for the host with g++ and
checked bit for bit: the FP32-parameter walk against the integer-parameter walk, and the walk clipped to
the support box of a perturbation (the tangent kernel's) against the whole walk.  Runs on the CPU."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "doi_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_walks_are_exact(tmp_path):
    exe = str(tmp_path / "walk_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, os.path.join(HERE, "walk_check.cpp"), "-o", exe],
                   check=True)
    out = subprocess.run([exe], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    fields = out.stdout.split()
    pairs, nonzero, bad = int(fields[1]), int(fields[3]), int(fields[5])
    assert pairs == 200000 and nonzero > 20000 and bad == 0, out.stdout
