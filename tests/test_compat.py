"""The reference-shaped C++ API (include/hc_compat.hpp) over the C ABI."""
import os
import subprocess

import numpy as np
import pytest

import hc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_compat(tmp_path):
    exe = str(tmp_path / "compat_verify")
    pkg = os.path.join(ROOT, "hetero-compute_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "compat", "compat_verify.cpp"), "-L", pkg, "-lhc",
                    f"-Wl,-rpath,{pkg}", "-o", exe], check=True)
    return exe


def test_compat_header_builds_and_links(tmp_path):
    assert os.path.exists(build_compat(tmp_path))


@pytest.mark.gpu
def test_compat_drivers_verify(tmp_path):
    exe = build_compat(tmp_path)
    g = hc.gen_kronecker(12, 16, 2, wtype=hc.W_I32)
    sg, wsg = str(tmp_path / "g.sg"), str(tmp_path / "g.wsg")
    hc.write_graph(sg, hc.HostCSR(g.index, g.neighbors))
    hc.write_graph(wsg, g)
    r = subprocess.run([exe, sg, wsg], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("success") == 3 + 3 + 4 + 4
