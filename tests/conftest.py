"""Shared test setup: import paths, the `gpu` marker, built libraries."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hetero-compute_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path through the C ABI")
    # Build what is missing (prebuilt .so files travel with the tree to the GPU box).
    if not os.path.exists(os.path.join(PKG, "libhc.so")):
        subprocess.run(["make", "-s", "-j8", "-C", PKG], check=True)
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True)


@pytest.fixture(scope="session")
def golden():
    import json

    import numpy as np
    gdir = os.path.join(ROOT, "tests", "golden")
    with open(os.path.join(gdir, "manifest.json")) as f:
        man = json.load(f)
    out = {}
    for name, rec in man.items():
        out[name] = (rec, dict(np.load(os.path.join(gdir, name + ".npz"))))
    return out


def make_graph(rec):
    import hc
    kind, args, wt = rec["kind"], rec["args"], rec["wtype"]
    if kind == "kronecker":
        return hc.gen_kronecker(*args, wtype=wt)
    if kind == "uniform":
        return hc.gen_uniform(*args, wtype=wt)
    return hc.gen_grid(*args, wtype=wt)
