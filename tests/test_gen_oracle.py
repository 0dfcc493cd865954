"""The graph generators are pinned by an independent restatement
(oracle/gen.py, whole-array numpy) of the construction the reference's gapbs
adapters describe (src/gapbs/generator.h:53-165, src/gapbs/builder.h:141-186,
:366-406): R-MAT / uniform endpoints, symmetrisation, self-loop and duplicate
removal keeping the lightest weight, relabelling by (degree desc, id desc),
sorted rows.  The library's host builder (and, on the GPU, its device builder,
tests/test_gpu_build.py) must produce the same CSR bit for bit.  CPU only."""
import hashlib
import os

import numpy as np
import pytest

import hc
from oracle import gen


def _same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("kind,scale,factor,seed,wtype", [
    ("kronecker", 10, 16, 1, hc.W_I32), ("kronecker", 12, 8, 7, hc.W_I32), ("kronecker", 13, 16, 2, hc.W_NONE),
    ("kronecker", 11, 8, 3, hc.W_F32), ("uniform", 10, 8, 3, hc.W_I32), ("uniform", 12, 4, 9, hc.W_F32),
    ("kronecker", 16, 16, 1, hc.W_I32), ("kronecker", 3, 2, 5, hc.W_I32)])
def test_library_generator_matches_numpy_restatement(kind, scale, factor, seed, wtype):
    idx, nbr, w = gen.build(kind, scale, factor, seed, wtype)
    h = hc.gen_kronecker(scale, factor, seed, wtype) if kind == "kronecker" else hc.gen_uniform(scale, factor, seed,
                                                                                              wtype)
    assert _same(idx, h.index) and _same(nbr, h.neighbors)
    if wtype == hc.W_NONE:
        assert w is None and h.weights is None
    else:
        assert _same(np.asarray(w).view(np.uint32), h.weights.view(np.uint32))


def test_restatement_properties():
    """Properties the construction promises, on the restatement itself: symmetric, no self-loops, no
    duplicates, sorted rows, degrees non-increasing, the lighter weight of a duplicate pair kept."""
    idx, nbr, w = gen.build("kronecker", 12, 16, 4, gen.W_I32)
    n = len(idx) - 1
    deg = np.diff(idx)
    assert (deg[:-1] >= deg[1:]).all()
    src = np.repeat(np.arange(n), deg)
    assert (src != nbr).all()
    key = src.astype(np.int64) * n + nbr
    assert (np.diff(key) > 0).all()  # rows sorted, no duplicate
    rev = nbr.astype(np.int64) * n + src
    pos = np.searchsorted(key, rev)
    assert (key[pos] == rev).all() and (w[pos] == w).all()  # every edge has its reverse, same weight
    assert w.min() >= 1 and w.max() <= 255


def test_written_files_load_in_the_library(tmp_path):
    idx, nbr, w = gen.build("kronecker", 10, 8, 2, gen.W_I32)
    sg, wsg = os.path.join(tmp_path, "g.sg"), os.path.join(tmp_path, "g.wsg")
    gen.write_graph(sg, idx, nbr)
    gen.write_graph(wsg, idx, nbr, w)
    a = hc.read_graph(sg)
    b = hc.read_graph(wsg, weighted=2)
    assert _same(a.index, idx) and _same(a.neighbors, nbr) and a.weights is None
    assert _same(b.neighbors, nbr) and _same(b.weights, w)
    # byte-identical to the library's writer
    hsg, hwsg = os.path.join(tmp_path, "h.sg"), os.path.join(tmp_path, "h.wsg")
    hc.write_graph(hsg, hc.HostCSR(idx, nbr))
    hc.write_graph(hwsg, hc.HostCSR(idx, nbr, w))
    for x, y in ((sg, hsg), (wsg, hwsg)):
        assert hashlib.sha256(open(x, "rb").read()).digest() == hashlib.sha256(open(y, "rb").read()).digest()
