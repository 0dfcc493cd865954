"""Graphs built on the device (hc_graph_generate) equal the host generator's CSR and the numpy
restatement's (oracle/gen.py) bit for bit, and the device source picker draws the host picker's sources."""
import hashlib

import numpy as np
import pytest

import hc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,scale,ef,wtype", [
    (hc.GEN_KRONECKER, 10, 16, hc.W_NONE),
    (hc.GEN_KRONECKER, 12, 16, hc.W_I32),
    (hc.GEN_KRONECKER, 11, 8, hc.W_F32),
    (hc.GEN_UNIFORM, 12, 8, hc.W_I32),
    (hc.GEN_KRONECKER, 16, 16, hc.W_I32),  # rows of a few thousand entries
])
def test_device_build_equals_host_build(kind, scale, ef, wtype):
    gen = hc.gen_kronecker if kind == hc.GEN_KRONECKER else hc.gen_uniform
    host = gen(scale, ef, 3, wtype=wtype)
    g = hc.Graph.generate(kind, scale, ef, 3, wtype)
    index, nbr, w = g.csr()
    assert g.num_nodes == host.num_nodes and g.num_edges == host.num_edges
    assert np.array_equal(index, host.index)
    assert np.array_equal(nbr, host.neighbors)
    if wtype == hc.W_NONE:
        assert w is None
    else:
        assert w.dtype == host.weights.dtype and np.array_equal(w.view(np.uint32), host.weights.view(np.uint32))
    assert np.array_equal(g.pick_sources(16), hc.pick_sources(host, 16))
    info = g.info()
    assert info.degree_sorted == 1


@pytest.mark.parametrize("kind,scale,ef,seed,wtype", [
    (hc.GEN_KRONECKER, 13, 16, 5, hc.W_I32), (hc.GEN_UNIFORM, 13, 8, 6, hc.W_F32),
    (hc.GEN_KRONECKER, 20, 16, 1, hc.W_I32)])
def test_device_build_equals_numpy_restatement(kind, scale, ef, seed, wtype):
    """The device builder against the independent numpy restatement of the construction (oracle/gen.py),
    up to scale 20 (33 M directed edges)."""
    from oracle import gen
    idx, nbr, w = gen.build("kronecker" if kind == hc.GEN_KRONECKER else "uniform", scale, ef, seed, wtype)
    g = hc.Graph.generate(kind, scale, ef, seed, wtype)
    index, neighbors, weights = g.csr()
    assert np.array_equal(index, idx) and np.array_equal(neighbors, nbr)
    assert np.array_equal(weights.view(np.uint32), np.asarray(w).view(np.uint32))


def test_device_build_repeatable_and_usable():
    """Two device builds agree (no dependence on atomic ordering), and the handle runs BFS like a host upload."""
    a = hc.Graph.generate(hc.GEN_KRONECKER, 14, 16, 7, hc.W_I32)
    b = hc.Graph.generate(hc.GEN_KRONECKER, 14, 16, 7, hc.W_I32)
    digest = [hashlib.sha256(np.concatenate([x.view(np.uint8) for x in g.csr()])).hexdigest() for g in (a, b)]
    assert digest[0] == digest[1]
    host = hc.gen_kronecker(14, 16, 7, wtype=hc.W_I32)
    hg = hc.Graph.from_host(host)
    src = a.pick_sources(4)
    da, _, _ = a.bfs(src)
    dh, _, _ = hg.bfs(src)
    assert np.array_equal(da, dh)


def test_device_build_rejects_bad_arguments():
    with pytest.raises(hc.HCError) as e:
        hc.Graph.generate(hc.GEN_KRONECKER, 0, 16)
    assert e.value.status == hc.INVALID_ARG
    with pytest.raises(hc.HCError) as e:
        hc.Graph.generate(7, 10, 16)
    assert e.value.status == hc.INVALID_ARG
