"""The oracle is pinned before it is trusted: its restatement (oracle/oracle.c)
must reproduce the reference's own CPU outputs stored in tests/golden/ (made by
tests/golden/make_golden.py from the reference compiled unchanged).  CPU only."""
import hashlib

import numpy as np
import pytest

import hc
import oracle
from conftest import make_graph


def graph_digest(g):
    h = hashlib.sha256()
    h.update(g.index.tobytes())
    h.update(g.neighbors.tobytes())
    if g.weights is not None:
        h.update(g.weights.tobytes())
    return h.hexdigest()


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


CASES = ["kron10", "kron12_ef8", "er10", "grid32", "kron16"]


@pytest.mark.parametrize("name", CASES)
def test_generator_reproduces_golden_graph(golden, name):
    rec, _ = golden[name]
    g = make_graph(rec)
    assert g.num_nodes == rec["num_nodes"] and g.num_edges == rec["num_edges"]
    assert graph_digest(g) == rec["graph_sha256"]


@pytest.mark.parametrize("name", CASES)
def test_source_picker_matches_reference(golden, name):
    rec, _ = golden[name]
    g = make_graph(rec)
    assert list(hc.pick_sources(g, len(rec["bfs_sources"]))) == rec["bfs_sources"]
    assert list(hc.pick_sources(g, len(rec["sssp_sources"]))) == rec["sssp_sources"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_bfs_depth_matches_reference(golden, name):
    rec, arr = golden[name]
    g = make_graph(rec)
    for i, s in enumerate(rec["bfs_sources"]):
        d = oracle.bfs_depth(g.index, g.neighbors, s)
        assert digest(d) == rec["bfs_depth_sha256"][i]
        if "bfs_parents" in arr:
            bad, counts = oracle.verify_bfs_parents(g.index, g.neighbors, d, arr["bfs_parents"][i], s)
            assert bad == 0, counts
        if "bfs_depth_i8" in arr:
            assert (d.astype(np.int8) == arr["bfs_depth_i8"][i]).all()


@pytest.mark.parametrize("name", CASES)
def test_oracle_dijkstra_matches_reference(golden, name):
    rec, arr = golden[name]
    g = make_graph(rec)
    for i, s in enumerate(rec["sssp_sources"]):
        d = oracle.sssp_dijkstra(g.index, g.neighbors, g.weights, s)
        assert digest(d) == rec["sssp_dist_sha256"][i]


@pytest.mark.parametrize("name", CASES)
def test_oracle_pagerank_matches_reference(golden, name):
    rec, arr = golden[name]
    g = make_graph(rec)
    s, it = oracle.pr_pull(g.index, g.neighbors)
    # Same float operations in the same order as the reference on one thread.
    assert np.array_equal(s, arr["pr_scores"]), np.abs(s - arr["pr_scores"]).max()


@pytest.mark.parametrize("name", ["kron10", "er10", "grid32"])
def test_fp64_fixed_point_close_to_reference(golden, name):
    rec, arr = golden[name]
    g = make_graph(rec)
    x, _ = oracle.pr_jacobi_f64(g.index, g.neighbors)
    # The reference stops once no vertex moves by more than 5e-8 in a sweep;
    # that leaves it a few 1e-6 (L-inf) from the fixed point on these graphs.
    err = np.abs(x - arr["pr_scores"]).max()
    assert err < 1e-5, err


def test_oracle_detects_planted_errors(golden):
    """Mistakes planted in outputs handed to the checker must be caught."""
    rec, arr = golden["kron10"]
    g = make_graph(rec)
    s = rec["bfs_sources"][0]
    d = oracle.bfs_depth(g.index, g.neighbors, s)
    par = arr["bfs_parents"][0].copy()
    v = int(np.flatnonzero((d > 1))[0])
    par[v] = s  # the source is not at depth d[v] - 1
    assert oracle.verify_bfs_parents(g.index, g.neighbors, d, par, s)[0] > 0
    par = arr["bfs_parents"][0].copy()
    par[v] = -1
    assert oracle.verify_bfs_parents(g.index, g.neighbors, d, par, s)[0] > 0
    dist = oracle.sssp_dijkstra(g.index, g.neighbors, g.weights, s)
    bad = np.full(g.num_nodes, -1, dtype=np.int32)
    bad[s] = s
    assert oracle.verify_sp_tree(g.index, g.neighbors, g.weights, dist, bad, s) > 0


def test_dense_adjoint_matches_finite_differences():
    """FP64 references for the adjoint (no reference counterpart) agree with central differences."""
    rng = np.random.default_rng(0)
    g = hc.gen_kronecker(6, 4, 11, wtype=hc.W_F32)
    n = g.num_nodes
    c = rng.standard_normal(n)
    t = rng.random(n)
    t /= t.sum()
    x, dt, dw = oracle.pr_dense_grad(g.index, g.neighbors, c, g.weights.astype(np.float64), t)
    h = 1e-6
    for j in rng.choice(n, 5, replace=False):
        tp, tm = t.copy(), t.copy()
        tp[j] += h
        tm[j] -= h
        fd = (c @ oracle.pr_dense(g.index, g.neighbors, g.weights.astype(np.float64), tp) -
              c @ oracle.pr_dense(g.index, g.neighbors, g.weights.astype(np.float64), tm)) / (2 * h)
        assert abs(fd - dt[j]) < 1e-6 * max(1.0, abs(fd))
    w = g.weights.astype(np.float64)
    for e in rng.choice(g.num_edges, 5, replace=False):
        wp, wm = w.copy(), w.copy()
        wp[e] += h
        wm[e] -= h
        fd = (c @ oracle.pr_dense(g.index, g.neighbors, wp, t) - c @ oracle.pr_dense(g.index, g.neighbors, wm, t)) / (2 * h)
        assert abs(fd - dw[e]) < 1e-6 * max(1.0, abs(fd))
