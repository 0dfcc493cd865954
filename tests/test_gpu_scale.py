"""Parity at the benchmark's own size: Kronecker scale 22 (4.2 M vertices, 128 M directed edges), built on
the device, BFS / SSSP / PageRank checked against the oracle for SourcePicker sources; batched BFS / SSSP
columns sampled at scale 20.  (bench.py checks the same configuration against the reference's own outputs
after its timed region.)"""
import numpy as np
import pytest

import hc
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big():
    g = hc.Graph.generate(hc.GEN_KRONECKER, 22, 16, 1, hc.W_I32)
    index, nbr, w = g.csr()
    return g, index, nbr, w


def test_scale22_bfs_sssp_against_oracle(big):
    g, index, nbr, w = big
    src = g.pick_sources(2)
    depth, parent, _ = g.bfs(src)
    dist, sparent, _ = g.sssp(src, want_parent=True)
    for i, s in enumerate(src):
        d = oracle.bfs_depth(index, nbr, s)
        assert np.array_equal(depth[i], d)
        assert oracle.verify_bfs_parents(index, nbr, d, parent[i], s)[0] == 0
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(index, nbr, w, s))
        assert oracle.verify_sp_tree(index, nbr, w, dist[i], sparent[i], s) == 0


def test_scale22_pagerank_against_fp64(big):
    g, index, nbr, _ = big
    s, st = g.pagerank(tol_l1=1e-4, max_iters=50)  # the benchmark's stopping rule
    assert st.converged
    x, _ = oracle.pr_jacobi_f64(index, nbr, tol=1e-11, max_iters=1000)
    err = float(np.abs(s - x).max())
    print(f"scale 22 PageRank (L1 1e-4): |GPU-FP64| {err:.3e}, max score {x.max():.3e}")
    assert err <= 1e-6


def test_scale20_batched_columns_against_oracle():
    g = hc.Graph.generate(hc.GEN_KRONECKER, 20, 16, 2, hc.W_I32)
    index, nbr, w = g.csr()
    src = g.pick_sources(128)
    depth, _ = g.bfs_batched(src)
    dist, st = g.sssp_batched(src)
    for i in (0, 37, 127):
        assert np.array_equal(depth[i], oracle.bfs_depth(index, nbr, src[i]))
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(index, nbr, w, src[i]))
