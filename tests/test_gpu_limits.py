"""The bounded device waits: each one made to run out with a short limit
(hc_set_time_limits), the call ending with HC_ERR_TIMEOUT and the handle
staying usable.  No wait here is unbounded: the held-back barrier and the
runs end after about a millisecond, and the defaults are restored after
every test."""
import numpy as np
import pytest

import hc
import oracle

pytestmark = pytest.mark.gpu

MS = 1_000_000


@pytest.fixture(autouse=True)
def restore_limits():
    yield
    hc.set_time_limits(0)


@pytest.fixture(scope="module")
def graph():
    host = hc.gen_kronecker(14, 16, 3, wtype=hc.W_I32)
    return host, hc.Graph.from_host(host)


def _status(call):
    with pytest.raises(hc.HCError) as e:
        call()
    return e.value.status


def test_grid_barrier_gives_up_when_a_block_never_arrives(graph):
    hc.set_time_limits(0, wait_ns=MS)
    assert hc.selftest_grid_barrier(0, 8, -1) == hc.OK
    assert hc.selftest_grid_barrier(0, 8, 3) == hc.TIMEOUT
    assert hc.selftest_grid_barrier(0, 1, 0) == hc.OK  # the only block returns before the barrier
    hc.set_time_limits(0)
    host, g = graph
    src = hc.pick_sources(host, 2)
    depth, _, _ = g.bfs(src)
    for i, s in enumerate(src):
        assert np.array_equal(depth[i], oracle.bfs_depth(host.index, host.neighbors, s))


def test_run_limit_ends_persistent_runs(graph):
    host, g = graph
    src = hc.pick_sources(host, 2)
    hc.set_time_limits(0, run_ns=1)
    assert _status(lambda: g.bfs(src)) == hc.TIMEOUT
    assert _status(lambda: g.sssp(src)) == hc.TIMEOUT
    assert _status(lambda: g.pagerank_ordered()) == hc.TIMEOUT
    hc.set_time_limits(0)
    depth, parent, _ = g.bfs(src)
    dist, _, _ = g.sssp(src)
    for i, s in enumerate(src):
        d = oracle.bfs_depth(host.index, host.neighbors, s)
        assert np.array_equal(depth[i], d)
        assert oracle.verify_bfs_parents(host.index, host.neighbors, d, parent[i], s)[0] == 0
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, s))
    s_, st = g.pagerank_ordered()
    ref, it = oracle.pr_pull(host.index, host.neighbors)
    assert np.array_equal(s_, ref) and st.iterations == it


@pytest.mark.parametrize("use_graph", [hc.GRAPH_ON, hc.GRAPH_OFF])
def test_loop_limit_ends_batched_groups(graph, use_graph):
    host, g = graph
    src = hc.pick_sources(host, 64)
    hc.set_time_limits(0, loop_ns=1)
    assert _status(lambda: g.bfs_batched(src, use_graph=use_graph)) == hc.TIMEOUT
    assert _status(lambda: g.sssp_batched(src, use_graph=use_graph)) == hc.TIMEOUT
    hc.set_time_limits(0)
    depth, _ = g.bfs_batched(src, use_graph=use_graph)
    dist, _ = g.sssp_batched(src, use_graph=use_graph)
    for i in (0, 17, 63):
        s = src[i]
        assert np.array_equal(depth[i], oracle.bfs_depth(host.index, host.neighbors, s))
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, s))
