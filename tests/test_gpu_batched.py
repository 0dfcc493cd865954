"""Batched multi-source BFS / SSSP and personalised PageRank against the oracle."""
import numpy as np
import pytest

import hc
import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scale,k", [(12, 512), (14, 100), (10, 7)])
def test_bfs_batched_depths(scale, k):
    host = hc.gen_kronecker(scale, 16, 31)
    g = hc.Graph.from_host(host)
    src = hc.pick_sources(host, k)
    depth, st = g.bfs_batched(src)
    assert st.groups == 1
    for i, s in enumerate(src):
        assert np.array_equal(depth[i], oracle.bfs_depth(host.index, host.neighbors, s)), i


@pytest.mark.parametrize("switch_alpha", [-1, 1000000])
def test_bfs_batched_pull_only_and_push_mostly(switch_alpha):
    host = hc.gen_kronecker(13, 16, 33)
    g = hc.Graph.from_host(host)
    src = hc.pick_sources(host, 70)
    depth, _ = g.bfs_batched(src, group=128, switch_alpha=switch_alpha)
    for i in range(0, 70, 7):
        assert np.array_equal(depth[i], oracle.bfs_depth(host.index, host.neighbors, src[i])), i


def test_bfs_batched_groups_and_duplicates():
    host = hc.gen_kronecker(11, 8, 2)
    g = hc.Graph.from_host(host)
    src = np.concatenate([hc.pick_sources(host, 300), hc.pick_sources(host, 5)])  # duplicates across groups
    depth, st = g.bfs_batched(src, group=128)
    assert st.groups == 3
    for i, s in enumerate(src):
        assert np.array_equal(depth[i], oracle.bfs_depth(host.index, host.neighbors, s))


@pytest.mark.parametrize("use_graph", [hc.GRAPH_ON, hc.GRAPH_OFF])
def test_bfs_batched_grid(use_graph):
    """~90 levels: the level loop as a CUDA graph (while node) and as a host loop."""
    host = hc.gen_grid(40, 50, 1)
    g = hc.Graph.from_host(host)
    src = np.array([0, 1999, 1000, 7], dtype=np.int32)
    depth, st = g.bfs_batched(src, use_graph=use_graph)
    assert st.epochs > 40
    for i, s in enumerate(src):
        assert np.array_equal(depth[i], oracle.bfs_depth(host.index, host.neighbors, s))
    with pytest.raises(hc.HCError) as e:
        g.bfs_batched(src, max_epochs=10, use_graph=use_graph)
    assert e.value.status == hc.NOT_CONVERGED
    depth2, _ = g.bfs_batched(src, use_graph=use_graph)  # handle still usable
    assert np.array_equal(depth2, depth)


@pytest.mark.parametrize("scale,k", [(12, 40), (10, 32), (13, 5)])
def test_sssp_batched_distances(scale, k):
    host = hc.gen_kronecker(scale, 16, 41, wtype=hc.W_I32)
    g = hc.Graph.from_host(host)
    src = hc.pick_sources(host, k)
    dist, st = g.sssp_batched(src)
    for i, s in enumerate(src):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, s)), i


@pytest.mark.parametrize("group", [32, 64, 128, 256, 512])
def test_sssp_batched_group_widths(group):
    host = hc.gen_kronecker(11, 16, 42, wtype=hc.W_I32)
    g = hc.Graph.from_host(host)
    src = np.concatenate([hc.pick_sources(host, 150), hc.pick_sources(host, 3)])  # ragged last group, duplicates
    dist, st = g.sssp_batched(src, group=group)
    assert st.groups == -(-len(src) // group)
    for i, s in enumerate(src):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, s)), i
    torch = pytest.importorskip("torch")
    dd = torch.empty((len(src), host.num_nodes), dtype=torch.int32, device="cuda")
    g.sssp_batched(src, dd, group=group)
    assert np.array_equal(dd.cpu().numpy(), dist)


@pytest.mark.parametrize("switch_alpha", [-1, 0, 1000000])
def test_sssp_batched_push_and_pull_epochs(switch_alpha):
    """Push only, the default switch, and pull for every epoch."""
    big = hc.gen_kronecker(16, 16, 3, wtype=hc.W_I32)  # rows above the chunk size
    g = hc.Graph.from_host(big)
    src = hc.pick_sources(big, 70)
    dist, _ = g.sssp_batched(src, group=64, switch_alpha=switch_alpha)
    for i in range(0, 70, 9):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(big.index, big.neighbors, big.weights, src[i])), i


@pytest.mark.parametrize("use_graph", [hc.GRAPH_ON, hc.GRAPH_OFF])
def test_sssp_batched_graph_and_host_loop(use_graph):
    """The epoch loop as a CUDA graph (while node) and as a host loop give the same distances."""
    host = hc.gen_grid(50, 40, 4, wtype=hc.W_I32)  # ~100 epochs
    g = hc.Graph.from_host(host)
    src = np.array([0, 1999, 1000, 7, 7, 1234], dtype=np.int32)
    dist, st = g.sssp_batched(src, group=32, use_graph=use_graph)
    assert st.epochs > 40
    for i, s in enumerate(src):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, s)), i
    before = hc.kernel_launches()
    g.sssp_batched(src, group=32, use_graph=use_graph)
    assert hc.kernel_launches() - before >= 6 * st.epochs  # launches inside the graph are counted too


@pytest.mark.parametrize("use_graph", [hc.GRAPH_ON, hc.GRAPH_OFF])
def test_sssp_batched_epoch_cap(use_graph):
    host = hc.gen_grid(50, 40, 4, wtype=hc.W_I32)
    g = hc.Graph.from_host(host)
    with pytest.raises(hc.HCError) as e:
        g.sssp_batched(np.array([0], dtype=np.int32), max_epochs=5, use_graph=use_graph)
    assert e.value.status == hc.NOT_CONVERGED
    dist, st = g.sssp_batched(np.array([0], dtype=np.int32), use_graph=use_graph)  # handle still usable
    assert np.array_equal(dist[0], oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, 0))


def test_sssp_batched_asymmetric_weights():
    """w(u->v) != w(v->u): epochs stay push, weights read from u's row."""
    host = hc.gen_kronecker(12, 8, 3)
    w = np.random.default_rng(0).integers(1, 256, size=host.num_edges).astype(np.int32)
    g = hc.Graph(host.index, host.neighbors, w)
    src = hc.pick_sources(host, 40)
    dist, _ = g.sssp_batched(src)
    for i, s in enumerate(src):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, w, s)), i


def test_sssp_batched_grid_and_hubs():
    host = hc.gen_grid(60, 70, 2, wtype=hc.W_I32)
    g = hc.Graph.from_host(host)
    src = np.array([0, 4199, 2100, 33, 33], dtype=np.int32)
    dist, _ = g.sssp_batched(src)
    for i, s in enumerate(src):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, s))
    big = hc.gen_kronecker(16, 16, 3, wtype=hc.W_I32)  # rows above the chunking threshold
    assert big.degrees().max() > 2048
    gb = hc.Graph.from_host(big)
    src = hc.pick_sources(big, 6)
    dist, _ = gb.sssp_batched(src)
    for i, s in enumerate(src):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(big.index, big.neighbors, big.weights, s))


@pytest.mark.parametrize("weighted", [False, True])
def test_ppr_batched_against_dense(weighted):
    host = hc.gen_kronecker(11, 16, 5, wtype=hc.W_F32)
    g = hc.Graph.from_host(host)
    rng = np.random.default_rng(2)
    k = 40
    sizes = rng.integers(1, 33, size=k)
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    seeds = np.concatenate([rng.choice(host.num_nodes, s, replace=False) for s in sizes]).astype(np.int32)
    scores, st = g.ppr_batched(off, seeds, tol_l1=1e-8, max_iters=300, weighted=weighted)
    w = host.weights.astype(np.float64) if weighted else None
    for c in range(0, k, 7):
        t = np.zeros(host.num_nodes)
        t[seeds[off[c]:off[c + 1]]] = 1.0 / sizes[c]
        x = oracle.pr_dense(host.index, host.neighbors, w, t)
        assert np.abs(scores[:, c] - x).max() < 1e-6, c


def test_ppr_batched_columns_stop_at_their_own_pace():
    """70 columns (three 32-column chunks) converging after different sweep counts: converged columns
    leave the packed state, host and device outputs agree, every column matches the FP64 solve."""
    torch = pytest.importorskip("torch")
    host = hc.gen_kronecker(12, 16, 8)
    g = hc.Graph.from_host(host)
    rng = np.random.default_rng(5)
    k = 70
    sizes = rng.integers(1, 33, size=k)
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    active = np.flatnonzero(host.degrees() > 0)
    seeds = np.concatenate([rng.choice(active, s, replace=False) for s in sizes]).astype(np.int32)
    scores, st = g.ppr_batched(off, seeds, tol_l1=1e-7, max_iters=300)
    assert st.converged
    dev = torch.empty((host.num_nodes, k), dtype=torch.float32, device="cuda")
    g.ppr_batched(off, seeds, dev, tol_l1=1e-7, max_iters=300)
    assert np.array_equal(dev.cpu().numpy(), scores)
    for c in range(0, k, 3):
        t = np.zeros(host.num_nodes)
        t[seeds[off[c]:off[c + 1]]] = 1.0 / sizes[c]
        x = oracle.pr_dense(host.index, host.neighbors, None, t)
        assert np.abs(scores[:, c] - x).max() < 1e-6, c


def test_dense_multicolumn_forward():
    host = hc.gen_kronecker(10, 16, 6)
    g = hc.Graph.from_host(host)
    rng = np.random.default_rng(4)
    T = rng.random((host.num_nodes, 8)).astype(np.float32)
    T /= T.sum(axis=0, keepdims=True)
    X, st = g.pagerank(T, tol_l1=1e-8, max_iters=300)
    for c in range(8):
        x = oracle.pr_dense(host.index, host.neighbors, None, T[:, c].astype(np.float64))
        assert np.abs(X[:, c] - x).max() < 1e-6
