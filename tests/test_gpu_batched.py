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


@pytest.mark.parametrize("dist_bits", [0, 32])
@pytest.mark.parametrize("group", [32, 64, 128, 256, 512])
def test_sssp_batched_group_widths(group, dist_bits):
    host = hc.gen_kronecker(11, 16, 42, wtype=hc.W_I32)
    g = hc.Graph.from_host(host)
    src = np.concatenate([hc.pick_sources(host, 150), hc.pick_sources(host, 3)])  # ragged last group, duplicates
    dist, st = g.sssp_batched(src, group=group, dist_bits=dist_bits)
    assert st.wide_groups == (st.groups if dist_bits == 32 or group == 32 else 0)
    assert st.groups == -(-len(src) // group)
    for i, s in enumerate(src):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, s)), i
    torch = pytest.importorskip("torch")
    dd = torch.empty((len(src), host.num_nodes), dtype=torch.int32, device="cuda")
    g.sssp_batched(src, dd, group=group, dist_bits=dist_bits)
    assert np.array_equal(dd.cpu().numpy(), dist)


@pytest.mark.parametrize("dist_bits", [0, 32])
@pytest.mark.parametrize("switch_alpha", [-1, 0, 1000000])
def test_sssp_batched_push_and_pull_epochs(switch_alpha, dist_bits):
    """Push only, the default switch, and pull for every epoch; 16- and 32-bit distances."""
    big = hc.gen_kronecker(16, 16, 3, wtype=hc.W_I32)  # rows above the chunk size
    g = hc.Graph.from_host(big)
    src = hc.pick_sources(big, 70)
    dist, _ = g.sssp_batched(src, group=64, switch_alpha=switch_alpha, dist_bits=dist_bits)
    for i in range(0, 70, 9):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(big.index, big.neighbors, big.weights, src[i])), i


@pytest.mark.parametrize("group", [32, 64])
@pytest.mark.parametrize("use_graph", [hc.GRAPH_ON, hc.GRAPH_OFF])
def test_sssp_batched_graph_and_host_loop(use_graph, group):
    """The epoch loop as a CUDA graph (while node) and as a host loop give the same distances
    (32-bit distances at 32 sources per group, 16-bit at 64)."""
    host = hc.gen_grid(50, 40, 4, wtype=hc.W_I32)  # ~100 epochs
    g = hc.Graph.from_host(host)
    src = np.array([0, 1999, 1000, 7, 7, 1234], dtype=np.int32)
    dist, st = g.sssp_batched(src, group=group, use_graph=use_graph)
    assert st.epochs > 40
    assert st.wide_groups == (1 if group == 32 else 0)
    for i, s in enumerate(src):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, s)), i
    before = hc.kernel_launches()
    g.sssp_batched(src, group=group, use_graph=use_graph)
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


def _line(n, w):
    """Path 0 - 1 - ... - n-1, every edge of weight w both ways."""
    deg = np.full(n, 2, dtype=np.int64)
    deg[0] = deg[-1] = 1
    index = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
    nbr = np.concatenate([[v for v in (u - 1, u + 1) if 0 <= v < n] for u in range(n)]).astype(np.int32)
    return index, nbr, np.full(len(nbr), w, dtype=np.int32)


def test_sssp_batched_16_and_32_bit_agree():
    """Kronecker, weights [1,255]: 16-bit working distances by default, 32-bit on request, same result."""
    host = hc.gen_kronecker(12, 16, 43, wtype=hc.W_I32)
    g = hc.Graph.from_host(host)
    src = hc.pick_sources(host, 130)
    d16, st16 = g.sssp_batched(src)
    assert (st16.wide_groups, st16.reruns) == (0, 0)
    d32, st32 = g.sssp_batched(src, dist_bits=32)
    assert st32.wide_groups == st32.groups and st32.reruns == 0
    assert np.array_equal(d16, d32)
    for i in range(0, len(src), 11):
        assert np.array_equal(d16[i], oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, src[i])), i


@pytest.mark.parametrize("use_graph", [hc.GRAPH_ON, hc.GRAPH_OFF])
@pytest.mark.parametrize("n,reruns", [(15, 0), (16, 1), (17, 1), (40, 1)])
def test_sssp_batched_16bit_range(n, reruns, use_graph):
    """Line of weight 4095 (the largest 16-bit weight): the farthest vertex sits at (n-1)*4095.
    Up to 15 vertices every distance plus the largest weight stays below the 16-bit
    unreachable mark (0xF000) and the group finishes 16-bit; from 16 on it runs again
    32-bit (17 and 40 have distances that 16 bits cannot hold).  The 40-vertex line stops
    its 16-bit run after a few epochs, as soon as a written distance comes within the
    largest weight of the mark."""
    index, nbr, w = _line(n, 4095)
    g = hc.Graph(index, nbr, w)
    src = np.array([0, n - 1, n // 2, 0], dtype=np.int32)
    dist, st = g.sssp_batched(src, use_graph=use_graph)
    assert st.reruns == reruns
    assert st.wide_groups == reruns
    for i, s in enumerate(src):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(index, nbr, w, s)), i
    if n == 40:
        assert st.epochs >= 39  # the 32-bit rerun walks the whole line


def test_sssp_batched_16bit_rerun_midway():
    """Two components: a Kronecker graph (short distances) and a long line of weight 4000.
    The first 64-source group stays 16-bit; the second holds a line vertex, runs again
    32-bit, and so do the groups after it; every row matches Dijkstra."""
    kr = hc.gen_kronecker(10, 8, 44, wtype=hc.W_I32)
    ln_index, ln_nbr, ln_w = _line(60, 4000)
    nk = kr.num_nodes
    index = np.concatenate([kr.index, kr.index[-1] + ln_index[1:]]).astype(np.int64)
    nbr = np.concatenate([kr.neighbors, ln_nbr + nk]).astype(np.int32)
    w = np.concatenate([kr.weights, ln_w]).astype(np.int32)
    g = hc.Graph(index, nbr, w)
    src = hc.pick_sources(kr, 200)
    src[70] = nk + 3  # in the second group of 64
    with_host = np.empty((len(src), nk + 60), dtype=np.int32)
    dist, st = g.sssp_batched(src, with_host, group=64)
    assert st.reruns == 1
    assert st.groups == 4 and st.wide_groups == 3
    for i in list(range(0, 64, 9)) + [70] + list(range(64, 200, 13)):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(index, nbr, w, src[i])), i


def test_sssp_batched_heavy_weights_stay_32bit():
    """Weights above 4095 never use 16-bit distances."""
    host = hc.gen_kronecker(10, 8, 45)
    # symmetric weights: w(u->v) = w(v->u) through a hash of the unordered pair
    u = np.repeat(np.arange(host.num_nodes), np.diff(host.index))
    v = host.neighbors
    lo, hi = np.minimum(u, v).astype(np.int64), np.maximum(u, v).astype(np.int64)
    w = (((lo * 1000003 + hi) * 2654435761) % 99991 + 4096).astype(np.int32)
    g = hc.Graph(host.index, host.neighbors, w)
    src = hc.pick_sources(host, 40)
    dist, st = g.sssp_batched(src)
    assert st.wide_groups == st.groups and st.reruns == 0
    for i in range(0, 40, 5):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, w, src[i])), i


@pytest.mark.parametrize("dist_bits", [0, 32])
def test_sssp_batched_zero_weights_and_isolated_sources(dist_bits):
    """All-zero weights (every reached distance 0) and sources without edges (only their own
    distance is finite) in the same group as ordinary sources."""
    host = hc.gen_kronecker(11, 8, 46)
    w = np.zeros(host.num_edges, dtype=np.int32)
    g = hc.Graph(host.index, host.neighbors, w)
    deg = host.degrees()
    isolated = np.flatnonzero(deg == 0)[:3].astype(np.int32)
    assert len(isolated) == 3
    src = np.concatenate([hc.pick_sources(host, 70), isolated, isolated[:1]])
    dist, st = g.sssp_batched(src, dist_bits=dist_bits)
    assert st.reruns == 0
    for i, s in enumerate(src):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, w, s)), i
    for i in range(70, len(src)):
        assert (dist[i] == 0).sum() == 1 and (dist[i] == np.iinfo(np.int32).max).sum() == host.num_nodes - 1


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
