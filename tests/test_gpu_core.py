"""GPU parity of the plain hot path (BFS, SSSP, PageRank) through the C ABI
against the oracle and the reference's golden outputs."""
import hashlib

import numpy as np
import pytest

import hc
import oracle
from conftest import make_graph

pytestmark = pytest.mark.gpu

CASES = ["kron10", "kron12_ef8", "er10", "grid32", "kron16"]


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def graphs(golden):
    out = {}
    for name in CASES:
        rec, arr = golden[name]
        host = make_graph(rec)
        out[name] = (rec, arr, host, hc.Graph.from_host(host))
    return out


# ------------------------------------------------------------------- BFS

@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("direction,bu", [(0, hc.VARIANT_AUTO), (1, hc.VARIANT_AUTO), (2, hc.VARIANT_THREAD),
                                          (2, hc.VARIANT_WARP), (0, hc.VARIANT_WARP)])
def test_bfs_depths_bit_exact(graphs, name, direction, bu):
    rec, arr, host, g = graphs[name]
    src = rec["bfs_sources"]
    depth, parent, st = g.bfs(src, direction=direction, bu_variant=bu)
    for i, s in enumerate(src):
        assert digest(depth[i]) == rec["bfs_depth_sha256"][i], (name, i)
        bad, counts = oracle.verify_bfs_parents(host.index, host.neighbors, depth[i], parent[i], s)
        assert bad == 0, counts


def test_bfs_larger_graph_against_oracle():
    host = hc.gen_kronecker(19, 16, 9)
    g = hc.Graph.from_host(host)
    src = hc.pick_sources(host, 6)
    depth, parent, st = g.bfs(src, stats=True)
    assert st.td_levels > 0 and st.bu_levels > 0
    for i, s in enumerate(src):
        d = oracle.bfs_depth(host.index, host.neighbors, s)
        assert np.array_equal(depth[i], d)
        assert oracle.verify_bfs_parents(host.index, host.neighbors, d, parent[i], s)[0] == 0


def _handmade(edges, n):
    """CSR from an edge list, kept as given (duplicates, self-loops, unsorted rows allowed)."""
    edges = np.array(edges, dtype=np.int64).reshape(-1, 2)
    order = np.argsort(edges[:, 0], kind="stable")
    e = edges[order]
    idx = np.zeros(n + 1, dtype=np.int64)
    np.add.at(idx, e[:, 0] + 1, 1)
    return np.cumsum(idx), e[:, 1].astype(np.int32)


def test_bfs_edge_cases():
    # path 0-1-...-299 (high diameter), a star around 300, isolated 400, self-loops, duplicates
    n = 401
    edges = []
    for i in range(299):
        edges += [(i, i + 1), (i + 1, i)]
    for j in range(301, 340):
        edges += [(300, j), (j, 300), (300, j)]
    edges += [(5, 5), (300, 300)]
    idx, nbr = _handmade(edges, n)
    g = hc.Graph(idx, nbr)
    for s in [0, 150, 300, 320, 400, 5]:
        for direction in (0, 1, 2):
            depth, parent, _ = g.bfs([s], direction=direction)
            d = oracle.bfs_depth(idx, nbr, s)
            assert np.array_equal(depth[0], d), (s, direction)
            assert oracle.verify_bfs_parents(idx, nbr, d, parent[0], s)[0] == 0
    # empty graph (no edges) and a single vertex
    g1 = hc.Graph(np.zeros(2, dtype=np.int64), np.zeros(0, dtype=np.int32))
    depth, parent, _ = g1.bfs([0])
    assert depth[0, 0] == 0 and parent[0, 0] == 0


def test_bfs_unsorted_degrees():
    host = hc.gen_kronecker(12, 8, 4)
    n = host.num_nodes
    perm = np.random.default_rng(1).permutation(n).astype(np.int32)  # old -> new
    inv = np.argsort(perm)
    deg = host.degrees()[inv]
    idx = np.concatenate([[0], np.cumsum(deg)]).astype(np.int64)
    nbr = np.concatenate([np.sort(perm[host.neighbors[host.index[o]:host.index[o + 1]]]) for o in inv]).astype(np.int32)
    g = hc.Graph(idx, nbr)
    assert g.info().degree_sorted == 0
    for s in hc.pick_sources(hc.HostCSR(idx, nbr), 3):
        depth, parent, _ = g.bfs([s])
        assert np.array_equal(depth[0], oracle.bfs_depth(idx, nbr, s))


def test_bfs_device_outputs():
    torch = pytest.importorskip("torch")
    host = hc.gen_kronecker(12, 16, 2)
    g = hc.Graph.from_host(host)
    src = hc.pick_sources(host, 3)
    depth = torch.empty((3, host.num_nodes), dtype=torch.int32, device="cuda")
    parent = torch.empty((3, host.num_nodes), dtype=torch.int32, device="cuda")
    g.bfs(torch.from_numpy(src).cuda(), depth, parent)
    torch.cuda.synchronize()
    for i, s in enumerate(src):
        assert np.array_equal(depth[i].cpu().numpy(), oracle.bfs_depth(host.index, host.neighbors, s))


def test_bfs_rejects_bad_sources(graphs):
    g = graphs["kron10"][3]
    with pytest.raises(hc.HCError) as e:
        g.bfs([5000])
    assert e.value.status == hc.INVALID_ARG


# ------------------------------------------------------------------ SSSP

@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("delta", [0, -1, 1, 64, 100000])
def test_sssp_distances_bit_exact(graphs, name, delta):
    rec, arr, host, g = graphs[name]
    src = rec["sssp_sources"]
    dist, parent, _ = g.sssp(src, delta=delta, want_parent=True)
    for i, s in enumerate(src):
        assert digest(dist[i]) == rec["sssp_dist_sha256"][i], (name, i, delta)
        assert oracle.verify_sp_tree(host.index, host.neighbors, host.weights, dist[i], parent[i], s) == 0


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("delta,pull_alpha", [(0, -1), (0, 1000000), (-1, 1000000), (64, 2)])
def test_sssp_push_pull_modes_bit_exact(graphs, name, delta, pull_alpha):
    """pull_alpha -1: push epochs only; 1e6: nearly every epoch is a pull sweep."""
    rec, arr, host, g = graphs[name]
    src = rec["sssp_sources"]
    dist, _, _ = g.sssp(src, delta=delta, pull_alpha=pull_alpha)
    for i, s in enumerate(src):
        assert digest(dist[i]) == rec["sssp_dist_sha256"][i], (name, i, delta, pull_alpha)


def test_sssp_asymmetric_weights_use_push():
    """With w(u->v) != w(v->u) the pull sweep is disabled; push semantics (weight from u's row) hold."""
    host = hc.gen_kronecker(12, 8, 3)
    rng = np.random.default_rng(0)
    w = rng.integers(1, 256, size=host.num_edges).astype(np.int32)
    g = hc.Graph(host.index, host.neighbors, w)
    src = hc.pick_sources(host, 3)
    dist, parent, _ = g.sssp(src, pull_alpha=1000000, want_parent=True)
    for i, s in enumerate(src):
        d = oracle.sssp_dijkstra(host.index, host.neighbors, w, s)
        assert np.array_equal(dist[i], d)
        assert oracle.verify_sp_tree(host.index, host.neighbors, w, d, parent[i], s) == 0


def test_sssp_one_asymmetric_weight_disables_pull():
    """A single edge whose reverse has another weight: the symmetry hash must see it (pull sweeps would read
    the reverse weight), and every epoch stays push."""
    host = hc.gen_kronecker(12, 8, 4, wtype=hc.W_I32)
    w = host.weights.copy()
    src = hc.pick_sources(host, 4)
    u = int(src[0])
    e = int(host.index[u])  # the first edge of a source row: on every shortest-path tree from it
    w[e] = 1 if w[e] != 1 else 2
    g = hc.Graph(host.index, host.neighbors, w)
    dist, _, _ = g.sssp(src, pull_alpha=1000000)
    for i, s in enumerate(src):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, w, s)), i


def test_sssp_pull_on_unsorted_rows():
    """Rows in shuffled order (symmetric weights): pull sweeps stay enabled and exact."""
    host = hc.gen_kronecker(12, 8, 5, wtype=hc.W_I32)
    rng = np.random.default_rng(3)
    nbr, w = host.neighbors.copy(), host.weights.copy()
    for v in range(host.num_nodes):
        b, e = host.index[v], host.index[v + 1]
        if e - b > 1:
            p = rng.permutation(e - b) + b
            nbr[b:e], w[b:e] = nbr[p], w[p]
    g = hc.Graph(host.index, nbr, w)
    src = hc.pick_sources(host, 4)
    dist, _, st = g.sssp(src, pull_alpha=1000000, stats=True)
    for i, s in enumerate(src):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, nbr, w, s)), i


def _sym_weights(host, kind):
    """Symmetric weights (a hash of the unordered pair) of a chosen distribution."""
    row = np.repeat(np.arange(host.num_nodes, dtype=np.int64), np.diff(host.index))
    col = host.neighbors.astype(np.int64)
    lo, hi = np.minimum(row, col), np.maximum(row, col)
    h = (lo * 1000003 + hi * 7919) % 2147483629
    h = (h * 48271) % 2147483647
    if kind == "zeros":
        return (h % 3).astype(np.int32)  # 0, 1, 2
    if kind == "wide":
        return (h % (1 << 20)).astype(np.int32)
    if kind == "equal":
        return np.full(host.num_edges, 7, dtype=np.int32)
    # skewed: mostly 1, one in 50 near the top of a wide range
    return np.where(h % 50 == 0, (1 << 18) + h % 1000, 1).astype(np.int32)


@pytest.mark.parametrize("kind", ["zeros", "wide", "equal", "skewed"])
def test_sssp_weight_ordered_pulls_exact(kind):
    """Pull sweeps read each row's pairs in weight-bucket order and stop a row once the bucket floor reaches its
    best distance: exact for zero weights, a wide range, equal weights (one bucket) and a skewed mix."""
    host = hc.gen_kronecker(12, 8, 11)
    w = _sym_weights(host, kind)
    g = hc.Graph(host.index, host.neighbors, w)
    src = hc.pick_sources(host, 4)
    ref = [oracle.sssp_dijkstra(host.index, host.neighbors, w, s) for s in src]
    for pull_alpha in (1000000, 0, 2):
        dist, parent, _ = g.sssp(src, pull_alpha=pull_alpha, want_parent=True)
        for i, s in enumerate(src):
            assert np.array_equal(dist[i], ref[i]), (kind, pull_alpha, i)
            assert oracle.verify_sp_tree(host.index, host.neighbors, w, ref[i], parent[i], s) == 0
    # Batched pulls skip a lane's words of a neighbour whose weight reaches the lane's largest distance.
    for switch_alpha, bits in ((1000000, 0), (0, 0), (1000000, 32)):
        db, _ = g.sssp_batched(src, switch_alpha=switch_alpha, dist_bits=bits)
        for i in range(len(src)):
            assert np.array_equal(db[i], ref[i]), (kind, "batched", switch_alpha, bits, i)


def test_sssp_grid_against_dijkstra():
    host = hc.gen_grid(200, 300, 3, wtype=hc.W_I32)
    g = hc.Graph.from_host(host)
    src = hc.pick_sources(host, 3)
    dist, _, st = g.sssp(src, stats=True)
    assert st.epochs > 200
    for i, s in enumerate(src):
        assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, s))


def test_sssp_larger_graph_against_dijkstra():
    host = hc.gen_kronecker(18, 16, 5, wtype=hc.W_I32)
    g = hc.Graph.from_host(host)
    src = hc.pick_sources(host, 4)
    for delta in (0, -1):
        dist, _, _ = g.sssp(src, delta=delta)
        for i, s in enumerate(src):
            assert np.array_equal(dist[i], oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, s))


def test_sssp_errors():
    host = hc.gen_kronecker(8, 4, 1)
    g = hc.Graph.from_host(host)  # unweighted
    with pytest.raises(hc.HCError) as e:
        g.sssp([0])
    assert e.value.status == hc.UNSUPPORTED
    w = np.ones(host.num_edges, dtype=np.int32)
    w[3] = -2
    g2 = hc.Graph(host.index, host.neighbors, w)
    with pytest.raises(hc.HCError) as e:
        g2.sssp([int(hc.pick_sources(host, 1)[0])])
    assert e.value.status == hc.INVALID_ARG
    # epoch cap reached -> NOT_CONVERGED, and the handle stays usable
    hg = hc.gen_grid(50, 50, 1, wtype=hc.W_I32)
    g3 = hc.Graph.from_host(hg)
    with pytest.raises(hc.HCError) as e:
        g3.sssp([0], max_epochs=5)
    assert e.value.status == hc.NOT_CONVERGED
    dist, _, _ = g3.sssp([0])
    assert np.array_equal(dist[0], oracle.sssp_dijkstra(hg.index, hg.neighbors, hg.weights, 0))


# -------------------------------------------------------------- PageRank

@pytest.mark.parametrize("name", CASES)
def test_pagerank_reference_order_bit_exact(graphs, name):
    """hc_pr_pull_ordered, the compat pr_pull_gpu, gives the reference's single-thread pr_pull_cpu scores (the
    golden fixture, made by the reference's own code) bit for bit, in the same number of sweeps."""
    rec, arr, host, g = graphs[name]
    ref = arr["pr_scores"]
    s, st = g.pagerank_ordered()
    _, sweeps = oracle.pr_pull(host.index, host.neighbors)
    assert st.converged and st.iterations == sweeps, (st.iterations, sweeps)
    assert np.array_equal(s.view(np.uint32), ref.view(np.uint32)), float(np.abs(s - ref).max())
    s2 = hc.pr_pull_gpu(g)  # at most 201 sweeps, as the reference's GPU driver; none of these needs more
    assert np.array_equal(s2.view(np.uint32), ref.view(np.uint32))


def test_pagerank_reference_order_caller_init_and_cap():
    """The caller's init_score (pr_pull_gpu's argument) and a sweep cap, against the oracle run the same way."""
    host = hc.gen_kronecker(12, 16, 11)
    g = hc.Graph.from_host(host)
    rng = np.random.default_rng(4)
    init = (rng.random(host.num_nodes) / host.num_nodes).astype(np.float32)
    for cap in (0, 3):
        s, st = g.pagerank_ordered(init, max_iters=cap)
        ref, it = oracle.pr_pull(host.index, host.neighbors, max_iters=cap, init=init)
        assert st.iterations == it and bool(st.converged) == (cap == 0)
        assert np.array_equal(s.view(np.uint32), ref.view(np.uint32))


def test_pagerank_reference_order_refuses_asymmetric():
    index, nbr = np.array([0, 1, 1], dtype=np.int64), np.array([1], dtype=np.int32)  # 0 -> 1 only
    g = hc.Graph(index, nbr)
    with pytest.raises(hc.HCError) as e:
        g.pagerank_ordered()
    assert e.value.status == hc.UNSUPPORTED


# Distance of the reference's scores from the FP64 fixed point, per golden graph (its per-vertex 5e-8 rule
# stops early; largest at scale 16): the engine's Jacobi sweeps land near the fixed point, so where this
# exceeds 1e-5 the Jacobi result cannot be within 1e-5 of the reference, and the test states the deviation.
@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("mode", ["eps_vertex 5e-8", "tol_l1 1e-6"])
def test_pagerank_jacobi_errors_stated(graphs, name, mode):
    """Jacobi PageRank (hc_pr_forward) against the reference and against FP64: |GPU-ref|, |ref-FP64| and
    |GPU-FP64| (L-inf) printed per graph.  |GPU-ref| <= 1e-5 wherever the reference is within 1e-5 of FP64;
    elsewhere (kron16: 3.7e-5) |GPU-FP64| <= 1e-6 and the deviation from the reference is stated."""
    rec, arr, host, g = graphs[name]
    ref = arr["pr_scores"]
    if mode.startswith("eps"):
        s, st = g.pagerank(tol_l1=0.0, eps_vertex=5e-8, max_iters=201)
    else:
        s, st = g.pagerank(tol_l1=1e-6, max_iters=500)
    assert st.converged
    x, _ = oracle.pr_jacobi_f64(host.index, host.neighbors, tol=1e-15, max_iters=3000)
    gpu_ref, ref_64, gpu_64 = (float(np.abs(s - ref).max()), float(np.abs(ref - x).max()),
                               float(np.abs(s - x).max()))
    print(f"pagerank {name} [{mode}]: |GPU-ref| {gpu_ref:.3e}  |ref-FP64| {ref_64:.3e}  |GPU-FP64| {gpu_64:.3e}")
    assert gpu_64 <= 1e-6, gpu_64
    if ref_64 <= 1e-5:
        assert gpu_ref <= 1e-5, gpu_ref


def test_pagerank_l1_tolerance_mode():
    host = hc.gen_kronecker(16, 16, 2)
    g = hc.Graph.from_host(host)
    s, st = g.pagerank(tol_l1=1e-4, max_iters=50)
    assert st.converged and st.iterations <= 50 and st.residual_l1 < 1e-4
    x, _ = oracle.pr_jacobi_f64(host.index, host.neighbors)
    assert np.abs(s - x).max() < 1e-5
    assert abs(s.sum() - x.sum()) < 1e-3


def test_pagerank_weighted_and_teleport():
    host = hc.gen_kronecker(11, 8, 3, wtype=hc.W_F32)
    g = hc.Graph.from_host(host)
    rng = np.random.default_rng(3)
    t = rng.random(host.num_nodes).astype(np.float32)
    t /= t.sum()
    s, st = g.pagerank(t, weighted=True, tol_l1=1e-9, max_iters=300)
    x = oracle.pr_dense(host.index, host.neighbors, host.weights.astype(np.float64), t.astype(np.float64))
    assert np.abs(s - x).max() < 1e-6
    s2, _ = g.pagerank(t, weighted=False, tol_l1=1e-9, max_iters=300)
    x2 = oracle.pr_dense(host.index, host.neighbors, None, t.astype(np.float64))
    assert np.abs(s2 - x2).max() < 1e-6


def test_pagerank_hub_rows_chunked():
    # scale 18 has rows above the hub threshold (16384 edges): exercises the chunked path
    host = hc.gen_kronecker(18, 16, 1)
    assert host.degrees().max() > 16384
    g = hc.Graph.from_host(host)
    s, st = g.pagerank(tol_l1=1e-7, max_iters=200)
    x, _ = oracle.pr_jacobi_f64(host.index, host.neighbors, tol=1e-12)
    assert np.abs(s - x).max() < 1e-6


def test_host_outputs_pinned_and_mixed():
    """Per-source results bound for host memory are staged and copied while the next source runs:
    pinned and pageable host outputs, and host/device mixes, give the device outputs' depths and distances
    and valid parent trees."""
    torch = pytest.importorskip("torch")
    host = hc.gen_kronecker(13, 16, 9, wtype=hc.W_I32)
    g = hc.Graph.from_host(host)
    src = hc.pick_sources(host, 7)
    n = host.num_nodes
    dd = torch.empty((7, n), dtype=torch.int32, device="cuda")
    g.bfs(src, dd, torch.empty((7, n), dtype=torch.int32, device="cuda"))
    pinned_d = torch.empty((7, n), dtype=torch.int32).pin_memory().numpy()
    pinned_p = torch.empty((7, n), dtype=torch.int32).pin_memory().numpy()
    g.bfs(src, pinned_d, pinned_p)
    assert np.array_equal(pinned_d, dd.cpu().numpy())
    mixed_p = np.empty((7, n), dtype=np.int32)
    dd2 = torch.empty((7, n), dtype=torch.int32, device="cuda")
    g.bfs(src, dd2, mixed_p)
    assert np.array_equal(dd2.cpu().numpy(), dd.cpu().numpy())
    only_p = torch.empty((7, n), dtype=torch.int32).pin_memory().numpy()
    d_none, _, _ = g.bfs(src, None, only_p, want_depth=False)  # parents only, as the reference's bfs_gpu
    assert d_none is None
    for i, s in enumerate(src):  # parents may differ between runs (any neighbour one level up is valid)
        for par in (pinned_p[i], mixed_p[i], only_p[i]):
            assert oracle.verify_bfs_parents(host.index, host.neighbors, pinned_d[i], par, s)[0] == 0
    sd = torch.empty((7, n), dtype=torch.int32, device="cuda")
    g.sssp(src, sd)
    pinned_s = torch.empty((7, n), dtype=torch.int32).pin_memory().numpy()
    pinned_sp = torch.empty((7, n), dtype=torch.int32).pin_memory().numpy()
    dist, parent, _ = g.sssp(src, pinned_s, pinned_sp, want_parent=True)
    assert np.array_equal(pinned_s, sd.cpu().numpy())
    for i, s in enumerate(src):
        assert oracle.verify_sp_tree(host.index, host.neighbors, host.weights, pinned_s[i], pinned_sp[i], s) == 0


def test_bfs_frontier_summary_with_a_shift():
    """Above 2^22 vertices a summary bit covers several frontier words (2^23 here: two); bottom-up levels
    probe global memory only where it is set.  Depths against the serial BFS, parents as BFS trees."""
    host = hc.gen_uniform(23, 2, 17)
    assert host.num_nodes == 1 << 23
    g = hc.Graph.from_host(host)
    src = hc.pick_sources(host, 2)
    for direction in (2, 0):  # every level bottom-up; Beamer's switching
        depth, parent, _ = g.bfs(src, direction=direction)
        for i, s in enumerate(src):
            d = oracle.bfs_depth(host.index, host.neighbors, s)
            assert np.array_equal(depth[i], d), (direction, i)
            assert oracle.verify_bfs_parents(host.index, host.neighbors, d, parent[i], s)[0] == 0
    g.close()


def test_sssp_weight_ordered_pulls_on_hub_chunks():
    """A hub row longer than the chunk size (its later chunks test their first window before reading it),
    with skewed weights, every epoch a pull: exact against Dijkstra."""
    rng = np.random.default_rng(5)
    n, hub_deg = 30000, 20000
    edges = {(0, int(v)) for v in rng.choice(np.arange(1, n), hub_deg, replace=False)}
    while len(edges) < hub_deg + 4 * n:
        a, b = (int(x) for x in rng.integers(1, n, 2))
        if a != b:
            edges.add((min(a, b), max(a, b)))
    src_l, dst_l = zip(*edges)
    src_a, dst_a = np.array(src_l + dst_l), np.array(dst_l + src_l)
    order = np.lexsort((dst_a, src_a))
    src_a, dst_a = src_a[order], dst_a[order]
    index = np.zeros(n + 1, dtype=np.int64)
    np.add.at(index, src_a + 1, 1)
    index = np.cumsum(index)
    nbr = dst_a.astype(np.int32)
    lo, hi = np.minimum(src_a, dst_a).astype(np.int64), np.maximum(src_a, dst_a).astype(np.int64)
    h = (lo * 1000003 + hi * 7919) % 2147483629
    w = np.where(h % 40 == 0, 1 + h % 3, 200 + h % 50).astype(np.int32)  # a few light edges, most heavy
    g = hc.Graph(index, nbr, w)
    srcs = np.array([0, 1, 12345], dtype=np.int32)
    for pull_alpha in (1000000, 0):
        dist, parent, _ = g.sssp(srcs, pull_alpha=pull_alpha, want_parent=True)
        for i, s in enumerate(srcs):
            d = oracle.sssp_dijkstra(index, nbr, w, int(s))
            assert np.array_equal(dist[i], d), (pull_alpha, i)
            assert oracle.verify_sp_tree(index, nbr, w, d, parent[i], int(s)) == 0
    g.close()
