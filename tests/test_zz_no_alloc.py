"""hc_bfs_noalloc: the BFS entry point for callers that cannot allocate device
memory (code inside another framework's memory pool, paths that must not
trigger an allocation's device synchronisation).  Its working set is a fixed
array inside the library, so it must give exactly what hc_bfs gives, call after
call, and refuse graphs beyond that array's size.  Kept in a file of its own
that pytest collects last."""
import numpy as np
import pytest

import hc
import oracle

pytestmark = pytest.mark.gpu


def _call(idx, nbr, n, m, src, depth, parent):
    return hc.lib().hc_bfs_noalloc(idx.data_ptr(), nbr.data_ptr(), n, m, int(src), depth.data_ptr(),
                                   parent.data_ptr(), None)


def test_noalloc_bfs_matches_hc_bfs_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    host = hc.gen_kronecker(16, 16, 3)
    n, m = host.num_nodes, host.num_edges
    g = hc.Graph.from_host(host)
    src = hc.pick_sources(host, 2)
    ref_depth, _, _ = g.bfs(src)
    idx = torch.from_numpy(host.index).cuda()
    nbr = torch.from_numpy(host.neighbors).cuda()
    for i, s in enumerate(src):  # two calls in a row share the fixed array
        depth = torch.full((n,), 7, dtype=torch.int32, device="cuda")
        parent = torch.full((n,), 7, dtype=torch.int32, device="cuda")
        st = _call(idx, nbr, n, m, s, depth, parent)
        assert st == hc.OK, hc.lib().hc_last_error().decode()
        d = depth.cpu().numpy()
        assert np.array_equal(d, ref_depth[i])  # depths are unique: exact
        bad, counts = oracle.verify_bfs_parents(host.index, host.neighbors, d, parent.cpu().numpy(), s)
        assert bad == 0, counts


def test_noalloc_bfs_rejects_what_does_not_fit():
    torch = pytest.importorskip("torch")
    idx = torch.zeros(4, dtype=torch.int64, device="cuda")
    nbr = torch.zeros(4, dtype=torch.int32, device="cuda")
    out = torch.zeros(4, dtype=torch.int32, device="cuda")
    assert _call(idx, nbr, (1 << 20) + 1, 0, 0, out, out) == hc.INVALID_ARG
    assert "exceeds" in hc.lib().hc_last_error().decode()
    assert _call(idx, nbr, 3, (1 << 24) + 1, 0, out, out) == hc.INVALID_ARG
    host_idx = np.zeros(4, dtype=np.int64)
    st = hc.lib().hc_bfs_noalloc(host_idx.ctypes.data, nbr.data_ptr(), 3, 0, 0, out.data_ptr(), out.data_ptr(),
                                 None)
    assert st == hc.INVALID_ARG


@pytest.mark.parametrize("kind", ["near_limit", "grid", "isolated_source"])
def test_noalloc_bfs_near_its_limits_and_odd_graphs(kind):
    """Near the fixed working set's limits (Kronecker scale 20, edge factor 8: 2^20 vertices, under 2^24
    edges), on a graph without degree ordering (a grid), and from a source without edges."""
    torch = pytest.importorskip("torch")
    if kind == "near_limit":
        host = hc.gen_kronecker(20, 8, 4)
        assert host.num_nodes == 1 << 20 and host.num_edges <= 1 << 24
        srcs = hc.pick_sources(host, 2)
    elif kind == "grid":
        host = hc.gen_grid(64, 48, 2)
        srcs = np.array([0, 1234], dtype=np.int32)
    else:
        host = hc.gen_kronecker(12, 4, 6)
        srcs = np.array([int(np.flatnonzero(host.degrees() == 0)[0])], dtype=np.int32)
    n, m = host.num_nodes, host.num_edges
    g = hc.Graph.from_host(host)
    idx = torch.from_numpy(host.index).cuda()
    nbr = torch.from_numpy(host.neighbors).cuda()
    for s in srcs:
        depth = torch.empty((n,), dtype=torch.int32, device="cuda")
        parent = torch.empty((n,), dtype=torch.int32, device="cuda")
        assert _call(idx, nbr, n, m, s, depth, parent) == hc.OK, hc.lib().hc_last_error().decode()
        d = depth.cpu().numpy()
        ref, _, _ = g.bfs(np.array([s], dtype=np.int32))
        assert np.array_equal(d, ref[0]) and np.array_equal(d, oracle.bfs_depth(host.index, host.neighbors, s))
        assert oracle.verify_bfs_parents(host.index, host.neighbors, d, parent.cpu().numpy(), s)[0] == 0
