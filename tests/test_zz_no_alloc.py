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
