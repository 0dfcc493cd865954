"""Input guards: bad CSR arrays are refused before any traversal kernel reads
them, and int32 distance overflow is reported instead of returned wrapped."""
import numpy as np
import pytest

import hc
import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

INT32_MAX = 2**31 - 1


def _path(weights):
    """Symmetric path 0 - 1 - ... - k with the given edge weights."""
    k = len(weights)
    rows = [[] for _ in range(k + 1)]
    for i, w in enumerate(weights):
        rows[i].append((i + 1, w))
        rows[i + 1].append((i, w))
    index = np.zeros(k + 2, dtype=np.int64)
    index[1:] = np.cumsum([len(r) for r in rows])
    nbr = np.array([v for r in rows for v, _ in sorted(r)], dtype=np.int32)
    w = np.array([x for r in rows for _, x in sorted(r)], dtype=np.int32)
    return index, nbr, w


def test_sssp_int32_overflow_is_reported():
    """Candidates clamp at INT32_MAX; a run whose distances come within the largest weight of it is refused
    (there a clamped candidate may have hidden a longer distance), one that stays below is exact."""
    for weights in ([2**30, 2**30], [2**30 - 1, 2**30 - 1, 1], [2**29, 2**29, 2**29, 2**29]):
        index, nbr, w = _path(weights)
        g = hc.Graph(index, nbr, w)
        with pytest.raises(hc.HCError) as e:
            g.sssp([0])
        assert e.value.status == hc.UNSUPPORTED
        with pytest.raises(hc.HCError) as e:
            g.sssp_batched(np.array([0, 1], dtype=np.int32))
        assert e.value.status == hc.UNSUPPORTED
    index, nbr, w = _path([2**29, 2**29, 2**28, 5])  # largest distance 2^30 + 2^28 + 5, + 2^29 < INT32_MAX
    g = hc.Graph(index, nbr, w)
    d, _, _ = g.sssp([0, 4])
    far = 2**30 + 2**28 + 5
    assert list(d[0]) == [0, 2**29, 2**30, 2**30 + 2**28, far]
    assert list(d[1]) == [far, 2**29 + 2**28 + 5, 2**28 + 5, 5, 0]
    db, _ = g.sssp_batched(np.array([0, 4], dtype=np.int32))
    assert np.array_equal(db, d)


def test_sssp_large_weights_below_the_limit_are_exact():
    host = hc.gen_kronecker(10, 8, 5, wtype=hc.W_I32)
    w = (host.weights.astype(np.int64) * 2**20).astype(np.int32)  # up to 255 * 2^20: the range check runs
    g = hc.Graph(host.index, host.neighbors, w)
    src = hc.pick_sources(host, 3)
    d, _, _ = g.sssp(src)  # the overflow check runs (w_max * (n - 1) >= INT32_MAX) and finds nothing
    for i, s in enumerate(src):
        assert np.array_equal(d[i], oracle.sssp_dijkstra(host.index, host.neighbors, w, s))


def _bad_csrs():
    host = hc.gen_kronecker(10, 8, 2)
    n, m = host.num_nodes, host.num_edges
    good = (host.index.copy(), host.neighbors.copy(), n, m)
    dec = host.index.copy()
    dec[5] = dec[6] + 1  # offsets fall
    out = host.neighbors.copy()
    out[m // 2] = n  # id outside [0, n)
    neg = host.neighbors.copy()
    neg[3] = -1
    short = host.index.copy()
    short[-1] = m - 1  # index[n] != num_edges
    start = host.index.copy()
    start[0] = 1  # index[0] != 0
    return good, [(dec, host.neighbors, n, m), (host.index, out, n, m), (host.index, neg, n, m),
                  (short, host.neighbors, n, m), (start, host.neighbors, n, m)]


def test_csr_check_refuses_bad_arrays():
    good, bad = _bad_csrs()
    idx, nbr, n, m = good
    ti, tn = torch.from_numpy(idx).cuda(), torch.from_numpy(nbr).cuda()
    assert hc.lib().hc_csr_check(ti.data_ptr(), tn.data_ptr(), 0, n, m, None) == hc.OK
    for idx, nbr, n, m in bad:
        ti, tn = torch.from_numpy(idx).cuda(), torch.from_numpy(nbr).cuda()
        assert hc.lib().hc_csr_check(ti.data_ptr(), tn.data_ptr(), 0, n, m, None) == hc.INVALID_ARG
    # interleaved {v, w} edges, as the reference's wnode_t
    idx, nbr, n, m = good
    wn = np.empty(2 * m, dtype=np.int32)
    wn[0::2], wn[1::2] = nbr, np.float32(1.0).view(np.int32)
    ti, tw = torch.from_numpy(idx).cuda(), torch.from_numpy(wn).cuda()
    assert hc.lib().hc_csr_check(ti.data_ptr(), tw.data_ptr(), 1, n, m, None) == hc.OK
    wn[2 * 7] = n + 5
    tw = torch.from_numpy(wn).cuda()
    assert hc.lib().hc_csr_check(ti.data_ptr(), tw.data_ptr(), 1, n, m, None) == hc.INVALID_ARG


def test_noalloc_refuses_bad_arrays_and_then_runs():
    good, bad = _bad_csrs()
    for idx, nbr, n, m in bad:
        ti, tn = torch.from_numpy(idx).cuda(), torch.from_numpy(nbr).cuda()
        d = torch.empty(n, dtype=torch.int32, device="cuda")
        p = torch.empty(n, dtype=torch.int32, device="cuda")
        st = hc.lib().hc_bfs_noalloc(ti.data_ptr(), tn.data_ptr(), n, m, 0, d.data_ptr(), p.data_ptr(), None)
        assert st == hc.INVALID_ARG
    idx, nbr, n, m = good
    ti, tn = torch.from_numpy(idx).cuda(), torch.from_numpy(nbr).cuda()
    d = torch.empty(n, dtype=torch.int32, device="cuda")
    p = torch.empty(n, dtype=torch.int32, device="cuda")
    src = int(hc.pick_sources(hc.HostCSR(idx, nbr), 1)[0])
    assert hc.lib().hc_bfs_noalloc(ti.data_ptr(), tn.data_ptr(), n, m, src, d.data_ptr(), p.data_ptr(), None) == hc.OK
    assert np.array_equal(d.cpu().numpy(), oracle.bfs_depth(idx, nbr, src))


def test_graph_create_refuses_bad_arrays():
    _, bad = _bad_csrs()
    for idx, nbr, n, m in bad:
        with pytest.raises(hc.HCError) as e:
            hc.Graph(idx, nbr)
        assert e.value.status == hc.INVALID_ARG
