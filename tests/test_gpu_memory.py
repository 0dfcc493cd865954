"""Device memory pressure: a call whose allocation fails releases the rebuildable derived arrays it does not
need (the SSSP pull sweeps' pair array here) and tries once more, and a later call builds them again."""
import numpy as np
import pytest

import hc
import oracle

pytestmark = pytest.mark.gpu


def test_weighted_pagerank_reclaims_the_sssp_pair_array():
    torch = pytest.importorskip("torch")
    host = hc.gen_kronecker(20, 16, 7, wtype=hc.W_I32)
    n, m = host.num_nodes, host.num_edges
    src = hc.pick_sources(host, 2)
    ref = hc.Graph.from_host(host)
    x_ref, st_ref = ref.pagerank(weighted=True, tol_l1=1e-6)
    ref.close()

    g = hc.Graph.from_host(host)
    d0, _, _ = g.sssp(src)  # builds the pair array: 8 (M + 64) bytes
    held_adj = g.info().device_bytes
    adj_bytes = 8 * (m + 64)
    weighted_bytes = 8 * (m + 64) + 4 * n  # fp32 weights, normalised weights, 1 / row sums
    free, _ = torch.cuda.mem_get_info()
    # Leave less than the weighted arrays need, and more than they need once the pair array is gone.
    leave = weighted_bytes - adj_bytes // 2
    filler = torch.empty(max(free - leave, 0), dtype=torch.uint8, device="cuda")
    try:
        x, st = g.pagerank(weighted=True, tol_l1=1e-6)
        held_after = g.info().device_bytes
    finally:
        del filler
        torch.cuda.empty_cache()
    assert held_after < held_adj - adj_bytes + weighted_bytes + adj_bytes // 2  # the pair array went
    assert st.iterations == st_ref.iterations
    assert np.allclose(x, x_ref, rtol=0, atol=1e-7)
    # SSSP builds the pair array again and stays exact.
    d1, _, _ = g.sssp(src)
    assert np.array_equal(d1, d0)
    for i, s in enumerate(src):
        assert np.array_equal(d1[i], oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, s))
    g.close()
