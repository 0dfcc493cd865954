"""hc_graph_load: .sg / .wsg files streamed into device memory through pinned
chunks equal the host loader's CSR, across chunk boundaries; bad files are
refused with HC_ERR_IO."""
import os

import numpy as np
import pytest

import hc
import oracle
from oracle import gen

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scale,weighted", [(12, 0), (12, 1), (12, 2), (20, 2), (20, 0)])
def test_load_equals_host_read(tmp_path, scale, weighted):
    wt = {0: gen.W_NONE, 1: gen.W_F32, 2: gen.W_I32}[weighted]
    idx, nbr, w = gen.build("kronecker", scale, 16, 3, wt)
    path = os.path.join(tmp_path, "g.wsg" if weighted else "g.sg")
    gen.write_graph(path, idx, nbr, w)
    g = hc.Graph.load(path, weighted)
    index, neighbors, weights = g.csr()
    assert np.array_equal(index, idx) and np.array_equal(neighbors, nbr)
    if weighted:
        assert np.array_equal(weights.view(np.uint32), np.asarray(w).view(np.uint32))
    else:
        assert weights is None
    if weighted == 2:
        src = g.pick_sources(2)
        d, _, _ = g.sssp(src)
        for i, s in enumerate(src):
            assert np.array_equal(d[i], oracle.sssp_dijkstra(idx, nbr, w, s))


def _status(path, weighted):
    with pytest.raises(hc.HCError) as e:
        hc.Graph.load(path, weighted)
    return e.value.status


def test_load_refuses_bad_files(tmp_path):
    idx, nbr, w = gen.build("kronecker", 10, 8, 2, gen.W_I32)
    good = os.path.join(tmp_path, "g.wsg")
    gen.write_graph(good, idx, nbr, w)
    data = open(good, "rb").read()
    short = os.path.join(tmp_path, "short.wsg")
    open(short, "wb").write(data[:-3])
    assert _status(short, 2) == hc.IO
    frac = os.path.join(tmp_path, "frac.wsg")
    wf = w.astype(np.float32)
    wf[5] = 2.5
    gen.write_graph(frac, idx, nbr, wf)
    assert _status(frac, 2) == hc.IO
    hc.Graph.load(frac, 1)  # as fp32 weights it is fine
    bad_idx = idx.copy()
    bad_idx[3] = bad_idx[4] + 1
    dec = os.path.join(tmp_path, "dec.wsg")
    gen.write_graph(dec, bad_idx, nbr, w)
    assert _status(dec, 2) == hc.IO
    bad_nbr = nbr.copy()
    bad_nbr[7] = len(idx) + 3
    out = os.path.join(tmp_path, "out.sg")
    gen.write_graph(out, idx, bad_nbr)
    assert _status(out, 0) == hc.IO
    assert _status(os.path.join(tmp_path, "missing.sg"), 0) == hc.IO
