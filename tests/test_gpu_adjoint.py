"""PageRank adjoint on the GPU: dL/d(teleport) and dL/d(edge weights) for
L = sum_i c_i x_i, checked against an FP64 dense-solve gradient and FP64 central
finite differences on a scale-12 graph (no counterpart in the reference)."""
import numpy as np
import pytest

import hc
import oracle

pytestmark = pytest.mark.gpu

D = 0.85


@pytest.fixture(scope="module")
def wgraph():
    host = hc.gen_kronecker(12, 16, 21, wtype=hc.W_F32)
    return host, hc.Graph.from_host(host)


@pytest.fixture(scope="module")
def ugraph():
    host = hc.gen_kronecker(12, 16, 22)
    return host, hc.Graph.from_host(host)


def _case(host, weighted, seed):
    rng = np.random.default_rng(seed)
    n = host.num_nodes
    c = rng.standard_normal(n)
    t = rng.random(n)
    t /= t.sum()
    w = host.weights.astype(np.float64) if weighted else None
    x, dt, dw = oracle.pr_dense_grad(host.index, host.neighbors, c, w, t, D)
    return c, t, x, dt, dw


@pytest.mark.parametrize("weighted", [True, False])
def test_adjoint_matches_dense_solve(wgraph, ugraph, weighted):
    host, g = wgraph if weighted else ugraph
    c, t, x64, dt64, dw64 = _case(host, weighted, 5)
    x, st = g.pagerank(t.astype(np.float32), weighted=weighted, tol_l1=1e-10, max_iters=400)
    assert np.abs(x - x64).max() < 1e-7
    dt, dw, bst = g.pagerank_backward(x, c.astype(np.float32), weighted=weighted, tol_l1=1e-9, max_iters=500)
    e_t = np.abs(dt - dt64).max() / np.abs(dt64).max()
    e_w = np.abs(dw - dw64).max() / np.abs(dw64).max()
    assert e_t < 1e-5, e_t
    assert e_w < 1e-4, e_w


def test_adjoint_matches_finite_differences(wgraph):
    host, g = wgraph
    c, t, x64, _, _ = _case(host, True, 6)
    x, _ = g.pagerank(t.astype(np.float32), weighted=True, tol_l1=1e-10, max_iters=400)
    dt, dw, _ = g.pagerank_backward(x, c.astype(np.float32), weighted=True, tol_l1=1e-9, max_iters=500)
    rng = np.random.default_rng(9)
    w = host.weights.astype(np.float64)
    h = 1e-6

    def loss(tt, ww):
        return c @ oracle.pr_dense(host.index, host.neighbors, ww, tt, D)

    for j in rng.choice(host.num_nodes, 4, replace=False):
        tp, tm = t.copy(), t.copy()
        tp[j] += h
        tm[j] -= h
        fd = (loss(tp, w) - loss(tm, w)) / (2 * h)
        assert abs(fd - dt[j]) <= 1e-4 * max(1.0, np.abs(dt).max()), (j, fd, dt[j])
    big = np.argsort(-np.abs(dw))[:3]
    for e in list(big) + list(rng.choice(host.num_edges, 3, replace=False)):
        wp, wm = w.copy(), w.copy()
        wp[e] += h
        wm[e] -= h
        fd = (loss(t, wp) - loss(t, wm)) / (2 * h)
        assert abs(fd - dw[e]) <= 1e-3 * np.abs(dw).max(), (e, fd, dw[e])


def test_autograd_function(wgraph):
    torch = pytest.importorskip("torch")
    from hc.autograd import pagerank
    host, g = wgraph
    c, t, x64, dt64, dw64 = _case(host, True, 7)
    tt = torch.tensor(t, dtype=torch.float32, device="cuda", requires_grad=True)
    ww = torch.tensor(host.weights, dtype=torch.float32, device="cuda", requires_grad=True)
    x = pagerank(g, tt, ww)
    loss = (torch.tensor(c, dtype=torch.float32, device="cuda") * x).sum()
    loss.backward()
    assert abs(loss.item() - float(c @ x64)) < 1e-5 * max(1, abs(float(c @ x64)))
    assert np.abs(tt.grad.cpu().numpy() - dt64).max() < 1e-5 * np.abs(dt64).max()
    assert np.abs(ww.grad.cpu().numpy() - dw64).max() < 1e-4 * np.abs(dw64).max()


def test_backward_requires_inputs(ugraph):
    host, g = ugraph
    st = hc.lib().hc_pr_backward(g.handle, None, None, None, None, None, None)
    assert st == hc.INVALID_ARG
    fg = hc.Graph.from_host(hc.gen_kronecker(8, 4, 1, wtype=hc.W_I32))  # int weights: no weighted PageRank
    x, _ = fg.pagerank()
    with pytest.raises(hc.HCError) as e:
        fg.pagerank_backward(x, np.ones_like(x), weighted=True)
    assert e.value.status == hc.UNSUPPORTED
