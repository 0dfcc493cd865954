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
    ug = hc.Graph.from_host(hc.gen_kronecker(8, 4, 1))  # no weights: no weighted PageRank
    x, _ = ug.pagerank()
    with pytest.raises(hc.HCError) as e:
        ug.pagerank_backward(x, np.ones_like(x), weighted=True)
    assert e.value.status == hc.UNSUPPORTED


def test_int32_weights_match_their_fp32_values():
    """Weighted PageRank and its adjoint on int32 weights equal the same run on the weights as fp32."""
    host = hc.gen_kronecker(11, 16, 23, wtype=hc.W_I32)
    gi = hc.Graph.from_host(host)
    gf = hc.Graph(host.index, host.neighbors, host.weights.astype(np.float32))
    rng = np.random.default_rng(3)
    c = rng.standard_normal(host.num_nodes).astype(np.float32)
    xi, _ = gi.pagerank(weighted=True, tol_l1=1e-8, max_iters=300)
    xf, _ = gf.pagerank(weighted=True, tol_l1=1e-8, max_iters=300)
    assert np.array_equal(xi, xf)
    dti, dwi, _ = gi.pagerank_backward(xi, c, weighted=True, tol_l1=1e-8, max_iters=300)
    dtf, dwf, _ = gf.pagerank_backward(xf, c, weighted=True, tol_l1=1e-8, max_iters=300)
    assert np.array_equal(dti, dtf) and np.array_equal(dwi, dwf)
    x64, dt64, dw64 = oracle.pr_dense_grad(host.index, host.neighbors, c.astype(np.float64),
                                           host.weights.astype(np.float64),
                                           np.full(host.num_nodes, 1.0 / host.num_nodes), D)
    assert np.abs(xi - x64).max() < 1e-7
    assert np.abs(dti - dt64).max() < 1e-5 * np.abs(dt64).max()


@pytest.mark.parametrize("weighted", [True, False])
def test_cg_chebyshev_and_jacobi_reach_the_same_gradient(wgraph, ugraph, weighted):
    """accel=0 (conjugate gradients on the symmetric system), 2 (Chebyshev semi-iteration) and -1 (plain
    Jacobi) all match the FP64 dense gradient; conjugate gradients need the fewest sweeps."""
    host, g = wgraph if weighted else ugraph
    c, t, x64, dt64, dw64 = _case(host, weighted, 8)
    x, _ = g.pagerank(t.astype(np.float32), weighted=weighted, tol_l1=1e-10, max_iters=400)
    runs = {}
    for accel in (0, 2, -1):
        dt, dw, st = g.pagerank_backward(x, c.astype(np.float32), weighted=weighted, tol_l1=1e-9, max_iters=500,
                                         accel=accel)
        assert np.abs(dt - dt64).max() < 1e-5 * np.abs(dt64).max(), accel
        assert np.abs(dw - dw64).max() < 1e-4 * np.abs(dw64).max(), accel
        # Sweeps to a tolerance above the fp32 rounding floor (1e-9 never stops before the cap).
        dt, _, st = g.pagerank_backward(x, c.astype(np.float32), weighted=weighted, tol_l1=1e-5, max_iters=500,
                                        accel=accel, want_dw=False)
        assert st.converged and np.abs(dt - dt64).max() < 1e-2 * np.abs(dt64).max(), accel
        runs[accel] = st.iterations
    assert runs[0] < runs[-1] and runs[2] <= 2 * runs[-1], runs


def test_chebyshev_forward(wgraph):
    """accel=1: Chebyshev weights on the forward sweeps reach the same fixed point (opt-in: from the
    uniform start the forward's error is already in fast modes, where plain sweeps do as well)."""
    host, g = wgraph
    _, t, x64, _, _ = _case(host, True, 9)
    x1, s1 = g.pagerank(t.astype(np.float32), weighted=True, tol_l1=1e-7, max_iters=400, accel=1)
    x0, s0 = g.pagerank(t.astype(np.float32), weighted=True, tol_l1=1e-7, max_iters=400, accel=-1)
    assert s1.converged and s0.converged
    assert np.abs(x1 - x64).max() < 1e-7 and np.abs(x0 - x64).max() < 1e-7


def test_asymmetric_weights_fall_back_to_jacobi():
    """w(u->v) != w(v->u): no Chebyshev weights (the walk is not reversible); the result still matches."""
    host = hc.gen_kronecker(11, 8, 7)
    w = np.random.default_rng(1).random(host.num_edges).astype(np.float32) + 0.01
    g = hc.Graph(host.index, host.neighbors, w)
    rng = np.random.default_rng(2)
    c = rng.standard_normal(host.num_nodes)
    t = np.full(host.num_nodes, 1.0 / host.num_nodes)
    x64, dt64, dw64 = oracle.pr_dense_grad(host.index, host.neighbors, c, w.astype(np.float64), t, D)
    x, _ = g.pagerank(t.astype(np.float32), weighted=True, tol_l1=1e-10, max_iters=400)
    dt, dw, _ = g.pagerank_backward(x, c.astype(np.float32), weighted=True, tol_l1=1e-9, max_iters=500)
    assert np.abs(dt - dt64).max() < 1e-5 * np.abs(dt64).max()
    assert np.abs(dw - dw64).max() < 1e-4 * np.abs(dw64).max()
