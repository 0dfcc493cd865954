"""torch.autograd binding of the PageRank forward and its hand-written adjoint.

`pagerank(graph, teleport, weights)` returns the scores x solving
x = (1-d) t + d A x on the device; backward calls hc_pr_backward, which solves
lambda = dL/dx + d A^T lambda on the GPU and returns dL/dt = (1-d) lambda and
dL/dw (raw edge weights, CSR slot order).  `weights` must be the tensor the
graph handle was created from: it carries the gradient, the handle holds the
values.  Test binding only -- the product entry points are the C ABI.
"""
from __future__ import annotations

import torch

from . import Graph


class _PageRank(torch.autograd.Function):
    @staticmethod
    def forward(ctx, teleport, weights, graph: Graph, damping, tol_l1, max_iters, weighted):
        scores = torch.empty_like(teleport)
        graph.pagerank(teleport.contiguous(), scores, damping=damping, tol_l1=tol_l1, max_iters=max_iters,
                       weighted=weighted)
        ctx.graph = graph
        ctx.opts = (damping, weighted, max_iters)
        ctx.save_for_backward(scores)
        return scores

    @staticmethod
    def backward(ctx, grad):
        (scores,) = ctx.saved_tensors
        damping, weighted, max_iters = ctx.opts
        g = ctx.graph
        dt = torch.empty_like(scores)
        dw = torch.empty(g.num_edges, dtype=torch.float32, device=scores.device) if ctx.needs_input_grad[1] else None
        g.pagerank_backward(scores, grad.contiguous(), damping=damping, tol_l1=1e-9, max_iters=max(max_iters, 500),
                            weighted=weighted, want_dw=dw is not None, dteleport=dt, dweights=dw)
        return dt, dw, None, None, None, None, None


def pagerank(graph: Graph, teleport: torch.Tensor, weights: torch.Tensor | None = None, *, damping=0.85,
             tol_l1=1e-9, max_iters=500):
    """Differentiable PageRank scores (fp32, on the graph's device)."""
    weighted = weights is not None
    if weights is None:
        weights = torch.zeros(0, device=teleport.device, requires_grad=False)
    return _PageRank.apply(teleport, weights, graph, damping, tol_l1, max_iters, weighted)
