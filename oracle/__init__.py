"""TEST INFRASTRUCTURE ONLY: Python access to the oracle.

Wraps oracle/liboracle.so (the plain-C restatement in oracle.c) and adds the
FP64 dense-solve references for the PageRank adjoint, which has no counterpart
in the reference.  Only tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline leg use this module, always as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")
INF = 0x7FFFFFFF

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.or_bfs_depth.argtypes = [P, P, C.c_int32, C.c_int32, P]
        L.or_bfs_depth.restype = C.c_int
        L.or_verify_bfs_parents.argtypes = [P, P, P, P, C.c_int32, C.c_int32, P]
        L.or_verify_bfs_parents.restype = C.c_int64
        L.or_sssp_dijkstra.argtypes = [P, P, P, C.c_int32, C.c_int32, P]
        L.or_sssp_dijkstra.restype = C.c_int
        L.or_verify_sp_tree.argtypes = [P, P, P, P, P, C.c_int32, C.c_int32]
        L.or_verify_sp_tree.restype = C.c_int64
        L.or_pr_pull.argtypes = [P, P, C.c_int32, C.c_float, C.c_float, C.c_int32, P, P]
        L.or_pr_pull.restype = C.c_int32
        L.or_pr_jacobi_f64.argtypes = [P, P, P, C.c_int32, P, C.c_double, C.c_double, C.c_int32, P]
        L.or_pr_jacobi_f64.restype = C.c_int32
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def bfs_depth(index, nbr, src):
    n = len(index) - 1
    d = np.empty(n, dtype=np.int32)
    assert lib().or_bfs_depth(_p(index), _p(nbr), n, int(src), _p(d)) == 0
    return d


def verify_bfs_parents(index, nbr, depth, parents, src):
    """Error count of tests/bfs/bfs_verify.cu:133-197 plus a neighbour check."""
    counts = np.zeros(5, dtype=np.int64)
    parents = np.ascontiguousarray(parents, dtype=np.int32)
    bad = lib().or_verify_bfs_parents(_p(index), _p(nbr), _p(depth), _p(parents), len(index) - 1, int(src),
                                      _p(counts))
    return int(bad), counts


def sssp_dijkstra(index, nbr, w, src):
    n = len(index) - 1
    d = np.empty(n, dtype=np.int32)
    assert lib().or_sssp_dijkstra(_p(index), _p(nbr), _p(np.ascontiguousarray(w, dtype=np.int32)), n, int(src),
                                  _p(d)) == 0
    return d


def verify_sp_tree(index, nbr, w, dist, parent, src):
    return int(lib().or_verify_sp_tree(_p(index), _p(nbr), _p(np.ascontiguousarray(w, dtype=np.int32)), _p(dist),
                                       _p(np.ascontiguousarray(parent, dtype=np.int32)), len(index) - 1, int(src)))


def pr_pull(index, nbr, damping=0.85, eps=5e-8, max_iters=0, init=None):
    """Reference CPU PageRank on one thread (src/kernels/cpu/pr.cuh:33-65); init (fp32 [N]) replaces the
    uniform 1/N start, as the caller's init_score of pr_pull_gpu (src/kernels/gpu/pr.cuh:42-46)."""
    n = len(index) - 1
    s = np.empty(n, dtype=np.float32)
    ini = None if init is None else np.ascontiguousarray(init, dtype=np.float32)
    it = lib().or_pr_pull(_p(index), _p(nbr), n, damping, eps, max_iters, _p(ini), _p(s))
    return s, int(it)


def pr_jacobi_f64(index, nbr, w=None, teleport=None, damping=0.85, tol=1e-14, max_iters=2000):
    n = len(index) - 1
    x = np.empty(n, dtype=np.float64)
    wf = None if w is None else np.ascontiguousarray(w, dtype=np.float32)
    t = None if teleport is None else np.ascontiguousarray(teleport, dtype=np.float64)
    it = lib().or_pr_jacobi_f64(_p(index), _p(nbr), _p(wf), n, _p(t), damping, tol, max_iters, _p(x))
    return x, int(it)


# ------------------------------------------------- adjoint (no reference)

def transition_dense(index, nbr, w=None):
    """A[v, u] = W_uv = w_uv / sum_k w_uk (w None: 1/deg u), FP64 dense."""
    n = len(index) - 1
    A = np.zeros((n, n), dtype=np.float64)
    for u in range(n):
        b, e = index[u], index[u + 1]
        if b == e:
            continue
        ws = np.ones(e - b) if w is None else w[b:e].astype(np.float64)
        A[nbr[b:e], u] = ws / ws.sum()
    return A


def pr_dense(index, nbr, w=None, teleport=None, damping=0.85):
    """x = (1-d) (I - d A)^-1 t by a dense FP64 solve."""
    n = len(index) - 1
    A = transition_dense(index, nbr, w)
    t = np.full(n, 1.0 / n) if teleport is None else np.asarray(teleport, dtype=np.float64)
    return np.linalg.solve(np.eye(n) - damping * A, (1 - damping) * t)


def pr_dense_grad(index, nbr, c, w=None, teleport=None, damping=0.85):
    """Gradients of L = c . x: dL/dt = (1-d) (I - d A)^-T c and dL/dw (CSR slot order of row u) via the
    exact chain rule through the row normalisation."""
    n = len(index) - 1
    A = transition_dense(index, nbr, w)
    M = np.eye(n) - damping * A
    x = pr_dense(index, nbr, w, teleport, damping)
    lam = np.linalg.solve(M.T, np.asarray(c, dtype=np.float64))
    dt = (1 - damping) * lam
    dw = np.zeros(len(nbr), dtype=np.float64)
    for u in range(n):
        b, e = index[u], index[u + 1]
        if b == e:
            continue
        ws = np.ones(e - b) if w is None else w[b:e].astype(np.float64)
        s = ws.sum()
        W = ws / s
        lk = lam[nbr[b:e]]
        dw[b:e] = damping * x[u] / s * (lk - np.dot(W, lk))
    return x, dt, dw


def run_reference(algo, graph_path, nsrc, out_path, threads=None, timeout=None, repeats=1, warmup=0):
    """Runs the reference's own CPU code (oracle/_ref/ref_driver); returns its JSON line as a dict.
    repeats: the source sequence runs that many times in one process (per-run ms for each); warmup: untimed
    runs from the first source before them."""
    import json
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    r = subprocess.run([REF_DRIVER, algo, graph_path, str(nsrc), out_path, str(repeats), str(warmup)],
                       capture_output=True, text=True, env=env, check=True, timeout=timeout)
    return json.loads(r.stdout.strip().splitlines()[-1])


def equal_edge_ranges_reference(index, num_segments, chunk_size=1):
    """compute_equal_edge_ranges (src/graph.cuh:156-201) step by step, with its array allowed to grow: returns
    (bounds written, in order; closures).  bounds[0] = 0; a closure at vertex v writes v; after the walk, if
    fewer than num_segments closures happened, num_nodes is written next; inner bounds 1 .. num_segments - 1
    are rounded to chunk_size.  Entries the reference leaves unwritten are absent."""
    n = len(index) - 1
    avg = int(index[n] - index[0]) // num_segments
    b = [0]
    acc, closures = 0, 0
    for v in range(n):
        acc += int(index[v + 1] - index[v])
        if acc >= avg:
            b.append(v)
            acc = 0
            closures += 1
    if closures != num_segments:
        b.append(n)
    for i in range(1, min(num_segments, len(b))):
        r = b[i] % chunk_size
        if r:
            b[i] = b[i] - r if r < chunk_size // 2 else b[i] - r + chunk_size
    return b, closures
