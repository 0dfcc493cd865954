"""Regenerates the golden fixtures in this directory.

Graphs come from this project's generator (libhc, host code); the outputs come
from the reference's OWN CPU implementation, compiled unchanged from its source
tree into oracle/_ref/ref_driver (see oracle/Makefile), run single-threaded so
PageRank is deterministic.  The fixtures pin the oracle restatement
(oracle/oracle.c) and, through it, the GPU kernels.

Needs the reference tree (it is not present on the GPU box); run here:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "hetero-compute_b200"))

import hc  # noqa: E402
import oracle  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# name: (generator, args, wtype, bfs sources, sssp sources, pagerank?, store full arrays?)
CASES = {
    "kron10": ("kronecker", (10, 16, 1), hc.W_I32, 16, 16, True, True),
    "kron12_ef8": ("kronecker", (12, 8, 7), hc.W_I32, 8, 8, True, True),
    "er10": ("uniform", (10, 8, 3), hc.W_I32, 8, 8, True, True),
    "grid32": ("grid", (32, 32, 5), hc.W_I32, 4, 4, True, True),
    # Kronecker scale 16, edge factor 16, 64 BFS sources.
    "kron16": ("kronecker", (16, 16, 1), hc.W_I32, 64, 4, True, False),
}


def make_graph(kind, args, wtype):
    if kind == "kronecker":
        return hc.gen_kronecker(*args, wtype=wtype)
    if kind == "uniform":
        return hc.gen_uniform(*args, wtype=wtype)
    return hc.gen_grid(*args, wtype=wtype)


def graph_digest(g: hc.HostCSR) -> str:
    h = hashlib.sha256()
    h.update(g.index.tobytes())
    h.update(g.neighbors.tobytes())
    if g.weights is not None:
        h.update(g.weights.tobytes())
    return h.hexdigest()


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def float_dist_to_int(dist: np.ndarray) -> np.ndarray:
    """Reference float distances (integer valued, inf = unreachable) -> int32, INT32_MAX unreachable."""
    fin = np.isfinite(dist)
    assert (np.round(dist[fin]) == dist[fin]).all()
    out = np.full(dist.shape, hc.INF_DIST, dtype=np.int32)
    out[fin] = dist[fin].astype(np.int64)
    return out


def depth_from_parents(parents: np.ndarray, src: int) -> np.ndarray:
    n = len(parents)
    d = np.full(n, -1, dtype=np.int32)
    d[src] = 0
    while True:
        p = parents
        ok = (d == -1) & (p >= 0)
        pd = np.where(ok, d[np.clip(p, 0, n - 1)], -1)
        upd = ok & (pd >= 0)
        if not upd.any():
            break
        d[upd] = pd[upd] + 1
    return d


def main():
    manifest = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, (kind, args, wtype, nb, ns, pr, full) in CASES.items():
            g = make_graph(kind, args, wtype)
            n = g.num_nodes
            sg = os.path.join(tmp, name + ".sg")
            wsg = os.path.join(tmp, name + ".wsg")
            hc.write_graph(sg, hc.HostCSR(g.index, g.neighbors, None))
            hc.write_graph(wsg, g)
            rec = {"kind": kind, "args": list(args), "wtype": wtype, "num_nodes": n, "num_edges": g.num_edges,
                   "graph_sha256": graph_digest(g)}
            arrays = {}
            # BFS: reference bfs_do_cpu parents -> depths implied by the tree.
            out = os.path.join(tmp, "bfs.bin")
            info = oracle.run_reference("bfs", sg, nb, out, threads=1)
            parents = np.fromfile(out, dtype=np.int32).reshape(nb, n)
            depths = np.stack([depth_from_parents(parents[i], s) for i, s in enumerate(info["sources"])])
            rec["bfs_sources"] = info["sources"]
            rec["bfs_depth_sha256"] = [digest(d) for d in depths]
            if full:
                arrays["bfs_depth"] = depths
                arrays["bfs_parents"] = parents
            else:
                arrays["bfs_depth_i8"] = depths.astype(np.int8)
            # SSSP: reference sssp_pull_cpu (float distances, integer valued).
            out = os.path.join(tmp, "sssp.bin")
            info = oracle.run_reference("sssp", wsg, ns, out, threads=1)
            dist = np.fromfile(out, dtype=np.float32).reshape(ns, n)
            idist = float_dist_to_int(dist)
            out2 = os.path.join(tmp, "dij.bin")
            info2 = oracle.run_reference("sssp_dijkstra", wsg, ns, out2, threads=1)
            dj = np.fromfile(out2, dtype=np.float32).reshape(ns, n)
            dj = float_dist_to_int(dj)
            assert (dj == idist).all(), "reference Bellman-Ford and Dijkstra disagree"
            assert info2["sources"] == info["sources"]
            rec["sssp_sources"] = info["sources"]
            rec["sssp_dist_sha256"] = [digest(d) for d in idist]
            if full:
                arrays["sssp_dist"] = idist
            # PageRank: reference pr_pull_cpu on one thread.
            if pr:
                out = os.path.join(tmp, "pr.bin")
                oracle.run_reference("pr", wsg, 0, out, threads=1)
                arrays["pr_scores"] = np.fromfile(out, dtype=np.float32)
            np.savez_compressed(os.path.join(OUT, name + ".npz"), **arrays)
            manifest[name] = rec
            print(name, n, g.num_edges, {k: v.shape for k, v in arrays.items()})
    with open(os.path.join(OUT, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)


if __name__ == "__main__":
    main()
