"""CPU check of the rule behind hc_pr_pull_ordered: on a graph whose edges all
have a reverse, updating the vertices level by level (level(v) = 1 + max level
of its lower neighbours), each level in one vectorised step, gives the scores of
the reference's sequential in-place sweep (src/kernels/cpu/pr.cuh:33-65,
:157-187; the oracle's or_pr_pull) bit for bit, when every row is summed in CSR
order in fp32.  Runs the level schedule in numpy, no GPU."""
import numpy as np
import pytest

import hc
import oracle


def level_schedule(index, nbr):
    n = len(index) - 1
    lev = np.zeros(n, dtype=np.int64)
    for v in range(n):
        nb = nbr[index[v]:index[v + 1]]
        nb = nb[nb < v]
        lev[v] = lev[nb].max() + 1 if len(nb) else 0
    return lev


def ordered_sweeps(index, nbr, damping=np.float32(0.85), eps=np.float32(5e-8), max_sweeps=10000):
    n = len(index) - 1
    lev = level_schedule(index, nbr)
    deg = np.diff(index)
    degf = deg.astype(np.float32)
    score = np.full(n, np.float32(1.0) / np.float32(n), dtype=np.float32)
    base = (np.float32(1.0) - damping) / np.float32(n)
    levels = [np.flatnonzero(lev == l) for l in range(int(lev.max()) + 1)]
    sweeps = 0
    with np.errstate(divide="ignore", invalid="ignore"):
        while sweeps < max_sweeps:
            updated = 0
            for verts in levels:
                d = deg[verts]
                total = np.zeros(len(verts), dtype=np.float32)
                # Row sums in CSR order: position j of every row at once.
                for j in range(int(d.max()) if len(d) else 0):
                    rows = d > j
                    u = nbr[index[verts[rows]] + j]
                    total[rows] = total[rows] + score[u] / degf[u]
                new = base + damping * total
                move = np.abs(new - score[verts]) > eps
                score[verts[move]] = new[move]
                updated += int(move.sum())
            sweeps += 1
            if updated == 0:
                break
    return score, sweeps


@pytest.mark.parametrize("maker", [lambda: hc.gen_kronecker(10, 16, 1), lambda: hc.gen_kronecker(11, 8, 4),
                                   lambda: hc.gen_uniform(10, 8, 3), lambda: hc.gen_grid(20, 30, 2)])
def test_level_schedule_reproduces_sequential_sweep(maker):
    g = maker()
    ref, it = oracle.pr_pull(g.index, g.neighbors)
    s, sweeps = ordered_sweeps(g.index, g.neighbors)
    assert sweeps == it
    assert np.array_equal(s.view(np.uint32), ref.view(np.uint32))


def test_level_schedule_separates_neighbours():
    g = hc.gen_kronecker(11, 16, 2)
    lev = level_schedule(g.index, g.neighbors)
    src = np.repeat(np.arange(g.num_nodes), np.diff(g.index))
    dst = g.neighbors
    keep = src != dst
    lo, hi = np.minimum(src, dst)[keep], np.maximum(src, dst)[keep]
    assert (lev[lo] < lev[hi]).all()  # a lower neighbour is always placed in an earlier level
