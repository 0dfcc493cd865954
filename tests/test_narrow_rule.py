"""The rule behind batched SSSP's 16-bit working distances, checked on the CPU.

Distances are kept below an unreachable mark INF (0xF000); a relaxation whose
candidate d[u] + w would reach INF is dropped, so a distance that does not fit
stays unreachable.  The claim: when the largest final finite distance plus the
largest weight is below INF, the result equals the true shortest distances,
whatever order the relaxations ran in.  Here a chaotic in-place relaxation with
that rule runs on random graphs (random edge order each pass) and is compared
with Dijkstra from the oracle; where the check fails, the caller would rerun
with 32-bit distances, so only the claim's direction is asserted, plus that the
check does fail whenever some reachable distance does not fit.
"""
import numpy as np
import pytest

import oracle

INF16 = 0xF000
I32_MAX = np.iinfo(np.int32).max


def _random_graph(rng, n, m, wmin, wmax, chain):
    u = rng.integers(0, n, size=m)
    v = rng.integers(0, n, size=m)
    if chain:  # a long path through every vertex, so distances grow with n
        u = np.concatenate([u, np.arange(n - 1)])
        v = np.concatenate([v, np.arange(1, n)])
    keep = u != v
    u, v = u[keep], v[keep]
    w = rng.integers(wmin, wmax + 1, size=len(u))
    # symmetric, deduplicated by keeping the lightest of parallel edges
    a = np.concatenate([u, v])
    b = np.concatenate([v, u])
    ww = np.concatenate([w, w])
    order = np.lexsort((ww, b, a))
    a, b, ww = a[order], b[order], ww[order]
    first = np.ones(len(a), dtype=bool)
    first[1:] = (a[1:] != a[:-1]) | (b[1:] != b[:-1])
    a, b, ww = a[first], b[first], ww[first]
    index = np.zeros(n + 1, dtype=np.int64)
    np.add.at(index, a + 1, 1)
    index = np.cumsum(index)
    return index, b.astype(np.int32), ww.astype(np.int32)


def _narrow_relax(index, nbr, w, src, rng):
    n = len(index) - 1
    d = np.full(n, INF16, dtype=np.int64)
    d[src] = 0
    rows = np.repeat(np.arange(n), np.diff(index))
    while True:
        changed = False
        for e in rng.permutation(len(nbr)):
            u, v = rows[e], nbr[e]
            if d[u] >= INF16:
                continue
            c = d[u] + w[e]
            if c < INF16 and c < d[v]:
                d[v] = c
                changed = True
        if not changed:
            return d


@pytest.mark.parametrize("seed", range(16))
def test_narrow_rule(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(8, 60))
    chain = bool(seed % 2)
    if chain:  # sparse heavy chains: distances from a few thousand to well past the mark
        index, nbr, w = _random_graph(rng, n, int(rng.integers(0, n // 6 + 1)), 1500, 4095, True)
    else:
        index, nbr, w = _random_graph(rng, n, int(rng.integers(n, 4 * n)), 1, int(rng.choice([255, 4095])), False)
    for src in rng.choice(n, size=3, replace=False):
        d16 = _narrow_relax(index, nbr, w, int(src), rng)
        exact = oracle.sssp_dijkstra(index, nbr, w, int(src)).astype(np.int64)
        finite = d16[d16 < INF16]
        fits = finite.max() + w.max() < INF16
        true_fits = exact[exact != I32_MAX].max() < INF16
        if fits:
            got = np.where(d16 >= INF16, I32_MAX, d16)
            assert np.array_equal(got, exact), (seed, src)
        if not true_fits:
            assert not fits, (seed, src)  # a distance that does not fit always fails the check


def test_narrow_rule_boundary():
    """A path of weight 4095: 15 vertices fit (largest distance 57330 + 4095 < 0xF000), 16 fail the
    check (61425 + 4095), 17 hold a distance that 16 bits cannot store."""
    rng = np.random.default_rng(0)
    for n, fits_expected in ((15, True), (16, False), (17, False)):
        index = np.concatenate([[0], np.cumsum([1] + [2] * (n - 2) + [1])]).astype(np.int64)
        nbr = np.concatenate([[v for v in (u - 1, u + 1) if 0 <= v < n] for u in range(n)]).astype(np.int32)
        w = np.full(len(nbr), 4095, dtype=np.int32)
        d16 = _narrow_relax(index, nbr, w, 0, rng)
        finite = d16[d16 < INF16]
        assert (finite.max() + 4095 < INF16) == fits_expected, n
