"""Equal-edge vertex ranges (hc_equal_edge_ranges) against a step-by-step
restatement of the reference's compute_equal_edge_ranges (src/graph.cuh:156-201)
wherever the reference's result is well defined, and the stated departures
where it is not.  CPU only."""
import numpy as np
import pytest

import hc
import oracle
from hc import profile


@pytest.mark.parametrize("maker", [lambda: hc.gen_kronecker(12, 16, 1), lambda: hc.gen_uniform(11, 8, 2),
                                   lambda: hc.gen_grid(30, 31, 1), lambda: hc.gen_kronecker(9, 4, 7)])
@pytest.mark.parametrize("segs", [1, 2, 3, 4, 7, 16, 64])
@pytest.mark.parametrize("chunk", [1, 32])
def test_ranges_match_the_reference_where_defined(maker, segs, chunk):
    g = maker()
    n = g.num_nodes
    ours = profile.equal_edge_ranges(g.index, segs, chunk)
    ref, closures = oracle.equal_edge_ranges_reference(g.index, segs, chunk)
    assert ours[0] == 0 and ours[-1] == n and (np.diff(ours) >= 0).all()  # a partition of [0, N)
    if closures < segs:
        # well defined in the reference: bounds written up to its final N
        assert list(ours[:len(ref)]) == ref
        assert (ours[len(ref):] == n).all()
    else:
        # the reference drops [v_last, N) (or writes past its array); ours closes at most segs - 1 times
        assert list(ours[:segs]) == ref[:segs]


def test_ranges_edge_totals_balance():
    g = hc.gen_kronecker(14, 16, 3)
    r = profile.equal_edge_ranges(g.index, 16)
    e = g.index[r[1:]] - g.index[r[:-1]]
    assert e.sum() == g.num_edges
    avg = g.num_edges // 16
    deg = np.diff(g.index)
    # A segment closes once its edges plus those of the closing vertex (which opens the next one) reach
    # the average.
    assert (e[:-1] + deg[r[1:-1]] >= avg).all()


def test_ranges_reject_bad_arguments():
    g = hc.gen_kronecker(8, 4, 1)
    with pytest.raises(hc.HCError):
        profile.equal_edge_ranges(g.index, 0)
