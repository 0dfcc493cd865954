"""Autotuner: the tuned parameters come from the candidate sets, results stay
exact under the tuned launch parameters, and explicit options still win."""
import math

import numpy as np
import pytest

import hc
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tuned():
    host = hc.gen_kronecker(14, 16, 51, wtype=hc.W_I32)
    g = hc.Graph.from_host(host)
    src = hc.pick_sources(host, 64)
    t = g.autotune(src)
    return host, g, src, t


def test_tuned_values_come_from_the_candidates(tuned):
    host, g, src, t = tuned
    assert t["trials"] > 20 and t["tune_ms"] > 0
    assert t["bfs_bu_variant"] in (hc.VARIANT_THREAD, hc.VARIANT_WARP, hc.VARIANT_BLOCK)
    # BFS alpha: a coarse pass, then floor(0.7 x) and floor(1.4 x) around the winner (double arithmetic,
    # as the tuner computes them); SSSP pull alpha: 2-16, then -1 / +1 / x1.5 around the winner.
    coarse = (4, 8, 15, 30, 45, 60, 90, 120, 240)
    alphas = set(coarse) | {max(1, math.floor(b * f)) for b in coarse for f in (0.7, 1.4)}
    assert t["bfs_alpha"] in alphas and t["bfs_beta"] in (6, 12, 18, 36, 72)
    assert t["sssp_delta"] > 0 and (t["sssp_pull_alpha"] == -1 or 1 <= t["sssp_pull_alpha"] <= 24)
    assert t["mbfs_group"] in (64, 128, 256, 512) and t["mbfs_switch_alpha"] in (5, 10, 20, 40, -1)
    assert t["mssp_group"] in (64, 128, 256, 512) and t["mssp_switch_alpha"] in (1, 2, 4, -1)
    assert 0 <= t["bfs_bu_split_levels"] <= 8 and len(t["bfs_bu_split"]) == t["bfs_bu_split_levels"]
    assert g.tuning == t


def test_results_exact_under_tuning(tuned):
    host, g, src, t = tuned
    s = src[:6]
    depth, parent, _ = g.bfs(s)
    dist, _, _ = g.sssp(s)
    mdepth, _ = g.bfs_batched(src)
    mdist, _ = g.sssp_batched(src)
    for i, v in enumerate(s):
        ref_d = oracle.bfs_depth(host.index, host.neighbors, v)
        ref_s = oracle.sssp_dijkstra(host.index, host.neighbors, host.weights, v)
        assert np.array_equal(depth[i], ref_d) and np.array_equal(mdepth[i], ref_d)
        assert np.array_equal(dist[i], ref_s) and np.array_equal(mdist[i], ref_s)


def test_set_tuning_round_trip_and_explicit_options_win(tuned):
    host, g, src, t = tuned
    saved = g.tuning
    g.set_tuning(dict(saved, mssp_group=32, mbfs_group=64))
    _, st = g.sssp_batched(src[:40])
    assert st.groups == 2  # tuned width 32
    _, st = g.sssp_batched(src[:40], group=64)
    assert st.groups == 1  # explicit option
    _, st = g.bfs_batched(np.resize(src, 100))  # 100 sources, duplicates allowed
    assert st.groups == 2
    with pytest.raises(hc.HCError) as e:
        g.set_tuning(dict(saved, bfs_bu_variant=9))
    assert e.value.status == hc.INVALID_ARG
    g.set_tuning(saved)
    assert g.tuning == saved


def test_per_level_split_table_exact_and_validated(tuned):
    """The per-bottom-up-level warp/thread split (the per-epoch granularity selector): tuned splits come
    from the equal-edge segment bounds, hand-set tables of every shape keep BFS exact, and bad tables are
    refused."""
    from hc import profile
    host, g, src, t = tuned
    bounds = set(profile.equal_edge_ranges(host.index[:g.info().num_active + 1], 16, 32).tolist())
    n_active = g.info().num_active
    for x in t["bfs_bu_split"]:
        assert x in bounds or x % 32 == 0, x
    saved = g.tuning
    s = src[:5]
    for table in ([0], [n_active], [n_active, 0, 1024], [64, 4096, 0, n_active]):
        g.set_tuning(dict(saved, bfs_bu_split=table, bfs_bu_split_levels=len(table)))
        depth, parent, st = g.bfs(s, stats=True)
        assert st.bu_levels > 0
        for i, v in enumerate(s):
            d = oracle.bfs_depth(host.index, host.neighbors, v)
            assert np.array_equal(depth[i], d)
            assert oracle.verify_bfs_parents(host.index, host.neighbors, d, parent[i], v)[0] == 0
    for bad in (dict(bfs_bu_split_levels=9), dict(bfs_bu_split=[-1], bfs_bu_split_levels=1),
                dict(bfs_bu_split=[host.num_nodes + 1], bfs_bu_split_levels=1)):
        with pytest.raises(hc.HCError) as e:
            g.set_tuning(dict(saved, **bad))
        assert e.value.status == hc.INVALID_ARG
    g.set_tuning(saved)
