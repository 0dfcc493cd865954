"""Segment profiling (hc_profile_segments): every segment of every layer timed,
edge counts and degree ranges consistent with the CSR, and the reference's YAML
layout (src/benchmarks/benchmark.cuh:156-240)."""
import numpy as np
import pytest
import yaml

import hc
from hc import profile

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graph():
    host = hc.gen_kronecker(14, 16, 2, wtype=hc.W_I32)
    return host, hc.Graph.from_host(host)


@pytest.mark.parametrize("algo,variant,sync", [(profile.SSSP, hc.VARIANT_WARP, 0), (profile.SSSP, hc.VARIANT_THREAD, 0),
                                               (profile.PR, hc.VARIANT_BLOCK, 0), (profile.BFS, hc.VARIANT_THREAD, 0),
                                               (profile.BFS, hc.VARIANT_WARP, 0), (profile.BFS, hc.VARIANT_WARP, 2)])
def test_tree_profile(graph, algo, variant, sync):
    host, g = graph
    src = int(hc.pick_sources(host, 1)[0])
    layers = profile.tree(g, host.index, algo, 3, variant=variant, sync_iters=sync, source=src, level=2,
                          block_count=64, thread_count=256, iters=3)
    assert [len(x) for x in layers] == [1, 2, 4, 8]
    deg = np.diff(host.index)
    for layer in layers:
        assert layer[0]["start_id"] == 0 and layer[-1]["end_id"] == host.num_nodes
        assert sum(s["num_edges"] for s in layer) == host.num_edges
        for s in layer:
            assert s["millis"] > 0 and np.isfinite(s["gteps"])
            assert s["epoch"] == (2 if algo == profile.BFS else -1)
            if s["end_id"] > s["start_id"]:
                d = deg[s["start_id"]:s["end_id"]]
                assert s["min_degree"] == d.min() and s["max_degree"] == d.max()
    doc = yaml.safe_load(profile.tree_yaml(layers, "NVIDIA B200", "sssp_gpu_warp_red"))
    assert doc["config"]["kernel"] == "sssp_gpu_warp_red"
    assert [r["depth"] for r in doc["results"]] == [0, 1, 2, 3]
    seg = doc["results"][3]["segments"][5]
    assert set(seg) == {"start", "end", "avg_deg", "min_deg", "max_deg", "num_edges", "millis", "gteps"}
    one = yaml.safe_load(profile.layer_yaml(layers[2], "NVIDIA B200", "k"))
    assert len(one["results"][0]["segments"]) == 4


def test_profile_rejects_bad_ranges(graph):
    host, g = graph
    with pytest.raises(hc.HCError):
        profile.segments(g, profile.PR, [0, host.num_nodes + 5])
    with pytest.raises(hc.HCError):
        profile.segments(g, profile.PR, [10, 5])
