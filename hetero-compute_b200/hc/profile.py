"""Segment profiling of the epoch kernels (hc_profile_segments), in the shape of
the reference's TreeBenchmark (src/benchmarks/benchmark.cuh:87-309): the
degree-ordered vertices cut into 2^d segments of about equal edge count for
each depth d, one epoch kernel launch timed per segment, and the results
written as the reference's YAML (segment_res_t / layer_res_t / tree_res_t
writers, src/benchmarks/benchmark.cuh:156-240)."""
from __future__ import annotations

import ctypes as C

import numpy as np

import hc

SSSP, PR, BFS = 0, 1, 2


class SegmentResult(C.Structure):
    _fields_ = [("start_id", C.c_int32), ("end_id", C.c_int32), ("num_edges", C.c_int64),
                ("avg_degree", C.c_float), ("min_degree", C.c_float), ("max_degree", C.c_float),
                ("epoch", C.c_int32), ("millis", C.c_double), ("gteps", C.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def _bind():
    L = hc.lib()
    P = C.c_void_p
    L.hc_equal_edge_ranges.argtypes = [P, C.c_int32, C.c_int32, C.c_int32, P]
    L.hc_equal_edge_ranges.restype = C.c_int
    L.hc_profile_segments.argtypes = [P, C.c_int, C.c_int, C.c_int32, P, C.c_int32, C.c_int32, C.c_int32,
                                      C.c_int32, C.c_int32, C.c_int32, C.POINTER(SegmentResult)]
    L.hc_profile_segments.restype = C.c_int
    return L


def equal_edge_ranges(index: np.ndarray, num_segments: int, chunk_size: int = 1) -> np.ndarray:
    """hc_equal_edge_ranges: num_segments + 1 vertex bounds of about equal edge count."""
    index = np.ascontiguousarray(index, dtype=np.int64)
    out = np.empty(num_segments + 1, dtype=np.int32)
    hc._check(_bind().hc_equal_edge_ranges(index.ctypes.data, len(index) - 1, num_segments, chunk_size,
                                           out.ctypes.data), "hc_equal_edge_ranges")
    return out


def segments(g: "hc.Graph", algo: int, ranges, *, variant=hc.VARIANT_WARP, sync_iters=0, source=0, level=0,
             block_count=64, thread_count=1024, iters=5) -> list:
    """hc_profile_segments: one result dict per segment [ranges[s], ranges[s+1])."""
    r = np.ascontiguousarray(ranges, dtype=np.int32)
    k = len(r) - 1
    out = (SegmentResult * k)()
    hc._check(_bind().hc_profile_segments(g.handle, algo, variant, sync_iters, r.ctypes.data, k, source, level,
                                          block_count, thread_count, iters, out), "hc_profile_segments")
    return [x.as_dict() for x in out]


def tree(g: "hc.Graph", index: np.ndarray, algo: int, depth: int, *, warmup=1, **kw) -> list:
    """tree_microbenchmark (src/benchmarks/benchmark.cuh:259-276): layers of 2^0 .. 2^depth segments,
    after `warmup` untimed passes over one segment."""
    for _ in range(warmup):
        segments(g, algo, equal_edge_ranges(index, 1), **kw)
    return [segments(g, algo, equal_edge_ranges(index, 1 << d), **kw) for d in range(depth + 1)]


def _segment_yaml(seg: dict, indent: str) -> list:
    p = lambda x: f"{x:.10g}"  # BENCHMARK_PRECISION 10
    return [f"{indent}- start: {seg['start_id']}", f"{indent}  end: {seg['end_id']}",
            f"{indent}  avg_deg: {p(seg['avg_degree'])}", f"{indent}  min_deg: {p(seg['min_degree'])}",
            f"{indent}  max_deg: {p(seg['max_degree'])}", f"{indent}  num_edges: {seg['num_edges']}",
            f"{indent}  millis: {p(seg['millis'])}", f"{indent}  gteps: {p(seg['gteps'])}"]


def tree_yaml(layers: list, device: str, kernel: str) -> str:
    """The reference's tree_res_t YAML (src/benchmarks/benchmark.cuh:216-240)."""
    lines = ["config:", f"  device: {device}", f"  kernel: {kernel}", "results:"]
    for d, layer in enumerate(layers):
        lines += [f"  - depth: {d}", "    segments:"]
        for seg in layer:
            lines += _segment_yaml(seg, "      ")
    return "\n".join(lines) + "\n"


def layer_yaml(layer: list, device: str, kernel: str) -> str:
    """The reference's layer_res_t YAML (src/benchmarks/benchmark.cuh:186-211)."""
    lines = ["config:", f"  device: {device}", f"  kernel: {kernel}", "results:", "  - segments: "]
    for seg in layer:
        lines += _segment_yaml(seg, "      ")
    return "\n".join(lines) + "\n"
