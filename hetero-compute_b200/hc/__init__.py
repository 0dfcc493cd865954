"""ctypes binding of the libhc C ABI (include/hc.h).

This is the Python side of the drop-in boundary: the same entry points a
C/C++ host links against, called through ctypes with numpy arrays (host
memory) or torch CUDA tensors (device memory, passed by data pointer).  There
is no fallback: if libhc.so is missing or a call fails, an exception says so.

Reference interfaces mirrored (chrisliu/hetero-compute):
  bfs_gpu           src/kernels/gpu/bfs.cuh:21-95
  sssp_pull_gpu     src/kernels/gpu/sssp.cuh:42-100
  pr_pull_gpu       src/kernels/gpu/pr.cuh:42-118
  SourcePicker      src/graph.cuh:106-141
  .sg / .wsg I/O    src/graph.cuh:207-239
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libhc.so")

OK, INVALID_ARG, OOM, CUDA, NOT_CONVERGED, TIMEOUT, NO_DEVICE, UNSUPPORTED, IO = range(9)
W_NONE, W_I32, W_F32 = 0, 1, 2
GEN_KRONECKER, GEN_UNIFORM = 0, 1  # hc_graph_generate
VARIANT_AUTO, VARIANT_THREAD, VARIANT_WARP, VARIANT_BLOCK = 0, 1, 2, 3
INF_DIST = 0x7FFFFFFF


class HCError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


class CSR(C.Structure):
    _fields_ = [("num_nodes", C.c_int32), ("num_edges", C.c_int64), ("index", C.POINTER(C.c_int64)),
                ("neighbors", C.POINTER(C.c_int32)), ("weights", C.c_void_p), ("wtype", C.c_int)]


class GraphInfo(C.Structure):
    _fields_ = [("num_nodes", C.c_int32), ("num_edges", C.c_int64), ("num_active", C.c_int32),
                ("degree_sorted", C.c_int32), ("max_degree", C.c_int32), ("device", C.c_int32),
                ("wtype", C.c_int), ("device_bytes", C.c_int64)]


class BfsOpts(C.Structure):
    _fields_ = [("alpha", C.c_int32), ("beta", C.c_int32), ("direction", C.c_int32), ("bu_variant", C.c_int),
                ("collect_stats", C.c_int32)]


class BfsStats(C.Structure):
    _fields_ = [("levels", C.c_int32), ("td_levels", C.c_int32), ("bu_levels", C.c_int32), ("reached", C.c_int32),
                ("vertices_scanned", C.c_int64), ("edges_scanned", C.c_int64), ("bytes_model", C.c_double),
                ("ms", C.c_double)]


class SsspOpts(C.Structure):
    _fields_ = [("delta", C.c_int32), ("max_epochs", C.c_int32), ("collect_stats", C.c_int32), ("pull_alpha", C.c_int32)]


class SsspStats(C.Structure):
    _fields_ = [("epochs", C.c_int32), ("reached", C.c_int32), ("vertices_processed", C.c_int64),
                ("edges_relaxed", C.c_int64), ("bytes_model", C.c_double), ("ms", C.c_double)]


class PrOpts(C.Structure):
    _fields_ = [("damping", C.c_float), ("tol_l1", C.c_float), ("eps_vertex", C.c_float), ("max_iters", C.c_int32),
                ("weighted", C.c_int32), ("variant", C.c_int), ("accel", C.c_int32)]


class PrStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("residual_l1", C.c_float),
                ("changed", C.c_int32), ("bytes_model", C.c_double), ("ms", C.c_double)]


GRAPH_AUTO, GRAPH_ON, GRAPH_OFF = 0, 1, 2  # hc_batch_opts.use_graph


class BatchOpts(C.Structure):
    _fields_ = [("group", C.c_int32), ("max_epochs", C.c_int32), ("use_graph", C.c_int32),
                ("switch_alpha", C.c_int32), ("dist_bits", C.c_int32)]


class Tuning(C.Structure):
    """hc_tuning: launch parameters picked by hc_autotune (0 = untuned)."""
    _fields_ = [("bfs_alpha", C.c_int32), ("bfs_beta", C.c_int32), ("bfs_bu_variant", C.c_int32),
                ("sssp_delta", C.c_int32), ("sssp_pull_alpha", C.c_int32), ("mbfs_group", C.c_int32),
                ("mbfs_switch_alpha", C.c_int32), ("mssp_group", C.c_int32), ("mssp_switch_alpha", C.c_int32),
                ("trials", C.c_int32), ("tune_ms", C.c_double), ("bfs_bu_split", C.c_int32 * 8),
                ("bfs_bu_split_levels", C.c_int32), ("sssp_blocks_per_sm", C.c_int32)]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["bfs_bu_split"] = list(d["bfs_bu_split"])[:self.bfs_bu_split_levels]
        return d


TUNE_BFS, TUNE_SSSP, TUNE_BFS_BATCHED, TUNE_SSSP_BATCHED, TUNE_BFS_LEVELS, TUNE_ALL = 1, 2, 4, 8, 16, 31


class BatchStats(C.Structure):
    _fields_ = [("epochs", C.c_int32), ("groups", C.c_int32), ("bytes_model", C.c_double), ("ms", C.c_double),
                ("wide_groups", C.c_int32), ("reruns", C.c_int32)]


_P = C.c_void_p
_SIGS = {
    "hc_last_error": (C.c_char_p, []),
    "hc_status_string": (C.c_char_p, [C.c_int]),
    "hc_abi_version": (C.c_int32, []),
    "hc_gen_kronecker": (C.c_int, [C.c_int32, C.c_int32, C.c_uint64, C.c_int, C.POINTER(CSR)]),
    "hc_gen_uniform": (C.c_int, [C.c_int32, C.c_int32, C.c_uint64, C.c_int, C.POINTER(CSR)]),
    "hc_gen_grid": (C.c_int, [C.c_int32, C.c_int32, C.c_uint64, C.c_int, C.POINTER(CSR)]),
    "hc_csr_free": (None, [C.POINTER(CSR)]),
    "hc_csr_read": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(CSR)]),
    "hc_csr_write": (C.c_int, [C.c_char_p, C.POINTER(CSR)]),
    "hc_pick_sources": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_int32, _P]),
    "hc_graph_create": (C.c_int, [_P, _P, _P, C.c_int, C.c_int32, C.c_int64, C.c_int32, C.POINTER(_P)]),
    "hc_graph_destroy": (C.c_int, [_P]),
    "hc_graph_set_stream": (C.c_int, [_P, _P]),
    "hc_graph_get_info": (C.c_int, [_P, C.POINTER(GraphInfo)]),
    "hc_graph_generate": (C.c_int, [C.c_int, C.c_int32, C.c_int32, C.c_uint64, C.c_int, C.c_int32, C.POINTER(_P)]),
    "hc_graph_get_csr": (C.c_int, [_P, _P, _P, _P]),
    "hc_graph_load": (C.c_int, [C.c_char_p, C.c_int32, C.c_int32, C.POINTER(_P)]),
    "hc_graph_pick_sources": (C.c_int, [_P, C.c_int32, _P]),
    "hc_bfs": (C.c_int, [_P, _P, C.c_int32, _P, _P, C.POINTER(BfsOpts), C.POINTER(BfsStats)]),
    "hc_sssp": (C.c_int, [_P, _P, C.c_int32, _P, _P, C.POINTER(SsspOpts), C.POINTER(SsspStats)]),
    "hc_pr_forward": (C.c_int, [_P, _P, C.c_int32, _P, C.POINTER(PrOpts), C.POINTER(PrStats)]),
    "hc_pr_backward": (C.c_int, [_P, _P, _P, _P, _P, C.POINTER(PrOpts), C.POINTER(PrStats)]),
    "hc_pr_pull_ordered": (C.c_int, [_P, _P, _P, C.POINTER(PrOpts), C.POINTER(PrStats)]),
    "hc_ppr_batched": (C.c_int, [_P, _P, _P, C.c_int32, _P, C.POINTER(PrOpts), C.POINTER(PrStats)]),
    "hc_bfs_batched": (C.c_int, [_P, _P, C.c_int32, _P, C.POINTER(BatchOpts), C.POINTER(BatchStats)]),
    "hc_sssp_batched": (C.c_int, [_P, _P, C.c_int32, _P, C.POINTER(BatchOpts), C.POINTER(BatchStats)]),
    "hc_dev_malloc": (C.c_int, [C.POINTER(_P), C.c_size_t, C.c_int32]),
    "hc_dev_free": (C.c_int, [_P]),
    "hc_memcpy": (C.c_int, [_P, _P, C.c_size_t]),
    "hc_dev_memset": (C.c_int, [_P, C.c_int32, C.c_size_t]),
    "hc_device_synchronize": (C.c_int, []),
    "hc_kernel_launches": (C.c_int64, []),
    "hc_autotune": (C.c_int, [_P, _P, C.c_int32, C.c_uint32, C.POINTER(Tuning)]),
    "hc_get_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "hc_set_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "hc_bfs_noalloc": (C.c_int, [_P, _P, C.c_int32, C.c_int64, C.c_int32, _P, _P, _P]),
    "hc_set_time_limits": (C.c_int, [C.c_int32, C.c_uint64, C.c_uint64, C.c_uint64]),
    "hc_csr_check": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_int64, _P]),
    "hc_selftest_grid_barrier": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "hc_epoch_sssp_pull": (C.c_int, [_P, _P, C.c_int32, C.c_int32, _P, _P, C.c_int, C.c_int32, C.c_int32, _P]),
    "hc_epoch_pr_pull": (C.c_int, [_P, _P, C.c_int32, C.c_int32, _P, _P, C.c_int32, _P, C.c_int, C.c_int32,
                                   C.c_int32, _P]),
    "hc_epoch_bfs_pull": (C.c_int, [_P, _P, _P, C.c_int32, C.c_int32, _P, _P, _P, C.c_int, C.c_int32, C.c_int32,
                                    _P]),
    "hc_epoch_bfs_sync_pull": (C.c_int, [_P, _P, _P, C.c_int32, C.c_int32, _P, _P, _P, C.c_int32, C.c_int32,
                                         C.c_int32, _P]),
}

_lib = None


def lib() -> C.CDLL:
    """Loads libhc.so (built in-tree by `make` in hetero-compute_b200/)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libhc.so not built at {LIB_PATH}; run make in hetero-compute_b200/ "
                               "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(status: int, where: str):
    if status != OK:
        raise HCError(status, where, lib().hc_last_error().decode(errors="replace"))


def _ptr(x):
    """Address of a numpy array or torch tensor (contiguous), or None."""
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        assert x.flags["C_CONTIGUOUS"], "arrays passed to libhc must be C-contiguous"
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        assert x.is_contiguous(), "tensors passed to libhc must be contiguous"
        return x.data_ptr()
    raise TypeError(f"cannot pass {type(x)} to libhc")


def kernel_launches() -> int:
    """Kernels this process has launched through libhc so far."""
    return int(lib().hc_kernel_launches())


def set_time_limits(device: int = 0, wait_ns: int = 0, run_ns: int = 0, loop_ns: int = 0):
    """hc_set_time_limits: bounds of the device-side waits on `device` (0 = default: 2 s per barrier wait,
    20 s per persistent run, 60 s per batched epoch loop)."""
    _check(lib().hc_set_time_limits(device, wait_ns, run_ns, loop_ns), "hc_set_time_limits")


def selftest_grid_barrier(device: int, blocks: int, withhold_block: int) -> int:
    """hc_selftest_grid_barrier: the grid barrier's recorded status with one block held back (-1: none)."""
    st = C.c_int32(-1)
    _check(lib().hc_selftest_grid_barrier(device, blocks, withhold_block, C.byref(st)), "hc_selftest_grid_barrier")
    return int(st.value)


# ------------------------------------------------------------------ graphs

@dataclass
class HostCSR:
    """Host CSR graph: int64 offsets, int32 neighbours, optional weights."""
    index: np.ndarray
    neighbors: np.ndarray
    weights: np.ndarray | None = None

    @property
    def num_nodes(self) -> int:
        return len(self.index) - 1

    @property
    def num_edges(self) -> int:
        return len(self.neighbors)

    @property
    def wtype(self) -> int:
        if self.weights is None:
            return W_NONE
        return W_I32 if self.weights.dtype == np.int32 else W_F32

    def degrees(self) -> np.ndarray:
        return np.diff(self.index)


def _take_csr(c: CSR) -> HostCSR:
    n, m = c.num_nodes, c.num_edges
    idx = np.ctypeslib.as_array(c.index, shape=(n + 1,)).copy()
    nbr = np.ctypeslib.as_array(c.neighbors, shape=(max(m, 1),))[:m].copy()
    w = None
    if c.wtype != W_NONE and c.weights:
        dt = C.c_int32 if c.wtype == W_I32 else C.c_float
        w = np.ctypeslib.as_array(C.cast(c.weights, C.POINTER(dt)), shape=(max(m, 1),))[:m].copy()
    lib().hc_csr_free(C.byref(c))
    return HostCSR(idx, nbr, w)


def gen_kronecker(scale: int, edge_factor: int = 16, seed: int = 1, wtype: int = W_NONE) -> HostCSR:
    c = CSR()
    _check(lib().hc_gen_kronecker(scale, edge_factor, seed, wtype, C.byref(c)), "hc_gen_kronecker")
    return _take_csr(c)


def gen_uniform(scale: int, degree: int = 16, seed: int = 1, wtype: int = W_NONE) -> HostCSR:
    c = CSR()
    _check(lib().hc_gen_uniform(scale, degree, seed, wtype, C.byref(c)), "hc_gen_uniform")
    return _take_csr(c)


def gen_grid(rows: int, cols: int, seed: int = 1, wtype: int = W_NONE) -> HostCSR:
    c = CSR()
    _check(lib().hc_gen_grid(rows, cols, seed, wtype, C.byref(c)), "hc_gen_grid")
    return _take_csr(c)


def read_graph(path: str, weighted: int = 0) -> HostCSR:
    """weighted: 0 = .sg, 1 = .wsg with fp32 weights, 2 = .wsg converted to int32."""
    c = CSR()
    _check(lib().hc_csr_read(path.encode(), weighted, C.byref(c)), "hc_csr_read")
    return _take_csr(c)


def write_graph(path: str, g: HostCSR):
    c = CSR()
    c.num_nodes = g.num_nodes
    c.num_edges = g.num_edges
    c.index = g.index.ctypes.data_as(C.POINTER(C.c_int64))
    c.neighbors = g.neighbors.ctypes.data_as(C.POINTER(C.c_int32))
    c.weights = g.weights.ctypes.data if g.weights is not None else None
    c.wtype = g.wtype
    _check(lib().hc_csr_write(path.encode(), C.byref(c)), "hc_csr_write")


def pick_sources(g: HostCSR, count: int, const_source: int = -1) -> np.ndarray:
    """SourcePicker (src/graph.cuh:106-141): mt19937(37525) draws, skipping isolated vertices."""
    out = np.empty(count, dtype=np.int32)
    _check(lib().hc_pick_sources(_ptr(g.index), _ptr(g.neighbors), g.num_nodes, count, const_source, _ptr(out)),
           "hc_pick_sources")
    return out


# ------------------------------------------------------------ device graph

class Graph:
    """A CSR graph resident in HBM (hc_graph handle)."""

    def __init__(self, index, neighbors, weights=None, device: int = 0):
        index = np.ascontiguousarray(index, dtype=np.int64) if isinstance(index, np.ndarray) else index
        neighbors = np.ascontiguousarray(neighbors, dtype=np.int32) if isinstance(neighbors, np.ndarray) else neighbors
        if weights is None:
            wt = W_NONE
        elif str(weights.dtype).endswith("int32"):
            wt = W_I32
        else:
            wt = W_F32
        self.num_nodes = len(index) - 1
        self.num_edges = len(neighbors)
        self.wtype = wt
        h = C.c_void_p()
        _check(lib().hc_graph_create(_ptr(index), _ptr(neighbors), _ptr(weights), wt, self.num_nodes,
                                     self.num_edges, device, C.byref(h)), "hc_graph_create")
        self._h = h

    @classmethod
    def from_host(cls, g: HostCSR, device: int = 0) -> "Graph":
        return cls(g.index, g.neighbors, g.weights, device)

    @classmethod
    def generate(cls, kind: int, scale: int, edge_factor: int, seed: int = 1, wtype: int = W_NONE,
                 device: int = 0) -> "Graph":
        """hc_graph_generate: the gen_kronecker / gen_uniform graph, built on the device."""
        h = C.c_void_p()
        _check(lib().hc_graph_generate(kind, scale, edge_factor, seed, wtype, device, C.byref(h)),
               "hc_graph_generate")
        self = cls.__new__(cls)
        self._h = h
        info = self.info()
        self.num_nodes, self.num_edges, self.wtype = info.num_nodes, info.num_edges, info.wtype
        return self

    @classmethod
    def load(cls, path: str, weighted: int = 0, device: int = 0) -> "Graph":
        """hc_graph_load: a .sg (weighted 0) or .wsg (1: fp32 weights, 2: int32) file streamed to the device."""
        h = C.c_void_p()
        _check(lib().hc_graph_load(path.encode(), weighted, device, C.byref(h)), "hc_graph_load")
        self = cls.__new__(cls)
        self._h = h
        info = self.info()
        self.num_nodes, self.num_edges, self.wtype = info.num_nodes, info.num_edges, info.wtype
        return self

    def csr(self):
        """(index int64[N+1], neighbors int32[M], weights or None) copied to host memory."""
        index = np.empty(self.num_nodes + 1, dtype=np.int64)
        nbr = np.empty(self.num_edges, dtype=np.int32)
        w = None
        if self.wtype != W_NONE:
            w = np.empty(self.num_edges, dtype=np.int32 if self.wtype == W_I32 else np.float32)
        _check(lib().hc_graph_get_csr(self._h, _ptr(index), _ptr(nbr), _ptr(w)), "hc_graph_get_csr")
        return index, nbr, w

    def pick_sources(self, count: int) -> np.ndarray:
        out = np.empty(count, dtype=np.int32)
        _check(lib().hc_graph_pick_sources(self._h, count, _ptr(out)), "hc_graph_pick_sources")
        return out

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().hc_graph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> GraphInfo:
        i = GraphInfo()
        _check(lib().hc_graph_get_info(self._h, C.byref(i)), "hc_graph_get_info")
        return i

    def set_stream(self, stream_ptr: int | None):
        _check(lib().hc_graph_set_stream(self._h, stream_ptr), "hc_graph_set_stream")

    # -- algorithms.  Outputs: numpy (host) unless torch CUDA tensors are given.
    def bfs(self, sources, depth=None, parent=None, *, alpha=0, beta=0, direction=0, bu_variant=VARIANT_AUTO,
            stats=False, want_parent=True, want_depth=True):
        """want_depth=False with depth=None returns parents only (the reference's bfs_gpu output)."""
        src = np.ascontiguousarray(sources, dtype=np.int32) if not hasattr(sources, "data_ptr") else sources
        k = len(src)
        if depth is None and want_depth:
            depth = np.empty((k, self.num_nodes), dtype=np.int32)
        if parent is None and want_parent:
            parent = np.empty((k, self.num_nodes), dtype=np.int32)
        o = BfsOpts(alpha, beta, direction, bu_variant, 1 if stats else 0)
        st = BfsStats()
        _check(lib().hc_bfs(self._h, _ptr(src), k, _ptr(depth), _ptr(parent), C.byref(o), C.byref(st)), "hc_bfs")
        return depth, parent, st

    def sssp(self, sources, dist=None, parent=None, *, delta=0, max_epochs=0, stats=False, want_parent=False,
             pull_alpha=0):
        src = np.ascontiguousarray(sources, dtype=np.int32) if not hasattr(sources, "data_ptr") else sources
        k = len(src)
        if dist is None:
            dist = np.empty((k, self.num_nodes), dtype=np.int32)
        if parent is None and want_parent:
            parent = np.empty((k, self.num_nodes), dtype=np.int32)
        o = SsspOpts(delta, max_epochs, 1 if stats else 0, pull_alpha)
        st = SsspStats()
        _check(lib().hc_sssp(self._h, _ptr(src), k, _ptr(dist), _ptr(parent), C.byref(o), C.byref(st)), "hc_sssp")
        return dist, parent, st

    def pagerank(self, teleport=None, scores=None, *, damping=0.85, tol_l1=1e-4, eps_vertex=0.0, max_iters=50,
                 weighted=False, accel=0):
        ncols = 1 if teleport is None or teleport.ndim == 1 else teleport.shape[1]
        if scores is None:
            scores = np.empty((self.num_nodes,) if ncols == 1 else (self.num_nodes, ncols), dtype=np.float32)
        o = PrOpts(damping, tol_l1, eps_vertex, max_iters, 1 if weighted else 0, VARIANT_AUTO, accel)
        st = PrStats()
        _check(lib().hc_pr_forward(self._h, _ptr(teleport), ncols, _ptr(scores), C.byref(o), C.byref(st)),
               "hc_pr_forward")
        return scores, st

    def pagerank_ordered(self, init=None, scores=None, *, damping=0.85, eps_vertex=5e-8, max_iters=0):
        """hc_pr_pull_ordered: in-place sweeps in vertex order with the per-vertex eps rule, the reference's
        single-thread pr_pull_cpu bit for bit (max_iters 0 = until a sweep stores nothing)."""
        if scores is None:
            scores = np.empty(self.num_nodes, dtype=np.float32)
        o = PrOpts(damping, 0.0, eps_vertex, max_iters, 0, VARIANT_AUTO, 0)
        st = PrStats()
        _check(lib().hc_pr_pull_ordered(self._h, _ptr(init), _ptr(scores), C.byref(o), C.byref(st)),
               "hc_pr_pull_ordered")
        return scores, st

    def pagerank_backward(self, scores, dL_dscores, *, damping=0.85, tol_l1=1e-7, eps_vertex=0.0, max_iters=500,
                          weighted=False, want_dw=True, dteleport=None, dweights=None, accel=0):
        if dteleport is None:
            dteleport = np.empty(self.num_nodes, dtype=np.float32)
        if dweights is None and want_dw:
            dweights = np.empty(self.num_edges, dtype=np.float32)
        o = PrOpts(damping, tol_l1, eps_vertex, max_iters, 1 if weighted else 0, VARIANT_AUTO, accel)
        st = PrStats()
        _check(lib().hc_pr_backward(self._h, _ptr(scores), _ptr(dL_dscores), _ptr(dteleport), _ptr(dweights),
                                    C.byref(o), C.byref(st)), "hc_pr_backward")
        return dteleport, dweights, st

    def ppr_batched(self, seed_offsets, seeds, scores=None, *, damping=0.85, tol_l1=1e-4, max_iters=50,
                    weighted=False):
        off = np.ascontiguousarray(seed_offsets, dtype=np.int32)
        sd = np.ascontiguousarray(seeds, dtype=np.int32)
        k = len(off) - 1
        if scores is None:
            scores = np.empty((self.num_nodes, k), dtype=np.float32)
        o = PrOpts(damping, tol_l1, 0.0, max_iters, 1 if weighted else 0, VARIANT_AUTO)
        st = PrStats()
        _check(lib().hc_ppr_batched(self._h, _ptr(off), _ptr(sd), k, _ptr(scores), C.byref(o), C.byref(st)),
               "hc_ppr_batched")
        return scores, st

    def bfs_batched(self, sources, depth=None, *, group=0, max_epochs=0, use_graph=GRAPH_AUTO, switch_alpha=0):
        src = np.ascontiguousarray(sources, dtype=np.int32)
        if depth is None:
            depth = np.empty((len(src), self.num_nodes), dtype=np.int32)
        o = BatchOpts(group, max_epochs, use_graph, switch_alpha)
        st = BatchStats()
        _check(lib().hc_bfs_batched(self._h, _ptr(src), len(src), _ptr(depth), C.byref(o), C.byref(st)),
               "hc_bfs_batched")
        return depth, st

    def sssp_batched(self, sources, dist=None, *, group=0, max_epochs=0, use_graph=GRAPH_AUTO, switch_alpha=0,
                     dist_bits=0):
        """dist_bits: working distances, 0/16 = 16-bit where they fit (else 32-bit), 32 = always 32-bit."""
        src = np.ascontiguousarray(sources, dtype=np.int32)
        if dist is None:
            dist = np.empty((len(src), self.num_nodes), dtype=np.int32)
        o = BatchOpts(group, max_epochs, use_graph, switch_alpha, dist_bits)
        st = BatchStats()
        _check(lib().hc_sssp_batched(self._h, _ptr(src), len(src), _ptr(dist), C.byref(o), C.byref(st)),
               "hc_sssp_batched")
        return dist, st

    def autotune(self, sample_sources, what=TUNE_ALL) -> dict:
        """Times candidate launch parameters on the sample sources and keeps the fastest on the handle."""
        src = np.ascontiguousarray(sample_sources, dtype=np.int32)
        t = Tuning()
        _check(lib().hc_autotune(self._h, _ptr(src), len(src), what, C.byref(t)), "hc_autotune")
        return t.as_dict()

    @property
    def tuning(self) -> dict:
        t = Tuning()
        _check(lib().hc_get_tuning(self._h, C.byref(t)), "hc_get_tuning")
        return t.as_dict()

    def set_tuning(self, values: dict):
        vals = {k: v for k, v in values.items() if k in dict(Tuning._fields_)}
        split = list(vals.pop("bfs_bu_split", []))
        t = Tuning(**vals)
        for i, x in enumerate(split[:8]):
            t.bfs_bu_split[i] = x
        _check(lib().hc_set_tuning(self._h, C.byref(t)), "hc_set_tuning")


# --------------------------------------------- reference-shaped entry points

def bfs_gpu(g: Graph, source_id: int, variant: int = VARIANT_AUTO):
    """bfs_gpu (src/kernels/gpu/bfs.cuh:21-95): parents from one source."""
    _, parent, _ = g.bfs([source_id], bu_variant=variant)
    return parent[0]


def sssp_pull_gpu(g: Graph, source_id: int):
    """sssp_pull_gpu (src/kernels/gpu/sssp.cuh:42-100): distances from one source (int32, INF_DIST unreachable)."""
    dist, _, _ = g.sssp([source_id])
    return dist[0]


def pr_pull_gpu(g: Graph, init_score=None, *, eps_vertex: float = 5e-8, max_iters: int = 201):
    """pr_pull_gpu (src/kernels/gpu/pr.cuh:42-118): the reference's in-place sweep and stopping rule (a score
    moves only by more than 5e-8; stop when a sweep moves none, at most 201 sweeps), in the single-thread
    vertex order of pr_pull_cpu (src/kernels/cpu/pr.cuh:33-65), so the scores equal that code's bit for bit."""
    scores, _ = g.pagerank_ordered(init_score, eps_vertex=eps_vertex, max_iters=max_iters)
    return scores
