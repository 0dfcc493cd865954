"""Host-side logic of libhc and the C ABI surface, on CPU (no compute calls)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import hc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "hc.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = C.CDLL(hc.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert hc.lib().hc_abi_version() == 1


def check_csr(g: hc.HostCSR, degree_sorted=True):
    idx, nb = g.index, g.neighbors
    assert idx[0] == 0 and idx[-1] == len(nb)
    deg = np.diff(idx)
    assert (deg >= 0).all()
    if degree_sorted:
        assert (np.diff(deg) <= 0).all()
    rows = np.repeat(np.arange(g.num_nodes), deg)
    assert (nb != rows).all(), "self-loop"
    # strictly increasing within rows => no duplicates
    same_row = rows[1:] == rows[:-1]
    assert (np.diff(nb)[same_row] > 0).all()
    # symmetric structure and symmetric weights
    key = rows.astype(np.int64) * g.num_nodes + nb
    rkey = nb.astype(np.int64) * g.num_nodes + rows
    order = np.argsort(key)
    pos = np.searchsorted(key[order], rkey)
    assert (key[order][pos] == rkey).all()
    if g.weights is not None:
        assert (g.weights[order][pos] == g.weights).all()


@pytest.mark.parametrize("wtype", [hc.W_NONE, hc.W_I32, hc.W_F32])
def test_kronecker_properties(wtype):
    g = hc.gen_kronecker(11, 16, 3, wtype=wtype)
    check_csr(g)
    if wtype == hc.W_I32:
        assert g.weights.min() >= 1 and g.weights.max() <= 255
    if wtype == hc.W_F32:
        assert g.weights.min() > 0 and g.weights.max() <= 1.0


def test_generators_deterministic_and_seeded():
    a = hc.gen_kronecker(10, 8, 5, wtype=hc.W_I32)
    b = hc.gen_kronecker(10, 8, 5, wtype=hc.W_I32)
    c = hc.gen_kronecker(10, 8, 6, wtype=hc.W_I32)
    assert np.array_equal(a.index, b.index) and np.array_equal(a.neighbors, b.neighbors)
    assert np.array_equal(a.weights, b.weights)
    assert not (np.array_equal(a.index, c.index) and np.array_equal(a.neighbors, c.neighbors))


def test_uniform_and_grid_properties():
    check_csr(hc.gen_uniform(10, 8, 2, wtype=hc.W_I32))
    g = hc.gen_grid(7, 9, 1, wtype=hc.W_I32)
    check_csr(g, degree_sorted=False)
    deg = g.degrees().reshape(7, 9)
    assert deg[0, 0] == 2 and deg[0, 4] == 3 and deg[3, 4] == 4
    assert g.num_edges == 2 * (7 * 8 + 6 * 9)


def test_graph_file_round_trip(tmp_path):
    g = hc.gen_kronecker(9, 8, 1, wtype=hc.W_I32)
    p = str(tmp_path / "g.wsg")
    hc.write_graph(p, g)
    assert os.path.getsize(p) == 4 + 8 + 8 * (g.num_nodes + 1) + 8 * g.num_edges
    h = hc.read_graph(p, weighted=2)
    assert np.array_equal(h.index, g.index) and np.array_equal(h.neighbors, g.neighbors)
    assert np.array_equal(h.weights, g.weights)
    f = hc.read_graph(p, weighted=1)
    assert np.array_equal(f.weights, g.weights.astype(np.float32))
    q = str(tmp_path / "g.sg")
    hc.write_graph(q, hc.HostCSR(g.index, g.neighbors))
    assert os.path.getsize(q) == 4 + 8 + 8 * (g.num_nodes + 1) + 4 * g.num_edges
    u = hc.read_graph(q)
    assert np.array_equal(u.neighbors, g.neighbors) and u.weights is None


def test_corrupt_graph_files_are_rejected(tmp_path):
    g = hc.gen_kronecker(8, 8, 1)
    p = str(tmp_path / "g.sg")
    hc.write_graph(p, g)
    raw = open(p, "rb").read()
    open(str(tmp_path / "short.sg"), "wb").write(raw[:len(raw) // 2])
    with pytest.raises(hc.HCError) as e:
        hc.read_graph(str(tmp_path / "short.sg"))
    assert e.value.status == hc.IO
    bad = bytearray(raw)
    off = 12 + 8 * (g.num_nodes + 1)
    bad[off:off + 4] = np.int32(10 ** 6).tobytes()  # neighbour out of range
    open(str(tmp_path / "bad.sg"), "wb").write(bytes(bad))
    with pytest.raises(hc.HCError):
        hc.read_graph(str(tmp_path / "bad.sg"))
    with pytest.raises(hc.HCError):
        hc.read_graph(str(tmp_path / "missing.sg"))


def test_source_picker_rules():
    # vertex 0 isolated, 1 self-loop only, 2-3 connected
    index = np.array([0, 0, 1, 2, 3], dtype=np.int64)
    nbr = np.array([1, 3, 2], dtype=np.int32)
    g = hc.HostCSR(index, nbr)
    s = hc.pick_sources(g, 50)
    assert set(s.tolist()) <= {2, 3}
    assert (hc.pick_sources(g, 3, const_source=1) == 1).all()


def test_invalid_arguments_report_status():
    with pytest.raises(hc.HCError) as e:
        hc.gen_kronecker(0, 16)
    assert e.value.status == hc.INVALID_ARG
    with pytest.raises(hc.HCError):
        hc.pick_sources(hc.HostCSR(np.zeros(3, dtype=np.int64), np.zeros(0, dtype=np.int32)), 1)


def test_no_device_is_an_error_not_a_fallback():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    g = hc.gen_kronecker(6, 4, 1)
    with pytest.raises(hc.HCError) as e:
        hc.Graph.from_host(g)
    assert e.value.status == hc.NO_DEVICE


# ctypes mirrors of the public structs in include/hc.h (class name -> C type).
_STRUCTS = {"CSR": "hc_csr", "GraphInfo": "hc_graph_info", "BfsOpts": "hc_bfs_opts", "BfsStats": "hc_bfs_stats",
            "SsspOpts": "hc_sssp_opts", "SsspStats": "hc_sssp_stats", "PrOpts": "hc_pr_opts",
            "PrStats": "hc_pr_stats", "BatchOpts": "hc_batch_opts", "BatchStats": "hc_batch_stats",
            "Tuning": "hc_tuning", "profile.SegmentResult": "hc_segment_result"}


def _resolve(name):
    import importlib
    mod, _, attr = name.rpartition(".")
    return getattr(importlib.import_module("hc." + mod) if mod else hc, attr)


def test_ctypes_structs_match_the_c_header(tmp_path):
    """Every ctypes struct the Python binding passes through the C ABI has the size and field
    offsets the C compiler gives the header's struct (a field added on one side only shifts
    every field after it)."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("gcc not found")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "hc.h"', "int main(void) {"]
    for py, c in _STRUCTS.items():
        cls = _resolve(py)
        lines.append(f'printf("{py} size %zu\\n", sizeof({c}));')
        for name, _ in cls._fields_:
            lines.append(f'printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            py, name, val = line.split()
            got[(py, name)] = int(val)
    for py in _STRUCTS:
        cls = _resolve(py)
        assert got[(py, "size")] == C.sizeof(cls), py
        for name, _ in cls._fields_:
            assert got[(py, name)] == getattr(cls, name).offset, (py, name)
