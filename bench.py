"""Benchmark of the epoch-kernel hot path: BFS, SSSP and PageRank on one
synthetic Kronecker graph, reported as GTEPS with the HBM roofline.

Workload (one step): Kronecker scale 22, edge factor 16, symmetrized, int32
weights in [1,255] (seeded synthetic; no dataset); BFS from 64 sources, SSSP
from the same 64 sources (SourcePicker seed 37525), PageRank d=0.85 with an L1
tolerance of 1e-4 and at most 50 iterations.  GTEPS follows the reference's
benchmark formula: every run (one source, or one PageRank solve) counts M/2
edges (src/benchmarks/gpu_benchmark.cuh:259), value = runs * M/2 / time.

  python bench.py [--gpus N --steps K --warmup W]          this engine
  python bench.py --impl reference [...]                   the reference's own
        OpenMP CPU code (oracle/_ref), host cores, the full workload per step

After the timed steps (N = 1): the reference's CPU step (cpu_baseline) with
parity checks of the GPU's outputs against the reference's (key "parity"),
512 batched BFS / SSSP sources against 512 sequential plain launches (key
"batched") and PageRank forward + adjoint against the forward (key
"adjoint"), each with its own parity check.

Under torchrun (N > 1) each rank holds a replica of the graph and runs its own
64 sources (weak scaling, no data-path collective); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "hetero-compute_b200"))

METRIC = "GTEPS & %HBM roofline, BFS/SSSP/PR: batched+adjoint vs plain, 1 B200"
L2_BYTES = 126 * 1024 * 1024


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--scale", type=int, default=22)
    p.add_argument("--edge-factor", type=int, default=16)
    p.add_argument("--sources", type=int, default=64)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--no-cpu-baseline", action="store_true",
                   help="skip the reference's CPU step and the parity checks against it")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the batched (512 sources) and adjoint sections of the default run")
    p.add_argument("--no-tune", dest="tune", action="store_false",
                   help="skip the (untimed) autotuner pass and use the built-in launch parameters")
    p.add_argument("--mode", choices=["bench", "profile"], default="bench",
                   help="profile: one BFS, one SSSP and one PageRank solve, untimed (for ncu captures)")
    p.add_argument("--suite", choices=["plain", "batched", "adjoint", "grid", "roofline", "large"], default="plain",
                   help="batched: 512 BFS / 512 SSSP sources and 256 PPR columns in batched launches vs "
                        "sequential plain launches (Kronecker scale 24); adjoint: PageRank forward vs "
                        "forward + adjoint (scale 24, fp32 weights, and an Erdos-Renyi 2^24 graph); "
                        "grid: SSSP on the 4096^2 grid from 16 sources")
    return p.parse_args()


def _time_cuda(fn, torch, dev, reps=1):
    """Device time of fn() in ms: events on the current stream, synchronised on both sides."""
    s = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    torch.cuda.synchronize(dev)
    return e0.elapsed_time(e1) / reps


def run_suite(a):
    """The batched / adjoint / grid comparisons (one JSON line each, rank 0, one GPU)."""
    import torch

    import hc
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    scale = a.scale if a.scale != 22 else {"roofline": 25, "large": 27}.get(a.suite, 24)
    out = {"suite": a.suite, "metric": METRIC, "unit": "GTEPS", "data": "synthetic", "warmup": a.warmup,
           "steps": a.steps}
    t0 = time.time()
    if a.suite == "batched":
        host = hc.gen_kronecker(scale, a.edge_factor, a.seed, hc.W_I32)
        g = hc.Graph.from_host(host)
        g.set_stream(stream.cuda_stream)
        n, m = host.num_nodes, host.num_edges
        k = 512
        src = hc.pick_sources(host, k)
        src_t = torch.from_numpy(src).to(dev)
        out["config"] = {"workload": f"kronecker-s{scale}-ef{a.edge_factor}: {k} BFS + {k} SSSP sources, "
                                     f"256 PPR teleports (1-32 seeds each)", "num_nodes": n, "num_edges": m,
                         "graph_gen_s": time.time() - t0}
        if a.tune:  # untimed: launch parameters for both arms (batched and sequential)
            out["tuning"] = g.autotune(src)
        depth = torch.empty((k, n), dtype=torch.int32, device=dev)
        for _ in range(max(1, a.warmup)):
            g.bfs_batched(src_t[:64].cpu().numpy(), depth[:64])
        tb = _time_cuda(lambda: g.bfs_batched(src, depth), torch, dev, a.steps)
        one = torch.empty((1, n), dtype=torch.int32, device=dev)
        par = torch.empty((1, n), dtype=torch.int32, device=dev)

        def seq_bfs():
            for s in src:
                g.bfs(np.array([s], dtype=np.int32), one, par)
        ts = _time_cuda(seq_bfs, torch, dev, 1)
        out["bfs"] = {"batched_ms": tb, "sequential_ms": ts, "batched_gteps": k * (m / 2) / tb / 1e6,
                      "sequential_gteps": k * (m / 2) / ts / 1e6, "speedup": ts / tb}
        del depth
        dist_b = torch.empty((k, n), dtype=torch.int32, device=dev)
        g.sssp_batched(src[:32], dist_b[:32])
        tb = _time_cuda(lambda: g.sssp_batched(src, dist_b), torch, dev, 1)

        def seq_sssp():
            for s in src:
                g.sssp(np.array([s], dtype=np.int32), one)
        g.sssp(src[:2], dist_b[:2])
        ts = _time_cuda(seq_sssp, torch, dev, 1)
        out["sssp"] = {"batched_ms": tb, "sequential_ms": ts, "batched_gteps": k * (m / 2) / tb / 1e6,
                       "sequential_gteps": k * (m / 2) / ts / 1e6, "speedup": ts / tb}
        del dist_b
        rng = np.random.default_rng(a.seed)
        cols = 256
        sizes = rng.integers(1, 33, size=cols)
        off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
        active = np.flatnonzero(host.degrees() > 0)
        seeds = np.concatenate([rng.choice(active, s, replace=False) for s in sizes]).astype(np.int32)
        sc = torch.empty((n, cols), dtype=torch.float32, device=dev)
        _, pst = g.ppr_batched(off, seeds, sc, tol_l1=1e-4, max_iters=50)
        tb = _time_cuda(lambda: g.ppr_batched(off, seeds, sc, tol_l1=1e-4, max_iters=50), torch, dev, 1)
        del sc
        x1 = torch.empty(n, dtype=torch.float32, device=dev)
        tele = torch.zeros(n, dtype=torch.float32, device=dev)

        def seq_ppr():
            for c in range(cols):
                tele.zero_()
                tele[torch.from_numpy(seeds[off[c]:off[c + 1]]).to(dev).long()] = 1.0 / sizes[c]
                g.pagerank(tele, x1, tol_l1=1e-4, max_iters=50)
        ts = _time_cuda(seq_ppr, torch, dev, 1)
        out["ppr"] = {"columns": cols, "batched_ms": tb, "sequential_ms": ts, "speedup": ts / tb,
                      "batched_iterations": int(pst.iterations),
                      "batched_gteps": cols * (m / 2) / tb / 1e6, "sequential_gteps": cols * (m / 2) / ts / 1e6}
        out["value"] = out["bfs"]["batched_gteps"]
    elif a.suite == "adjoint":
        res = {}
        for name, maker in [("kronecker", lambda: hc.gen_kronecker(scale, a.edge_factor, a.seed, hc.W_F32)),
                            ("erdos_renyi", lambda: hc.gen_uniform(24, 8, a.seed, hc.W_F32))]:
            host = maker()
            g = hc.Graph.from_host(host)
            g.set_stream(stream.cuda_stream)
            n, m = host.num_nodes, host.num_edges
            rng = np.random.default_rng(a.seed)
            c = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).to(dev)
            t = torch.full((n,), 1.0 / n, dtype=torch.float32, device=dev)
            x = torch.empty(n, dtype=torch.float32, device=dev)
            dt = torch.empty(n, dtype=torch.float32, device=dev)
            dw = torch.empty(m, dtype=torch.float32, device=dev)
            opts = dict(tol_l1=1e-6, max_iters=200, weighted=True)
            g.pagerank(t, x, **opts)
            g.pagerank_backward(x, c, dteleport=dt, dweights=dw, tol_l1=1e-6, max_iters=200, weighted=True)
            tf = _time_cuda(lambda: g.pagerank(t, x, **opts), torch, dev, a.steps)
            _, fst = g.pagerank(t, x, **opts)
            tfb = _time_cuda(lambda: (g.pagerank(t, x, **opts),
                                      g.pagerank_backward(x, c, dteleport=dt, dweights=dw, tol_l1=1e-6,
                                                          max_iters=200, weighted=True)), torch, dev, a.steps)
            _, _, bst = g.pagerank_backward(x, c, dteleport=dt, dweights=dw, tol_l1=1e-6, max_iters=200,
                                            weighted=True)
            res[name] = {"num_nodes": n, "num_edges": m, "forward_ms": tf, "forward_adjoint_ms": tfb,
                         "ratio": tfb / tf, "forward_iterations": int(fst.iterations),
                         "adjoint_iterations": int(bst.iterations),
                         "forward_gbs": fst.bytes_model / (fst.ms / 1e3) / 1e9 if fst.ms else None}
            g.close()
        out["config"] = {"workload": f"pagerank fp32 weights row-normalised, L = c.x, tol_l1 1e-6: "
                                     f"kronecker-s{scale}-ef{a.edge_factor} and erdos-renyi 2^24 (8 pairs/vertex)"}
        out["adjoint"] = res
        out["value"] = res["kronecker"]["ratio"]
        out["unit"] = "forward+adjoint / forward"
    elif a.suite == "large":
        # One graph resident in HBM (int32 weights [1,255]): BFS and SSSP from
        # 64 sources, one batched 128-source BFS, PageRank forward + adjoint
        # (the int32 weights as fp32), each as GTEPS and the bytes model
        # against the measured HBM peak.
        # Built on the device (the same CSR as the host generator, in seconds).
        g = hc.Graph.generate(hc.GEN_KRONECKER, scale, a.edge_factor, a.seed, hc.W_I32)
        torch.cuda.synchronize(dev)
        gen_s = time.time() - t0
        g.set_stream(stream.cuda_stream)
        n, m = g.num_nodes, g.num_edges
        src = g.pick_sources(128)
        hbm, peak_kind = peaks()
        tuning = g.autotune(src[:64], hc.TUNE_BFS | hc.TUNE_SSSP) if a.tune else None
        res = {}

        def record(name, ms, runs, st=None, st_runs=None):
            # st: a pass over st_runs of the same units (default: runs), for its bytes model; the
            # achieved bandwidth is that model scaled to the timed call, over the timed call's time.
            r = {"ms": ms, "runs": runs, "gteps": runs * (m / 2) / ms / 1e6}
            if st is not None and st.bytes_model:
                r["bytes_model"] = st.bytes_model * runs / (st_runs or runs)
                r["achieved_gbs"] = r["bytes_model"] / (ms / 1e3) / 1e9
                r["frac"] = r["achieved_gbs"] / hbm
            res[name] = r
        out4 = torch.empty((4, n), dtype=torch.int32, device=dev)
        par4 = torch.empty((4, n), dtype=torch.int32, device=dev)
        out_i, par = out4[:1], par4[:1]
        s64 = src[:64]
        g.bfs(s64[:2], out4[:2], par4[:2])
        ms = _time_cuda(lambda: [g.bfs(s64[i:i + 1], out_i, par) for i in range(64)], torch, dev, 1)
        record("bfs_x64", ms, 64, g.bfs(s64[:4], out4, par4, stats=True)[2], 4)
        g.sssp(s64[:1], out_i)
        ms = _time_cuda(lambda: [g.sssp(s64[i:i + 1], out_i) for i in range(64)], torch, dev, 1)
        record("sssp_x64", ms, 64, g.sssp(s64[:4], out4, stats=True)[2], 4)
        depth = torch.empty((128, n), dtype=torch.int32, device=dev)
        g.bfs_batched(src, depth)  # warm-up with the timed call's shape (workspace sized once)
        ms = _time_cuda(lambda: g.bfs_batched(src, depth), torch, dev, 1)
        _, bst = g.bfs_batched(src, depth)
        record("bfs_batched_x128", ms, 128, bst)
        del depth, out_i, par, out4, par4
        x = torch.empty(n, dtype=torch.float32, device=dev)
        rng = np.random.default_rng(a.seed)
        c = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).to(dev)
        dt = torch.empty(n, dtype=torch.float32, device=dev)
        dw = torch.empty(m, dtype=torch.float32, device=dev)
        popts = dict(tol_l1=1e-6, max_iters=200, weighted=True)
        # Warm-ups: the one-time setup (fp32 weights, transposed weights, the
        # symmetry check, workspaces) stays out of the timed calls.
        g.pagerank(None, x, **popts)
        g.pagerank_backward(x, c, dteleport=dt, dweights=dw, **popts)
        tf = _time_cuda(lambda: g.pagerank(None, x, **popts), torch, dev, 1)
        _, fst = g.pagerank(None, x, **popts)
        tb = _time_cuda(lambda: g.pagerank_backward(x, c, dteleport=dt, dweights=dw, **popts), torch, dev, 1)
        _, _, bst2 = g.pagerank_backward(x, c, dteleport=dt, dweights=dw, **popts)
        record("pagerank_forward", tf, 1, fst)
        res["pagerank_forward"]["iterations"] = int(fst.iterations)
        record("pagerank_adjoint", tb, 1, bst2)
        res["pagerank_adjoint"]["iterations"] = int(bst2.iterations)
        res["pagerank_forward_plus_adjoint_over_forward"] = (tf + tb) / tf
        out["config"] = {"workload": f"kronecker-s{scale}-ef{a.edge_factor} int32 weights [1,255] built and resident in HBM: "
                                     f"bfs x64, sssp x64, batched bfs x128, weighted pagerank forward + adjoint "
                                     f"(L1 tol 1e-6, max 200)", "num_nodes": n, "num_edges": m,
                         "graph_gen_s": gen_s, "device_bytes_held": int(g.info().device_bytes),
                         "peak_gbs": hbm, "peak_kind": peak_kind}
        out["tuning"] = tuning
        out["large"] = res
        out["value"] = res["bfs_batched_x128"]["gteps"]
    elif a.suite == "roofline":
        # Plain BFS / SSSP / PageRank on one large Kronecker graph: GTEPS and
        # the bytes model of each call against the measured HBM peak.
        host = hc.gen_kronecker(scale, a.edge_factor, a.seed, hc.W_I32)
        gen_s = time.time() - t0
        g = hc.Graph.from_host(host)
        g.set_stream(stream.cuda_stream)
        n, m = host.num_nodes, host.num_edges
        src = hc.pick_sources(host, 16)
        del host
        tuning = g.autotune(src, hc.TUNE_BFS | hc.TUNE_SSSP) if a.tune else None
        depth = torch.empty((16, n), dtype=torch.int32, device=dev)
        parent = torch.empty((16, n), dtype=torch.int32, device=dev)
        scores = torch.empty(n, dtype=torch.float32, device=dev)
        hbm, peak_kind = peaks()
        res = {}
        for name, call, runs in [
                ("bfs", lambda st=False: g.bfs(src, depth, parent, stats=st)[2], 16),
                ("sssp", lambda st=False: g.sssp(src[:8], depth[:8], stats=st)[2], 8),
                ("pagerank", lambda st=False: g.pagerank(None, scores, tol_l1=1e-4, max_iters=50)[1], 1)]:
            for _ in range(max(1, a.warmup)):
                call()
            ms = _time_cuda(call, torch, dev, max(1, a.steps))
            st = call(True)  # instrumented pass: the bytes model (its statistics-keeping kernels run slower)
            res[name] = {"ms": ms, "gteps": runs * (m / 2) / ms / 1e6, "runs": runs, "instrumented_ms": st.ms,
                         "bytes_model": st.bytes_model,
                         "achieved_gbs": st.bytes_model / (ms / 1e3) / 1e9 if ms else None}
            res[name]["frac"] = res[name]["achieved_gbs"] / hbm if res[name]["achieved_gbs"] else None
        res["pagerank"]["iterations"] = int(st.iterations)
        # One pass over the CSR (offsets + neighbours, + weights for SSSP), the floor of any full sweep,
        # against the time per source (BFS, SSSP) or per iteration (PageRank).
        res["pagerank"]["per_iteration_ms"] = res["pagerank"]["ms"] / max(1, int(st.iterations))
        for name, wb, per in (("bfs", 0, res["bfs"]["ms"] / 16), ("sssp", 4, res["sssp"]["ms"] / 8),
                              ("pagerank", 0, res["pagerank"]["per_iteration_ms"])):
            one = (8.0 * (n + 1) + (4.0 + wb) * m) / (hbm * 1e9) * 1e3
            res[name]["one_pass_ms_at_peak"] = one
            res[name]["one_pass_frac"] = one / per if per > 0 else None
        out["config"] = {"workload": f"kronecker-s{scale}-ef{a.edge_factor}: bfs x16, sssp x8, pagerank "
                                     f"(d=0.85, L1 tol 1e-4, max 50)", "num_nodes": n, "num_edges": m,
                         "graph_gen_s": gen_s, "peak_gbs": hbm, "peak_kind": peak_kind}
        out["tuning"] = tuning
        out["roofline"] = res
        out["value"] = res["pagerank"]["frac"]
        out["unit"] = "fraction of measured HBM peak (pagerank)"
    else:
        host = hc.gen_grid(4096, 4096, a.seed, hc.W_I32)
        g = hc.Graph.from_host(host)
        g.set_stream(stream.cuda_stream)
        n, m = host.num_nodes, host.num_edges
        src = hc.pick_sources(host, 16)
        d = torch.empty((16, n), dtype=torch.int32, device=dev)
        g.sssp(src[:1], d[:1])
        res = {}
        for delta in [0, 256, 1024, 4096]:
            ms = _time_cuda(lambda: g.sssp(src, d, delta=delta), torch, dev, 1)
            _, _, st = g.sssp(src[:1], d[:1], delta=delta, stats=True)
            res[str(delta)] = {"ms_per_source": ms / 16, "gteps": 16 * (m / 2) / ms / 1e6, "epochs": int(st.epochs)}
        out["config"] = {"workload": "grid 4096x4096, 4-neighbour, int32 weights [1,255], SSSP x16",
                         "num_nodes": n, "num_edges": m}
        out["grid_sssp"] = res
        out["value"] = max(r["gteps"] for r in res.values())
    print(json.dumps(out), flush=True)


def profile_case(a):
    """One source of BFS and SSSP, then one PageRank solve: the launches an ncu
    capture of bfs_persistent / sssp_persistent / sssp_pull_kernel / pr_sweep
    selects.  With --suite batched: one 512-source batched BFS, one 512-source
    batched SSSP group on 16-bit distances and one 256-source group on int32
    distances (device outputs).  Under a profiler that replays each captured
    launch dozens of times a whole persistent run takes far longer than it
    does alone, so the run and loop limits are raised to 10 minutes here (the
    per-barrier wait limit stays at its default)."""
    import hc
    hc.set_time_limits(0, 0, 600 * 10**9, 600 * 10**9)
    if a.suite == "batched":
        import torch
        host = hc.gen_kronecker(a.scale, a.edge_factor, a.seed, hc.W_I32)
        g = hc.Graph.from_host(host)
        src = hc.pick_sources(host, 512)
        out = torch.empty((512, host.num_nodes), dtype=torch.int32, device="cuda")
        # Host-driven epoch loops, so that each kernel is a plain launch for the profiler.
        g.bfs_batched(src, out, use_graph=hc.GRAPH_OFF)
        g.sssp_batched(src, out, group=512, use_graph=hc.GRAPH_OFF)  # 16-bit distances
        g.sssp_batched(src[:256], out[:256], group=256, dist_bits=32, use_graph=hc.GRAPH_OFF)
        torch.cuda.synchronize()
        g.close()
        print(json.dumps({"mode": "profile", "suite": "batched", "scale": a.scale, "num_edges": host.num_edges}))
        return
    host = hc.gen_kronecker(a.scale, a.edge_factor, a.seed, hc.W_I32)
    g = hc.Graph.from_host(host)
    src = hc.pick_sources(host, 1)
    g.bfs(src)
    g.sssp(src)
    g.pagerank(tol_l1=1e-4, max_iters=50)
    g.close()
    print(json.dumps({"mode": "profile", "scale": a.scale, "num_edges": host.num_edges, "source": int(src[0])}))


def gpu_local_cpus(dev) -> set | None:
    """Host CPUs on the GPU's own NUMA node (sysfs local_cpulist of its PCI
    function), within this process's allowed set; None when unknown."""
    try:
        import torch
        p = torch.cuda.get_device_properties(dev)
        bdf = "%04x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
        text = open(f"/sys/bus/pci/devices/{bdf}/local_cpulist").read().strip()
        cpus = set()
        for part in text.split(","):
            lo, _, hi = part.partition("-")
            cpus.update(range(int(lo), int(hi or lo) + 1))
        cpus &= os.sched_getaffinity(0)
        return cpus or None
    except Exception:
        return None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload(a):
    return {"workload": f"kronecker-s{a.scale}-ef{a.edge_factor}: bfs x{a.sources} + sssp x{a.sources} + pagerank",
            "scale": a.scale, "edge_factor": a.edge_factor, "sources_per_gpu": a.sources,
            "weights": "int32 uniform [1,255]", "pagerank": "d=0.85, L1 tol 1e-4, max 50 iters",
            "l2": "CSR (>= 0.5 GB) larger than L2; L2 flushed between timed steps"}


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ----------------------------------------------------------- CPU legs

def _ref_graph_files(tmp, index, nbr, weights, writer):
    """.sg (BFS) and .wsg (SSSP, PageRank) files of the benchmark graph for the reference's loader."""
    sg, wsg = os.path.join(tmp, "g.sg"), os.path.join(tmp, "g.wsg")
    writer(sg, index, nbr, None)
    writer(wsg, index, nbr, weights)
    return sg, wsg


def _ref_step_ms(sg, wsg, k, threads, repeats, warmup):
    """The reference's own CPU code (oracle/_ref) on the step's workload: bfs_do_cpu and sssp_pull_cpu from
    the first k SourcePicker sources, then pr_pull_cpu, `repeats` times with the graph loaded once per
    algorithm; returns per-step milliseconds (sum of the reference drivers' own timings) and the raw runs."""
    import oracle
    bfs = oracle.run_reference("bfs", sg, k, "-", threads=threads, repeats=repeats, warmup=warmup)
    sssp = oracle.run_reference("sssp", wsg, k, "-", threads=threads, repeats=repeats, warmup=warmup)
    pr = oracle.run_reference("pr", wsg, 0, "-", threads=threads, repeats=repeats, warmup=min(warmup, 1))
    steps = []
    for r in range(repeats):
        steps.append(sum(bfs["ms"][r * k:(r + 1) * k]) + sum(sssp["ms"][r * k:(r + 1) * k]) + pr["ms"][r])
    per_run = {"bfs_ms": float(np.mean(bfs["ms"])), "sssp_ms": float(np.mean(sssp["ms"])),
               "pagerank_ms": float(np.mean(pr["ms"]))}
    return steps, per_run, bfs["sources"]


def cpu_leg(host, a, gpu):
    """cpu_baseline: one full step of the reference's own OpenMP code (oracle/_ref) on all host cores, timed
    by the reference's drivers, with nothing extrapolated.  The same leg checks the GPU's results against the
    reference's outputs for the first sources (and the oracle, as the checker):
      BFS   GPU depths == the oracle's serial BFS depths; GPU parents a valid BFS tree; the reference's
            bfs_do_cpu parents a valid tree for the GPU's depths (tests/bfs/bfs_verify.cu:133-233 rules)
      SSSP  GPU distances == the reference's sssp_pull_cpu distances, bit for bit (inf as INT32_MAX)
      PR    the reference-order sweep (hc_pr_pull_ordered) == the reference's pr_pull_cpu on one thread, bit
            for bit; the timed Jacobi PageRank's L-inf distance to the reference and to the FP64 fixed point
    `gpu` holds host copies of the GPU outputs."""
    import oracle
    import hc
    threads = os.cpu_count() or 1
    m = host.num_edges
    with tempfile.TemporaryDirectory() as tmp:
        sg, wsg = _ref_graph_files(tmp, host.index, host.neighbors, host.weights,
                                   lambda p, i, n, w: hc.write_graph(p, hc.HostCSR(i, n, w)))
        if not os.path.exists(oracle.REF_DRIVER):
            return ({"value": None, "unit": "GTEPS", "cores": None, "kind": "unavailable",
                     "sample": "the reference's CPU code was not built (oracle/_ref absent)"}, None)
        steps, per_run, _ = _ref_step_ms(sg, wsg, a.sources, threads, 1, 1)
        runs = 2 * a.sources + 1
        cpu = {"value": runs * (m / 2) / (steps[0] / 1e3) / 1e9, "unit": "GTEPS", "cores": threads,
               "kind": "reference",
               "sample": f"one full step (bfs_do_cpu x{a.sources} + sssp_pull_cpu x{a.sources} + pr_pull_cpu x1) "
                         f"on {threads} OpenMP threads, {steps[0]:.0f} ms by the reference's own timers",
               "per_run_ms": per_run}
        # Parity on the first sources, against the reference's own outputs.
        kp = min(4, a.sources)
        par = {}
        out = os.path.join(tmp, "out.bin")
        n = host.num_nodes
        ref = oracle.run_reference("bfs", sg, kp, out, threads=threads)
        ref_par = np.fromfile(out, dtype=np.int32).reshape(kp, n)
        ok = list(ref["sources"]) == list(gpu["sources"])  # both sides drew the same SourcePicker sources
        for i, s in enumerate(ref["sources"]):
            d = oracle.bfs_depth(host.index, host.neighbors, s)
            ok &= bool(np.array_equal(gpu["depth"][i], d))
            ok &= oracle.verify_bfs_parents(host.index, host.neighbors, d, gpu["parent"][i], s)[0] == 0
            ok &= oracle.verify_bfs_parents(host.index, host.neighbors, d, ref_par[i], s)[0] == 0
        par["bfs"] = {"sources": kp, "ok": bool(ok),
                      "check": "depths == serial BFS; GPU parents and the reference's bfs_do_cpu parents valid trees"}
        ref = oracle.run_reference("sssp", wsg, kp, out, threads=threads)
        ref_d = np.fromfile(out, dtype=np.float32).reshape(kp, n).astype(np.float64)
        ref_d[np.isinf(ref_d)] = 0x7FFFFFFF  # the reference's inf is this engine's INT32_MAX
        want = ref_d.astype(np.int64)
        ok = bool(np.array_equal(gpu["dist"][:kp].astype(np.int64), want))
        par["sssp"] = {"sources": kp, "ok": ok, "check": "bit-exact vs the reference's sssp_pull_cpu"}
        ref = oracle.run_reference("pr", wsg, 0, out, threads=1)
        ref_pr = np.fromfile(out, dtype=np.float32)
        ordered = gpu["pr_ordered"]
        par["pagerank_reference_order"] = {
            "ok": bool(np.array_equal(ordered.view(np.uint32), ref_pr.view(np.uint32))),
            "sweeps": gpu["pr_ordered_sweeps"],
            "check": "hc_pr_pull_ordered bit-exact vs the reference's pr_pull_cpu on one thread"}
        x64, it64 = oracle.pr_jacobi_f64(host.index, host.neighbors, tol=1e-11, max_iters=1000)
        s = gpu["pr"]
        e_ref, e_64, r_64 = (float(np.abs(s - ref_pr).max()), float(np.abs(s - x64).max()),
                             float(np.abs(ref_pr - x64).max()))
        par["pagerank"] = {"ok": e_64 <= 1e-5, "gpu_vs_reference_linf": e_ref, "gpu_vs_fp64_linf": e_64,
                           "reference_vs_fp64_linf": r_64, "max_score": float(x64.max()),
                           "check": "timed Jacobi PageRank (L1 tol 1e-4) within 1e-5 of the FP64 fixed point; its "
                                    "distance to the reference is the reference's own stopping error (its "
                                    "per-vertex 5e-8 rule)"}
    return cpu, par


def run_reference_arm(a):
    """--impl reference: the reference's own OpenMP CPU code (oracle/_ref) on all host cores, on the same
    workload and config as the GPU arm.  Every timed step is a full step (64 bfs_do_cpu + 64 sssp_pull_cpu
    + 1 pr_pull_cpu) timed by the reference's own drivers; the graph is built by the numpy restatement of
    the generator (oracle/gen.py, bit-identical to the library's) and written as the .sg/.wsg files the
    reference loads, so no part of this project's library is loaded in this process."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import gen
    import oracle
    t0 = time.time()
    index, nbr, w = gen.build("kronecker", a.scale, a.edge_factor, a.seed, gen.W_I32)
    gen_s = time.time() - t0
    n, m = len(index) - 1, len(nbr)
    threads = os.cpu_count() or 1
    if not os.path.exists(oracle.REF_DRIVER):
        print(json.dumps({"impl": "reference", "unavailable": "the reference's CPU code was not built here "
                                                              "(oracle/_ref/ref_driver absent)"}))
        return
    t1 = time.time()
    with tempfile.TemporaryDirectory() as tmp:
        sg, wsg = _ref_graph_files(tmp, index, nbr, w, gen.write_graph)
        del index, nbr, w
        # Warm-up: one run per algorithm from the first source (the CPU needs no more); then K full steps.
        steps, per_run, _ = _ref_step_ms(sg, wsg, a.sources, threads, a.steps, max(1, a.warmup))
    wall = time.time() - t1
    total = float(np.sum(steps))
    runs = 2 * a.sources + 1
    value = a.steps * runs * (m / 2) / (total / 1e3) / 1e9
    sample = (f"every step the full workload: bfs_do_cpu x{a.sources} + sssp_pull_cpu x{a.sources} + "
              f"pr_pull_cpu x1 on {threads} OpenMP threads, timed by the reference's drivers; warm-up: "
              f"{max(1, a.warmup)} run(s) of each from the first source")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": total / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32/f32", "data": "synthetic",
        "config": workload(a) | {"num_nodes": n, "num_edges": m, "parallelism": f"replicas x{a.gpus}"},
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "detail": {"per_run_ms": per_run, "step_ms": steps, "graph_gen_s": gen_s, "timed_wall_s": wall,
                   "graph": "oracle/gen.py (numpy restatement; bit-identical to the library's generator)"}}))


# ----------------------------------------------------------- extra sections

def batched_section(g, host, a, torch, dev, stream, k=512):
    """Batched multi-source BFS and SSSP (one launch sequence for all sources of a group) against k
    sequential plain launches, on the benchmark graph; parity: every batched row equals the plain run's
    (the plain path itself is checked against the reference in the CPU leg and the tests)."""
    import hc
    n, m = host.num_nodes, host.num_edges
    src = hc.pick_sources(host, k)
    out = {"sources": k}
    if a.tune:  # untimed: group widths and switch points for both batched paths
        out["tuning"] = g.autotune(src, hc.TUNE_BFS_BATCHED | hc.TUNE_SSSP_BATCHED)
    seq = torch.empty((k, n), dtype=torch.int32, device=dev)
    bat = torch.empty((k, n), dtype=torch.int32, device=dev)
    par1 = torch.empty((1, n), dtype=torch.int32, device=dev)
    for name, run_b, run_p in [
            ("bfs", lambda: g.bfs_batched(src, bat), lambda i: g.bfs(src[i:i + 1], seq[i:i + 1], par1)),
            ("sssp", lambda: g.sssp_batched(src, bat), lambda i: g.sssp(src[i:i + 1], seq[i:i + 1]))]:
        run_b()  # warm-up: workspaces and plans sized once
        run_p(0)
        tb = min(_time_cuda(run_b, torch, dev, 1) for _ in range(2))
        tp = _time_cuda(lambda: [run_p(i) for i in range(k)], torch, dev, 1)
        out[name] = {"batched_ms": tb, "sequential_ms": tp, "speedup": tp / tb,
                     "batched_gteps": k * (m / 2) / tb / 1e6, "sequential_gteps": k * (m / 2) / tp / 1e6,
                     "parity": bool(torch.equal(bat, seq))}
    del seq, bat
    torch.cuda.empty_cache()
    out["ok"] = out["bfs"]["parity"] and out["sssp"]["parity"]
    out["config"] = (f"kronecker-s{a.scale}-ef{a.edge_factor}: {k} BFS and {k} SSSP sources batched vs {k} "
                     f"sequential plain launches (device outputs [{k}][N] int32)")
    return out


def batched_ranks_section(g, host, a, torch, dev, rank, world, k=512):
    """N > 1: the batched engine sharded by source (weak scaling, no data-path collective): every rank runs
    k sources of its own (picks [r*k, (r+1)*k) of the SourcePicker sequence) in one batched BFS and one
    batched SSSP call; time = max over ranks; parity: the first rows against the plain runs on each rank."""
    import hc
    from hc.shard import max_over_ranks, rank_sources
    n, m = host.num_nodes, host.num_edges
    src = rank_sources(host, k, rank)
    bat = torch.empty((k, n), dtype=torch.int32, device=dev)
    one = torch.empty((1, n), dtype=torch.int32, device=dev)
    par1 = torch.empty((1, n), dtype=torch.int32, device=dev)
    out = {"sources_per_rank": k, "ranks": world}
    ok = True
    for name, run_b, run_p in [("bfs", lambda: g.bfs_batched(src, bat), lambda i: g.bfs(src[i:i + 1], one, par1)),
                               ("sssp", lambda: g.sssp_batched(src, bat), lambda i: g.sssp(src[i:i + 1], one))]:
        run_b()
        ms = max_over_ranks(_time_cuda(run_b, torch, dev, 1), dev)
        for i in (0, k // 2, k - 1):
            run_p(i)
            ok &= bool(torch.equal(bat[i:i + 1], one))
        out[name] = {"batched_ms": ms, "batched_gteps": world * k * (m / 2) / ms / 1e6}
    t = torch.tensor([1.0 if ok else 0.0], device=dev)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
    out["ok"] = bool(t.item() == 1.0)
    del bat
    torch.cuda.empty_cache()
    return out


def adjoint_section(g, host, a, torch, dev):
    """PageRank forward + hand-written adjoint against the forward alone (weighted: the int32 weights as
    fp32, row-normalised; L = c . x with seeded Gaussian c; L1 tolerance 1e-6 forward, 1e-6 relative
    adjoint).  Parity at full size through two exact identities:
      linearity        x is linear in the teleport t, so c . x = (dL/dt) . t
      row scaling      A does not change when one row's weights are scaled, so sum_k w_uk dL/dw_uk = 0
                       for every row u"""
    n, m = host.num_nodes, host.num_edges
    rng = np.random.default_rng(a.seed)
    c = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).to(dev)
    x = torch.empty(n, dtype=torch.float32, device=dev)
    dt = torch.empty(n, dtype=torch.float32, device=dev)
    dw = torch.empty(m, dtype=torch.float32, device=dev)
    opts = dict(tol_l1=1e-6, max_iters=200, weighted=True)

    def fwd():
        return g.pagerank(None, x, **opts)

    def bwd():
        return g.pagerank_backward(x, c, dteleport=dt, dweights=dw, **opts)
    fwd()
    bwd()  # warm-up: fp32 weights, transposed weights, symmetry check, workspaces
    tf = min(_time_cuda(fwd, torch, dev, 1) for _ in range(3))
    tfb = min(_time_cuda(lambda: (fwd(), bwd()), torch, dev, 1) for _ in range(3))
    _, fst = fwd()
    _, _, bst = bwd()
    x64, c64 = x.double(), c.double()
    lhs = float((c64 * x64).sum())
    rhs = float(dt.double().sum() / n)  # t = 1/N everywhere
    lin = abs(lhs - rhs) / float((c64 * x64).abs().sum())
    deg = torch.from_numpy(np.diff(host.index)).to(dev)
    rows = torch.repeat_interleave(torch.arange(n, device=dev), deg)
    w = torch.from_numpy(host.weights.astype(np.float32)).to(dev).double()
    wg = w * dw.double()
    row_sum = torch.zeros(n, dtype=torch.float64, device=dev).index_add_(0, rows, wg)
    row_abs = torch.zeros(n, dtype=torch.float64, device=dev).index_add_(0, rows, wg.abs())
    scale_inv = float(row_sum.abs().max() / row_abs.max())
    del rows, w, wg, row_sum, row_abs, dw
    torch.cuda.empty_cache()
    return {"forward_ms": tf, "forward_adjoint_ms": tfb, "ratio": tfb / tf,
            "forward_iterations": int(fst.iterations), "adjoint_iterations": int(bst.iterations),
            "parity": {"linearity_rel_err": lin, "row_scaling_rel_err": scale_inv,
                       "ok": lin <= 1e-4 and scale_inv <= 1e-4, "tolerance": 1e-4},
            "config": f"kronecker-s{a.scale}-ef{a.edge_factor}: weighted PageRank (int32 weights as fp32, "
                      f"row-normalised), L = c.x, c ~ N(0,1) seed {a.seed}; tol 1e-6"}


# ----------------------------------------------------------- GPU arm

def main():
    a = parse()
    if a.impl == "reference":
        run_reference_arm(a)
        return
    if a.mode == "profile":
        profile_case(a)
        return
    if a.suite != "plain":
        run_suite(a)
        return
    import torch
    import torch.distributed as dist

    import hc

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)

    t0 = time.time()
    host = hc.gen_kronecker(a.scale, a.edge_factor, a.seed, hc.W_I32)
    gen_s = time.time() - t0
    n, m = host.num_nodes, host.num_edges
    g = hc.Graph.from_host(host, device=local)
    # One side stream for the library and the timing events.
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    g.set_stream(stream.cuda_stream)
    k = a.sources
    from hc.shard import max_over_ranks, rank_sources
    src = rank_sources(host, k, rank)
    src_dev = torch.from_numpy(src).to(dev)
    # Untimed: the autotuner picks the BFS / SSSP launch parameters on this graph.
    tuning = g.autotune(src, hc.TUNE_BFS | hc.TUNE_BFS_LEVELS | hc.TUNE_SSSP) if a.tune else None

    depth = torch.empty((k, n), dtype=torch.int32, device=dev)
    parent = torch.empty((k, n), dtype=torch.int32, device=dev)
    dist_o = torch.empty((k, n), dtype=torch.int32, device=dev)
    scores = torch.empty(n, dtype=torch.float32, device=dev)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device=dev)

    def step(times):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        _, _, sb = g.bfs(src_dev, depth, parent)
        ev[1].record(stream)
        _, _, ss = g.sssp(src_dev, dist_o)
        ev[2].record(stream)
        _, sp = g.pagerank(None, scores, tol_l1=1e-4, max_iters=50)
        ev[3].record(stream)
        torch.cuda.synchronize(dev)
        times.append([ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]), ev[2].elapsed_time(ev[3])])
        return sb, ss, sp

    for _ in range(a.warmup):
        step([])
    # Instrumented pass (not timed), after the warm-up so that one-time setup
    # (row plans, weight statistics) is not in its kernel times: algorithmic
    # byte counts and device times of the launches.
    _, _, bst = g.bfs(src_dev, depth, parent, stats=True)
    _, _, sst = g.sssp(src_dev, dist_o, stats=True)
    _, pst = g.pagerank(None, scores, tol_l1=1e-4, max_iters=50)
    # Timed region: K steps, L2 flushed (untimed) between steps.
    times = []
    pr_iters = []
    launch_ms = []  # device time of each algorithm's launches (the library's events) per timed step
    launches0 = hc.kernel_launches()
    with ClockSampler(local) as clk:
        for _ in range(a.steps):
            flush.fill_(1)
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize(dev)
            sb, ss, sp = step(times)
            pr_iters.append(sp.iterations)
            launch_ms.append([sb.ms, ss.ms, sp.ms])
    # Kernels the library launched in the timed steps (its own launch counter).
    launches = hc.kernel_launches() - launches0
    t = np.array(times)  # ms per algorithm per step
    step_ms = t.sum(axis=1)
    total_ms = float(step_ms.sum())
    total_ms = max_over_ranks(total_ms, dev)
    runs = 2 * k + 1
    value = world * a.steps * runs * (m / 2) / (total_ms / 1e3) / 1e9

    # End to end through the public API with host buffers: sources from pinned
    # host memory in, and back to pinned host memory what the reference's
    # drivers return: BFS parents (bfs_gpu), SSSP distances (sssp_pull_gpu),
    # PageRank scores (pr_pull_gpu).
    # The host buffers are placed (and the calls made) from the CPUs of the
    # GPU's NUMA node, where copies to and from the GPU are fastest; the
    # thread's CPU set is restored afterwards.
    saved_cpus = os.sched_getaffinity(0)
    near = gpu_local_cpus(dev)
    if near:
        os.sched_setaffinity(0, near)
    src_pin = torch.from_numpy(src.copy()).pin_memory()
    h_parent = torch.empty((k, n), dtype=torch.int32).pin_memory().numpy()
    h_dist = torch.empty((k, n), dtype=torch.int32).pin_memory().numpy()
    h_scores = torch.empty(n, dtype=torch.float32).pin_memory().numpy()
    e2e_ms = []
    e2e_phase = []  # per step: BFS, SSSP, PageRank calls (host clock)
    for _ in range(max(1, a.steps)):
        flush.fill_(1)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        s_np = src_pin.numpy()
        g.bfs(s_np, None, h_parent, want_depth=False)
        t1 = time.perf_counter()
        g.sssp(s_np, h_dist)
        t2 = time.perf_counter()
        g.pagerank(None, h_scores, tol_l1=1e-4, max_iters=50)
        t3 = time.perf_counter()
        e2e_ms.append((t3 - t0) * 1e3)
        e2e_phase.append([(t1 - t0) * 1e3, (t2 - t1) * 1e3, (t3 - t2) * 1e3])
    os.sched_setaffinity(0, saved_cpus)
    e2e_total = float(np.sum(e2e_ms))
    e2e_total = max_over_ranks(e2e_total, dev)
    e2e_value = world * len(e2e_ms) * runs * (m / 2) / (e2e_total / 1e3) / 1e9

    # Roofline of the dominant kernel (largest share of the step).
    hbm, peak_kind = peaks()
    per_algo = {}
    share = t.sum(axis=0) / t.sum()
    lm = np.array(launch_ms)
    for i, (name, st) in enumerate([("bfs", bst), ("sssp", sst), ("pagerank", pst)]):
        # Device time of the launches themselves in the timed steps (library
        # events on the launching stream); the instrumented pass gives only
        # the byte counts (its statistics-keeping kernels run slower).
        ms_kernel = float(lm[:, i].mean())
        runs_a = k if name != "pagerank" else 1
        per_algo[name] = {
            "gteps": runs_a * (m / 2) / (float(t[:, i].mean()) / 1e3) / 1e9,
            "ms_per_step": float(t[:, i].mean()),
            "share": float(share[i]),
            "kernel_ms": ms_kernel,
            "bytes_model": st.bytes_model,
            "achieved_gbs": st.bytes_model / (ms_kernel / 1e3) / 1e9 if ms_kernel > 0 else None,
        }
    per_algo["pagerank"]["iterations"] = int(pst.iterations)
    per_algo["bfs"]["levels"] = int(bst.levels)
    per_algo["sssp"]["epochs"] = int(sst.epochs)
    # One streaming pass over the CSR at the measured peak: the floor of any algorithm that reads every
    # edge once (8(N+1) offsets + 4M neighbours, + 4M weights for SSSP), per source / per iteration.
    for name, wb in (("bfs", 0), ("sssp", 4), ("pagerank", 0)):
        one = (8.0 * (n + 1) + (4.0 + wb) * m) / (peaks()[0] * 1e9) * 1e3
        unit_ms = per_algo[name]["ms_per_step"] / (k if name != "pagerank" else max(1, int(pst.iterations)))
        per_algo[name]["one_pass_ms"] = one
        per_algo[name]["one_pass_frac"] = one / unit_ms if unit_ms > 0 else None
    dom = max(per_algo, key=lambda x: per_algo[x]["share"])
    achieved = per_algo[dom]["achieved_gbs"]
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(f"s{a.scale}", {}).get(dom)
        except Exception:
            traffic = None
    roof = {"bound": "hbm", "kernel": {"bfs": "bfs_persistent",
                                       "sssp": "sssp_persistent + sssp_pull_kernel",
                                       "pagerank": "pr_sweep"}[dom],
            "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm if achieved else None, "peak_kind": peak_kind, "traffic": traffic,
            "traffic_unit": "DRAM bytes per source (per solve for pagerank), one ncu capture "
                            "(profiles/traffic.json)" if traffic else None,
            "bytes_model_per_unit": per_algo[dom]["bytes_model"] / (k if dom != "pagerank" else 1)}

    # The GPU's outputs for the parity checks: what the last end-to-end step returned to host memory
    # (parents, distances, scores) and the timed steps' depths, for the first sources; and the
    # reference-order PageRank (untimed).
    extras = {}
    cpu = None
    parity = None
    if rank == 0 and world == 1:
        kp = min(4, k)
        gpu_out = {"sources": src[:kp].tolist(), "depth": depth[:kp].cpu().numpy(), "parent": h_parent[:kp].copy(),
                   "dist": h_dist[:kp].copy(), "pr": h_scores.copy()}
        if not a.no_cpu_baseline:  # the reference-order PageRank is checked against the reference's run
            ordered, ost = g.pagerank_ordered()
            gpu_out.update(pr_ordered=ordered, pr_ordered_sweeps=int(ost.iterations), pr_ordered_ms=ost.ms)
        del depth, parent, dist_o, flush
        torch.cuda.empty_cache()
        if not a.no_extras:
            extras["batched"] = batched_section(g, host, a, torch, dev, stream)
            extras["adjoint"] = adjoint_section(g, host, a, torch, dev)
        if not a.no_cpu_baseline:
            try:
                cpu, parity = cpu_leg(host, a, gpu_out)
            except Exception as ex:  # reported, not fatal
                cpu = {"value": None, "unit": "GTEPS", "cores": None, "kind": "unavailable", "sample": repr(ex)}
        if parity is not None:
            parity["pagerank_reference_order"]["ms"] = gpu_out["pr_ordered_ms"]
            for key in ("batched", "adjoint"):
                if key in extras:
                    parity[key] = {"ok": extras[key]["ok"] if key == "batched" else extras[key]["parity"]["ok"]}
            parity["ok"] = all(v["ok"] for v in parity.values() if isinstance(v, dict))

    if world > 1 and not a.no_extras:
        # Every rank takes the same collective steps here (max-over-ranks timings, the parity reduction).
        extras["batched"] = batched_ranks_section(g, host, a, torch, dev, rank, world)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": float(step_ms.mean()), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32/f32", "data": "synthetic",
            "config": workload(a) | {"num_nodes": n, "num_edges": m, "parallelism": f"replicas x{world}"},
            "roofline": roof, "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "GTEPS", "h2d_bytes_per_step": int(src.nbytes),
                    "d2h_bytes_per_step": int(2 * k * n * 4 + n * 4),
                    "host_cpus": (f"{len(near)} of {len(saved_cpus)}, the GPU's NUMA node" if near
                                  else f"all {len(saved_cpus)}"),
                    "phase_ms": dict(zip(("bfs", "sssp", "pagerank"),
                                         np.array(e2e_phase).mean(axis=0).round(3).tolist()))},
            "gpu_launches": launches, "clocks": clk.summary(), "parity": parity, "per_algo": per_algo,
            **extras, "tuning": tuning, "graph_gen_s": gen_s}), flush=True)
    g.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
