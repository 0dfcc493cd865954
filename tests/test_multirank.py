"""Multi-rank source sharding on CPU: two gloo ranks, each running the oracle
on its own slice of sources (the stand-in for its GPU), must reproduce the
single-process result, and the timing reduction must be the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "hetero-compute_b200")]
    import hc
    import oracle
    from hc.shard import gather_rows, max_over_ranks, rank_sources, run_sharded, split_batch
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        host = hc.gen_kronecker(10, 8, 3)
        src = rank_sources(host, 5, rank)
        depth = np.stack([oracle.bfs_depth(host.index, host.neighbors, s) for s in src])
        allsrc = gather_rows(src[None, :], world).reshape(-1)
        alld = gather_rows(depth, world)
        t = max_over_ranks(1.0 + rank)
        # split_batch: pad each rank's slice to a common width with -1 before gathering
        part = split_batch(np.arange(11), rank, world)
        parts = gather_rows(np.pad(part, (0, 6 - len(part)), constant_values=-1)[None, :], world)
        # One batch of 11 sources split over the ranks (uneven shares), each rank's share run by a stand-in
        # for the batched BFS (the oracle, row per source), rows gathered in source order.
        batch = hc.pick_sources(host, 11)
        rows = run_sharded(lambda ss: np.stack([oracle.bfs_depth(host.index, host.neighbors, s) for s in ss]),
                           batch, rank, world)
        if rank == 0:
            q.put((allsrc, alld, t, parts, rows))
    finally:
        dist.destroy_process_group()


def test_two_rank_source_sharding():
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "hetero-compute_b200")]
    import hc
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    allsrc, alld, t, parts, rows = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    host = hc.gen_kronecker(10, 8, 3)
    ref_src = hc.pick_sources(host, 10)
    assert np.array_equal(allsrc, ref_src)
    for i, s in enumerate(ref_src):
        assert np.array_equal(alld[i], oracle.bfs_depth(host.index, host.neighbors, s))
    assert t == 2.0
    got = parts[parts >= 0]
    assert np.array_equal(np.sort(got), np.arange(11))
    batch = hc.pick_sources(host, 11)
    assert rows.shape == (11, host.num_nodes)
    for i, s in enumerate(batch):
        assert np.array_equal(rows[i], oracle.bfs_depth(host.index, host.neighbors, s))
