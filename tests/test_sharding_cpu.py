"""The N-GPU bench path on CPU ranks: first-SNP slabs of equal work, one
all-gather of the per-rank candidate lists, merge -> the one-rank answer.

Runs two gloo ranks on 127.0.0.1 with the CPU oracle standing in for the GPU
search of each slab."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "oracle")]
    import bench
    import pyoracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.default_rng(3)
    M = 40
    g_cases = rng.integers(0, 3, size=(M, 300))
    g_controls = rng.integers(0, 3, size=(M, 280))
    cases, controls = pyoracle.pack(g_cases), pyoracle.pack(g_controls)
    bench.M = M  # slabs over this small dataset
    fb, fe = bench.work_slabs(world)[rank]
    r = pyoracle.search(cases, controls, 300, 280, order=3, score="k2", top_k=32, first_begin=fb, first_end=fe)
    mine = (np.array(r["top"], dtype=np.int64), r["top_fp32"], r["top_fp64"])
    allv = [None] * world
    dist.all_gather_object(allv, mine)
    rows, best = bench.merge_candidates(allv)
    if rank == 0:
        full = pyoracle.search(cases, controls, 300, 280, order=3, score="k2", top_k=32)
        out.put((tuple(best[1]), best[2], tuple(full["best"]), full["best_fp64"],
                 [r[1] for r in rows[:32]], full["top"], sum(1 for _ in range(1))))
    dist.barrier()
    dist.destroy_process_group()


def test_work_slabs_balance():
    import bench

    s = bench.work_slabs(4)
    assert s[0][0] == 0 and s[-1][1] == bench.M - 2
    assert all(a[1] == b[0] for a, b in zip(s, s[1:]))
    import math

    w = [sum(math.comb(bench.M - 1 - x, 2) for x in range(a, b)) for a, b in s]
    assert max(w) / min(w) < 1.01


def test_two_rank_merge_equals_one_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    best, best64, full_best, full64, top, full_top, _ = res
    assert best == full_best and best64 == full64
    assert [tuple(t) for t in top] == [tuple(t) for t in full_top]
