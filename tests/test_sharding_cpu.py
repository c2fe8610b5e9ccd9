"""The multi-GPU path on CPU ranks (sharded.py): first-SNP slabs of equal
work, one all-gather of the per-rank candidate lists, merge -> the one-rank
answer.

Runs gloo ranks on 127.0.0.1 with the CPU oracle standing in for the GPU
search of each slab (the `search` argument of search_sharded)."""
import math
import os
import socket
import sys
from types import SimpleNamespace

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_search(cases, controls, nc, nn, *, num_snps, order, score, top_k, device, first_begin, first_end):
    import pyoracle

    o = pyoracle.search(cases, controls, nc, nn, order=order, score=score, top_k=top_k, first_begin=first_begin,
                        first_end=first_end)
    return SimpleNamespace(top_snps=np.array(o["top"], dtype=np.int64).reshape(-1, order), top_fp32=o["top_fp32"],
                           top_fp64=o["top_fp64"], sets_evaluated=o["sets"])


def _rank(rank, world, port, order, score, out):
    sys.path[:0] = [os.path.join(ROOT, "tensor-episdet_b200"), os.path.join(ROOT, "oracle")]
    import pyoracle
    import sharded

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.default_rng(3 + order)
    M = 40 if order == 3 else 90
    g_cases = rng.integers(0, 3, size=(M, 300))
    g_controls = rng.integers(0, 3, size=(M, 280))
    cases, controls = pyoracle.pack(g_cases), pyoracle.pack(g_controls)
    r = sharded.search_sharded(cases, controls, 300, 280, num_snps=M, order=order, score=score, top_k=32,
                               search=_oracle_search)
    if rank == 0:
        full = pyoracle.search(cases, controls, 300, 280, order=order, score=score, top_k=32)
        out.put((tuple(r.snps), r.score, tuple(full["best"]), full["best_fp64"], [tuple(t) for t in r.top_snps],
                 [tuple(t) for t in full["top"]], r.top_fp32.tobytes(), np.asarray(full["top_fp32"]).tobytes(),
                 r.sets_evaluated, full["sets"]))
    dist.barrier()
    dist.destroy_process_group()


def test_work_slabs_balance():
    sys.path.insert(0, os.path.join(ROOT, "tensor-episdet_b200"))
    import sharded

    M = 4096
    s = sharded.work_slabs(M, 3, 4)
    assert s[0][0] == 0 and s[-1][1] == M - 2
    assert all(a[1] == b[0] for a, b in zip(s, s[1:]))
    w = [sum(math.comb(M - 1 - x, 2) for x in range(a, b)) for a, b in s]
    assert max(w) / min(w) < 1.01
    # Pairs, a sub-range, and more ranks than first SNPs.
    s = sharded.work_slabs(100, 2, 3, first_begin=10, first_end=40)
    assert s[0][0] == 10 and s[-1][1] == 40
    s = sharded.work_slabs(5, 3, 6)
    assert s[-1][1] == 3 and sum(b - a for a, b in s) == 3 and all(b >= a for a, b in s)


def test_merge_orders_like_the_engines():
    sys.path.insert(0, os.path.join(ROOT, "tensor-episdet_b200"))
    import sharded

    a = (np.array([[0, 1], [2, 3]]), np.array([5.0, 7.0], np.float32), np.array([5.1, 6.9]))
    b = (np.array([[0, 2], [1, 4]]), np.array([5.0, 6.0], np.float32), np.array([5.05, 6.9]))
    rows, best = sharded.merge_candidates([a, b], "k2")
    assert [r[1] for r in rows] == [(0, 1), (0, 2), (1, 4), (2, 3)]
    assert best[1] == (0, 2)  # FP64 minimum
    rows, best = sharded.merge_candidates([a, b], "mi", top_k=3)
    assert [r[1] for r in rows] == [(2, 3), (1, 4), (0, 1)]
    assert best[1] == (1, 4)  # FP64 maximum 6.9, tie with (2, 3): lower set


@pytest.mark.parametrize("world,order,score", [(2, 3, "k2"), (3, 2, "mi")])
def test_sharded_equals_one_rank(world, order, score):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, order, score, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    best, best64, full_best, full64, top, full_top, f32, full_f32, sets, full_sets = res
    assert best == full_best and best64 == full64
    assert top == full_top and f32 == full_f32
    assert sets == full_sets


@pytest.mark.parametrize("score", ["k2", "mi"])
def test_slab_topk_lists_merge_to_the_global_topk(score):
    """The property the sharded search and the resume cursor rely on: keeping
    each slab's top-k by (FP32 key, set) and merging the kept lists gives the
    top-k of the whole set of candidates, ties on the FP32 score included."""
    sys.path.insert(0, os.path.join(ROOT, "tensor-episdet_b200"))
    import sharded

    rng = np.random.default_rng(11)
    for trial in range(20):
        n = int(rng.integers(50, 400))
        sets = rng.choice(10**6, size=n, replace=False)
        snps = np.stack([sets // 10000, (sets // 100) % 100, sets % 100], axis=1)
        f32 = rng.integers(0, 40, size=n).astype(np.float32) * np.float32(0.5)  # many ties
        f64 = f32.astype(np.float64) + rng.normal(0, 0.01, size=n)
        k = int(rng.integers(1, 60))
        rows_all, best_all = sharded.merge_candidates([(snps, f32, f64)], score, k)
        cuts = np.sort(rng.choice(np.arange(1, n), size=int(rng.integers(1, 6)), replace=False))
        parts = []
        for idx in np.split(np.arange(n), cuts):
            r, _ = sharded.merge_candidates([(snps[idx], f32[idx], f64[idx])], score, k)
            parts.append((np.array([x[1] for x in r]).reshape(-1, 3), np.array([x[0] for x in r], np.float32),
                          np.array([x[2] for x in r])))
        rows, best = sharded.merge_candidates(parts, score, k)
        assert rows == rows_all and best == best_all
