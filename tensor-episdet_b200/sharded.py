"""Multi-GPU exhaustive search: one process per GPU over torch.distributed.

The search shards without a data-path collective: each rank searches the
sets whose first SNP lies in its slab of the first-SNP range (slabs of equal
work, C(M-1-x, k-1) sets for first SNP x), and one all-gather of the k-entry
candidate lists (SNP set, FP32 score, FP64 re-score) lets every rank merge
them into the single-GPU answer: the union of the slabs' top-k lists holds the
global top-k in the engines' order (FP32 score, then set), and the FP64
optimum over it is the same best set (ties to the lowest set).

The reference runs on one GPU (src/search-triplets.cu:8); this is the
replacement's scale-out path.  Planes are replicated: every rank passes the
whole dataset (host arrays or its own GPU's tensors).
"""
from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np

import episdet


def work_slabs(num_snps: int, order: int, n: int, first_begin: int = 0, first_end: int = 0) -> list:
    """Splits the first SNPs that start a set, [first_begin, min(first_end, M-order+1)),
    into n contiguous (begin, end) slabs of about equal work; trailing slabs
    may be empty (begin == end) when n exceeds the number of first SNPs."""
    M = num_snps
    fe = M if first_end <= 0 or first_end > M else first_end
    last = min(fe, M - order + 1)
    fb = max(0, first_begin)
    w = [math.comb(M - 1 - x, order - 1) for x in range(fb, last)]
    total = sum(w)
    bounds, acc, r = [fb], 0, 1
    for i, v in enumerate(w):
        acc += v
        if r < n and acc >= total * r / n:
            bounds.append(fb + i + 1)
            r += 1
    while len(bounds) < n:
        bounds.append(last)
    bounds.append(last)
    return [(bounds[i], bounds[i + 1]) for i in range(n)]


def _fp32_key(score_fp32: float, maximize: bool) -> int:
    """The engines' candidate key (lower is better for both scores)."""
    s = np.float32(-score_fp32 if maximize else score_fp32)
    u = int(s.view(np.uint32))
    return (~u & 0xFFFFFFFF) if u & 0x80000000 else (u | 0x80000000)


def merge_candidates(tops, score="k2", top_k=None):
    """tops: per-rank (top_snps [n][order], top_fp32 [n], top_fp64 [n]).
    Returns (rows, best): rows = (fp32, set, fp64) in the engines' order
    (FP32 score key, then set), cut to top_k; best = the FP64 optimum of rows
    (lowest set on ties)."""
    maximize = (score == "mi") if isinstance(score, str) else int(score) == episdet.SCORE_MI
    rows = []
    for snps, f32, f64 in tops:
        for s, a, b in zip(np.asarray(snps).tolist(), np.asarray(f32).tolist(), np.asarray(f64).tolist()):
            rows.append((float(a), tuple(int(v) for v in s), float(b)))
    rows.sort(key=lambda r: (_fp32_key(r[0], maximize), r[1]))
    if top_k is not None:
        rows = rows[:top_k]
    if not rows:
        return rows, None
    best = (max if maximize else min)(rows, key=lambda r: (r[2], tuple(-v for v in r[1])) if maximize
                                      else (r[2], r[1]))
    return rows, best


def gather_candidates(top_snps, top_fp32, top_fp64, top_k: int, order: int, group=None, device=None):
    """All-gathers each rank's candidate list (at most top_k entries) as one
    [top_k][5] float64 tensor per rank (3 SNP indices, FP32 score, FP64
    score; unused rows marked by a NaN FP64 score).  device: where the
    collective's tensors live (a CUDA device for NCCL, None -> CPU for gloo)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    t = torch.full((top_k, 5), float("nan"), dtype=torch.float64)
    n = len(top_fp32)
    snps = np.zeros((n, 3), dtype=np.float64)
    snps[:, :order] = np.asarray(top_snps)[:, :order]
    t[:n, 0:3] = torch.from_numpy(snps)
    t[:n, 3] = torch.from_numpy(np.asarray(top_fp32, dtype=np.float64))
    t[:n, 4] = torch.from_numpy(np.asarray(top_fp64, dtype=np.float64))
    if device is not None:
        t = t.to(device)
    out = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(out, t, group=group)
    tops = []
    for o in out:
        o = o.cpu().numpy()
        o = o[~np.isnan(o[:, 4])]
        tops.append((o[:, 0:order].astype(np.int64), o[:, 3].astype(np.float32), o[:, 4]))
    return tops


def search_sharded(cases, controls, num_cases: int, num_controls: int, *, num_snps=None, order: int = 3,
                   score="k2", top_k: int = 1024, group=None, device: int = 0, collective_device=None,
                   search=None, **kwargs):
    """The search of episdet.search sharded over the ranks of `group` (every
    rank calls it with the same arguments and its own GPU `device`).  Returns
    the merged answer on every rank: snps, score, score_fp32, top_snps,
    top_fp32, top_fp64, sets_evaluated (summed over ranks).  The collective
    runs on `collective_device` (default: this rank's GPU under NCCL, the CPU
    under gloo).  `search` replaces episdet.search (same keyword arguments),
    e.g. to run the merge logic against another implementation."""
    import torch
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    if collective_device is None and dist.get_backend(group) == "nccl":
        collective_device = torch.device("cuda", device)  # NCCL collectives take device tensors
    M = num_snps if num_snps is not None else int(cases.shape[0])
    fb, fe = work_slabs(M, order, world, kwargs.pop("first_begin", 0), kwargs.pop("first_end", 0))[rank]
    run = search or episdet.search
    if fe > fb:
        r = run(cases, controls, num_cases, num_controls, num_snps=M, order=order, score=score, top_k=top_k,
                device=device, first_begin=fb, first_end=fe, **kwargs)
        mine = (r.top_snps, r.top_fp32, r.top_fp64, int(r.sets_evaluated))
    else:
        mine = (np.zeros((0, order), np.int64), np.zeros(0, np.float32), np.zeros(0), 0)
    tops = gather_candidates(mine[0], mine[1], mine[2], top_k, order, group=group, device=collective_device)
    sets = torch.tensor([mine[3]], dtype=torch.int64)
    if collective_device is not None:
        sets = sets.to(collective_device)
    dist.all_reduce(sets, group=group)
    rows, best = merge_candidates(tops, score, top_k)
    if best is None:
        raise episdet.EpisdetError(9, "no candidate survived the sharded search")
    return SimpleNamespace(
        snps=best[1], score=best[2], score_fp32=best[0], sets_evaluated=int(sets.item()),
        top_snps=np.array([r[1] for r in rows], dtype=np.int64).reshape(-1, order),
        top_fp32=np.array([r[0] for r in rows], dtype=np.float32), top_fp64=np.array([r[2] for r in rows]),
        slab=(fb, fe))
