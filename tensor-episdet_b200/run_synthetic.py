"""Runs one search on a seeded synthetic dataset and prints a JSON summary.

  python tensor-episdet_b200/run_synthetic.py --snps 2048 --cases 65536 --controls 65536 \
      --order 3 --score k2 [--first-begin 0 --first-end 1] [--engine tensor|simt] [--repeat 1]

Useful to reproduce a workload, to time one configuration, or as the
command of a profiler capture of a single counting launch (a one-SNP slab
with --first-end 1 launches the triplet kernel once).
"""
import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import episdet  # noqa: E402


def perm(a):
    """Permutation batch: one cohort, a.permutations label vectors, 2-way or 3-way."""
    import time

    import numpy as np

    n = a.cases + a.controls
    planes = episdet.generate_cohort(a.seed, a.snps, n, maf=tuple(a.maf))
    labels = episdet.generate_labels(a.seed + 1, n, a.cases, a.permutations)
    t0 = time.perf_counter()
    res = episdet.search_perm(planes, n, labels, order=a.order, score=a.score, top_k=a.top_k, flags=a.flags)
    dt = time.perf_counter() - t0
    best = np.array([r.score for r in res])
    sets = sum(r.sets_evaluated for r in res)
    print(json.dumps({"permutations": len(res), "seconds": dt, "device_ms": sum(r.device_ms for r in res),
                      "count_kernel_ms": sum(r.count_kernel_ms for r in res),
                      "executed_macs": sum(r.executed_macs for r in res),
                      "sets": sets, "tera_sets_samples_per_s": sets * n / dt / 1e12,
                      "label0_best": [list(res[0].snps), res[0].score],
                      "null_best_scores": {"min": float(best[1:].min()), "median": float(np.median(best[1:])),
                                           "max": float(best[1:].max())} if len(res) > 1 else None,
                      # Max-statistic adjusted p-values of label 0's five best sets.
                      "label0_top5_pvalues": [float(p) for p in episdet.perm_pvalues(res, a.score)[:5]]
                      if len(res) > 1 else None}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--snps", type=int, default=1024)
    ap.add_argument("--cases", type=int, default=8192)
    ap.add_argument("--controls", type=int, default=8192)
    ap.add_argument("--order", type=int, default=3)
    ap.add_argument("--score", default="k2")
    ap.add_argument("--engine", default="auto")
    ap.add_argument("--first-begin", type=int, default=0)
    ap.add_argument("--first-end", type=int, default=0)
    ap.add_argument("--top-k", type=int, default=1024)
    ap.add_argument("--seed", type=lambda v: int(v, 0), default=0xE917)
    ap.add_argument("--maf", type=float, nargs=2, default=(0.05, 0.5))
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--planted", default="",
                    help="planted sets, comma-separated SNP indices, sets separated by ';' (e.g. 137,2048,3901)")
    ap.add_argument("--base-risk", type=float, default=0.5)
    ap.add_argument("--effect", type=float, default=0.25)
    ap.add_argument("--flags", type=lambda v: int(v, 0), default=0,
                    help="extra EPISDET_FLAG_* bits (e.g. 0x20 forces the K2 triplet scoring filter on)")
    ap.add_argument("--permutations", type=int, default=0,
                    help="search one cohort of cases+controls samples under this many label vectors "
                         "(label 0 the first half of the samples, the rest seeded permutations)")
    a = ap.parse_args()
    if a.permutations:
        perm(a)
        return
    planted = [tuple(int(v) for v in ps.split(",")) for ps in a.planted.split(";")] if a.planted else []
    cases, controls = episdet.generate(a.seed, a.snps, a.cases, a.controls, maf=tuple(a.maf), planted=planted,
                                       base_risk=a.base_risk, effect=a.effect)
    for i in range(a.repeat):
        r = episdet.search(cases, controls, a.cases, a.controls, order=a.order, score=a.score, top_k=a.top_k,
                           engine=a.engine, first_begin=a.first_begin, first_end=a.first_end,
                           flags=episdet.FLAG_TIMING | a.flags)
    n = a.cases + a.controls
    out = {"snps": list(r.snps), "score": r.score, "sets": r.sets_evaluated, "device_ms": r.device_ms,
           "count_kernel_ms": r.count_kernel_ms, "count_launches": r.count_kernel_launches,
           "executed_macs": r.executed_macs, "launches": r.kernel_launches,
           "tera_sets_samples_per_s": r.sets_evaluated * n / (r.device_ms * 1e-3) / 1e12}
    # FP32 ranking score against the FP64 re-score over the candidate list.
    f32 = r.top_fp32.astype("float64")
    err = abs(f32 - r.top_fp64)
    rel = err / abs(r.top_fp64).clip(min=1e-300)
    out["fp32_vs_fp64"] = {"candidates": int(len(f32)), "max_abs": float(err.max()) if len(err) else 0.0,
                           "max_rel": float(rel.max()) if len(rel) else 0.0}
    out["top5"] = [[[int(v) for v in t], float(f)] for t, f in zip(r.top_snps[:5], r.top_fp64[:5])]
    print(json.dumps(out))

if __name__ == "__main__":
    main()
