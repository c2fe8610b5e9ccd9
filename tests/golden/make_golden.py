"""Writes the known-answer fixtures in tests/golden/ (run: python tests/golden/make_golden.py).

hiperbio/tensor-episdet ships no tests, fixtures or expected outputs, so these
fixtures come from an independent restatement written here in plain Python:
genotypes are drawn with numpy from a fixed seed, every contingency table is
counted directly from the genotype matrix (no AND/derivation tricks), and the
scores apply include/scoring.hpp's formulas (K2: |sum lnG(ctrl+1) + lnG(case+1)
- lnG(ctrl+case+2)|, minimised; MI: H(X) + H(Y) - H(X,Y) in log2, maximised)
in double precision.  The CPU oracle is checked against them.
"""
from __future__ import annotations

import itertools
import json
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def hwe_genotypes(rng, M, n, maf=(0.05, 0.5)):
    p = rng.uniform(maf[0], maf[1], size=M)
    u = rng.random((M, n))
    q0 = (1 - p) ** 2
    q1 = 1 - p ** 2
    return np.where(u < q0[:, None], 0, np.where(u < q1[:, None], 1, 2)).astype(np.int8)


def table(g_cases, g_controls, snps):
    k = len(snps)
    shape = (3,) * k
    cs = np.zeros(shape, dtype=np.int64)
    cn = np.zeros(shape, dtype=np.int64)
    for s in range(g_cases.shape[1]):
        cs[tuple(int(g_cases[v, s]) for v in snps)] += 1
    for s in range(g_controls.shape[1]):
        cn[tuple(int(g_controls[v, s]) for v in snps)] += 1
    return cs.reshape(-1), cn.reshape(-1)


def k2(cs, cn):
    s = 0.0
    for a, b in zip(cs, cn):
        s = s + ((math.lgamma(b + 1.0) + math.lgamma(a + 1.0)) - math.lgamma(a + b + 2.0))
    return abs(s)


def mi(cs, cn, nc, nn):
    N = nc + nn

    def lg(v):
        return 0.0 if v == 0 else math.log2(v / N)

    hy = -((nc / N) * lg(nc)) - ((nn / N) * lg(nn))
    ha = hx = 0.0
    for a, b in zip(cs, cn):
        pa, pb = a / N, b / N
        ha -= pa * lg(a)
        ha -= pb * lg(b)
        hx -= (pa + pb) * lg(a + b)
    return (hx + hy) - ha


def case(name, g_cases, g_controls, order, top=10):
    nc, nn = g_cases.shape[1], g_controls.shape[1]
    M = g_cases.shape[0]
    rows = []
    for snps in itertools.combinations(range(M), order):
        cs, cn = table(g_cases, g_controls, snps)
        rows.append((snps, cs, cn, k2(cs, cn), mi(cs, cn, nc, nn)))
    best_k2 = min(rows, key=lambda r: (r[3], r[0]))
    best_mi = min(rows, key=lambda r: (-r[4], r[0]))
    by_k2 = sorted(rows, key=lambda r: (r[3], r[0]))[:top]
    by_mi = sorted(rows, key=lambda r: (-r[4], r[0]))[:top]
    sample = rows[:: max(1, len(rows) // 12)]
    return {
        "name": name,
        "order": order,
        "num_cases": nc,
        "num_controls": nn,
        "cases": g_cases.tolist(),
        "controls": g_controls.tolist(),
        "best_k2": {"snps": list(best_k2[0]), "score": best_k2[3]},
        "best_mi": {"snps": list(best_mi[0]), "score": best_mi[4]},
        "top_k2": [{"snps": list(r[0]), "score": r[3]} for r in by_k2],
        "top_mi": [{"snps": list(r[0]), "score": r[4]} for r in by_mi],
        "tables": [{"snps": list(r[0]), "cases": r[1].tolist(), "controls": r[2].tolist(), "k2": r[3], "mi": r[4]}
                   for r in sample],
    }


def main():
    rng = np.random.default_rng(0xE915)
    cases = []
    # Hand-sized tables: every genotype combination present.
    cases.append(case("tiny_pairs", hwe_genotypes(rng, 5, 9), hwe_genotypes(rng, 5, 7), 2))
    cases.append(case("tiny_triplets", hwe_genotypes(rng, 6, 13), hwe_genotypes(rng, 6, 11), 3))
    # Word and padding edges: class sizes 1, 31, 32, 33 and 1025 samples.
    cases.append(case("edge_pairs_1_33", hwe_genotypes(rng, 9, 1), hwe_genotypes(rng, 9, 33), 2))
    cases.append(case("edge_triplets_31_32", hwe_genotypes(rng, 8, 31), hwe_genotypes(rng, 8, 32), 3))
    cases.append(case("edge_triplets_1025_40", hwe_genotypes(rng, 7, 1025), hwe_genotypes(rng, 7, 40), 3))
    # A planted interaction the scores must find.
    g_all = hwe_genotypes(rng, 12, 400, maf=(0.2, 0.5))
    risk = 0.25 + 0.6 * ((g_all[3] >= 1) & (g_all[7] >= 1) & (g_all[10] >= 1))
    lab = rng.random(400) < risk
    cases.append(case("planted_triplet_3_7_10", g_all[:, lab], g_all[:, ~lab], 3))
    cases.append(case("random_pairs", hwe_genotypes(rng, 20, 150), hwe_genotypes(rng, 20, 170), 2))
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "seed": 0xE915, "cases": cases}, f)
    print(f"wrote {len(cases)} cases")


if __name__ == "__main__":
    main()
