"""CPU oracle against the known-answer fixtures and algebraic invariants.

The fixtures (tests/golden/known_answers.json, written by
tests/golden/make_golden.py) count every contingency table directly from the
genotype matrix and score it with include/scoring.hpp's formulas in plain
Python, independently of the oracle's AND-count + derivation route
(src/helper.cu:480-548, :634-662).
"""
import json
import math
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")


def _cases():
    with open(GOLDEN) as f:
        return json.load(f)["cases"]


CASES = _cases()


def _planes(oracle, c):
    return (oracle.pack(np.array(c["cases"])), oracle.pack(np.array(c["controls"])), c["num_cases"],
            c["num_controls"])


def test_pack_roundtrip(oracle):
    rng = np.random.default_rng(1)
    for n in (1, 31, 32, 33, 1023, 1024, 1025):
        g = rng.integers(0, 3, size=(5, n))
        p = oracle.pack(g)
        assert p.shape == (5, 2, oracle.class_words(n))
        assert np.array_equal(oracle.unpack(p, n), g)
        assert oracle.validate(p, n)


def test_msb_first_bit_order(oracle):
    # Sample 0 is the most significant bit of word 0 (src/helper.cu:72-73 masks the low bits).
    g = np.full((1, 33), 2)
    g[0, 0] = 0
    g[0, 32] = 1
    p = oracle.pack(g)
    assert p[0, 0, 0] == 0x80000000 and p[0, 1, 1] == 0x80000000


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
def test_tables_match_direct_count(oracle, c):
    cases, controls, nc, nn = _planes(oracle, c)
    for t in c["tables"]:
        if c["order"] == 2:
            cs, cn = oracle.table2(cases, controls, nc, nn, *t["snps"])
        else:
            cs, cn = oracle.table3(cases, controls, nc, nn, *t["snps"])
        assert cs.tolist() == t["cases"], t["snps"]
        assert cn.tolist() == t["controls"], t["snps"]
        assert cs.sum() == nc and cn.sum() == nn
        assert (cs >= 0).all() and (cn >= 0).all()


@pytest.mark.parametrize("c", CASES, ids=[c["name"] for c in CASES])
@pytest.mark.parametrize("score", ["k2", "mi"])
def test_search_best_matches_fixture(oracle, c, score):
    cases, controls, nc, nn = _planes(oracle, c)
    r = oracle.search(cases, controls, nc, nn, order=c["order"], score=score, top_k=64, threads=4)
    M = len(c["cases"])
    assert r["sets"] == math.comb(M, c["order"])
    want = c["best_" + score]
    assert list(r["best"]) == want["snps"]
    assert r["best_fp64"] == pytest.approx(want["score"], rel=1e-12, abs=1e-12)
    # FP64 scores of the fixture's top sets, recomputed by the oracle.
    by_set = {tuple(s): v for s, v in zip(r["top"], r["top_fp64"])}
    for e in c["top_" + score][:5]:
        if tuple(e["snps"]) in by_set:
            assert by_set[tuple(e["snps"])] == pytest.approx(e["score"], rel=1e-12, abs=1e-12)


@pytest.mark.parametrize("c", CASES[:4], ids=[c["name"] for c in CASES[:4]])
def test_top_list_is_sorted_and_complete(oracle, c):
    cases, controls, nc, nn = _planes(oracle, c)
    M = len(c["cases"])
    total = math.comb(M, c["order"])
    r = oracle.search(cases, controls, nc, nn, order=c["order"], score="k2", top_k=total + 5, threads=3)
    assert len(r["top"]) == total
    f = r["top_fp32"]
    assert all(f[i] <= f[i + 1] for i in range(len(f) - 1))
    assert len(set(r["top"])) == total


def test_planted_triplet_found(oracle):
    c = next(x for x in CASES if x["name"].startswith("planted"))
    cases, controls, nc, nn = _planes(oracle, c)
    for score in ("k2", "mi"):
        r = oracle.search(cases, controls, nc, nn, order=3, score=score, top_k=8)
        assert tuple(r["best"]) == (3, 7, 10)


def test_thread_count_does_not_change_answer(oracle):
    c = CASES[-1]
    cases, controls, nc, nn = _planes(oracle, c)
    a = oracle.search(cases, controls, nc, nn, order=2, score="k2", top_k=50, threads=1)
    b = oracle.search(cases, controls, nc, nn, order=2, score="k2", top_k=50, threads=7)
    assert a["top"] == b["top"] and a["best"] == b["best"]
    assert np.array_equal(a["top_fp32"], b["top_fp32"])


def test_slab_partitions_the_search(oracle):
    c = next(x for x in CASES if x["name"] == "tiny_triplets")
    cases, controls, nc, nn = _planes(oracle, c)
    M = len(c["cases"])
    full = oracle.search(cases, controls, nc, nn, order=3, score="k2", top_k=100)
    parts = [oracle.search(cases, controls, nc, nn, order=3, score="k2", top_k=100, first_begin=a, first_end=a + 1)
             for a in range(M - 2)]
    assert sum(p["sets"] for p in parts) == full["sets"]
    merged = sorted(((float(v), s) for p in parts for s, v in zip(p["top"], p["top_fp64"])))
    assert merged[0][1] == tuple(full["best"])


def test_validate_rejects_bad_planes(oracle):
    g = np.random.default_rng(3).integers(0, 3, size=(4, 40))
    p = oracle.pack(g)
    assert oracle.validate(p, 40)
    bad = p.copy()
    bad[1, 0, 1] |= 1  # sample 63: beyond n = 40 -> padding bit
    assert not oracle.validate(bad, 40)
    bad = p.copy()
    bad[2, 0, 0] |= p[2, 1, 0] | 0x80000000
    bad[2, 1, 0] |= 0x80000000  # sample 0 in both planes
    assert not oracle.validate(bad, 40)


def test_label_split_matches_repacked_classes(oracle):
    rng = np.random.default_rng(7)
    n = 77
    g = rng.integers(0, 3, size=(6, n))
    lab = rng.random(n) < 0.4
    label = oracle.pack(np.where(lab, 0, 2)[None, :])[0, 0]
    cases, controls, nc, nn = oracle.split_by_label(oracle.pack(g), n, label)
    assert nc == lab.sum() and nn == n - lab.sum()
    assert np.array_equal(cases, oracle.pack(g[:, lab]))
    assert np.array_equal(controls, oracle.pack(g[:, ~lab]))


def test_fp32_error_is_small(oracle):
    c = next(x for x in CASES if x["name"].startswith("edge_triplets_1025"))
    cases, controls, nc, nn = _planes(oracle, c)
    r = oracle.search(cases, controls, nc, nn, order=3, score="k2", top_k=35)
    rel = np.abs(r["top_fp32"].astype(np.float64) - r["top_fp64"]) / np.abs(r["top_fp64"])
    assert rel.max() < 1e-5


@pytest.mark.parametrize("score", ["k2", "mi"])
def test_fp32_error_with_large_counts(oracle, score):
    """Cells holding thousands of samples (table values near 1e5 for K2): the
    FP32 ranking score stays within 1e-5 of the exact FP64 score and the
    reported optimum is the FP64 optimum of the candidate list."""
    rng = np.random.default_rng(11)
    M, nc, nn = 10, 9000, 11000
    g = rng.integers(0, 3, size=(M, nc + nn)).astype(np.int8)
    g[:, : (nc + nn) // 2] = 0  # large cells: many counts well above 8192
    cases, controls = oracle.pack(g[:, :nc]), oracle.pack(g[:, nc:])
    r = oracle.search(cases, controls, nc, nn, order=2, score=score, top_k=math.comb(M, 2))
    rel = np.abs(r["top_fp32"].astype(np.float64) - r["top_fp64"]) / np.abs(r["top_fp64"])
    assert rel.max() < 1e-5
    best = min(range(len(r["top"])), key=lambda i: (r["top_fp64"][i] * (1 if score == "k2" else -1), r["top"][i]))
    assert tuple(r["best"]) == tuple(r["top"][best])


def test_tables_equal_direct_counts_on_random_data(oracle):
    """The oracle's 9- and 27-cell tables against numpy histograms of the
    genotype codes, and the cell-sum invariants: a triplet table summed over
    Z is the (X, Y) pair table, summed over Y and Z it is X's marginal."""
    rng = np.random.default_rng(23)
    M, nc, nn = 12, 301, 277
    g_cases = rng.integers(0, 3, size=(M, nc))
    g_controls = rng.integers(0, 3, size=(M, nn))
    cases, controls = oracle.pack(g_cases), oracle.pack(g_controls)
    m_cases = oracle.marginals(cases, nc)
    for _ in range(10):
        x, y, z = sorted(rng.choice(M, size=3, replace=False).tolist())
        cs3, cn3 = oracle.table3(cases, controls, nc, nn, x, y, z)
        for got, g in ((cs3, g_cases), (cn3, g_controls)):
            want = np.bincount(9 * g[x] + 3 * g[y] + g[z], minlength=27)
            assert got.tolist() == want.tolist()
        cs2, cn2 = oracle.table2(cases, controls, nc, nn, x, y)
        assert cs2.tolist() == np.bincount(3 * g_cases[x] + g_cases[y], minlength=9).tolist()
        assert cn2.tolist() == np.bincount(3 * g_controls[x] + g_controls[y], minlength=9).tolist()
        assert cs3.reshape(9, 3).sum(axis=1).tolist() == cs2.tolist()
        assert cn3.reshape(9, 3).sum(axis=1).tolist() == cn2.tolist()
        assert cs3.reshape(3, 9).sum(axis=1).tolist() == m_cases[:, x].tolist()


def _round_f32(x):
    """Exact rational x rounded to the nearest float32 (ties to even)."""
    from fractions import Fraction

    f = np.float32(float(x))
    best = None
    for c in (np.nextafter(f, np.float32(-np.inf)), f, np.nextafter(f, np.float32(np.inf))):
        d = abs(Fraction(float(c)) - x)
        key = (d, int(np.array([c], dtype=np.float32).view(np.uint32)[0]) & 1)
        if best is None or key < best[0]:
            best = (key, c)
    return np.float32(best[1])


def test_mi_fp32_score_follows_the_references_evaluation_order(oracle):
    """The oracle's FP32 MI score is the reference's device arithmetic
    (include/scoring.hpp:9-16, :18-51): per cell p = n * (1/N) in float and
    fused multiply-adds into the two entropies, and H(Y) as the device
    evaluates scoring.hpp:29-30 (float p, a double product rounded to float,
    then a double multiply-add rounded to float).  Emulated here exactly with
    rationals for the best pair of a dataset whose class sizes (2990, 4990)
    round H(Y) differently from a double evaluation."""
    from fractions import Fraction as F

    nc, nn = 2990, 4990
    N = nc + nn
    inv = np.float32(1.0 / N)
    t32 = lambda v: np.float32(0.0) if v == 0 else np.float32(math.log2(float(v) * float(inv)))
    p1 = np.float32(np.float32(nc) * inv)
    hy = np.float32(-(float(p1) * float(t32(nc))))
    p2 = np.float32(np.float32(nn) * inv)
    hy = np.float32(float(F(float(hy)) - F(float(p2)) * F(float(t32(nn)))))
    hy_double = np.float32(-(nc / N * math.log2(nc / N)) - (nn / N * math.log2(nn / N)))
    assert hy != hy_double  # the case discriminates between the two orders

    cases, controls = oracle.generate(11, 40, nc, nn)
    o = oracle.search(cases, controls, nc, nn, order=2, score="mi", top_k=4)
    a, b = o["top"][0]
    cs, cn = oracle.table2(cases, controls, nc, nn, a, b)

    def fmaf(x, y, z):
        return _round_f32(F(float(x)) * F(float(y)) + F(float(z)))

    ha = np.float32(0.0)
    hx = np.float32(0.0)
    for s_, n_ in zip(cs.tolist(), cn.tolist()):
        pc = np.float32(np.float32(s_) * inv)
        ha = fmaf(-pc, t32(s_), ha)
        pn = np.float32(np.float32(n_) * inv)
        ha = fmaf(-pn, t32(n_), ha)
        hx = fmaf(-np.float32(pc + pn), t32(s_ + n_), hx)
    score = np.float32(np.float32(hx + hy) - ha)
    assert np.array([score], dtype=np.float32).view(np.uint32)[0] == o["top_fp32"][:1].view(np.uint32)[0]
