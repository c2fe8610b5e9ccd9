"""GPU engines against the CPU oracle, through the C-ABI.

Bar: the best set, the FP32 candidate list (sets and FP32 score bits) and the
FP64 re-scores are identical to the oracle's, because every count is exact
and both sides evaluate the same score tables with the same operation order.
"""
import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "known_answers.json")))["cases"]
ENGINES = ["simt", "tensor"]


def assert_same(r, o, k):
    assert tuple(r.snps) == tuple(o["best"])
    assert r.score == o["best_fp64"]
    n = min(k, len(o["top"]))
    assert [tuple(s) for s in r.top_snps[:n]] == [tuple(s) for s in o["top"][:n]]
    assert np.array_equal(r.top_fp32[:n].view(np.uint32), o["top_fp32"][:n].view(np.uint32))
    assert np.array_equal(r.top_fp64[:n], o["top_fp64"][:n])


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("score", ["k2", "mi"])
@pytest.mark.parametrize("c", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_known_answers(episdet, oracle, c, score, engine):
    cases, controls = oracle.pack(np.array(c["cases"])), oracle.pack(np.array(c["controls"]))
    nc, nn = c["num_cases"], c["num_controls"]
    k = 64
    r = episdet.search(cases, controls, nc, nn, order=c["order"], score=score, top_k=k, engine=engine)
    o = oracle.search(cases, controls, nc, nn, order=c["order"], score=score, top_k=k)
    assert_same(r, o, k)
    assert list(r.snps) == c["best_" + score]["snps"]


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("order,M,nc,nn", [(2, 200, 3000, 2500), (3, 60, 700, 1300), (2, 70, 1, 4097),
                                           (3, 40, 31, 1025), (3, 45, 4097, 33), (2, 129, 1023, 1024),
                                           (2, 100, 9000, 11000), (3, 40, 12000, 9000)])
@pytest.mark.parametrize("score", ["k2", "mi"])
def test_random_datasets(episdet, oracle, order, M, nc, nn, score, engine):
    cases, controls = episdet.generate(100 + M + nc, M, nc, nn)
    k = 256
    r = episdet.search(cases, controls, nc, nn, order=order, score=score, top_k=k, engine=engine)
    o = oracle.search(cases, controls, nc, nn, order=order, score=score, top_k=k)
    assert_same(r, o, k)
    assert r.sets_evaluated == o["sets"]
    if order == 3 and score == "k2" and engine == "tensor":
        # The kernel with the K2 scoring filter, forced on at this small size.
        r = episdet.search(cases, controls, nc, nn, order=3, score="k2", top_k=k, engine="tensor",
                           flags=episdet.FLAG_FILTER_ON)
        assert_same(r, o, k)


@pytest.mark.parametrize("engine", ENGINES)
def test_config1_pairs_k2(episdet, oracle, engine):
    """512 SNPs x 4,096 samples (2,048 + 2,048), independent labels, 2-way K2."""
    cases, controls = episdet.generate(0xE916, 512, 2048, 2048, maf=(0.05, 0.5))
    r = episdet.search(cases, controls, 2048, 2048, order=2, score="k2", top_k=1024, engine=engine)
    o = oracle.search(cases, controls, 2048, 2048, order=2, score="k2", top_k=1024)
    assert_same(r, o, 1024)


@pytest.mark.parametrize("score", ["k2", "mi"])
def test_large_classes_triplets(episdet, oracle, score):
    """Classes of >= 32,768 samples: the triplet launches use the kernel that
    copies count segment 0 out of TMEM early; first SNPs whose segment 0 holds
    fewer than 8,192 samples (low MAF) run it without the copy, so both paths
    meet in one launch."""
    cases, controls = episdet.generate(0xE91A, 44, 70000, 66000, maf=(0.02, 0.5))
    k = 256
    o = oracle.search(cases, controls, 70000, 66000, order=3, score=score, top_k=k)
    for flags in ((episdet.FLAG_FILTER_OFF, episdet.FLAG_FILTER_ON) if score == "k2" else (0,)):
        r = episdet.search(cases, controls, 70000, 66000, order=3, score=score, top_k=k, engine="tensor",
                           flags=flags)
        assert_same(r, o, k)
        assert r.sets_evaluated == o["sets"]


@pytest.mark.parametrize("engine", ENGINES)
def test_planted_triplet(episdet, oracle, engine):
    cases, controls = episdet.generate(0xE917, 96, 8192, 8192, planted=[(5, 40, 77)], base_risk=0.5, effect=0.25)
    r = episdet.search(cases, controls, 8192, 8192, order=3, score="k2", top_k=512, engine=engine)
    assert tuple(r.snps) == (5, 40, 77)
    o = oracle.search(cases, controls, 8192, 8192, order=3, score="k2", top_k=512)
    assert_same(r, o, 512)


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("order", [2, 3])
def test_slab(episdet, oracle, order, engine):
    cases, controls = episdet.generate(77, 90, 1500, 1600)
    r = episdet.search(cases, controls, 1500, 1600, order=order, top_k=128, first_begin=17, first_end=41,
                       engine=engine)
    o = oracle.search(cases, controls, 1500, 1600, order=order, top_k=128, first_begin=17, first_end=41)
    assert_same(r, o, 128)


def test_engines_agree(episdet):
    cases, controls = episdet.generate(5, 150, 2500, 2600)
    a = episdet.search(cases, controls, 2500, 2600, order=3, top_k=1024, engine="simt")
    b = episdet.search(cases, controls, 2500, 2600, order=3, top_k=1024, engine="tensor")
    assert a.snps == b.snps and a.score == b.score
    assert np.array_equal(a.top_snps, b.top_snps)
    assert np.array_equal(a.top_fp32.view(np.uint32), b.top_fp32.view(np.uint32))


def test_device_resident_inputs(episdet):
    import torch

    cases, controls = episdet.generate(8, 64, 3000, 2000)
    h = episdet.search(cases, controls, 3000, 2000, order=3, top_k=64)
    dc = torch.from_numpy(cases.view(np.int32)).cuda()
    dn = torch.from_numpy(controls.view(np.int32)).cuda()
    d = episdet.search(dc, dn, 3000, 2000, num_snps=64, order=3, top_k=64)
    assert h.snps == d.snps and h.score == d.score and np.array_equal(h.top_snps, d.top_snps)


def test_repeat_is_deterministic(episdet):
    cases, controls = episdet.generate(9, 120, 2000, 2000)
    a = episdet.search(cases, controls, 2000, 2000, order=2, score="mi", top_k=300)
    b = episdet.search(cases, controls, 2000, 2000, order=2, score="mi", top_k=300)
    assert np.array_equal(a.top_snps, b.top_snps) and np.array_equal(a.top_fp64, b.top_fp64)


def test_invalid_planes_rejected(episdet):
    cases, controls = episdet.generate(3, 20, 100, 100)
    bad = cases.copy()
    bad[4, 1, 3] |= 1  # a padding bit (sample 127 >= 100)
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.search(bad, controls, 100, 100, order=2)
    assert e.value.name == "EPISDET_ERR_INVALID_INPUT"
    bad = controls.copy()
    bad[7, 0, 0] |= 0x80000000
    bad[7, 1, 0] |= 0x80000000  # sample 0 in both planes
    with pytest.raises(episdet.EpisdetError):
        episdet.search(cases, bad, 100, 100, order=3)
    # the context is still usable afterwards
    r = episdet.search(cases, controls, 100, 100, order=2, top_k=8)
    assert len(r.snps) == 2


@pytest.mark.parametrize("score", ["k2", "mi"])
@pytest.mark.parametrize("n,M,ncase,nl", [(3000, 80, 1400, 4), (20011, 300, 6100, 5)])
def test_permutations_match_split_searches(episdet, oracle, n, M, ncase, nl, score):
    """Label mode (the label as a third AND operand: only the cases' cells are
    counted per label, the controls' derived from the label-free totals), a
    plain two-class search per label, and the integer-pipe engine, each against
    the oracle on the split of every label."""
    planes = episdet.generate_cohort(21 + n, M, n)
    labels = episdet.generate_labels(22 + n, n, ncase, nl)
    want = []
    for lab in labels:
        cases, controls, nc, nn = oracle.split_by_label(planes, n, lab)
        want.append(oracle.search(cases, controls, nc, nn, order=2, score=score, top_k=64))
    for engine, flags in (("auto", 0), ("auto", episdet.FLAG_PERM_SPLIT), ("simt", 0)):
        res = episdet.search_perm(planes, n, labels, order=2, score=score, top_k=64, engine=engine, flags=flags)
        for r, o in zip(res, want):
            assert_same(r, o, 64)


def test_perm_pvalues_of_a_permutation_search(episdet):
    n, M, nl = 3000, 50, 24
    planes = episdet.generate_cohort(31, M, n)
    labels = episdet.generate_labels(32, n, 1400, nl)
    res = episdet.search_perm(planes, n, labels, order=2, score="k2", top_k=16)
    pv = episdet.perm_pvalues(res, "k2")
    null = np.array([r.score for r in res[1:]])
    assert pv.shape == (16,)
    for s, p in zip(res[0].top_fp64, pv):
        assert p == (1 + (null <= s).sum()) / nl
    # The C entry point over the same scores.
    rs = (episdet.Result * nl)()
    top = np.ascontiguousarray(res[0].top_fp64)
    rs[0].score, rs[0].top_count = res[0].score, len(top)
    rs[0].top_fp64 = top.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    for i in range(1, nl):
        rs[i].score = res[i].score
    out = np.zeros(16)
    cnt = ctypes.c_int32()
    assert episdet.lib().episdet_perm_pvalues(rs, nl, episdet.SCORE_K2, out.ctypes.data_as(
        ctypes.POINTER(ctypes.c_double)), 16, ctypes.byref(cnt)) == 0
    assert cnt.value == 16 and np.array_equal(out, pv)


@pytest.mark.parametrize("order,M,nc,nn,device", [(3, 60, 700, 1300, False), (2, 300, 900, 1100, True),
                                                  (3, 44, 70000, 66000, False)])
def test_resumable_equals_one_search(episdet, tmp_path, order, M, nc, nn, device):
    """A search interrupted after every two slabs and resumed from its
    checkpoint gives the uninterrupted search's answer bit for bit."""
    import torch
    cases, controls = episdet.generate(0xE91B + M, M, nc, nn)
    k = 128
    plain = episdet.search(cases, controls, nc, nn, order=order, top_k=k, engine="tensor")
    if device:
        cases, controls = torch.from_numpy(cases.view(np.int32)).cuda(), torch.from_numpy(controls.view(np.int32)).cuda()
    path = str(tmp_path / "run.ckpt")
    calls = 0
    while True:
        r, done, nxt = episdet.search_resumable(cases, controls, nc, nn, path, num_snps=M, order=order, top_k=k,
                                                engine="tensor", num_slabs=7, max_slabs=2)
        calls += 1
        if done:
            break
        assert 0 < nxt < M and calls < 8
    assert calls >= 2
    assert r.snps == plain.snps and r.score == plain.score and r.score_fp32 == plain.score_fp32
    assert r.packed_indices == plain.packed_indices and r.sets_evaluated == plain.sets_evaluated
    assert np.array_equal(r.top_snps, plain.top_snps)
    assert np.array_equal(r.top_fp32.view(np.uint32), plain.top_fp32.view(np.uint32))
    assert np.array_equal(r.top_fp64, plain.top_fp64)
    # A finished checkpoint answers again without searching.
    again, done, _ = episdet.search_resumable(cases, controls, nc, nn, path, num_snps=M, order=order, top_k=k,
                                              engine="tensor", num_slabs=7)
    assert done and again.snps == r.snps and again.kernel_launches == r.kernel_launches


def test_batched_equals_plain(episdet):
    rng = np.random.default_rng(4)
    cohorts, opts = [], []
    for i in range(6):
        M = int(rng.integers(30, 90))
        nc, nn = int(rng.integers(500, 3000)), int(rng.integers(500, 3000))
        c, k = episdet.generate(1000 + i, M, nc, nn)
        cohorts.append((c, k, nc, nn))
        opts.append({"order": 2 + i % 2, "score": "k2", "top_k": 32})
    batched = episdet.search_batched(cohorts, opts)
    for (c, k, nc, nn), opt, b in zip(cohorts, opts, batched):
        p = episdet.search(c, k, nc, nn, **opt)
        assert p.snps == b.snps and p.score == b.score
        assert np.array_equal(p.top_snps, b.top_snps)


@pytest.mark.parametrize("n", [1, 33, 1024, 1025, 5000])
def test_binarize_matches_packing(episdet, oracle, n):
    """Genotype matrix -> planes on the GPU equals packing each class's columns."""
    rng = np.random.default_rng(n)
    M = 37
    g = rng.integers(0, 3, size=(M, n + 1)).astype(np.uint8)
    flags = rng.random(n + 1) < 0.4
    flags[0], flags[-1] = True, False  # both classes non-empty
    cases, controls, nc, nn = episdet.binarize(g, flags)
    assert (nc, nn) == (int(flags.sum()), int((~flags).sum()))
    assert np.array_equal(cases, oracle.pack(g[:, flags]))
    assert np.array_equal(controls, oracle.pack(g[:, ~flags]))


def test_binarize_device_and_search(episdet, oracle):
    import torch

    rng = np.random.default_rng(5)
    M, n = 48, 3000
    g = rng.integers(0, 3, size=(M, n)).astype(np.uint8)
    flags = rng.random(n) < 0.5
    dc, dn, nc, nn = episdet.binarize(torch.from_numpy(g).cuda(), torch.from_numpy(flags).cuda())
    hc, hn, _, _ = episdet.binarize(g, flags)
    assert np.array_equal(dc.cpu().numpy().view(np.uint32), hc.reshape(-1))
    r = episdet.search(dc, dn, nc, nn, num_snps=M, order=2, top_k=32)
    o = oracle.search(hc, hn, nc, nn, order=2, top_k=32)
    assert tuple(r.snps) == tuple(o["best"])


def test_binarize_rejects_bad_values(episdet):
    g = np.zeros((4, 100), dtype=np.uint8)
    g[2, 50] = 3
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.binarize(g, np.arange(100) % 2 == 0)
    assert e.value.name == "EPISDET_ERR_INVALID_INPUT"
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.binarize(np.zeros((4, 100), dtype=np.uint8), np.zeros(100, dtype=bool))
    assert e.value.name == "EPISDET_ERR_INVALID_ARGUMENT"


def test_batched_concurrent_lanes_equal_plain(episdet):
    """More cohorts than worker lanes, uneven sizes, both orders and scores:
    every result equals the plain call bit for bit."""
    rng = np.random.default_rng(12)
    cohorts, opts = [], []
    for i in range(12):
        M = int(rng.integers(20, 140))
        nc, nn = int(rng.integers(64, 6000)), int(rng.integers(64, 6000))
        c, k = episdet.generate(2000 + i, M, nc, nn)
        cohorts.append((c, k, nc, nn))
        opts.append({"order": 2 + (i % 3 == 0), "score": "mi" if i % 4 == 1 else "k2", "top_k": 48})
    batched = episdet.search_batched(cohorts, opts)
    for (c, k, nc, nn), opt, b in zip(cohorts, opts, batched):
        p = episdet.search(c, k, nc, nn, **opt)
        assert p.snps == b.snps and p.score == b.score
        assert np.array_equal(p.top_snps, b.top_snps)
        assert np.array_equal(p.top_fp32.view(np.uint32), b.top_fp32.view(np.uint32))
        assert np.array_equal(p.top_fp64, b.top_fp64)


def test_batched_reports_the_failing_cohort(episdet):
    cohorts = []
    for i in range(6):
        c, k = episdet.generate(3000 + i, 30, 200, 200)
        cohorts.append((c, k, 200, 200))
    bad = cohorts[3][0].copy()
    bad[2, 1, 7] |= 1  # a padding bit: sample 255 >= 200
    cohorts[3] = (bad, cohorts[3][1], 200, 200)
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.search_batched(cohorts, [{"order": 2, "top_k": 16}] * 6)
    assert e.value.name == "EPISDET_ERR_INVALID_INPUT"
    assert "cohort 3" in str(e.value)
    r = episdet.search(*cohorts[0], order=2, top_k=16)  # the library stays usable
    assert len(r.snps) == 2


@pytest.mark.parametrize("variant,order,score", [("pairs.k2", 2, "k2"), ("triplets.mi", 3, "mi"),
                                                 ("triplets.k2", 3, "k2"), ("pairs.mi", 2, "mi")])
def test_cli_output(episdet, oracle, tmp_path, variant, order, score):
    cases, controls = episdet.generate(31, 70, 1800, 1300)
    path = str(tmp_path / "data.txt")
    episdet.write_dataset(path, cases, controls, 1800, 1300)
    exe = os.path.join(ROOT, "tensor-episdet_b200", "bin", f"tensor-episdet.{variant}.bin")
    p = subprocess.run([exe, path], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    lines = p.stdout.splitlines()
    assert lines[0] == "Num. SNPs: 70" and lines[1] == "Num. Blocks of SNPs: 1"
    assert lines[2] == "Num. Cases: 1800" and lines[3] == "Num. Controls: 1300"
    assert "Outer loop iteration 0 out of 1" in lines
    best = [l for l in lines if "SCORE\t->\t{" in l][0]
    o = oracle.search(cases, controls, 1800, 1300, order=order, score=score, top_k=16)
    want = "{" + ", ".join(str(v) for v in o["best"]) + "}: " + f"{np.float32(o['best_fp64']):.6f}"
    assert best.endswith(want), (best, want)
    assert "Num. of rounds processed: %d" % (1 if order == 2 else 70) in lines  # BLOCK_SIZE 256 rounds
    assert any(l.startswith("Unique sets of SNPs evaluated (k=%d): " % order) for l in lines)


@pytest.mark.parametrize("variant", ["triplets.k2", "pairs.mi"])
def test_cli_checkpoint(episdet, tmp_path, variant):
    """--checkpoint runs the search in slabs through the resumable entry
    point and prints the plain run's best-set and round lines."""
    cases, controls = episdet.generate(33, 70, 1800, 1300)
    path = str(tmp_path / "data.txt")
    episdet.write_dataset(path, cases, controls, 1800, 1300)
    exe = os.path.join(ROOT, "tensor-episdet_b200", "bin", f"tensor-episdet.{variant}.bin")
    plain = subprocess.run([exe, path], capture_output=True, text=True, timeout=300)
    ck = str(tmp_path / "run.ckpt")
    slabs = subprocess.run([exe, path, "--checkpoint", ck, "--slabs", "5"], capture_output=True, text=True,
                           timeout=300)
    assert plain.returncode == 0 and slabs.returncode == 0, slabs.stderr
    pick = lambda out: [l for l in out.splitlines() if "SCORE\t->\t{" in l or l.startswith("Num. of rounds")]
    assert pick(slabs.stdout) == pick(plain.stdout) and len(pick(plain.stdout)) == 2
    assert os.path.getsize(ck) > 0


def test_autotune_picks_and_caches_an_instance(tmp_path):
    """EPISDET_FLAG_AUTOTUNE: the first search of a shape times both triplet
    instances, caches the faster one (one line in EPISDET_TUNE_CACHE) and gives
    the same answer as a search without the flag; the next search of the same
    shape reuses the cached choice."""
    cache = tmp_path / "tune.txt"
    code = f"""
import sys
sys.path.insert(0, {os.path.join(ROOT, "tensor-episdet_b200")!r})
import numpy as np, episdet
cases, controls = episdet.generate(0xE91C, 40, 40000, 36000)
plain = episdet.search(cases, controls, 40000, 36000, order=3, top_k=128, engine="tensor")
assert episdet.tuned_stage(3, "k2", 40000, 36000) == -1
tuned = episdet.search(cases, controls, 40000, 36000, order=3, top_k=128, engine="tensor", flags=episdet.FLAG_AUTOTUNE)
choice = episdet.tuned_stage(3, "k2", 40000, 36000)
assert choice in (0, 1), choice
again = episdet.search(cases, controls, 40000, 36000, order=3, top_k=128, engine="tensor", flags=episdet.FLAG_AUTOTUNE)
for r in (tuned, again):
    assert r.snps == plain.snps and r.score == plain.score
    assert np.array_equal(r.top_snps, plain.top_snps)
    assert np.array_equal(r.top_fp32.view(np.uint32), plain.top_fp32.view(np.uint32))
print(choice)
"""
    env = dict(os.environ, EPISDET_TUNE_CACHE=str(cache))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=600)
    assert p.returncode == 0, p.stderr
    choice = int(p.stdout.strip().splitlines()[-1])
    assert cache.read_text().splitlines() == [f"3 0 15 {choice}"]
