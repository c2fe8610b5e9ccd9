"""Tensor engine against the oracle at the benchmark's own sizes.

The exhaustive searches of the large configurations take hours on the host
cores, so the oracle checks first-SNP slabs of them (every triplet whose
first SNP X lies in the slab, all Y < Z after it) -- the slabs that reach the
parts of the engine only large inputs reach:

* 4096 SNPs x 262,144 samples (3-way K2, planted triplet): X = 0, the
  heaviest first SNP (8.4 M triplets, every tile of the first tile list), and
  X in {126, 127}, which straddles the boundary between the first and second
  per-first-SNP tile lists inside one launch group;
* 8192 SNPs x 65,536 samples (3-way MI, MAF down to 0.01, two planted
  triplets): X = 0 (33.5 M triplets);
* 1024 SNPs x 20,000 samples: X in [250, 260), whose launch groups mix
  members of two tile lists, over lists that cross the band edges of the tile
  order in both directions.

The bar is the one of every parity test: the same best set, the same FP32
candidate list (sets and score bits) and the same FP64 re-scores.
"""
import numpy as np
import pytest

from test_parity_gpu import assert_same

pytestmark = pytest.mark.gpu

CFG2 = dict(seed=0xE917, M=4096, nc=131072, nn=131072, planted=[(137, 2048, 3901)])


@pytest.fixture(scope="module")
def cfg2(episdet):
    c, k = episdet.generate(CFG2["seed"], CFG2["M"], CFG2["nc"], CFG2["nn"], maf=(0.05, 0.5),
                            planted=CFG2["planted"], base_risk=0.5, effect=0.25)
    return c, k


@pytest.mark.parametrize("slab", [(0, 1), (126, 128)], ids=["x0", "x126-127"])
def test_bench_workload_slabs(episdet, oracle, cfg2, slab):
    cases, controls = cfg2
    fb, fe = slab
    k = 1024
    o = oracle.search(cases, controls, CFG2["nc"], CFG2["nn"], order=3, score="k2", top_k=k, first_begin=fb,
                      first_end=fe)
    # Both K2 triplet kernels: exact scoring, and the scoring filter (which a
    # full search of this size runs).
    for flags in (episdet.FLAG_FILTER_OFF, episdet.FLAG_FILTER_ON):
        r = episdet.search(cases, controls, CFG2["nc"], CFG2["nn"], order=3, score="k2", top_k=k, engine="tensor",
                           first_begin=fb, first_end=fe, flags=flags)
        assert_same(r, o, k)
        assert r.sets_evaluated == o["sets"]


def test_mi_workload_slab(episdet, oracle):
    M, nc, nn = 8192, 32768, 32768
    cases, controls = episdet.generate(0xE918, M, nc, nn, maf=(0.01, 0.5),
                                       planted=[(1000, 3000, 5000), (2000, 4000, 6000)])
    k = 1024
    r = episdet.search(cases, controls, nc, nn, order=3, score="mi", top_k=k, engine="tensor", first_begin=0,
                       first_end=1)
    o = oracle.search(cases, controls, nc, nn, order=3, score="mi", top_k=k, first_begin=0, first_end=1)
    assert_same(r, o, k)
    # FP32 epilogue scores against their FP64 re-scores over the candidate list.
    err = np.abs(r.top_fp32.astype(np.float64) - r.top_fp64)
    assert err.max() < 1e-4 and (err / np.abs(r.top_fp64)).max() < 1e-2


@pytest.mark.parametrize("score", ["k2", "mi"])
def test_tile_list_and_band_edges(episdet, oracle, score):
    M, nc, nn = 1024, 10000, 10000
    cases, controls = episdet.generate(0x5CA1E, M, nc, nn)
    k = 1024
    o = oracle.search(cases, controls, nc, nn, order=3, score=score, top_k=k, first_begin=250, first_end=260)
    for flags in ((episdet.FLAG_FILTER_OFF, episdet.FLAG_FILTER_ON) if score == "k2" else (0,)):
        r = episdet.search(cases, controls, nc, nn, order=3, score=score, top_k=k, engine="tensor",
                           first_begin=250, first_end=260, flags=flags)
        assert_same(r, o, k)
        assert r.sets_evaluated == o["sets"]


def test_class_past_fp32_exactness_goes_to_the_integer_engine(episdet, oracle):
    """A class of 2^24 + 1 samples is past what the tensor engine's FP32
    accumulators count exactly; the default engine hands the search to the
    integer-pipe engine, whose counts match the oracle's."""
    M, nc, nn = 8, (1 << 24) + 1, 3000
    cases, controls = episdet.generate(0xB16, M, nc, nn)
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.search(cases, controls, nc, nn, order=3, engine="tensor")
    assert e.value.name == "EPISDET_ERR_UNSUPPORTED"
    for order in (2, 3):
        r = episdet.search(cases, controls, nc, nn, order=order, score="k2", top_k=16)
        o = oracle.search(cases, controls, nc, nn, order=order, score="k2", top_k=16)
        assert_same(r, o, 16)
