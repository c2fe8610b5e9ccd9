"""3-way searches with the pair table held in blocks of second SNPs Y.

When the whole [M][M] pair table (32 x M^2 bytes) does not fit beside the
tensor engine's other buffers -- or when options.pair_block_snps asks -- the
triplet search holds the Y-Z pair rows of one block of second SNPs at a time
plus the pair rows of the current first SNPs, and sweeps its first SNPs once
per block.  The results must not change: the same best set, FP32 candidate
list and FP64 re-scores as the oracle, for every block size.
"""
import numpy as np
import pytest

from test_parity_gpu import assert_same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def data1000(episdet):
    return episdet.generate(0xB10C, 1000, 3000, 2800, planted=[(111, 500, 901)])


@pytest.mark.parametrize("score", ["k2", "mi"])
@pytest.mark.parametrize("slab", [(0, 0), (250, 260), (600, 700)], ids=["all", "x250-259", "x600-699"])
def test_y_blocks_give_the_whole_table_answer(episdet, oracle, data1000, score, slab):
    cases, controls = data1000
    fb, fe = slab
    k = 512
    o = oracle.search(cases, controls, 3000, 2800, order=3, score=score, top_k=k, first_begin=fb, first_end=fe)
    # 128 (the smallest block), 384 (a block edge inside a band of tiles) and a
    # block of the whole range (the whole table); K2 also with the scoring filter.
    for blk in (128, 384, 1000):
        for flags in ((0, episdet.FLAG_FILTER_ON) if score == "k2" else (0,)):
            r = episdet.search(cases, controls, 3000, 2800, order=3, score=score, top_k=k, engine="tensor",
                               first_begin=fb, first_end=fe, flags=flags, pair_block_snps=blk)
            assert_same(r, o, k)
            assert r.sets_evaluated == o["sets"]


def test_pair_table_larger_than_the_gpu_is_blocked(episdet, oracle):
    """80,000 SNPs: the whole pair table would take 32 x 80000^2 = 205 GB, more
    than a B200 holds; the engine picks a block size itself, and the first
    SNP's slab (3.2e9 triplets) matches the oracle."""
    import torch

    M, nc, nn = 80000, 1024, 1000
    assert 32 * M * M > torch.cuda.get_device_properties(0).total_memory
    cases, controls = episdet.generate(0xB1C, M, nc, nn, planted=[(0, 41234, 79000)])
    k = 256
    try:
        r = episdet.search(cases, controls, nc, nn, order=3, score="k2", top_k=k, engine="tensor", first_begin=0,
                           first_end=1)
    finally:
        episdet.release_workspace(0)  # the block took most of the device; later tests allocate afresh
    o = oracle.search(cases, controls, nc, nn, order=3, score="k2", top_k=k, first_begin=0, first_end=1)
    assert_same(r, o, k)
    assert r.sets_evaluated == o["sets"]
