"""The entry point that allocates no device memory, against the ordinary one.

episdet_search_pairs_noalloc exists for callers that cannot let the library
allocate: a process whose memory pool already owns the GPU's memory, or one
that cannot absorb the device-wide synchronisation of cudaFree.  It keeps all
its intermediate buffers in one fixed 8 MiB device array.  This file is named
to be collected last, so that a run that stops at the first failure has run
every other test before it; it also passes on its own in a fresh process
(the first call sets the array up).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_search_twice(episdet):
    import torch

    M, nc, nn = 300, 2100, 1900
    cases, controls = episdet.generate(0xA110C, M, nc, nn)
    dc = torch.from_numpy(cases.view(np.int32)).cuda()
    dn = torch.from_numpy(controls.view(np.int32)).cuda()
    for score in ("k2", "mi"):
        ref = episdet.search(cases, controls, nc, nn, order=2, score=score, top_k=256)
        for _ in range(2):  # the array keeps the previous call's contents
            r = episdet.search_pairs_noalloc(dc, dn, nc, nn, num_snps=M, score=score, top_k=256)
            assert r.snps == ref.snps and r.score == ref.score
            assert np.array_equal(r.top_snps, ref.top_snps)
            assert np.array_equal(r.top_fp32.view(np.uint32), ref.top_fp32.view(np.uint32))
            assert np.array_equal(r.top_fp64, ref.top_fp64)
            assert r.sets_evaluated == ref.sets_evaluated


@pytest.mark.parametrize("M,nc,nn,k,fb,fe", [(300, 2100, 1900, 128, 37, 100), (4096, 60000, 71072, 1024, 0, 0),
                                              (1000, 1, 131071, 1024, 990, 999)],
                         ids=["slab", "at-every-limit", "one-case"])
def test_noalloc_slabs_and_limits(episdet, M, nc, nn, k, fb, fe):
    """A first-SNP slab, and a search at the documented limits (4096 SNPs,
    131,072 samples, top_k 1024), which fill the fixed regions of the array to
    capacity, against the ordinary entry point."""
    import torch

    cases, controls = episdet.generate(0xA110C + M, M, nc, nn)
    dc = torch.from_numpy(cases.view(np.int32)).cuda()
    dn = torch.from_numpy(controls.view(np.int32)).cuda()
    ref = episdet.search(cases, controls, nc, nn, order=2, top_k=k, first_begin=fb, first_end=fe)
    for _ in range(2):
        r = episdet.search_pairs_noalloc(dc, dn, nc, nn, num_snps=M, top_k=k, first_begin=fb, first_end=fe)
        assert r.snps == ref.snps and r.score == ref.score
        assert np.array_equal(r.top_snps, ref.top_snps)
        assert np.array_equal(r.top_fp32.view(np.uint32), ref.top_fp32.view(np.uint32))
        assert np.array_equal(r.top_fp64, ref.top_fp64)
        assert r.sets_evaluated == ref.sets_evaluated


def test_noalloc_rejects_oversize_and_host_inputs(episdet):
    import torch

    cases, controls = episdet.generate(7, 64, 500, 500)
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.search_pairs_noalloc(cases, controls, 500, 500, num_snps=64)
    assert e.value.name == "EPISDET_ERR_INVALID_ARGUMENT"
    dc = torch.from_numpy(cases.view(np.int32)).cuda()
    dn = torch.from_numpy(controls.view(np.int32)).cuda()
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.search_pairs_noalloc(dc, dn, 500, 500, num_snps=64, top_k=1200)
    assert "no-alloc limits" in str(e.value)
    big = torch.zeros((4097 * 2 * 32,), dtype=torch.int32, device="cuda")
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.search_pairs_noalloc(big, big, 1000, 1000, num_snps=4097)
    assert "no-alloc limits" in str(e.value)
