"""Failure detection on the GPU, without a GPU fault.

Every wait inside the tensor engine's kernels is bounded.  These tests make
the waits run out on purpose -- the scoring warps first wait for a device word
that nothing sets (EPISDET_FLAG_INJECT_STALL) under a short wait limit -- and
check that the call reports EPISDET_ERR_TIMEOUT, that the launches drained
their copies and MMAs and freed their tensor memory (the next search on the
same context is correct), and that an allocation failure injected on the host
is reported as EPISDET_ERR_OUT_OF_MEMORY and leaves the library usable.
"""
import numpy as np
import pytest

from test_parity_gpu import assert_same

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order,M,nc,nn", [(3, 40, 3000, 2500), (3, 12, 33000, 34000), (2, 300, 5000, 4000)],
                         ids=["triplets", "triplets-staged", "pairs"])
def test_stalled_launches_time_out_and_the_device_recovers(episdet, oracle, order, M, nc, nn):
    cases, controls = episdet.generate(0xFA11 + M, M, nc, nn)
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.search(cases, controls, nc, nn, order=order, top_k=64, engine="tensor",
                       flags=episdet.FLAG_INJECT_STALL, wait_limit_ms=100)
    assert e.value.name == "EPISDET_ERR_TIMEOUT"
    for _ in range(2):
        r = episdet.search(cases, controls, nc, nn, order=order, top_k=64, engine="tensor")
        o = oracle.search(cases, controls, nc, nn, order=order, top_k=64)
        assert_same(r, o, 64)


def test_allocation_failure_is_reported_and_the_library_recovers(episdet, oracle):
    M, nc, nn = 50, 2000, 2200
    cases, controls = episdet.generate(0xA10C, M, nc, nn)
    o = oracle.search(cases, controls, nc, nn, order=3, top_k=64)
    for after in (1, 3, 8):
        episdet.release_workspace(0)  # the next search allocates its buffers again
        episdet.test_fail_allocation(after)
        with pytest.raises(episdet.EpisdetError) as e:
            episdet.search(cases, controls, nc, nn, order=3, top_k=64, engine="tensor")
        assert e.value.name == "EPISDET_ERR_OUT_OF_MEMORY"
        r = episdet.search(cases, controls, nc, nn, order=3, top_k=64, engine="tensor")
        assert_same(r, o, 64)
    episdet.test_fail_allocation(0)
