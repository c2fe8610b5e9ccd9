"""Python binding of libepisdet.so (the B200 epistasis-search C-ABI).

Mirrors the reference's search entry point, ``EpistasisDetectionSearch``
(hiperbio/tensor-episdet src/search-pairs.cu:9, src/search-triplets.cu:8),
with the same argument meanings, plus keyword-style helpers used by the tests
and the benchmark.  Every call goes through the C-ABI declared in
include/episdet.h; there is no Python or CPU fallback -- if the shared library
is missing or was not built for this GPU, calls raise.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libepisdet.so")

SCORE_K2, SCORE_MI = 0, 1
HOST, DEVICE = 0, 1
ENGINE_AUTO, ENGINE_TENSOR, ENGINE_SIMT = 0, 1, 2
FLAG_PROGRESS, FLAG_NO_VALIDATE, FLAG_TIMING = 0x1, 0x2, 0x4
FLAG_AUTOTUNE = 0x8  # measure the triplet instance per shape and cache the choice
FLAG_INJECT_STALL = 0x10  # testing aid: every tensor launch waits on a word nothing sets and times out
FLAG_FILTER_ON, FLAG_FILTER_OFF = 0x20, 0x40  # force the K2 triplet scoring filter on / off
FLAG_PERM_SPLIT = 0x80  # permutation search: a plain two-class search per label instead of label mode

STATUS = {
    0: "EPISDET_OK",
    1: "EPISDET_ERR_INVALID_ARGUMENT",
    2: "EPISDET_ERR_INVALID_INPUT",
    3: "EPISDET_ERR_NO_DEVICE",
    4: "EPISDET_ERR_CUDA",
    5: "EPISDET_ERR_OUT_OF_MEMORY",
    6: "EPISDET_ERR_TIMEOUT",
    7: "EPISDET_ERR_IO",
    8: "EPISDET_ERR_UNSUPPORTED",
    9: "EPISDET_ERR_INTERNAL",
}

# Every symbol include/episdet.h declares with C linkage.
EXPORTED = [
    "episdet_class_words", "episdet_default_options", "episdet_search", "episdet_search_batched",
    "episdet_search_perm", "episdet_read_dataset", "episdet_free_dataset", "episdet_write_dataset",
    "episdet_generate", "episdet_generate_cohort", "episdet_generate_labels", "episdet_n_choose_k",
    "episdet_status_string", "episdet_last_error", "episdet_abi_version", "episdet_release_workspace",
    "episdet_search_pairs_noalloc", "episdet_binarize", "episdet_perm_pvalues", "episdet_search_resumable",
    "episdet_tuned_stage", "episdet_test_fail_allocation", "episdet_last_launch_profile",
]


class EpisdetError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.name = STATUS.get(status, str(status))


class Dataset(ctypes.Structure):
    _fields_ = [("cases", ctypes.c_void_p), ("controls", ctypes.c_void_p), ("num_snps", ctypes.c_int32),
                ("num_cases", ctypes.c_int32), ("num_controls", ctypes.c_int32), ("memory", ctypes.c_int32)]


class Cohort(ctypes.Structure):
    _fields_ = [("planes", ctypes.c_void_p), ("num_snps", ctypes.c_int32), ("num_samples", ctypes.c_int32),
                ("memory", ctypes.c_int32)]


class Options(ctypes.Structure):
    _fields_ = [("order", ctypes.c_int32), ("score", ctypes.c_int32), ("top_k", ctypes.c_int32),
                ("device", ctypes.c_int32), ("engine", ctypes.c_int32), ("first_begin", ctypes.c_int32),
                ("first_end", ctypes.c_int32), ("flags", ctypes.c_uint32), ("stream", ctypes.c_uint64),
                ("wait_limit_ms", ctypes.c_int32), ("pair_block_snps", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 4)]


class Result(ctypes.Structure):
    _fields_ = [("snps", ctypes.c_uint32 * 3), ("packed_indices", ctypes.c_uint64), ("score", ctypes.c_double),
                ("score_fp32", ctypes.c_float), ("top_count", ctypes.c_int32), ("sets_evaluated", ctypes.c_int64),
                ("rounds", ctypes.c_int64), ("seconds", ctypes.c_double), ("device_ms", ctypes.c_double),
                ("kernel_launches", ctypes.c_uint64), ("count_kernel_ms", ctypes.c_double),
                ("count_kernel_launches", ctypes.c_int64), ("executed_macs", ctypes.c_double),
                ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64), ("top_capacity", ctypes.c_int32),
                ("top_snps", ctypes.POINTER(ctypes.c_uint32)), ("top_fp32", ctypes.POINTER(ctypes.c_float)),
                ("top_fp64", ctypes.POINTER(ctypes.c_double))]


class Resume(ctypes.Structure):
    _fields_ = [("path", ctypes.c_char_p), ("num_slabs", ctypes.c_int32), ("max_slabs", ctypes.c_int32),
                ("done", ctypes.c_int32), ("next_first", ctypes.c_int32), ("slabs_run", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 3)]


class Synth(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("num_snps", ctypes.c_int32), ("num_cases", ctypes.c_int32),
                ("num_controls", ctypes.c_int32), ("maf_min", ctypes.c_float), ("maf_max", ctypes.c_float),
                ("num_planted", ctypes.c_int32), ("planted_order", ctypes.c_int32),
                ("planted", (ctypes.c_int32 * 3) * 2), ("planted_maf", ctypes.c_float),
                ("base_risk", ctypes.c_float), ("effect", ctypes.c_float)]


_lib = None


def lib() -> ctypes.CDLL:
    """Loads libepisdet.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `make -C {HERE}`")
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    L.episdet_class_words.argtypes = [ctypes.c_int32]
    L.episdet_class_words.restype = ctypes.c_int32
    L.episdet_default_options.argtypes = [P(Options)]
    L.episdet_search.argtypes = [P(Dataset), P(Options), P(Result)]
    L.episdet_search.restype = ctypes.c_int
    L.episdet_search_batched.argtypes = [P(Dataset), P(Options), ctypes.c_int32, P(Result)]
    L.episdet_search_batched.restype = ctypes.c_int
    L.episdet_search_perm.argtypes = [P(Cohort), ctypes.c_void_p, ctypes.c_int32, P(Options), P(Result)]
    L.episdet_search_perm.restype = ctypes.c_int
    L.episdet_read_dataset.argtypes = [ctypes.c_char_p, P(Dataset)]
    L.episdet_read_dataset.restype = ctypes.c_int
    L.episdet_free_dataset.argtypes = [P(Dataset)]
    L.episdet_write_dataset.argtypes = [ctypes.c_char_p, P(Dataset)]
    L.episdet_write_dataset.restype = ctypes.c_int
    L.episdet_generate.argtypes = [P(Synth), ctypes.c_void_p, ctypes.c_void_p]
    L.episdet_generate.restype = ctypes.c_int
    L.episdet_generate_cohort.argtypes = [ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32, ctypes.c_float,
                                          ctypes.c_float, ctypes.c_void_p]
    L.episdet_generate_cohort.restype = ctypes.c_int
    L.episdet_generate_labels.argtypes = [ctypes.c_uint64, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                          ctypes.c_void_p]
    L.episdet_generate_labels.restype = ctypes.c_int
    L.episdet_binarize.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]
    L.episdet_binarize.restype = ctypes.c_int
    L.episdet_n_choose_k.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
    L.episdet_n_choose_k.restype = ctypes.c_uint64
    L.episdet_status_string.argtypes = [ctypes.c_int]
    L.episdet_status_string.restype = ctypes.c_char_p
    L.episdet_last_error.restype = ctypes.c_char_p
    L.episdet_abi_version.restype = ctypes.c_int32
    L.episdet_release_workspace.argtypes = [ctypes.c_int32]
    L.episdet_release_workspace.restype = ctypes.c_int
    L.episdet_last_launch_profile.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
    L.episdet_last_launch_profile.restype = ctypes.c_int64
    L.episdet_test_fail_allocation.argtypes = [ctypes.c_int32]
    L.episdet_test_fail_allocation.restype = None
    L.episdet_search_pairs_noalloc.argtypes = [P(Dataset), P(Options), P(Result)]
    L.episdet_search_pairs_noalloc.restype = ctypes.c_int
    _lib = L
    return L


def _check(status: int) -> None:
    if status != 0:
        raise EpisdetError(status, lib().episdet_last_error().decode(errors="replace"))


def class_words(n: int) -> int:
    return ((n + 1023) // 1024) * 32


def n_choose_k(n: int, k: int) -> int:
    return int(lib().episdet_n_choose_k(n, k))


# ------------------------------------------------------------------ data
def empty_planes(num_snps: int, num_samples: int) -> np.ndarray:
    return np.zeros((num_snps, 2, class_words(num_samples)), dtype=np.uint32)


def generate(seed: int, num_snps: int, num_cases: int, num_controls: int, maf=(0.05, 0.5), planted=(),
             planted_maf: float = 0.0, base_risk: float = 0.5, effect: float = 0.25):
    """Seeded Hardy-Weinberg dataset in the reference's per-class plane format.

    planted: up to two tuples of 2 or 3 SNP indices carrying the penetrance
    effect.  Returns (cases, controls) uint32 arrays [M][2][W].
    """
    s = Synth()
    s.seed, s.num_snps, s.num_cases, s.num_controls = seed, num_snps, num_cases, num_controls
    s.maf_min, s.maf_max = maf
    s.num_planted = len(planted)
    s.planted_order = len(planted[0]) if planted else 3
    for q, ps in enumerate(planted):
        for e, v in enumerate(ps):
            s.planted[q][e] = v
    s.planted_maf, s.base_risk, s.effect = planted_maf, base_risk, effect
    cases = empty_planes(num_snps, num_cases)
    controls = empty_planes(num_snps, num_controls)
    _check(lib().episdet_generate(ctypes.byref(s), cases.ctypes.data, controls.ctypes.data))
    return cases, controls


def generate_cohort(seed: int, num_snps: int, num_samples: int, maf=(0.05, 0.5)) -> np.ndarray:
    planes = empty_planes(num_snps, num_samples)
    _check(lib().episdet_generate_cohort(seed, num_snps, num_samples, maf[0], maf[1], planes.ctypes.data))
    return planes


def generate_labels(seed: int, num_samples: int, num_cases: int, num_labels: int) -> np.ndarray:
    labels = np.zeros((num_labels, class_words(num_samples)), dtype=np.uint32)
    _check(lib().episdet_generate_labels(seed, num_samples, num_cases, num_labels, labels.ctypes.data))
    return labels


def binarize(genotypes, is_case, device: int = 0):
    """Dense [SNP][sample] genotype matrix (values 0/1/2, uint8) and a per-sample
    case flag -> (cases, controls, num_cases, num_controls) in the reference's
    plane format, built on the GPU.  numpy inputs give numpy outputs; CUDA
    tensors give CUDA tensors (int32 views of the words)."""
    M, n = int(genotypes.shape[0]), int(genotypes.shape[1])
    flags = is_case
    if hasattr(is_case, "is_cuda"):
        nc = int(is_case.count_nonzero().item())
    else:
        flags = np.ascontiguousarray(np.asarray(is_case).astype(np.uint8) != 0).astype(np.uint8)
        nc = int(flags.sum())
    nn = n - nc
    wc, wn = class_words(max(nc, 1)), class_words(max(nn, 1))
    if hasattr(genotypes, "is_cuda"):
        import torch

        g = genotypes.contiguous()
        f = (flags != 0).to(torch.uint8).contiguous()
        cases = torch.zeros((M * 2 * wc,), dtype=torch.int32, device=g.device)
        controls = torch.zeros((M * 2 * wn,), dtype=torch.int32, device=g.device)
        _check(lib().episdet_binarize(g.data_ptr(), M, n, f.data_ptr(), cases.data_ptr(), controls.data_ptr(),
                                      DEVICE, device))
        return cases, controls, nc, nn
    g = np.ascontiguousarray(genotypes, dtype=np.uint8)
    cases = np.zeros((M, 2, wc), dtype=np.uint32)
    controls = np.zeros((M, 2, wn), dtype=np.uint32)
    _check(lib().episdet_binarize(g.ctypes.data, M, n, flags.ctypes.data, cases.ctypes.data, controls.ctypes.data,
                                  HOST, device))
    return cases, controls, nc, nn


def read_dataset(path: str):
    d = Dataset()
    _check(lib().episdet_read_dataset(path.encode(), ctypes.byref(d)))
    try:
        M, nc, nn = d.num_snps, d.num_cases, d.num_controls
        wc, wn = class_words(nc), class_words(nn)
        cases = np.ctypeslib.as_array(ctypes.cast(d.cases, ctypes.POINTER(ctypes.c_uint32)),
                                      shape=(M * 2 * wc,)).copy().reshape(M, 2, wc)
        controls = np.ctypeslib.as_array(ctypes.cast(d.controls, ctypes.POINTER(ctypes.c_uint32)),
                                         shape=(M * 2 * wn,)).copy().reshape(M, 2, wn)
    finally:
        lib().episdet_free_dataset(ctypes.byref(d))
    return cases, controls, nc, nn


def write_dataset(path: str, cases: np.ndarray, controls: np.ndarray, num_cases: int, num_controls: int) -> None:
    cases = np.ascontiguousarray(cases, dtype=np.uint32)
    controls = np.ascontiguousarray(controls, dtype=np.uint32)
    d = Dataset(cases.ctypes.data, controls.ctypes.data, cases.shape[0], num_cases, num_controls, HOST)
    _check(lib().episdet_write_dataset(path.encode(), ctypes.byref(d)))


# ---------------------------------------------------------------- search
@dataclass
class SearchResult:
    snps: tuple
    score: float
    score_fp32: float
    packed_indices: int
    sets_evaluated: int
    rounds: int
    seconds: float
    device_ms: float
    kernel_launches: int
    count_kernel_ms: float
    count_kernel_launches: int
    executed_macs: float
    h2d_bytes: int
    d2h_bytes: int
    top_snps: np.ndarray = field(repr=False)
    top_fp32: np.ndarray = field(repr=False)
    top_fp64: np.ndarray = field(repr=False)


def _ptr(a):
    """(pointer, memory kind) of a numpy array, a CUDA tensor or a (pinned) host tensor."""
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous() or a.element_size() != 4:
            raise TypeError("tensors must be contiguous 32-bit")
        return a.data_ptr(), (DEVICE if a.is_cuda else HOST)
    if not (isinstance(a, np.ndarray) and a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]):
        raise TypeError("planes must be C-contiguous uint32 numpy arrays or CUDA tensors")
    return a.ctypes.data, HOST


def make_options(order=3, score="k2", top_k=1024, device=0, engine="auto", first_begin=0, first_end=0,
                 flags=0, stream=0, wait_limit_ms=0, pair_block_snps=0) -> Options:
    o = Options()
    lib().episdet_default_options(ctypes.byref(o))
    o.order = order
    o.score = {"k2": SCORE_K2, "mi": SCORE_MI}[score] if isinstance(score, str) else int(score)
    o.top_k = top_k
    o.device = device
    o.engine = {"auto": ENGINE_AUTO, "tensor": ENGINE_TENSOR, "simt": ENGINE_SIMT}[engine] \
        if isinstance(engine, str) else int(engine)
    o.first_begin, o.first_end, o.flags = first_begin, first_end, flags
    o.stream = int(stream)
    o.wait_limit_ms = int(wait_limit_ms)
    o.pair_block_snps = int(pair_block_snps)
    return o


def _result_buffers(cap: int) -> Result:
    r = Result()
    r.top_capacity = cap
    bufs = (np.zeros((cap, 3), dtype=np.uint32), np.zeros(cap, dtype=np.float32), np.zeros(cap, dtype=np.float64))
    r.top_snps = bufs[0].ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
    r.top_fp32 = bufs[1].ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    r.top_fp64 = bufs[2].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    return r, bufs


def _to_result(order: int, r: Result, bufs) -> SearchResult:
    n = r.top_count
    return SearchResult(snps=tuple(int(v) for v in r.snps[:order]), score=r.score, score_fp32=r.score_fp32,
                        packed_indices=int(r.packed_indices), sets_evaluated=int(r.sets_evaluated),
                        rounds=int(r.rounds), seconds=r.seconds, device_ms=r.device_ms,
                        kernel_launches=int(r.kernel_launches), count_kernel_ms=r.count_kernel_ms,
                        count_kernel_launches=int(r.count_kernel_launches), executed_macs=r.executed_macs,
                        h2d_bytes=int(r.h2d_bytes), d2h_bytes=int(r.d2h_bytes), top_snps=bufs[0][:n, :order].copy(),
                        top_fp32=bufs[1][:n].copy(), top_fp64=bufs[2][:n].copy())


def search(cases, controls, num_cases: int, num_controls: int, *, num_snps: Optional[int] = None, order: int = 3,
           score="k2", top_k: int = 1024, device: int = 0, engine="auto", first_begin: int = 0, first_end: int = 0,
           flags: int = 0, stream: int = 0, wait_limit_ms: int = 0, pair_block_snps: int = 0) -> SearchResult:
    """Exhaustive search; cases/controls are host uint32 arrays or CUDA tensors in the plane format."""
    pc, mc = _ptr(cases)
    pn, mn = _ptr(controls)
    if mc != mn:
        raise TypeError("cases and controls must live in the same memory")
    M = num_snps if num_snps is not None else int(cases.shape[0])
    d = Dataset(pc, pn, M, num_cases, num_controls, mc)
    o = make_options(order, score, top_k, device, engine, first_begin, first_end, flags, stream, wait_limit_ms,
                     pair_block_snps)
    r, bufs = _result_buffers(top_k)
    _check(lib().episdet_search(ctypes.byref(d), ctypes.byref(o), ctypes.byref(r)))
    return _to_result(order, r, bufs)


def search_resumable(cases, controls, num_cases: int, num_controls: int, checkpoint: str, *,
                     num_snps: Optional[int] = None, order: int = 3, score="k2", top_k: int = 1024, device: int = 0,
                     engine="auto", first_begin: int = 0, first_end: int = 0, flags: int = 0, num_slabs: int = 16,
                     max_slabs: int = 0):
    """Search in first-SNP slabs with a checkpoint file after each slab;
    rerunning with the same arguments continues from the checkpoint.
    Returns (SearchResult, done, next_first): the answer when done, else the
    best set and list of the slabs searched so far."""
    pc, mc = _ptr(cases)
    pn, mn = _ptr(controls)
    if mc != mn:
        raise TypeError("cases and controls must live in the same memory")
    M = num_snps if num_snps is not None else int(cases.shape[0])
    d = Dataset(pc, pn, M, num_cases, num_controls, mc)
    o = make_options(order, score, top_k, device, engine, first_begin, first_end, flags)
    rs = Resume()
    rs.path = os.fsencode(checkpoint)
    rs.num_slabs, rs.max_slabs = num_slabs, max_slabs
    r, bufs = _result_buffers(top_k)
    _check(lib().episdet_search_resumable(ctypes.byref(d), ctypes.byref(o), ctypes.byref(rs), ctypes.byref(r)))
    return _to_result(order, r, bufs), bool(rs.done), int(rs.next_first)


def release_workspace(device: int = 0) -> None:
    _check(lib().episdet_release_workspace(device))


def last_launch_profile(device: int = 0):
    """Per counting launch of the last search with FLAG_TIMING on `device`:
    (device ms, tensor MACs issued), two float64 arrays in launch order."""
    n = int(lib().episdet_last_launch_profile(device, None, None, 0))
    ms = np.zeros(n, dtype=np.float64)
    macs = np.zeros(n, dtype=np.float64)
    if n:
        lib().episdet_last_launch_profile(device, ms.ctypes.data, macs.ctypes.data, n)
    return ms, macs


def test_fail_allocation(after: int) -> None:
    """Testing aid: the after-th device allocation from now on fails once as
    out of memory (after <= 0 disarms)."""
    lib().episdet_test_fail_allocation(after)


def tuned_stage(order: int, score, num_cases: int, num_controls: int) -> int:
    """The cached FLAG_AUTOTUNE choice for a shape: 1 staged triplet instance,
    0 plain, -1 not tuned yet."""
    sc = {"k2": SCORE_K2, "mi": SCORE_MI}[score] if isinstance(score, str) else int(score)
    return int(lib().episdet_tuned_stage(order, sc, num_cases, num_controls))


def perm_pvalues(results, score="k2") -> np.ndarray:
    """Single-step max-statistic adjusted p-values of the observed labels'
    top list (results[0], as search_perm returns it) against the best scores
    of the permuted labels results[1:]: (1 + #{perm best at least as extreme})
    / len(results); lower is more extreme for K2, higher for MI.  Same rule as
    episdet_perm_pvalues."""
    if len(results) < 2:
        raise ValueError("need the observed labels and at least one permutation")
    maximize = (score == "mi") if isinstance(score, str) else int(score) == SCORE_MI
    obs = results[0]
    s = obs.top_fp64 if len(obs.top_fp64) else np.array([obs.score])
    null = np.array([r.score for r in results[1:]])
    hits = (null[None, :] >= s[:, None]) if maximize else (null[None, :] <= s[:, None])
    return (1.0 + hits.sum(axis=1)) / len(results)


def search_pairs_noalloc(cases, controls, num_cases: int, num_controls: int, *, num_snps: int, score="k2",
                         top_k: int = 1024, device: int = 0, first_begin: int = 0, first_end: int = 0,
                         stream: int = 0) -> SearchResult:
    """Pairs search through the entry point that allocates no device memory
    (for callers whose memory is owned by a pool or that cannot synchronise
    for cudaFree).  cases/controls must be device-resident (CUDA tensors);
    limits: 4096 SNPs, 131072 samples, top_k 1024."""
    pc, mc = _ptr(cases)
    pn, mn = _ptr(controls)
    d = Dataset(pc, pn, num_snps, num_cases, num_controls, mc)
    o = make_options(2, score, top_k, device, "simt", first_begin, first_end, 0, stream)
    r, bufs = _result_buffers(top_k)
    _check(lib().episdet_search_pairs_noalloc(ctypes.byref(d), ctypes.byref(o), ctypes.byref(r)))
    return _to_result(2, r, bufs)


def search_batched(cohorts, options) -> list:
    """cohorts: list of (cases, controls, num_cases, num_controls[, num_snps]) (num_snps is needed
    for flat device tensors); options: list of dicts for make_options.  The cohorts run
    concurrently; each result equals the one a plain search() call returns."""
    n = len(cohorts)
    ds = (Dataset * n)()
    os_ = (Options * n)()
    rs = (Result * n)()
    keep = []
    for i, (co, opt) in enumerate(zip(cohorts, options)):
        c, k, nc, nn = co[:4]
        m = int(co[4]) if len(co) > 4 else int(c.shape[0])
        pc, mc = _ptr(c)
        pn, _ = _ptr(k)
        ds[i] = Dataset(pc, pn, m, nc, nn, mc)
        os_[i] = make_options(**opt)
        r, bufs = _result_buffers(os_[i].top_k)
        rs[i] = r
        keep.append(bufs)
    _check(lib().episdet_search_batched(ds, os_, n, rs))
    return [_to_result(os_[i].order, rs[i], keep[i]) for i in range(n)]


def search_perm(planes, num_samples: int, labels, *, order: int = 2, score="k2", top_k: int = 1024, device: int = 0,
                engine="auto", flags: int = 0) -> list:
    pp, mp = _ptr(planes)
    pl, ml = _ptr(labels)
    if mp != ml:
        raise TypeError("planes and labels must live in the same memory")
    nl = int(labels.shape[0])
    c = Cohort(pp, int(planes.shape[0]), num_samples, mp)
    o = make_options(order, score, top_k, device, engine, flags=flags)
    rs = (Result * nl)()
    keep = []
    for i in range(nl):
        r, bufs = _result_buffers(top_k)
        rs[i] = r
        keep.append(bufs)
    _check(lib().episdet_search_perm(ctypes.byref(c), ctypes.c_void_p(pl), nl, ctypes.byref(o), rs))
    return [_to_result(order, rs[i], keep[i]) for i in range(nl)]


def EpistasisDetectionSearch(datasetCases, datasetControls, numSNPs, numCases, numControls, numSNPsWithPadding,
                             numCasesWithPadding, numControlsWithPadding, *, triplets=True, mi_score=False):
    """The reference's entry point (src/search-triplets.cu:8): returns
    (status, roundsCounter, searchTime, outputFromGpu, packedIndices).

    status is 0 on success like cudaSuccess; the padded sizes must be the ones
    the reference's loader computes (src/tensor-episdet.cu:87-95)."""
    if numCasesWithPadding != class_words(numCases) * 32 or numControlsWithPadding != class_words(numControls) * 32 \
            or numSNPsWithPadding < numSNPs:
        return 1, 0, 0.0, 0.0, 0
    try:
        r = search(datasetCases, datasetControls, numCases, numControls, num_snps=numSNPs,
                   order=3 if triplets else 2, score="mi" if mi_score else "k2")
    except EpisdetError as e:
        return e.status, 0, 0.0, 0.0, 0
    return 0, r.rounds, r.seconds, float(np.float32(r.score)), r.packed_indices
