"""ctypes binding of the CPU oracle (oracle/build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product.  See oracle.h for what the
oracle restates from hiperbio/tensor-episdet and for its parity status.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboracle.so")
K2, MI = 0, 1


class _Dataset(ctypes.Structure):
    _fields_ = [("cases", ctypes.c_void_p), ("controls", ctypes.c_void_p), ("num_snps", ctypes.c_int32),
                ("num_cases", ctypes.c_int32), ("num_controls", ctypes.c_int32)]


class _Options(ctypes.Structure):
    _fields_ = [("order", ctypes.c_int32), ("score", ctypes.c_int32), ("top_k", ctypes.c_int32),
                ("threads", ctypes.c_int32), ("first_begin", ctypes.c_int32), ("first_end", ctypes.c_int32),
                ("second_begin", ctypes.c_int32), ("second_end", ctypes.c_int32)]


class _Result(ctypes.Structure):
    _fields_ = [("top_sets", ctypes.POINTER(ctypes.c_uint64)), ("top_fp32", ctypes.POINTER(ctypes.c_float)),
                ("top_fp64", ctypes.POINTER(ctypes.c_double)), ("top_count", ctypes.c_int32),
                ("best_set", ctypes.c_uint64), ("best_fp64", ctypes.c_double), ("best_fp32", ctypes.c_float),
                ("sets", ctypes.c_uint64)]


class _Synth(ctypes.Structure):
    _fields_ = [("seed", ctypes.c_uint64), ("num_snps", ctypes.c_int32), ("num_cases", ctypes.c_int32),
                ("num_controls", ctypes.c_int32), ("maf_min", ctypes.c_float), ("maf_max", ctypes.c_float),
                ("num_planted", ctypes.c_int32), ("planted_order", ctypes.c_int32),
                ("planted", (ctypes.c_int32 * 3) * 2), ("planted_maf", ctypes.c_float),
                ("base_risk", ctypes.c_float), ("effect", ctypes.c_float)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        L.od_search.argtypes = [P(_Dataset), P(_Options), P(_Result)]
        L.od_search.restype = ctypes.c_int
        L.od_table2.argtypes = [P(_Dataset), ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
        L.od_table3.argtypes = [P(_Dataset), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                ctypes.c_void_p]
        L.od_marginals.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]
        L.od_validate.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]
        L.od_validate.restype = ctypes.c_int
        L.od_pair9.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]
        L.od_class_words.argtypes = [ctypes.c_int32]
        L.od_class_words.restype = ctypes.c_int32
        L.od_split_by_label.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p, P(ctypes.c_int32)]
        L.od_split_by_label.restype = ctypes.c_int32
        L.od_generate.argtypes = [P(_Synth), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.od_generate.restype = ctypes.c_int
        _lib = L
    return _lib


def class_words(n: int) -> int:
    return ((n + 1023) // 1024) * 32


def unkey(order: int, key: int) -> tuple:
    if order == 2:
        return (key >> 32, key & 0xFFFFFFFF)
    return ((key >> 42) & 0x1FFFFF, (key >> 21) & 0x1FFFFF, key & 0x1FFFFF)


def _ds(cases, controls, nc, nn):
    cases = np.ascontiguousarray(cases, dtype=np.uint32)
    controls = np.ascontiguousarray(controls, dtype=np.uint32)
    return _Dataset(cases.ctypes.data, controls.ctypes.data, cases.shape[0], nc, nn), (cases, controls)


def search(cases, controls, nc, nn, order=3, score="k2", top_k=1024, threads=0, first_begin=0, first_end=0,
           second_begin=0, second_end=0) -> dict:
    d, keep = _ds(cases, controls, nc, nn)
    o = _Options(order, K2 if score == "k2" else MI, top_k, threads, first_begin, first_end, second_begin,
                 second_end)
    sets = np.zeros(top_k, dtype=np.uint64)
    f32 = np.zeros(top_k, dtype=np.float32)
    f64 = np.zeros(top_k, dtype=np.float64)
    r = _Result(sets.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                f32.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                f64.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0, 0, 0.0, 0.0, 0)
    rc = lib().od_search(ctypes.byref(d), ctypes.byref(o), ctypes.byref(r))
    if rc != 0:
        raise RuntimeError(f"oracle search failed ({rc})")
    n = r.top_count
    return {
        "best": unkey(order, int(r.best_set)),
        "best_fp64": r.best_fp64,
        "best_fp32": r.best_fp32,
        "sets": int(r.sets),
        "top": [unkey(order, int(s)) for s in sets[:n]],
        "top_fp32": f32[:n].copy(),
        "top_fp64": f64[:n].copy(),
    }


def generate(seed, num_snps, num_cases, num_controls, maf=(0.05, 0.5), planted=(), planted_maf=0.0,
             base_risk=0.5, effect=0.25, threads=0):
    """The product generator's dataset, made by the oracle library alone
    (same arguments and bits as episdet.generate)."""
    s = _Synth()
    s.seed, s.num_snps, s.num_cases, s.num_controls = seed, num_snps, num_cases, num_controls
    s.maf_min, s.maf_max = maf
    s.num_planted = len(planted)
    s.planted_order = len(planted[0]) if planted else 3
    for q, ps in enumerate(planted):
        for e, v in enumerate(ps):
            s.planted[q][e] = v
    s.planted_maf, s.base_risk, s.effect = planted_maf, base_risk, effect
    cases = np.zeros((num_snps, 2, class_words(num_cases)), dtype=np.uint32)
    controls = np.zeros((num_snps, 2, class_words(num_controls)), dtype=np.uint32)
    rc = lib().od_generate(ctypes.byref(s), cases.ctypes.data, controls.ctypes.data, threads)
    if rc != 0:
        raise ValueError(f"bad synthetic spec ({rc})")
    return cases, controls


def table2(cases, controls, nc, nn, a, b):
    d, keep = _ds(cases, controls, nc, nn)
    cs = np.zeros(9, dtype=np.int32)
    cn = np.zeros(9, dtype=np.int32)
    lib().od_table2(ctypes.byref(d), a, b, cs.ctypes.data, cn.ctypes.data)
    return cs, cn


def table3(cases, controls, nc, nn, x, y, z):
    d, keep = _ds(cases, controls, nc, nn)
    cs = np.zeros(27, dtype=np.int32)
    cn = np.zeros(27, dtype=np.int32)
    lib().od_table3(ctypes.byref(d), x, y, z, cs.ctypes.data, cn.ctypes.data)
    return cs, cn


def marginals(planes, n):
    planes = np.ascontiguousarray(planes, dtype=np.uint32)
    out = np.zeros((3, planes.shape[0]), dtype=np.uint32)
    lib().od_marginals(planes.ctypes.data, planes.shape[0], n, out.ctypes.data)
    return out


def validate(planes, n) -> bool:
    planes = np.ascontiguousarray(planes, dtype=np.uint32)
    return lib().od_validate(planes.ctypes.data, planes.shape[0], n) == 0


def split_by_label(planes, n, label):
    planes = np.ascontiguousarray(planes, dtype=np.uint32)
    label = np.ascontiguousarray(label, dtype=np.uint32)
    M = planes.shape[0]
    nc = int(sum(((int(label[s // 32]) >> (31 - s % 32)) & 1) for s in range(n)))
    nn = n - nc
    cases = np.zeros((M, 2, class_words(max(nc, 1))), dtype=np.uint32)
    controls = np.zeros((M, 2, class_words(max(nn, 1))), dtype=np.uint32)
    got_nn = ctypes.c_int32(0)
    got = lib().od_split_by_label(planes.ctypes.data, M, n, label.ctypes.data, cases.ctypes.data,
                                  controls.ctypes.data, ctypes.byref(got_nn))
    assert got == nc and got_nn.value == nn
    return cases, controls, nc, nn


# -------------------------------------------------------- plane packing
def pack(geno: np.ndarray) -> np.ndarray:
    """Genotype matrix [M][n] with values in {0,1,2} -> reference planes [M][2][W] (MSB-first)."""
    geno = np.asarray(geno)
    M, n = geno.shape
    W = class_words(n)
    out = np.zeros((M, 2, W), dtype=np.uint32)
    for g in (0, 1):
        bits = np.zeros((M, W * 32), dtype=np.uint8)
        bits[:, :n] = (geno == g)
        packed = np.packbits(bits, axis=1, bitorder="big").reshape(M, W, 4)
        out[:, g, :] = (packed[..., 0].astype(np.uint32) << 24) | (packed[..., 1].astype(np.uint32) << 16) | \
                       (packed[..., 2].astype(np.uint32) << 8) | packed[..., 3].astype(np.uint32)
    return out


def unpack(planes: np.ndarray, n: int) -> np.ndarray:
    """Reference planes [M][2][W] -> genotype matrix [M][n] (2 where neither plane is set)."""
    planes = np.asarray(planes, dtype=np.uint32)
    M, _, W = planes.shape
    b = np.stack([(planes >> (31 - k)) & 1 for k in range(32)], axis=-1).reshape(M, 2, W * 32)[:, :, :n]
    geno = np.full((M, n), 2, dtype=np.int8)
    geno[b[:, 1] == 1] = 1
    geno[b[:, 0] == 1] = 0
    return geno
