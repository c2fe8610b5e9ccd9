"""C-ABI surface on the CPU: exported symbols, host helpers, generator, I/O and
argument errors.  No kernel runs here."""
import ctypes
import math
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "episdet.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(episdet_[a-z_0-9]+)\s*\(", src)))


def test_every_declared_symbol_is_exported(episdet):
    names = _declared()
    assert "episdet_search" in names and "episdet_search_perm" in names
    L = episdet.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(episdet.EXPORTED)


def test_abi_version_and_helpers(episdet):
    L = episdet.lib()
    assert L.episdet_abi_version() == 1
    for n in (1, 31, 32, 1023, 1024, 1025, 131072, 262143):
        assert L.episdet_class_words(n) == episdet.class_words(n) == ((n + 1023) // 1024) * 32
    # README.md:54 of the reference: 11,444,858,880 triplets for 4096 SNPs.
    assert episdet.n_choose_k(4096, 3) == 11444858880 == math.comb(4096, 3)
    assert episdet.n_choose_k(512, 2) == math.comb(512, 2)
    assert L.episdet_status_string(2) == b"invalid input planes"


def test_generator_is_deterministic_and_valid(episdet, oracle):
    a = episdet.generate(11, 40, 100, 70)
    b = episdet.generate(11, 40, 100, 70)
    c = episdet.generate(12, 40, 100, 70)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[0], c[0])
    assert oracle.validate(a[0], 100) and oracle.validate(a[1], 70)
    g = oracle.unpack(a[0], 100)
    assert set(np.unique(g)) <= {0, 1, 2}


def test_generator_hwe_frequencies(episdet, oracle):
    cases, controls = episdet.generate(5, 50, 4000, 4000, maf=(0.3, 0.3))
    g = np.concatenate([oracle.unpack(cases, 4000), oracle.unpack(controls, 4000)], axis=1)
    freq = [(g == k).mean() for k in range(3)]
    assert freq == pytest.approx([0.49, 0.42, 0.09], abs=0.01)


def test_generator_planted_classes_full(episdet, oracle):
    cases, controls = episdet.generate(3, 30, 500, 600, planted=[(2, 9, 17)], base_risk=0.5, effect=0.25)
    m_c = oracle.marginals(cases, 500)
    m_n = oracle.marginals(controls, 600)
    assert (m_c.sum(axis=0) == 500).all() and (m_n.sum(axis=0) == 600).all()


def test_labels(episdet):
    n, nc = 1000, 400
    lab = episdet.generate_labels(9, n, nc, 5)
    bits = np.unpackbits(lab.astype(">u4").view(np.uint8), bitorder="big").reshape(5, -1)[:, :n]
    assert (bits.sum(axis=1) == nc).all()
    assert bits[0, :nc].all() and not bits[0, nc:].any()
    assert not np.array_equal(bits[1], bits[2])


def test_dataset_file_roundtrip(episdet, tmp_path):
    cases, controls = episdet.generate(2, 17, 1500, 900)
    path = str(tmp_path / "ds.txt")
    episdet.write_dataset(path, cases, controls, 1500, 900)
    lines = open(path).read().split("\n")
    assert lines[0] == "17" and lines[2] == "900" and lines[4] == "1500"  # src/tensor-episdet.cu:68-83
    c2, n2, nc, nn = episdet.read_dataset(path)
    assert (nc, nn) == (1500, 900)
    assert np.array_equal(c2, cases) and np.array_equal(n2, controls)


def test_short_bin_file_is_an_io_error(episdet, tmp_path):
    cases, controls = episdet.generate(2, 8, 100, 100)
    path = str(tmp_path / "ds.txt")
    episdet.write_dataset(path, cases, controls, 100, 100)
    with open(str(tmp_path / "ds.cases.bin"), "r+b") as f:
        f.truncate(100)
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.read_dataset(path)
    assert e.value.name == "EPISDET_ERR_IO"
    with pytest.raises(episdet.EpisdetError):
        episdet.read_dataset(str(tmp_path / "missing.txt"))


def test_argument_errors(episdet):
    L = episdet.lib()
    cases, controls = episdet.generate(1, 10, 64, 64)
    r = episdet.Result()
    o = episdet.make_options(order=3)
    assert L.episdet_search(None, ctypes.byref(o), ctypes.byref(r)) == 1
    d = episdet.Dataset(cases.ctypes.data, controls.ctypes.data, 10, 0, 64, 0)
    assert L.episdet_search(ctypes.byref(d), ctypes.byref(o), ctypes.byref(r)) == 1
    d = episdet.Dataset(cases.ctypes.data, controls.ctypes.data, 2, 64, 64, 0)
    assert L.episdet_search(ctypes.byref(d), ctypes.byref(o), ctypes.byref(r)) == 1  # 2 SNPs, order 3
    o.order = 4
    d = episdet.Dataset(cases.ctypes.data, controls.ctypes.data, 10, 64, 64, 0)
    assert L.episdet_search(ctypes.byref(d), ctypes.byref(o), ctypes.byref(r)) == 1
    o = episdet.make_options(order=2, top_k=100000)
    assert L.episdet_search(ctypes.byref(d), ctypes.byref(o), ctypes.byref(r)) == 1
    assert b"top_k" in L.episdet_last_error()


def test_reference_signature_rejects_inconsistent_padding(episdet):
    cases, controls = episdet.generate(1, 10, 100, 100)
    st, *_ = episdet.EpistasisDetectionSearch(cases, controls, 10, 100, 100, 256, 1000, 1024)
    assert st != 0


def _gpu_present():
    try:
        return subprocess.run(["nvidia-smi", "-L"], capture_output=True, timeout=20).returncode == 0
    except Exception:
        return False


@pytest.mark.skipif(_gpu_present(), reason="checks the no-device error path")
def test_no_device_is_reported(episdet):
    cases, controls = episdet.generate(1, 10, 64, 64)
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.search(cases, controls, 64, 64, order=2)
    assert e.value.name == "EPISDET_ERR_NO_DEVICE"


@pytest.mark.skipif(_gpu_present(), reason="checks the no-device error path")
def test_cli_reports_missing_device_and_usage(tmp_path):
    exe = os.path.join(ROOT, "tensor-episdet_b200", "bin", "tensor-episdet.pairs.k2.bin")
    p = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1


def test_tensor_engine_refuses_classes_past_fp32_exactness(episdet):
    """The tensor engine accumulates a class's counts in FP32, exact up to 2^24
    samples; a larger class is refused for the tensor engine before any device
    work (EPISDET_ENGINE_AUTO hands it to the integer-pipe engine instead)."""
    L = episdet.lib()
    cases, controls = episdet.generate(1, 10, 64, 64)
    r = episdet.Result()
    for big in ((1 << 24) + 1, 1 << 25):
        for order in (2, 3):
            o = episdet.make_options(order=order, engine="tensor")
            d = episdet.Dataset(cases.ctypes.data, controls.ctypes.data, 10, big, 64, 0)
            assert L.episdet_search(ctypes.byref(d), ctypes.byref(o), ctypes.byref(r)) == 8  # UNSUPPORTED
            assert b"2^24" in L.episdet_last_error() or b"16777216" in L.episdet_last_error()
            d = episdet.Dataset(cases.ctypes.data, controls.ctypes.data, 10, 64, big, 0)
            assert L.episdet_search(ctypes.byref(d), ctypes.byref(o), ctypes.byref(r)) == 8
