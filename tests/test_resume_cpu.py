"""Host logic of the significance and resume entry points, on the CPU: the
C p-values against the documented rule, and the checkpoint file (format,
fingerprint, refusal of another search's checkpoint, the answer assembled from
a completed checkpoint).  No kernel runs here."""
import ctypes
import struct

import numpy as np
import pytest

MASK = (1 << 64) - 1
# Layout of the checkpoint header and entries (native alignment, as written).
HEADER = struct.Struct("@8s8iQii5qQ4d")
ENTRY = struct.Struct("@3Ifd")


def _mix_int(x):
    x = (x + 0x9E3779B97F4A7C15) & MASK
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & MASK
    return x ^ (x >> 31)


def _mix_words(words, salt):
    """Sum over i of mix((w_i << 32) ^ i ^ salt) mod 2^64."""
    with np.errstate(over="ignore"):
        w = words.reshape(-1).astype(np.uint64)
        x = (w << np.uint64(32)) ^ np.arange(w.size, dtype=np.uint64) ^ np.uint64(salt)
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    return int(x.sum(dtype=np.uint64))


def _fingerprint(cases, controls, M, nc, nn, order, score, k, fb, fe):
    fp = _mix_int((M * 1000003 + order * 7 + score) & MASK) ^ _mix_int(((nc << 32) | nn) & MASK) \
        ^ _mix_int(((k << 40) ^ (fb << 20) ^ fe) & MASK)
    fp = (fp + _mix_words(cases, 1 << 62)) & MASK
    return (fp + _mix_words(controls, 2 << 62)) & MASK


def _write_checkpoint(path, *, M, nc, nn, order, score, k, fb, fe, fingerprint, cursor, entries, sets=0):
    with open(path, "wb") as f:
        f.write(HEADER.pack(b"EPISCKP1", M, nc, nn, order, score, k, fb, fe, fingerprint, cursor, len(entries),
                            sets, 7, 3, 100, 200, 11, 1.5, 2.5, 0.5, 1e9))
        for snps, f32, f64 in entries:
            f.write(ENTRY.pack(*snps, f32, f64))


def _results(episdet, obs_top, obs_score, null_scores, keep):
    n = 1 + len(null_scores)
    rs = (episdet.Result * n)()
    top = np.array(obs_top, dtype=np.float64)
    keep.append(top)
    rs[0].score = obs_score
    rs[0].top_count = len(top)
    rs[0].top_fp64 = top.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if len(top) else None
    for i, s in enumerate(null_scores):
        rs[i + 1].score = s
    return rs


class _R:
    def __init__(self, score, top=()):
        self.score = score
        self.top_fp64 = np.array(top, dtype=np.float64)


@pytest.mark.parametrize("score", ["k2", "mi"])
def test_perm_pvalues_c_matches_rule(episdet, score):
    rng = np.random.default_rng(5)
    obs_top = np.sort(rng.normal(100.0, 5.0, size=12))
    if score == "mi":
        obs_top = obs_top[::-1].copy()
    null = list(rng.normal(100.0, 5.0, size=40))
    null[3] = float(obs_top[2])  # a tie counts as at least as extreme
    keep = []
    rs = _results(episdet, obs_top, float(obs_top[0]), null, keep)
    pv = np.zeros(12)
    cnt = ctypes.c_int32()
    sc = episdet.SCORE_MI if score == "mi" else episdet.SCORE_K2
    st = episdet.lib().episdet_perm_pvalues(rs, 41, sc, pv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 12,
                                            ctypes.byref(cnt))
    assert st == 0 and cnt.value == 12
    want = episdet.perm_pvalues([_R(float(obs_top[0]), obs_top)] + [_R(s) for s in null], score)
    np.testing.assert_array_equal(pv, want)
    nul = np.array(null)
    for j, s in enumerate(obs_top):
        hits = (nul >= s).sum() if score == "mi" else (nul <= s).sum()
        assert pv[j] == (1 + hits) / 41
    assert np.all(np.diff(pv) >= 0)  # the list is in rank order
    # Without a top list the best set's score is used.
    rs = _results(episdet, [], 90.0, [95.0, 85.0, 90.0], keep)
    st = episdet.lib().episdet_perm_pvalues(rs, 4, episdet.SCORE_K2, pv.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                            12, ctypes.byref(cnt))
    assert st == 0 and cnt.value == 1 and pv[0] == 3 / 4


def test_perm_pvalues_argument_errors(episdet):
    keep = []
    rs = _results(episdet, [], 1.0, [], keep)
    pv = np.zeros(4)
    cnt = ctypes.c_int32()
    L = episdet.lib()
    p = pv.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert L.episdet_perm_pvalues(rs, 1, 0, p, 4, ctypes.byref(cnt)) == 1
    assert b"permutation" in L.episdet_last_error()
    assert L.episdet_perm_pvalues(None, 3, 0, p, 4, ctypes.byref(cnt)) == 1
    assert L.episdet_perm_pvalues(rs, 3, 5, p, 4, ctypes.byref(cnt)) == 1


def _dataset(episdet):
    M, nc, nn = 12, 100, 90
    cases, controls = episdet.generate(42, M, nc, nn)
    return cases, controls, M, nc, nn


def test_completed_checkpoint_is_answered_without_a_search(episdet, tmp_path):
    cases, controls, M, nc, nn = _dataset(episdet)
    order, k = 3, 8
    fp = _fingerprint(cases, controls, M, nc, nn, order, 0, k, 0, M)
    # FP32 rank order; two sets tie on the FP64 minimum, the lower set wins.
    entries = [((0, 1, 2), 10.0, 10.25), ((0, 3, 9), 10.5, 10.125), ((0, 2, 5), 11.0, 10.125),
               ((4, 6, 7), 12.0, 12.0)]
    path = str(tmp_path / "search.ckpt")
    _write_checkpoint(path, M=M, nc=nc, nn=nn, order=order, score=0, k=k, fb=0, fe=M, fingerprint=fp,
                      cursor=M - order + 1, entries=entries, sets=220)
    r, done, nxt = episdet.search_resumable(cases, controls, nc, nn, path, order=order, top_k=k)
    assert done and nxt == M - order + 1
    assert r.snps == (0, 2, 5) and r.score == 10.125 and r.score_fp32 == 11.0
    assert r.packed_indices == 0 | (2 << 21) | (5 << 42)
    assert [tuple(s) for s in r.top_snps] == [e[0] for e in entries]
    assert list(r.top_fp64) == [e[2] for e in entries]
    assert r.sets_evaluated == 220 and r.kernel_launches == 11


def test_checkpoint_of_another_search_is_refused(episdet, tmp_path):
    cases, controls, M, nc, nn = _dataset(episdet)
    path = str(tmp_path / "other.ckpt")
    fp = _fingerprint(cases, controls, M, nc, nn, 3, 0, 8, 0, M)
    # Same sizes and options, one plane word different.
    other = cases.copy()
    other[5, 0, 0] ^= np.uint32(0x80000000)
    _write_checkpoint(path, M=M, nc=nc, nn=nn, order=3, score=0, k=8, fb=0, fe=M,
                      fingerprint=_fingerprint(other, controls, M, nc, nn, 3, 0, 8, 0, M), cursor=M - 2, entries=[])
    assert fp != _fingerprint(other, controls, M, nc, nn, 3, 0, 8, 0, M)
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.search_resumable(cases, controls, nc, nn, path, order=3, top_k=8)
    assert e.value.status == 1 and "another search" in str(e.value)
    # Another top_k is another search too.
    _write_checkpoint(path, M=M, nc=nc, nn=nn, order=3, score=0, k=8, fb=0, fe=M, fingerprint=fp, cursor=M - 2,
                      entries=[])
    with pytest.raises(episdet.EpisdetError):
        episdet.search_resumable(cases, controls, nc, nn, path, order=3, top_k=16)


def test_corrupt_checkpoint_is_an_io_error(episdet, tmp_path):
    cases, controls, M, nc, nn = _dataset(episdet)
    path = tmp_path / "bad.ckpt"
    path.write_bytes(b"not a checkpoint at all" * 8)
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.search_resumable(cases, controls, nc, nn, str(path), order=3, top_k=8)
    assert e.value.name == "EPISDET_ERR_IO"
    # A header promising entries the file does not hold.
    fp = _fingerprint(cases, controls, M, nc, nn, 3, 0, 8, 0, M)
    _write_checkpoint(str(path), M=M, nc=nc, nn=nn, order=3, score=0, k=8, fb=0, fe=M, fingerprint=fp,
                      cursor=M - 2, entries=[((0, 1, 2), 1.0, 1.0)] * 3)
    data = path.read_bytes()
    path.write_bytes(data[:-10])
    with pytest.raises(episdet.EpisdetError) as e:
        episdet.search_resumable(cases, controls, nc, nn, str(path), order=3, top_k=8)
    assert "truncated" in str(e.value)
