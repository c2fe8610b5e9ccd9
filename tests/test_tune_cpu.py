"""The EPISDET_FLAG_AUTOTUNE cache on the CPU: the file named by
EPISDET_TUNE_CACHE is read once per process ("order score bucket choice"
lines, bucket = floor(log2(smaller class))); malformed lines are skipped.
Each case runs in a fresh process, since the cache is loaded once."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "tensor-episdet_b200")


def _query(cache, queries):
    code = ("import sys; sys.path.insert(0, %r); import episdet; "
            "print([episdet.tuned_stage(*q) for q in %r])" % (PKG, queries))
    env = dict(os.environ, EPISDET_TUNE_CACHE=str(cache))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=120)
    assert p.returncode == 0, p.stderr
    return eval(p.stdout.strip())


def test_cache_file_is_read(tmp_path):
    cache = tmp_path / "tune.txt"
    cache.write_text("3 0 16 1\n3 1 15 0\nnot a line\n3 0 14 7\n2 0 12 1\n")
    got = _query(cache, [(3, "k2", 70000, 66000),   # min class 66000 -> bucket 16
                         (3, "mi", 40000, 36000),   # bucket 15
                         (3, "k2", 20000, 30000),   # bucket 14: choice 7 is malformed
                         (3, "k2", 5000, 5000),     # bucket 12, no triplet entry
                         (2, "k2", 4096, 8000)])    # bucket 12 for pairs
    assert got == [1, 0, -1, -1, 1]


def test_missing_cache_file_means_untuned(tmp_path):
    assert _query(tmp_path / "absent.txt", [(3, "k2", 70000, 66000)]) == [-1]
