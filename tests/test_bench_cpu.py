"""bench.py's reference arm on the CPU: one step of the oracle's bounded
sample, printed as the one JSON line the benchmark contract asks for."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 0
    assert d["value"] > 0 and d["higher_is_better"] is True and d["unit"] == d["e2e"]["unit"]
    assert d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert "workload" in d["config"]
    # The arm runs the oracle alone: no library of the product is mapped.
    assert d["libraries_loaded"] == ["oracle/build/liboracle.so"], d["libraries_loaded"]


def test_oracle_generator_matches_the_product_generator():
    """The reference arm makes the bench planes with the oracle's generator;
    they must be the product generator's bits (bench.py's spec, in full)."""
    sys.path.insert(0, ROOT)
    import hashlib
    import numpy as np
    import bench

    a = bench.generate_oracle()
    b = bench.generate()
    for x, y in zip(a, b):
        assert x.shape == y.shape and x.dtype == y.dtype == np.uint32
        assert hashlib.sha256(x.tobytes()).hexdigest() == hashlib.sha256(y.tobytes()).hexdigest()
