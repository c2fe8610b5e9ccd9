"""The reference's own main, unmodified, linked against the library.

`make -C tensor-episdet_b200 reference-main` compiles src/tensor-episdet.cu of
the reference as it is (with the CUTLASS 1.3 names its include/helper.hpp
needs supplied by the interface stand-in under tensor-episdet_b200/compat/)
and links it against libepisdet_compat_{pairs,triplets}_{k2,mi}.a and
libepisdet.so, without src/helper.cu or any CUTLASS code.  The executables are
built where the reference tree is present and travel with the other built
files; these tests check the link on the CPU and, on a B200, that the
reference's main prints what the project's own executables print.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "tensor-episdet_b200")
REF_MAIN = os.path.join(PKG, "bin", "reference-main")
REF_TREE = os.environ.get("EPISDET_REFERENCE_TREE", "/root/reference")
VARIANTS = ["pairs.k2", "pairs.mi", "triplets.k2", "triplets.mi"]
# Lines that depend on the run's wall time.
TIMED = ("Wall-clock time", "Tensor TOPS", "Num. unique sets per sec.")


def _exe(v):
    return os.path.join(REF_MAIN, f"tensor-episdet.{v}.bin")


def _built():
    if os.path.isdir(os.path.join(REF_TREE, "src")):
        subprocess.run(["make", "-s", "-C", PKG, "reference-main"], check=True, capture_output=True, timeout=900)
    return all(os.path.exists(_exe(v)) for v in VARIANTS)


def test_reference_main_links_against_the_shims():
    if not _built():
        pytest.skip("the reference tree is not here and its main was not built")
    for v in VARIANTS:
        syms = subprocess.run(["nm", "-C", _exe(v)], capture_output=True, text=True, check=True).stdout
        # Both C++ symbols the reference's main calls are defined by the shim.
        assert any(" T EpistasisDetectionSearch(unsigned int*" in l for l in syms.splitlines()), v
        assert any(" n_choose_k(unsigned int, unsigned int)" in l and " U " not in l for l in syms.splitlines()), v
        deps = subprocess.run(["ldd", _exe(v)], capture_output=True, text=True).stdout
        assert os.path.join(PKG, "lib", "libepisdet.so") in deps or "libepisdet.so =>" in deps


@pytest.mark.gpu
@pytest.mark.parametrize("variant", VARIANTS)
def test_reference_main_prints_what_the_project_executable_prints(episdet, tmp_path, variant):
    if not all(os.path.exists(_exe(v)) for v in VARIANTS):
        pytest.skip("reference main not built (needs the reference tree at build time)")
    # 300 SNPs: not a multiple of the reference's BLOCK_SIZE, so its main reads
    # fewer rows than it pads to (and says so on stderr), as it does for any
    # such dataset.
    cases, controls = episdet.generate(41, 300, 2500, 2300)
    path = str(tmp_path / "data.txt")
    episdet.write_dataset(path, cases, controls, 2500, 2300)
    ours = subprocess.run([os.path.join(PKG, "bin", f"tensor-episdet.{variant}.bin"), path], capture_output=True,
                          text=True, timeout=600)
    ref = subprocess.run([_exe(variant), path], capture_output=True, text=True, timeout=600)
    assert ours.returncode == 0 and ref.returncode == 0, (ours.stderr, ref.stderr)
    keep = lambda out: [l for l in out.splitlines() if not l.startswith(TIMED)]
    assert keep(ref.stdout) == keep(ours.stdout)
    assert len(keep(ref.stdout)) >= 9
    assert any("SCORE\t->\t{" in l for l in keep(ref.stdout))
