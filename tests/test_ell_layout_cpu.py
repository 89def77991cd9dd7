"""The sliced-ELL layout built on the host (csrc/setup.hpp), checked on the CPU against CSR
products by a C++ emulation of the kernels' lane order and shuffle tree (tests/cpp/ell_check.cpp):
every entry in its slot, exact sums on integer data, and the per-window row permutation
leaving every row's bits unchanged while it cuts the padding."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_sliced_ell_layout_and_permutation(tmp_path):
    exe = str(tmp_path / "ell_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(ROOT, "parallel_admm_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "ell_check.cpp"), "-o", exe], check=True, capture_output=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip().endswith("ok")
