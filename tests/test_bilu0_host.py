"""Block ILU(0)'s numeric factorisation (factor_bilu0, h33_setup.cpp) on the host: the
level-parallel form (rows of one level of the lower pattern at once, with four or more
threads) against the natural-order sweep (one thread), bit for bit on seeded random
profiles and 27-point boxes, and the zero-pivot code 9001 in both
(tests/c_driver/bilu0_parallel_check.cpp, compiled with the library's h33_setup.cpp)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "frontistr_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_level_parallel_factors_equal_natural_order(tmp_path):
    exe = str(tmp_path / "bilu0_parallel_check")
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-fopenmp", "-I", CSRC,
                           os.path.join(ROOT, "tests", "c_driver", "bilu0_parallel_check.cpp"),
                           os.path.join(CSRC, "h33_setup.cpp"), "-o", exe])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
