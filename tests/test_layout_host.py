"""The layout split behind the device fill, checked on the host: the shape from row
counts (sell_shape) against build_sell, the fill kernels' placement rule, the row
order from counts, and the reordered SSOR layouts built the device's way (counts per
part, rank of each block among the part's smaller new columns) against the host chain
reordered_rows -> permute_rows -> build_sell, on seeded random profiles
(tests/c_driver/layout_shape_check.cpp, compiled with the library's h33_setup.cpp)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "frontistr_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_layout_shape_and_device_placement_match_host_builders(tmp_path):
    exe = str(tmp_path / "layout_shape_check")
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-fopenmp", "-I", CSRC,
                           os.path.join(ROOT, "tests", "c_driver", "layout_shape_check.cpp"),
                           os.path.join(CSRC, "h33_setup.cpp"), "-o", exe])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
