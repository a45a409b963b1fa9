"""The C ABI called from C (the way the Fortran iso_c_binding shim calls it) and the
two launch modes of the CG loop (one conditional-WHILE graph vs host-driven stream)."""
import os
import subprocess

import numpy as np
import pytest

from frontistr_b200.mesh import box_system
from frontistr_b200.solver import GpuSolver
from oracle_ctypes import Oracle

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "frontistr_b200", "lib")


def test_c_driver(tmp_path):
    exe = str(tmp_path / "drop_in_driver")
    subprocess.check_call(["gcc", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "c_driver", "drop_in_driver.c"), "-o", exe,
                           "-L", LIB, "-lhecmw33_gpu", "-lfistr_assemble", "-Wl,-rpath," + LIB])
    out = subprocess.run([exe, "8"], capture_output=True, text=True, check=True).stdout.split("\n")
    first = out[0].split()
    second = out[1].split()
    m = box_system(8, 8, 16)
    m.set_iter(20000)
    ref = Oracle(m).solve()
    assert int(first[3]) == 0 and int(first[2]) == 1
    assert abs(int(first[0]) - ref["iter"]) <= 2
    assert float(first[1]) <= 1e-8
    assert int(second[0]) == int(first[0])  # same matrix, recycled preconditioner


def test_stream_mode_matches_graph_mode(monkeypatch):
    m = box_system(12, 10, 20, jitter=0.1, seed=5)
    m.set_iter(20000)
    with GpuSolver() as s:
        a = m.copy()
        ia = s.solve(a)
        monkeypatch.setenv("HECMW33_GRAPH", "0")
        b = m.copy()
        ib = s.solve(b)
    assert ia["iter"] == ib["iter"]
    assert np.array_equal(a.X, b.X)
