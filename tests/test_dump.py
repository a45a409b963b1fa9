"""Dump files of hecmw_matrix_dump.f90 (DUMPTYPE=MM/CSR/BSR, .rhs/.sol, DUMPEXIT):
the Fortran e20.12e3 value format, write/read round trips of all three matrix
formats, the file names and calls of hecmw_solve_iterative, and a dumped matrix
solving to the same answer as the original."""
import os

import numpy as np
import pytest

from frontistr_b200 import dump
from frontistr_b200.matrix import IDX_I_DUMP, IDX_I_DUMP_EXIT
from frontistr_b200.mesh import box_system
from oracle_ctypes import Oracle


def test_fortran_e_format():
    assert dump.fortran_e(210000.0) == " 0.210000000000E+006"
    assert dump.fortran_e(-1.5e-10) == "-0.150000000000E-009"
    assert dump.fortran_e(0.0) == " 0.000000000000E+000"
    assert dump.fortran_e(1.0) == " 0.100000000000E+001"
    assert dump.fortran_e(9.9999999999996) == " 0.100000000000E+002"
    rng = np.random.default_rng(0)
    for v in rng.standard_normal(200) * 10.0 ** rng.integers(-200, 200, 200):
        s = dump.fortran_e(v)
        assert len(s) == 20
        assert abs(float(s) - v) <= 5e-12 * abs(v)


@pytest.mark.parametrize("fmt", ["bsr", "csr", "mm"])
def test_round_trip(tmp_path, fmt):
    m = box_system(3, 4, 2, jitter=0.2, sigma_E=1.0, seed=1)
    path = str(tmp_path / ("a." + fmt))
    {"bsr": dump.write_bsr, "csr": dump.write_csr, "mm": dump.write_mm}[fmt](m, path)
    r = dump.read_matrix(path)
    assert r.N == m.N
    for a in ("indexL", "indexU"):
        assert np.array_equal(getattr(r, a), getattr(m, a))
    assert np.array_equal(r.itemL[:m.NPL], m.itemL[:m.NPL])
    assert np.array_equal(r.itemU[:m.NPU], m.itemU[:m.NPU])
    for a, n in (("D", 9 * m.N), ("AL", 9 * m.NPL), ("AU", 9 * m.NPU)):
        x, y = getattr(r, a)[:n], getattr(m, a)[:n]
        assert np.all(np.abs(x - y) <= 5e-12 * np.abs(y))


def test_dumper_calls(tmp_path):
    m = box_system(3, 3, 3, seed=2)
    d = dump.Dumper(str(tmp_path), rank=0)
    m.Iarray[IDX_I_DUMP - 1] = 0
    d.dump(m)  # NumCall still counts the call
    m.Iarray[IDX_I_DUMP - 1] = dump.DUMP_BSR
    d.dump(m)
    m.X[:] = np.arange(3 * m.N)
    d.dump_solution(m)
    names = sorted(os.listdir(tmp_path))
    assert names == ["dump_matrix_2_0.bsr", "dump_matrix_2_0.rhs", "dump_matrix_2_0.sol"]
    assert np.allclose(dump.read_vector(str(tmp_path / "dump_matrix_2_0.rhs")), m.B, rtol=5e-12, atol=0)
    assert np.array_equal(dump.read_vector(str(tmp_path / "dump_matrix_2_0.sol")), m.X)
    m.Iarray[IDX_I_DUMP_EXIT - 1] = 1
    with pytest.raises(SystemExit):
        d.dump(m)


def test_dumped_matrix_solves_alike(tmp_path):
    m = box_system(6, 5, 7, jitter=0.1, seed=4)
    path = str(tmp_path / "m.bsr")
    dump.write_bsr(m, path)
    dump.write_vector(m.B, str(tmp_path / "m.rhs"))
    r = dump.read_bsr(path)
    r.B = dump.read_vector(str(tmp_path / "m.rhs"))
    a = Oracle(m).solve()
    b = Oracle(r).solve()
    assert a["error"] == b["error"] == 0
    assert abs(a["iter"] - b["iter"]) <= 1
    assert np.linalg.norm(a["X"] - b["X"]) <= 1e-9 * np.linalg.norm(a["X"])


@pytest.mark.gpu
def test_gpu_hecmw_solve_dumps(tmp_path):
    from frontistr_b200.solver import GpuSolver, hecmw_solve
    m = box_system(6, 5, 7, seed=4)
    m.Iarray[IDX_I_DUMP - 1] = dump.DUMP_BSR
    d = dump.Dumper(str(tmp_path))
    with GpuSolver() as s:
        info = hecmw_solve(m, solver=s, dumper=d)
        r = dump.read_bsr(str(tmp_path / "dump_matrix_1_0.bsr"))
        r.B = dump.read_vector(str(tmp_path / "dump_matrix_1_0.rhs"))
        info2 = s.solve(r)
    assert info["error"] == info2["error"] == 0
    assert abs(info["iter"] - info2["iter"]) <= 1
    sol = dump.read_vector(str(tmp_path / "dump_matrix_1_0.sol"))
    assert np.all(np.abs(sol - m.X) <= 5e-12 * np.abs(m.X))
    assert np.linalg.norm(r.X - m.X) <= 1e-9 * np.linalg.norm(m.X)
