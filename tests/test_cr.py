"""Preconditioned conjugate residual (METHOD = 7, hecmw_solver_CR.f90): recursive
residual with explicit true-residual checks every 100th iteration, at RESID_REC <=
TOL and at MAXIT.  CPU: the oracle's CR converges like CG and stops at MAXIT with
3001.  GPU: the CUDA CR matches the oracle (iterations within 2, solution within
1e-8 relative, the same flags)."""
import numpy as np
import pytest

from frontistr_b200.mesh import box_system
from oracle_ctypes import Oracle
from test_bicgstab import _flags, _rel


@pytest.mark.parametrize("precond", [1, 3, 10])
def test_oracle_cr(precond):
    m = box_system(8, 7, 9, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=3)
    gc, gr = _flags(m, precond, 1), _flags(m, precond, 7)
    cg = Oracle(m).solve(Iarray=gc.Iarray, Rarray=gc.Rarray)
    cr = Oracle(m).solve(Iarray=gr.Iarray, Rarray=gr.Rarray)
    assert cg["error"] == 0 and cr["error"] == 0
    assert cr["resid"] <= 1e-8 and cr["Iarray"][80] == 1
    assert abs(cr["iter"] - cg["iter"]) <= max(5, cg["iter"] // 10)
    assert _rel(cr["X"], cg["X"]) <= 1e-5


def test_oracle_cr_maxit():
    m = box_system(8, 7, 9, seed=3)
    g = _flags(m, 3, 7, 0, 25)
    r = Oracle(m).solve(Iarray=g.Iarray, Rarray=g.Rarray)
    assert r["error"] == 3001 and r["iter"] == 25


@pytest.mark.gpu
@pytest.mark.parametrize("precond", [1, 3, 10])
def test_gpu_cr_matches_oracle(precond):
    from frontistr_b200.solver import GpuSolver
    m = box_system(10, 9, 11, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=7)
    g = _flags(m, precond, 7)
    ref = Oracle(m).solve(Iarray=g.Iarray, Rarray=g.Rarray)
    h = _flags(m, precond, 7, 0, 25)
    ref2 = Oracle(m).solve(Iarray=h.Iarray, Rarray=h.Rarray)
    with GpuSolver() as s:
        info = s.solve(g)
        info2 = s.solve(h)
    assert info["error"] == 0 and ref["error"] == 0
    assert abs(info["iter"] - ref["iter"]) <= 2, (info["iter"], ref["iter"])
    assert _rel(g.X, ref["X"]) <= 1e-8
    assert g.get_flag_converged() == ref["Iarray"][80] == 1
    assert info2["error"] == ref2["error"] == 3001 and info2["iter"] == ref2["iter"] == 25
    assert _rel(h.X, ref2["X"]) <= 1e-9
