"""GMRESR (METHOD = 5, hecmw_solver_GMRESR.f90, with NBFGS = Iarray(60) quasi-Newton
pairs correcting the preconditioned residual) and GMRESREN (METHOD = 6,
hecmw_solver_GMRESREN.f90), both restarted after NREST = Iarray(6) steps, and the
METHOD2 = 5 fallback of a diverged CG.  Both solvers clear the preconditioner when
they return (hecmw_precond_clear), so the next solve builds it again whatever the
recycle flags say.

GMRESREN's second orthogonalisation uses the coefficient left by the previous step
(the reference computes, then ignores, the dot it should use); it is kept, so
GMRESREN converges more slowly than GMRESR, as the reference's does.

CPU: the oracle's GMRESR / GMRESREN reach the tolerance and agree with its CG; the
ITER > MAXIT exit; the fallback.  GPU: the CUDA solvers match the oracle (iterations
within 5 % and at least 2, solutions within 1e-6 relative -- restarted methods
carry rounding differences from one cycle into the next -- and the true residual
below the tolerance), and a CG solve after GMRESR builds a new preconditioner.
"""
import numpy as np
import pytest

from frontistr_b200.mesh import box_system
from oracle_ctypes import Oracle
from test_bicgstab import _flags, _rel, shifted


def _gmresr(m, precond, method=5, nrest=10, nbfgs=0, maxit=20000, method2=0):
    g = _flags(m, precond, method, method2, maxit)
    g.Iarray[5] = nrest
    g.Iarray[59] = nbfgs
    return g


CASES = [(5, 1, 10, 0), (5, 1, 10, 3), (5, 10, 30, 0), (5, 3, 10, 3), (6, 1, 10, 0), (6, 10, 10, 0)]


@pytest.mark.parametrize("method,precond,nrest,nbfgs", CASES)
def test_oracle_gmresr(method, precond, nrest, nbfgs):
    m = box_system(8, 7, 9, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=3)
    gc, gg = _flags(m, precond, 1), _gmresr(m, precond, method, nrest, nbfgs)
    cg = Oracle(m).solve(Iarray=gc.Iarray, Rarray=gc.Rarray)
    gm = Oracle(m).solve(Iarray=gg.Iarray, Rarray=gg.Rarray)
    assert cg["error"] == 0 and gm["error"] == 0
    assert gm["resid"] <= 1e-8 and gm["Iarray"][80] == 1
    assert _rel(gm["X"], cg["X"]) <= 1e-5


def test_oracle_gmresr_maxit_and_fallback():
    m = box_system(8, 7, 9, seed=3)
    g = _gmresr(m, 3, 5, 10, 2, maxit=25)
    r = Oracle(m).solve(Iarray=g.Iarray, Rarray=g.Rarray)
    assert r["error"] == 3001 and r["iter"] == 26  # ITER > MAXIT ends the loop
    ms = shifted(box_system(5, 5, 6, seed=3), 0.05)
    h = _flags(ms, 1, 1, 5, 3000)
    h.Iarray[5] = 30
    fb = Oracle(ms).solve(Iarray=h.Iarray, Rarray=h.Rarray)
    assert fb["error"] == 0 and fb["Iarray"][80] == 1 and fb["Iarray"][81] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("method,precond,nrest,nbfgs", CASES)
def test_gpu_gmresr_matches_oracle(method, precond, nrest, nbfgs):
    from frontistr_b200.solver import GpuSolver
    m = box_system(10, 9, 11, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=7)
    g = _gmresr(m, precond, method, nrest, nbfgs)
    ref = Oracle(m).solve(Iarray=g.Iarray, Rarray=g.Rarray)
    with GpuSolver() as s:
        info = s.solve(g)
    assert info["error"] == 0 and ref["error"] == 0
    assert abs(info["iter"] - ref["iter"]) <= max(2, ref["iter"] // 20), (info["iter"], ref["iter"])
    assert _rel(g.X, ref["X"]) <= 1e-6
    assert Oracle(m).rel_resid(g.X, m.B) < 1e-8
    assert g.get_flag_converged() == ref["Iarray"][80] == 1


@pytest.mark.gpu
def test_gpu_gmresr_maxit_fallback_and_precond_clear():
    from frontistr_b200.solver import GpuSolver
    m = box_system(8, 7, 9, seed=3)
    g = _gmresr(m, 3, 5, 10, 2, maxit=25)
    ref = Oracle(m).solve(Iarray=g.Iarray, Rarray=g.Rarray)
    ms = shifted(box_system(5, 5, 6, seed=3), 0.05)
    h = _flags(ms, 1, 1, 5, 3000)
    h.Iarray[5] = 30
    ref2 = Oracle(ms).solve(Iarray=h.Iarray, Rarray=h.Rarray)
    with GpuSolver() as s:
        info = s.solve(g)
        info2 = s.solve(h)
    assert info["error"] == ref["error"] == 3001 and info["iter"] == ref["iter"] == 26
    assert _rel(g.X, ref["X"]) <= 1e-6
    assert info2["error"] == ref2["error"] == 0
    assert abs(info2["iter"] - ref2["iter"]) <= max(2, ref2["iter"] // 20)
    assert Oracle(ms).rel_resid(h.X, ms.B) < 1e-8

    # GMRESR clears the preconditioner: a CG solve that asks to recycle it (flag 96
    # set, under maxrecycle) still runs on a new SSOR of its own matrix
    m1 = box_system(8, 7, 9, seed=3)
    m2 = m1.copy()
    m2.D *= 1.5
    a = _gmresr(m1, 1, 5, 10, 0)
    ia, ra = a.Iarray, a.Rarray
    fresh = _flags(m2, 1, 1)
    ref3 = Oracle(m2).solve(Iarray=fresh.Iarray, Rarray=fresh.Rarray)
    with GpuSolver() as s:
        assert s.solve(a)["error"] == 0
        b = m2.copy()
        ia[1] = 1
        ia[96] = 1
        b.Iarray, b.Rarray = ia, ra
        info3 = s.solve(b)
    assert info3["error"] == 0
    assert abs(info3["iter"] - ref3["iter"]) <= 2
    assert _rel(b.X, ref3["X"]) <= 1e-8
