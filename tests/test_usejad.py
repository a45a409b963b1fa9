"""USEJAD=YES (Iarray(33)): while hecmw_solve_CG holds its jagged-diagonal copy, every
product is hecmw_JAD_MATVEC_33 (hecmw_jadm_33.f90:57-211) -- D x row by row, plus the
row's off-diagonal blocks summed from zero in L-then-U order.  It is the same
product in another summation order; the device keeps its sliced layout for it.

CPU: the oracle's JAD product agrees with the plain one to rounding (1e-14 relative)
and a USEJAD solve converges to the same solution.  GPU: the device product agrees
with the JAD product within 1e-14 relative, and a USEJAD solve matches the oracle's
USEJAD solve (iterations within 2, solution within 1e-8 relative, true residual
below the tolerance).
"""
import numpy as np
import pytest

from frontistr_b200.matrix import IDX_I_USEJAD
from frontistr_b200.mesh import box_system
from oracle_ctypes import Oracle


def _system():
    m = box_system(9, 8, 10, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=11)
    m.set_iter(20000)
    return m


def _x(m, seed=5):
    return np.random.default_rng(seed).standard_normal(3 * m.NP)


def test_oracle_jad_product_is_the_product():
    m = _system()
    o = Oracle(m)
    x = _x(m)
    y, yj = o.matvec(x), o.matvec_jad(x)
    assert np.linalg.norm(yj - y) <= 1e-14 * np.linalg.norm(y)


@pytest.mark.parametrize("precond", [1, 10])
def test_oracle_usejad_solve(precond):
    m = _system()
    m.set_precond(precond)
    a = Oracle(m).solve()
    j = m.copy()
    j.Iarray[IDX_I_USEJAD - 1] = 1
    b = Oracle(j).solve()
    assert a["error"] == b["error"] == 0
    assert abs(a["iter"] - b["iter"]) <= 2
    assert np.linalg.norm(b["X"] - a["X"]) <= 1e-8 * np.linalg.norm(a["X"])
    assert b["resid_true"] < 1e-8


@pytest.mark.gpu
def test_gpu_product_matches_jad():
    from frontistr_b200.solver import GpuSolver
    m = _system()
    x = _x(m)
    with GpuSolver() as s:
        s.set_matrix(m)
        y = s.matvec(x)
    yj = Oracle(m).matvec_jad(x)
    assert np.linalg.norm(y - yj) <= 1e-14 * np.linalg.norm(yj)


@pytest.mark.gpu
@pytest.mark.parametrize("precond", [1, 10])
def test_gpu_usejad_solve_matches_oracle(precond):
    from frontistr_b200.solver import GpuSolver
    m = _system()
    m.set_precond(precond)
    m.Iarray[IDX_I_USEJAD - 1] = 1
    ref = Oracle(m).solve()
    g = m.copy()
    with GpuSolver() as s:
        info = s.solve(g)
    assert info["error"] == ref["error"] == 0
    assert abs(info["iter"] - ref["iter"]) <= 2
    assert np.linalg.norm(g.X - ref["X"]) <= 1e-8 * np.linalg.norm(ref["X"])
    assert Oracle(m).rel_resid(g.X, m.B) < 1e-8
    assert g.get_flag_converged() == 1
