"""Block ILU(1) and ILU(2) (PRECOND = 11, 12; hecmw_precond_BILU_33.f90 FORM_ILU1_33,
FORM_ILU2_33).  The fill of row i: level 1 = original L(i,k) x original U(k,j) not in
row i; level 2 (ILU(2)) = original L(i,k) x level-1 U(k,j) and level-1 L(i,k) x
original U(k,j).  The elimination uses L(i,k), U(k,j) whose levels sum below the ILU
level and, unlike ILU(0), updates the diagonal block too.

CPU: the oracle's factor pattern equals an independent restatement of that rule (sets
in Python); its ILU(1) / ILU(2) solves converge in fewer iterations than ILU(0) to the
same solution.  GPU: z = M^-1 r of the device factor agrees with the oracle's
(1e-12 relative), and the solves match the oracle's (iterations within 2, solution
within 1e-8 relative, true residual below the tolerance), also with the factor
stored in BF16 (Iarray(42) = 1).
"""
import numpy as np
import pytest

from frontistr_b200.mesh import box_system
from oracle_ctypes import Oracle
from test_bicgstab import _flags


def _rule(m, level):
    """Row patterns (1-based columns) of the reference's block ILU(level)."""
    n = m.NP
    L = [set(int(c) for c in m.itemL[m.indexL[i]:m.indexL[i + 1]]) for i in range(n)]
    U = [set(int(c) for c in m.itemU[m.indexU[i]:m.indexU[i + 1]]) for i in range(n)]
    f1 = [set() for _ in range(n)]
    for i in range(1, n):
        have = {i + 1} | L[i] | U[i]
        for k in sorted(L[i]):
            for j in sorted(U[k - 1]):
                if j not in have:
                    f1[i].add(j)
                    have.add(j)
    f2 = [set() for _ in range(n)]
    if level >= 2:
        for i in range(1, n):
            have = {i + 1} | L[i] | U[i] | f1[i]
            for k in sorted(L[i]):
                for j in sorted(c for c in f1[k - 1] if c > k):
                    if j not in have:
                        f2[i].add(j)
                        have.add(j)
            for k in sorted(c for c in f1[i] if c < i + 1):
                for j in sorted(U[k - 1]):
                    if j not in have:
                        f2[i].add(j)
                        have.add(j)
    lo = [sorted(L[i] | {c for c in f1[i] | f2[i] if c < i + 1}) for i in range(n)]
    up = [sorted(U[i] | {c for c in f1[i] | f2[i] if c > i + 1}) for i in range(n)]
    return lo, up


def _system(seed=3, dims=(8, 7, 9)):
    return box_system(*dims, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=seed)


@pytest.mark.parametrize("level", [1, 2])
@pytest.mark.parametrize("seed", [3, 8])
def test_oracle_fill_pattern(level, seed):
    m = _system(seed, (5, 4, 6))
    pc = Oracle(m).precond(10 + level)
    assert pc.error == 0
    inL, iaL, inU, iaU = pc.bilu_pattern()
    lo, up = _rule(m, level)
    for i in range(m.NP):
        assert list(iaL[inL[i]:inL[i + 1]]) == lo[i]
        assert list(iaU[inU[i]:inU[i + 1]]) == up[i]
    assert inL[-1] + inU[-1] > m.NPL + m.NPU  # the fill is there


def test_oracle_fill_solves():
    m = _system()
    out = {}
    for pc in (10, 11, 12):
        g = _flags(m, pc, 1)
        out[pc] = Oracle(m).solve(Iarray=g.Iarray, Rarray=g.Rarray)
        assert out[pc]["error"] == 0 and out[pc]["resid_true"] < 1e-8
    assert out[12]["iter"] < out[11]["iter"] < out[10]["iter"]
    for pc in (11, 12):
        assert np.linalg.norm(out[pc]["X"] - out[10]["X"]) <= 1e-6 * np.linalg.norm(out[10]["X"])


@pytest.mark.gpu
@pytest.mark.parametrize("level", [1, 2])
def test_gpu_fill_apply_matches_oracle(level):
    from frontistr_b200.solver import GpuSolver
    m = _system(seed=7, dims=(10, 9, 11))
    g = _flags(m, 10 + level, 1)
    r = np.random.default_rng(2).standard_normal(3 * m.NP)
    with GpuSolver() as s:
        s.set_matrix(m)
        z = s.precond_apply(r, g.Iarray.copy(), g.Rarray.copy())
    zo = Oracle(m).precond(10 + level).apply(r)
    assert np.linalg.norm(z - zo) <= 1e-12 * np.linalg.norm(zo)


@pytest.mark.gpu
@pytest.mark.parametrize("level,mode", [(1, 0), (2, 0), (1, 1)])
def test_gpu_fill_solve_matches_oracle(level, mode):
    from frontistr_b200.solver import GpuSolver
    m = _system(seed=7, dims=(10, 9, 11))
    g = _flags(m, 10 + level, 1)
    g.Iarray[41] = mode
    ref = Oracle(m).solve(Iarray=g.Iarray, Rarray=g.Rarray)
    with GpuSolver() as s:
        info = s.solve(g)
    assert info["error"] == ref["error"] == 0
    assert abs(info["iter"] - ref["iter"]) <= 2, (info["iter"], ref["iter"])
    assert np.linalg.norm(g.X - ref["X"]) <= 1e-8 * np.linalg.norm(ref["X"])
    assert Oracle(m).rel_resid(g.X, m.B) < 1e-8
    assert g.get_flag_converged() == 1
