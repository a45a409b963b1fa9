"""SCALING=YES (Iarray(7)): symmetric diagonal scaling around the CG
(hecmw_solver_scaling_33.f90:20-208, called from hecmw_solver_CG.f90:102,283).

CPU: the oracle's scaled solve reaches the tolerance on the scaled residual, its
solution agrees with the unscaled solve to the accuracy both solves reach, and
the caller's arrays are left exactly as they were.  GPU: the CUDA solve with
scaling matches the oracle's scaled solve (iterations +-2, solution 1e-8
relative, the same converged flag).
"""
import numpy as np
import pytest

from frontistr_b200.mesh import box_system
from oracle_ctypes import Oracle


def _scaled(m, precond, scaling):
    g = m.copy()
    g.set_iter(20000)
    g.set_resid(1e-8)
    g.set_precond(precond)
    g.set_scaling(scaling)
    return g


@pytest.mark.parametrize("precond", [1, 3, 10])
def test_oracle_scaling(precond):
    m = box_system(6, 7, 9, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=3)
    arrays = [a.copy() for a in (m.D, m.AL, m.AU, m.B)]
    gp = _scaled(m, precond, 0)
    plain = Oracle(m).solve(Iarray=gp.Iarray, Rarray=gp.Rarray)
    gs = _scaled(m, precond, 1)
    sc = Oracle(m).solve(Iarray=gs.Iarray, Rarray=gs.Rarray)
    assert plain["error"] == 0 and sc["error"] == 0
    for a, b in zip(arrays, (m.D, m.AL, m.AU, m.B)):
        assert np.array_equal(a, b)
    err = np.linalg.norm(sc["X"] - plain["X"]) / np.linalg.norm(plain["X"])
    assert err <= 1e-5, err
    # the scaled iteration converges on the scaled residual; the driver's flag is
    # set from the unscaled true residual
    assert sc["resid"] <= 1e-8
    assert (sc["Iarray"][80] == 1) == (Oracle(m).rel_resid(sc["X"], m.B) < 1e-8)
    assert sc["resid_true"] == Oracle(m).rel_resid(sc["X"], m.B)
    if precond == 3:
        # block-diagonal preconditioning is invariant under diagonal scaling in
        # exact arithmetic: the same iteration count up to rounding
        assert abs(sc["iter"] - plain["iter"]) <= max(2, plain["iter"] // 20)


@pytest.mark.gpu
@pytest.mark.parametrize("precond", [1, 3, 10])
def test_gpu_scaling_matches_oracle(precond):
    from frontistr_b200.solver import GpuSolver
    m = box_system(10, 9, 11, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=7)
    g = _scaled(m, precond, 1)
    arrays = [a.copy() for a in (g.D, g.AL, g.AU, g.B)]
    ref = Oracle(m).solve(Iarray=g.Iarray, Rarray=g.Rarray)
    with GpuSolver() as s:
        info = s.solve(g)
        rec = s.last_solve_info()
        # the same handle without scaling afterwards: the resident values are unscaled again
        h = _scaled(m, precond, 0)
        h.Iarray[97] = 1
        info2 = s.solve(h)
    gp = _scaled(m, precond, 0)
    plain = Oracle(m).solve(Iarray=gp.Iarray, Rarray=gp.Rarray)
    for a, b in zip(arrays, (g.D, g.AL, g.AU, g.B)):
        assert np.array_equal(a, b)
    assert info["error"] == 0 and ref["error"] == 0
    assert abs(info["iter"] - ref["iter"]) <= 2, (info["iter"], ref["iter"])
    assert np.linalg.norm(g.X - ref["X"]) <= 1e-8 * np.linalg.norm(ref["X"])
    if abs(ref["resid_true"] - 1e-8) > 1e-9:  # not at the threshold itself
        assert g.get_flag_converged() == ref["Iarray"][80]
    assert abs(rec["true_resid"] - Oracle(m).rel_resid(g.X, m.B)) <= 1e-3 * rec["true_resid"] + 1e-16
    assert info2["error"] == 0 and abs(info2["iter"] - plain["iter"]) <= 2
    assert np.linalg.norm(h.X - plain["X"]) <= 1e-8 * np.linalg.norm(plain["X"])
