"""MPC-CG (MPC_METHOD = Iarray(13) = 2; hecmw_solver_Iterative.f90:79-84,
hecmw_TtmatTvec_33 in hecmw_solver_las_33.F90:442-586).  With the mesh's MPCs (the
first term of each is its slave) every product of the solve is T^T A T x: T sets each
slave DOF to -sum val_j x(master_j), T^T zeroes the slave and moves -val_j times its
value onto the masters.  The caller hands the solver T^T b; the physical solution is
T x.

CPU: the oracle's MPC-CG converges, and T x equals a dense solve of the reduced system
(the non-slave DOFs of T^T A T) and satisfies every MPC.  GPU: the device MPC-CG
matches the oracle (iterations within 2, T x within 1e-8 relative, its true residual
below the tolerance); registered MPCs with another MPC_METHOD leave the solve as it is.
Both: the MPC constants enter the zero-RHS check (a zero B with nonzero constants is
solved, X = 0, without the 2002 warning).
"""
import numpy as np
import pytest

from frontistr_b200.matrix import IDX_I_MPC_METHOD
from frontistr_b200.mesh import box_system
from oracle_ctypes import Oracle

NX, NY, NZ = 6, 5, 8


def _mpcs():
    """Ties on the loaded top face: u_y of some nodes equal to a neighbour's, u_x of
    others the mean of two neighbours' (1-based nodes, x fastest)."""
    nxn, nyn = NX + 1, NY + 1
    top = NZ * nxn * nyn  # first node of the top layer, 0-based
    node = lambda i, j: top + j * nxn + i + 1
    terms = []
    for i in range(1, NX, 2):
        terms.append([(node(i, 2), 2, 1.0), (node(i - 1, 2), 2, -1.0)])
    for i in range(1, NX - 1, 2):
        terms.append([(node(i, 4), 1, 1.0), (node(i - 1, 4), 1, -0.5), (node(i + 1, 4), 1, -0.5)])
    terms.append([(node(2, 0), 4, 1.0), (node(3, 0), 4, -1.0)])  # a rotational DOF: left out
    index, item, dof, val = [0], [], [], []
    for t in terms:
        for n, d, v in t:
            item.append(n)
            dof.append(d)
            val.append(v)
        index.append(len(item))
    return (np.array(index, np.int32), np.array(item, np.int32), np.array(dof, np.int32),
            np.array(val, np.float64), np.zeros(len(terms)))


def _t(x, mpc, transpose=False):
    index, item, dof, val, _ = mpc
    y = x.copy()
    for i in range(len(index) - 1):
        js = range(index[i], index[i + 1])
        if any(dof[j] > 3 for j in js):
            continue
        k = index[i]
        kk = 3 * (item[k] - 1) + dof[k] - 1
        y[kk] = 0.0
        for j in range(k + 1, index[i + 1]):
            jj = 3 * (item[j] - 1) + dof[j] - 1
            if transpose:
                y[jj] -= val[j] * x[kk]
            else:
                y[kk] -= val[j] * x[jj]
    return y


def _system():
    m = box_system(NX, NY, NZ, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=5)
    m.set_iter(20000)
    mpc = _mpcs()
    m.B = _t(m.B, mpc, transpose=True)  # T^T b
    m.mpc = mpc
    m.Iarray[IDX_I_MPC_METHOD - 1] = 2
    return m, mpc


def _slaves(mpc):
    index, item, dof, _, _ = mpc
    return [3 * (item[index[i]] - 1) + dof[index[i]] - 1 for i in range(len(index) - 1)
            if all(dof[j] <= 3 for j in range(index[i], index[i + 1]))]


@pytest.mark.parametrize("precond", [1, 3])
def test_oracle_mpc_cg(precond):
    m, mpc = _system()
    m.set_precond(precond)
    r = Oracle(m).solve()
    assert r["error"] == 0 and r["resid_true"] < 1e-8
    u = _t(r["X"], mpc)
    # dense reduced solve: the non-slave DOFs of T^T A T
    n = 3 * m.N
    A = m.to_scipy().toarray()
    T = np.column_stack([_t(np.eye(n)[:, j], mpc) for j in range(n)])
    keep = np.setdiff1d(np.arange(n), _slaves(mpc))
    K = (T.T @ A @ T)[np.ix_(keep, keep)]
    xr = np.zeros(n)
    xr[keep] = np.linalg.solve(K, m.B[keep])
    ud = T @ xr
    assert np.linalg.norm(u - ud) <= 1e-7 * np.linalg.norm(ud)
    index, item, dof, val, _ = mpc
    for i in range(len(index) - 1):  # every MPC with DOFs 1-3 holds in T x
        js = range(index[i], index[i + 1])
        if any(dof[j] > 3 for j in js):
            continue
        s = sum(val[j] * u[3 * (item[j] - 1) + dof[j] - 1] for j in js)
        assert abs(s) <= 1e-12 * np.abs(u).max()


@pytest.mark.gpu
@pytest.mark.parametrize("precond", [1, 3, 10])
def test_gpu_mpc_cg_matches_oracle(precond):
    from frontistr_b200.solver import GpuSolver
    m, mpc = _system()
    m.set_precond(precond)
    ref = Oracle(m).solve()
    g = m.copy()
    with GpuSolver() as s:
        s.set_matrix(g)
        s.set_mpc(*mpc)
        info = s.solve_resident(g.B, g.X, g.Iarray, g.Rarray)
    assert info["error"] == ref["error"] == 0
    assert abs(info["iter"] - ref["iter"]) <= 2, (info["iter"], ref["iter"])
    u, uo = _t(g.X, mpc), _t(ref["X"], mpc)
    assert np.linalg.norm(u - uo) <= 1e-8 * np.linalg.norm(uo)
    assert g.get_flag_converged() == 1


@pytest.mark.gpu
def test_gpu_mpc_other_method_is_the_plain_solve():
    from frontistr_b200.solver import GpuSolver
    m, mpc = _system()
    m.Iarray[IDX_I_MPC_METHOD - 1] = 0
    plain = m.copy()
    plain.mpc = None
    ref = Oracle(plain).solve()
    g = m.copy()
    with GpuSolver() as s:
        s.set_matrix(g)
        s.set_mpc(*mpc)
        info = s.solve_resident(g.B, g.X, g.Iarray, g.Rarray)
    assert info["error"] == 0 and abs(info["iter"] - ref["iter"]) <= 2
    assert np.linalg.norm(g.X - ref["X"]) <= 1e-8 * np.linalg.norm(ref["X"])


def _zero_rhs_case(const):
    m, mpc = _system()
    m.B[:] = 0.0
    mpc = mpc[:4] + (np.full(len(mpc[0]) - 1, const),)
    m.mpc = mpc
    return m, mpc


def test_oracle_mpc_constants_in_the_zero_rhs_check():
    """hecmw_solve_check_zerorhs adds sum mpc_const^2 (hecmw_solver_Iterative.f90:305-309)."""
    m, _ = _zero_rhs_case(0.0)
    assert Oracle(m).solve()["error"] == 2002
    m, _ = _zero_rhs_case(0.5)
    r = Oracle(m).solve()
    assert r["error"] == 0 and not np.any(r["X"])


@pytest.mark.gpu
def test_gpu_mpc_constants_in_the_zero_rhs_check():
    from frontistr_b200.solver import GpuSolver
    for const, code in ((0.0, 2002), (0.5, 0)):
        m, mpc = _zero_rhs_case(const)
        ref = Oracle(m).solve()
        with GpuSolver() as s:
            s.set_matrix(m)
            s.set_mpc(*mpc)
            info = s.solve_resident(m.B, m.X, m.Iarray, m.Rarray)
        assert info["error"] == ref["error"] == code
        assert not np.any(m.X)


@pytest.mark.gpu
def test_gpu_hecmw_solve_passes_the_mpc_table():
    """The Python hecmw_solve hands hecMAT.mpc to the solver, as the shim does hecMESH%mpc."""
    from frontistr_b200.solver import GpuSolver, hecmw_solve
    m, mpc = _system()
    ref = Oracle(m).solve()
    g = m.copy()
    with GpuSolver() as s:
        info = hecmw_solve(g, solver=s)
    assert info["error"] == ref["error"] == 0
    assert abs(info["iter"] - ref["iter"]) <= 2
    assert np.linalg.norm(_t(g.X, mpc) - _t(ref["X"], mpc)) <= 1e-8 * np.linalg.norm(_t(ref["X"], mpc))
