"""ESTCOND (Iarray(14)): the Lanczos condition estimate of hecmw_solve_CG
(hecmw_solver_CG.f90:256-264, 299-301; hecmw_estimate_condition.F90:14-99).  The CG's
ALPHA / BETA give the tridiagonal D(k) = 1/ALPHA(k) + BETA(k)/ALPHA(k-1),
E(k-1) = sqrt(BETA(k))/ALPHA(k-1); its extreme eigenvalues estimate those of M^-1 A.

CPU: on a small box the oracle's Lanczos extremes approach the extreme eigenvalues of
M^-1 A from a dense eigen-decomposition.  GPU: the device records ALPHA / BETA in the
graph-captured CG; its estimate (bisection on the Sturm count) matches numpy's
eigenvalues of the oracle's tridiagonal, the "emin=..., emax=..., emax/emin=..." lines
are printed every ESTCOND iterations and at the end, and nothing is recorded when
ESTCOND is 0.
"""
import re

import numpy as np
import pytest

from frontistr_b200.matrix import IDX_I_ESTCOND
from frontistr_b200.mesh import box_system
from oracle_ctypes import Oracle


def _lanczos_extremes(alpha, beta):
    n = len(alpha)
    d = np.empty(n)
    e = np.empty(max(n - 1, 0))
    d[0] = 1.0 / alpha[0]
    for k in range(1, n):
        d[k] = 1.0 / alpha[k] + beta[k] / alpha[k - 1]
        e[k - 1] = np.sqrt(beta[k]) / alpha[k - 1]
    T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    w = np.linalg.eigvalsh(T)
    return w[0], w[-1]


def test_oracle_lanczos_estimates_the_spectrum():
    m = box_system(4, 3, 5, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=2)
    o = Oracle(m)
    pc = o.precond(1)
    r = pc.cg_lanczos(m.B, tol=1e-12)
    assert r["error"] == 0
    lo, hi = _lanczos_extremes(r["alpha"], r["beta"])
    n = 3 * m.N
    A = np.column_stack([o.matvec(np.eye(n)[:, j]) for j in range(n)])
    MA = np.column_stack([pc.apply(A[:, j]) for j in range(n)])
    w = np.sort(np.linalg.eigvals(MA).real)
    # (the largest eigenvalue, 1, belongs to the constrained rows, which the right-hand
    # side does not excite: Lanczos approaches it from below)
    assert abs(hi - w[-1]) <= 1e-3 * w[-1]
    assert abs(lo - w[0]) <= 1e-3 * w[0]


@pytest.mark.gpu
def test_gpu_estcond(capfd):
    from frontistr_b200.solver import GpuSolver
    m = box_system(9, 8, 10, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=11)
    m.set_iter(20000)
    ref = Oracle(m).precond(1).cg_lanczos(m.B)
    lo, hi = _lanczos_extremes(ref["alpha"], ref["beta"])
    with GpuSolver() as s:
        g = m.copy()
        info0 = s.solve(g)
        assert s.condition_estimate()[0] == 0
        g = m.copy()
        g.Iarray[IDX_I_ESTCOND - 1] = 20
        capfd.readouterr()
        info = s.solve(g)
        n, emin, emax = s.condition_estimate()
    out = capfd.readouterr().out
    assert info["error"] == 0 and info["iter"] == info0["iter"]
    assert abs(n - ref["iter"]) <= 2 and n == info["iter"]
    assert abs(emin - lo) <= 1e-6 * lo and abs(emax - hi) <= 1e-6 * hi
    lines = [l for l in out.splitlines() if l.startswith("emin=")]
    assert len(lines) == n // 20 + 1
    last = re.match(r"emin= ?([-+0-9.E]+), emax= ?([-+0-9.E]+), emax/emin= ?([-+0-9.E]+)", lines[-1])
    assert last and abs(float(last.group(1)) - emin) <= 1e-6 * emin


@pytest.mark.gpu
def test_gpu_estcond_gmres(capfd):
    """GMRES (hecmw_solver_GMRES.f90:290-291, 416-417): the extreme singular values of the
    rotated Hessenberg's leading I x I block, every ESTCOND iterations and at the end."""
    from frontistr_b200.solver import GpuSolver
    m = box_system(9, 8, 10, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=11)
    m.set_iter(20000)
    m.set_method(3)
    m.Iarray[5] = 40  # NREST
    ref = Oracle(m).precond(1).gmres_hess(m.B, 40)
    n = ref["I"]
    H = ref["H"][:n, :n].copy()
    H[np.tril_indices(n, -2)] = 0.0
    sv = np.linalg.svd(H, compute_uv=False)
    g = m.copy()
    g.Iarray[IDX_I_ESTCOND - 1] = 7
    with GpuSolver() as s:
        capfd.readouterr()
        info = s.solve(g)
        k, emin, emax = s.condition_estimate()
    out = capfd.readouterr().out
    assert info["error"] == 0 and info["iter"] == ref["iter"]
    assert k == n
    assert abs(emin - sv.min()) <= 1e-6 * sv.min() and abs(emax - sv.max()) <= 1e-6 * sv.max()
    lines = [l for l in out.splitlines() if l.startswith("emin=")]
    assert len(lines) == info["iter"] // 7 + 1


@pytest.mark.gpu
def test_gpu_iterlog(capfd):
    """ITERLOG (Iarray(21) = 1): the CG's ITERATION HISTORY lines, ITER and RESID in the
    reference's '(i7, 1pe16.6)' (hecmw_solver_CG.f90:251-253): one per iteration, the
    recursive residual (every 50th iteration the recomputed one), as the oracle's."""
    from frontistr_b200.solver import GpuSolver
    m = box_system(9, 8, 10, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=11)
    m.set_iter(20000)
    ref = Oracle(m).precond(1).cg(m.B, hist=True)
    with GpuSolver() as s:
        capfd.readouterr()
        info0 = s.solve(m.copy())
        quiet = capfd.readouterr().out
        g = m.copy()
        g.Iarray[20] = 1
        info = s.solve(g)
        out = capfd.readouterr().out
    assert not re.search(r"^ *\d+ +[-+0-9.]+E[-+]\d+$", quiet, re.M)
    lines = [l for l in out.splitlines() if re.match(r"^ *\d+ +[-+0-9.]+E[-+]\d+$", l)]
    assert info["iter"] == info0["iter"] and len(lines) == info["iter"]
    assert abs(info["iter"] - ref["iter"]) <= 2
    # every line, the recomputed true residuals of iterations 50, 100, ... and the
    # last (recompute-on-convergence) among them; the device and the oracle sum in
    # different orders, so late values agree to a looser bound than early ones
    n = min(len(lines), ref["iter"])
    for k, l in enumerate(lines[:n]):
        it, res = l.split()
        assert int(it) == k + 1 and len(l) == 23
        bound = 1e-5 if k < 20 else 1e-3
        assert abs(float(res) - ref["hist"][k]) <= bound * ref["hist"][k], (k + 1, res, ref["hist"][k])
    for k in (48, 49, 50):
        if k < n:
            assert abs(float(lines[k].split()[1]) - ref["hist"][k]) <= 1e-4 * ref["hist"][k], k + 1
    assert float(lines[-1].split()[1]) <= 1e-8 and ref["hist"][ref["iter"] - 1] <= 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("method,width", [(2, 23), (3, 32), (4, 21), (5, 23), (6, 23), (7, 23)])
def test_gpu_iterlog_other_methods(capfd, method, width):
    """ITERLOG with the other methods: one history line per iteration in each
    reference's format -- BiCGSTAB, CR, GMRESR, GMRESREN '(i7, 1pe16.6)', GMRES
    '(2i8, 1pe16.6)' (iter, step, RESID), GPBiCG '(i5, 1pe16.6)'."""
    from frontistr_b200.solver import GpuSolver
    m = box_system(7, 6, 8, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=13)
    m.set_iter(20000)
    m.set_method(method)
    m.Iarray[5] = 30
    m.Iarray[20] = 1
    with GpuSolver() as s:
        capfd.readouterr()
        info = s.solve(m)
        out = capfd.readouterr().out
    lines = [l for l in out.splitlines() if re.match(r"^ *\d+( +\d+)? +[-+0-9.]+E[-+]\d+$", l)]
    assert info["error"] == 0 and len(lines) == info["iter"]
    assert all(len(l) == width for l in lines)
    assert [int(l.split()[0]) for l in lines] == list(range(1, info["iter"] + 1))
