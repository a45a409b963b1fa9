"""Host generator of the Neo-Hookean Newton systems (no GPU): the element tangent is
the exact derivative of the residual (central finite differences), symmetric, zero
residual at rest, and at zero displacement equals the linear-elastic stiffness with
E = 9 kappa mu / (3 kappa + mu), nu = (3 kappa - 2 mu) / (2 (3 kappa + mu)),
mu = 2 C10, kappa = 2 / D1; a short Newton sequence converges quadratically with a
direct solver."""
import numpy as np
import scipy.sparse.linalg as spla

from frontistr_b200.mesh import box_system
from frontistr_b200.newton import NeoHookeBox, newton_sequence


def test_tangent_is_the_residual_derivative():
    b = NeoHookeBox(2, 2, 3, C10=1.0, D1=0.01)
    rng = np.random.default_rng(0)
    U = 0.05 * rng.standard_normal(3 * b.N)
    K = b.tangent(U).to_scipy().toarray()
    assert np.abs(K - K.T).max() <= 1e-12 * np.abs(K).max()
    du = rng.standard_normal(3 * b.N)
    eps = 1e-6
    fd = -(b.tangent(U + eps * du).B - b.tangent(U - eps * du).B) / (2 * eps)
    assert np.linalg.norm(K @ du - fd) <= 1e-7 * np.linalg.norm(fd)


def test_small_strain_limit_is_linear_elasticity():
    C10, D1 = 1.0, 0.01
    b = NeoHookeBox(2, 2, 2, C10=C10, D1=D1)
    m0 = b.tangent(np.zeros(3 * b.N))
    assert np.abs(m0.B).max() == 0.0
    mu, kappa = 2 * C10, 2 / D1
    E = 9 * kappa * mu / (3 * kappa + mu)
    nu = (3 * kappa - 2 * mu) / (2 * (3 * kappa + mu))
    lin = box_system(2, 2, 2, E=E, nu=nu)  # clamped bottom: compare nodes above it
    top = slice(9 * 9, 9 * b.N)
    assert np.allclose(m0.D[top], lin.D[top], rtol=1e-12, atol=1e-12 * np.abs(lin.D).max())


def test_newton_converges_quadratically():
    b = NeoHookeBox(2, 2, 4, C10=1.0, D1=0.01)

    def solve(inc, it, m):
        return spla.spsolve(m.to_scipy().tocsc(), m.B)

    recs = list(newton_sequence(b, solve, top_uz=-0.4, n_incr=2, max_newton=8, tol=1e-9))
    for inc in (1, 2):
        r = [x["residual"] for x in recs if x["increment"] == inc]
        assert recs[-1]["converged"] or r[-1] < 1e-8
        assert len(r) <= 6
    # the top face ended at -0.4 in z
    assert np.allclose(b.U[3 * b.top + 2], -0.4)
