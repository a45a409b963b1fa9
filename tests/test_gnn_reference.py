"""The CPU reference of the learned preconditioner's network checks itself:
analytic gradients against central finite differences, oddness and positive
homogeneity in the residual, and z = SSOR(r) when the output layer is zero."""
import numpy as np

import gnn_reference as G
from frontistr_b200.mesh import box_system
from oracle_ctypes import Oracle


def small_case(seed=0):
    m = box_system(3, 3, 4, jitter=0.15, sigma_E=0.5, seed=seed)
    g = G.Graph(m)
    A = m.to_scipy()
    rng = np.random.default_rng(seed)
    e = rng.standard_normal(3 * m.N)
    r = A @ e
    zs = Oracle(m).precond(1).apply(r)
    return m, g, A, e, r, zs


def loss_of(theta, g, A, e, r, zs):
    z, _ = G.forward(theta, g, zs, r)
    return G.energy_loss(A, z, e, r)[0]


def test_gradient_matches_finite_differences():
    m, g, A, e, r, zs = small_case()
    theta = G.init_params(seed=1, scale_out=0.3)
    z, cache = G.forward(theta, g, zs, r)
    L, dz = G.energy_loss(A, z, e, r)
    grad = G.backward(theta, g, cache, dz)
    rng = np.random.default_rng(2)
    idx = rng.choice(theta.size, 60, replace=False)
    for k in idx:
        h = 1e-6 * max(1.0, abs(theta[k]))
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (loss_of(tp, g, A, e, r, zs) - loss_of(tm, g, A, e, r, zs)) / (2 * h)
        assert abs(fd - grad[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, grad[k])


def test_odd_and_homogeneous_and_identity_start():
    m, g, A, e, r, zs = small_case(seed=3)
    theta = G.init_params(seed=4, scale_out=0.5)
    z1, _ = G.forward(theta, g, zs, r)
    z2, _ = G.forward(theta, g, -zs, -r)
    z3, _ = G.forward(theta, g, 3.0 * zs, 3.0 * r)
    assert np.allclose(z2, -z1, rtol=1e-12, atol=1e-14 * np.abs(z1).max())
    assert np.allclose(z3, 3.0 * z1, rtol=1e-12, atol=1e-14 * np.abs(z1).max())
    theta0 = G.init_params(seed=4, scale_out=0.0)
    z0, _ = G.forward(theta0, g, zs, r)
    assert np.array_equal(z0, zs)
