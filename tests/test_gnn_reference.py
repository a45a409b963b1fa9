"""The CPU reference of the learned two-level preconditioner checks itself: the
coarse-space loss's gradient in omega and the whole chain's gradient in the network
weights against central finite differences, omega = 1/2 from an untrained output
layer, and the coarse correction's algebra (an A-orthogonal projection).  Also the
library's host aggregation (through the C ABI) on small meshes: every node in one
connected aggregate, 3x3x3-node aggregates after one pass on a box."""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.csgraph as csg

import gnn_reference as G
from frontistr_b200.mesh import box_system
from frontistr_b200.solver import coarse_aggregates


def small_case(seed=0, n=(3, 3, 4)):
    m = box_system(*n, jitter=0.15, sigma_E=0.5, seed=seed)
    g = G.Graph(m)
    _, agg = coarse_aggregates(m)
    c = G.Coarse(m, g, agg)
    A = m.to_scipy()
    rng = np.random.default_rng(seed)
    pairs = []
    for _ in range(2):
        e = rng.standard_normal(3 * m.N) * c.mask
        pairs.append((A @ e, e))
    return m, g, c, pairs


def test_omega_gradient_matches_finite_differences():
    m, g, c, pairs = small_case()
    rng = np.random.default_rng(1)
    om = rng.uniform(0.2, 0.8, 3 * m.N)
    L, grad = c.loss_and_grad(om, pairs)
    assert 0.0 < L < 1.0
    for k in rng.choice(om.size, 40, replace=False):
        h = 1e-6
        op, omm = om.copy(), om.copy()
        op[k] += h
        omm[k] -= h
        fd = (c.loss_and_grad(op, pairs)[0] - c.loss_and_grad(omm, pairs)[0]) / (2 * h)
        assert abs(fd - grad[k]) <= 1e-6 * max(1e-3, abs(fd)) + 1e-9, (k, fd, grad[k])


def test_theta_gradient_matches_finite_differences():
    m, g, c, pairs = small_case(seed=2)
    theta = G.init_params(seed=3, scale_out=0.3)
    L, grad, _ = G.loss_and_theta_grad(theta, g, c, pairs)
    rng = np.random.default_rng(4)
    for k in rng.choice(theta.size, 40, replace=False):
        h = 1e-6 * max(1.0, abs(theta[k]))
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (G.loss_and_theta_grad(tp, g, c, pairs)[0] - G.loss_and_theta_grad(tm, g, c, pairs)[0]) / (2 * h)
        assert abs(fd - grad[k]) <= 1e-5 * max(1e-3, abs(fd)) + 1e-9, (k, fd, grad[k])


def test_untrained_network_gives_half_and_projection():
    m, g, c, pairs = small_case(seed=5)
    out, _ = G.forward(G.init_params(seed=6, scale_out=0.0), g, c.x)
    assert np.array_equal(G.omega_of(out), np.full_like(out, 0.5))
    # P Ac^-1 P^T A is an A-orthogonal projection: applying it twice changes nothing
    P = c.prolongator(np.full(3 * m.N, 0.5))
    A = c.A
    Ac = (P.T @ A @ P).toarray()
    v = np.random.default_rng(7).standard_normal(3 * m.N)
    pv = P @ np.linalg.solve(Ac, P.T @ (A @ v))
    ppv = P @ np.linalg.solve(Ac, P.T @ (A @ pv))
    assert np.linalg.norm(ppv - pv) <= 1e-10 * np.linalg.norm(pv)
    # constrained DOFs carry no coarse basis
    assert np.all(np.abs(P.toarray()[c.mask == 0]) == 0.0)


def test_host_aggregation_covers_connected_aggregates():
    for n, mx in (((6, 5, 8), 0), ((10, 10, 10), 40), ((4, 4, 4), 1)):
        m = box_system(*n)
        na, agg = coarse_aggregates(m, mx)
        assert agg.min() == 0 and agg.max() == na - 1
        assert np.all(np.bincount(agg, minlength=na) > 0)
        A = m.to_scipy().tocsr()
        B = sp.csr_matrix((np.ones(A.nnz), A.indices, A.indptr), shape=A.shape)
        nodes = sp.kron(sp.eye(m.N), np.ones((1, 3))).tocsr()  # node <- DOF map
        Gn = (nodes @ B @ nodes.T).tocsr()
        for a in range(na):  # the node graph restricted to an aggregate is connected
            idx = np.nonzero(agg == a)[0]
            ncomp, _ = csg.connected_components(Gn[idx][:, idx], directed=False)
            assert ncomp == 1, (n, a)
        if mx == 0:
            assert na < m.N  # the first pass always runs
    # one pass on a box: root neighbourhoods of 3x3x3 nodes
    m = box_system(8, 8, 8)
    na, agg = coarse_aggregates(m, 100000)
    assert na == 27 and np.median(np.bincount(agg)) == 27
