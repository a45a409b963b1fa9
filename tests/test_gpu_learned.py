"""Learned preconditioner (Iarray(43) = 1): GPU forward/backward against the CPU
reference (tests/gnn_reference.py, itself checked by finite differences), training
on pairs recorded from earlier solves, what the trained network gains over SSOR
alone, the SSOR-CG fallback, and its use inside mixed precision.

Tolerances: the GPU network runs in FP32 (weights, activations, FP32 SSOR copy)
against the FP64 reference, so values agree to ~1e-5 relative and gradients to
~1e-3 of the largest component."""
import numpy as np
import pytest

import gnn_reference as G
from frontistr_b200.mesh import box_system
from frontistr_b200.solver import GpuSolver
from oracle_ctypes import Oracle

pytestmark = pytest.mark.gpu


def build_ssor(s, m):
    m = m.copy()
    s.set_matrix(m)
    s.precond_apply(np.zeros(3 * m.N), m.Iarray.copy(), m.Rarray.copy())


def test_forward_and_gradient_match_cpu_reference():
    m = box_system(3, 3, 4, jitter=0.15, sigma_E=0.5, seed=0)
    g = G.Graph(m)
    A = m.to_scipy()
    rng = np.random.default_rng(1)
    e = rng.standard_normal(3 * m.N)
    r = A @ e
    theta = G.init_params(seed=1, scale_out=0.3).astype(np.float32)
    zs = Oracle(m).precond(1).apply(r)
    z_ref, cache = G.forward(theta.astype(np.float64), g, zs, r)
    L_ref, dz = G.energy_loss(A, z_ref, e, r)
    grad_ref = G.backward(theta.astype(np.float64), g, cache, dz)
    with GpuSolver() as s:
        build_ssor(s, m)
        z, L, grad = s.learn_eval(theta, r, e)
    assert np.linalg.norm(z - z_ref) <= 1e-5 * np.linalg.norm(z_ref)
    assert abs(L - L_ref) <= 1e-4 * abs(L_ref)
    scale = np.abs(grad_ref).max()
    assert np.abs(grad - grad_ref).max() <= 2e-3 * scale
    assert np.dot(grad, grad_ref) / (np.linalg.norm(grad) * np.linalg.norm(grad_ref)) > 0.9999


def _solve(s, m, learned=0, mixed=0, tol=1e-8):
    g = m.copy()
    g.set_iter(20000)
    g.set_resid(tol)
    g.Iarray[42] = learned
    g.Iarray[41] = mixed
    info = s.solve(g)
    return g, info, s.last_solve_info()


def _load_cases(m, k, seed):
    """k right-hand sides: the cantilever load plus random top-face tractions."""
    rng = np.random.default_rng(seed)
    out = [m.B.copy()]
    top = np.nonzero(np.abs(m.B) > 0)[0] // 3
    for _ in range(k - 1):
        b = np.zeros_like(m.B)
        t = rng.standard_normal(3)
        t /= np.linalg.norm(t)
        for node in np.unique(top):
            b[3 * node:3 * node + 3] = t
        out.append(b)
    return out


def test_training_gain_fallback_and_mixed():
    m = box_system(10, 10, 24, jitter=0.15, sigma_E=0.5, nu_range=(0.25, 0.4), seed=2)
    loads = _load_cases(m, 6, seed=3)
    with GpuSolver() as s:
        # increments 1-3: plain FP64 SSOR-CG, recording (r, e) pairs
        s.learn_record(1, max_pairs=24)
        plain_iters = []
        for b in loads[:3]:
            mm = m.copy()
            mm.B = b
            g, info, rec = _solve(s, mm)
            assert info["error"] == 0
            plain_iters.append(info["iter"])
        n_pairs = s.learn_record(0)
        assert n_pairs >= 10
        l0, l1 = s.learn_train(steps=150, lr=2e-3)
        assert np.isfinite(l1) and l1 < l0, (l0, l1)
        theta = s.learn_get_weights()
        assert theta is not None and theta.size == G.n_params()

        # what the network gains over SSOR alone on held-out pairs (from a new load case)
        mm = m.copy()
        mm.B = loads[4]
        ref = Oracle(mm).precond(1).cg(mm.B, maxit=20000, hist=False)
        xstar = ref["X"]
        A = mm.to_scipy()
        gains = []
        zero = theta.copy()
        zero[-3 * G.WIDTH:] = 0.0  # W_out = 0: the preconditioner reduces to SSOR
        pc = Oracle(mm).precond(1)
        for k in (2, 8, 32):
            x = pc.cg(mm.B, maxit=k)["X"]  # the k-th SSOR-CG iterate of a new load case
            e = xstar - x
            r = A @ e
            _, L_net, _ = s.learn_eval(theta, r, e)
            _, L_ssor, _ = s.learn_eval(zero, r, e)
            gains.append((L_ssor, L_net))
        s.learn_set_weights(theta)
        assert all(Ln < Ls for Ls, Ln in gains), gains

        # increments 4-6 with the learned preconditioner, FP64 and mixed
        for b in loads[3:]:
            mm = m.copy()
            mm.B = b
            g, info, rec = _solve(s, mm, learned=1)
            assert info["error"] == 0 and rec["learned"] == 1
            assert Oracle(mm).rel_resid(g.X, mm.B) <= 1e-8
            g2, info2, rec2 = _solve(s, mm, learned=1, mixed=1)
            assert info2["error"] == 0
            assert Oracle(mm).rel_resid(g2.X, mm.B) <= 1e-8

        # a deliberately bad network: the device falls back to SSOR-CG and converges
        bad = theta.copy()
        bad[-3 * G.WIDTH:] = 50.0 * np.random.default_rng(4).standard_normal(3 * G.WIDTH)
        s.learn_set_weights(bad)
        mm = m.copy()
        g, info, rec = _solve(s, mm, learned=1)
        assert info["error"] == 0
        assert rec["fallback"] > 0
        assert Oracle(mm).rel_resid(g.X, mm.B) <= 1e-8
