"""Learned two-level preconditioner (Iarray(43) = 1): the symmetric two-grid cycle of
SSOR and a coarse correction whose prolongator smoothing weights come from the network
(h33_gnn.cuh, h33_coarse.cuh).

  * the GPU network output (omega), training loss and weight gradient against the CPU
    reference (tests/gnn_reference.py, itself checked by finite differences);
  * training on (r, e) pairs recorded from earlier solves lowers the loss;
  * on held-out load cases the learned preconditioner needs far fewer CG iterations
    than the method without it (SSOR-CG, the drop-in), and no more than the same
    coarse space without the network's smoothing (Iarray(44) = 1); the solution meets
    the FP64 true residual, also with the BF16-stored SSOR of precision mode 1;
  * a coarse space from a deliberately bad network still converges.

Tolerances: the GPU network runs in FP32 (weights, activations) against the FP64
reference, so omega agrees to ~1e-5, the loss to ~1e-4 and the gradient to ~1e-3 of
its largest component."""
import numpy as np
import pytest

import gnn_reference as G
from frontistr_b200.mesh import box_system
from frontistr_b200.solver import GpuSolver, coarse_aggregates
from oracle_ctypes import Oracle

pytestmark = pytest.mark.gpu


def build_ssor(s, m):
    m = m.copy()
    s.set_matrix(m)
    s.precond_apply(np.zeros(3 * m.N), m.Iarray.copy(), m.Rarray.copy())


def test_forward_and_gradient_match_cpu_reference():
    m = box_system(4, 3, 5, jitter=0.15, sigma_E=0.5, seed=0)
    g = G.Graph(m)
    _, agg = coarse_aggregates(m)
    c = G.Coarse(m, g, agg)
    A = m.to_scipy()
    rng = np.random.default_rng(1)
    e = rng.standard_normal(3 * m.N) * c.mask
    r = A @ e
    r32 = r.astype(np.float32).astype(np.float64)  # the GPU keeps pairs in FP32
    e32 = e.astype(np.float32).astype(np.float64)
    theta = G.init_params(seed=1, scale_out=0.3).astype(np.float32)
    L_ref, grad_ref, om_ref = G.loss_and_theta_grad(theta.astype(np.float64), g, c, [(r32, e32)])
    with GpuSolver() as s:
        build_ssor(s, m)
        om, L, grad = s.learn_eval(theta, r, e)
    assert np.abs(om - om_ref).max() <= 1e-5
    assert abs(L - L_ref) <= 1e-4 * abs(L_ref)
    scale = np.abs(grad_ref).max()
    assert np.abs(grad - grad_ref).max() <= 2e-3 * scale
    assert np.dot(grad, grad_ref) / (np.linalg.norm(grad) * np.linalg.norm(grad_ref)) > 0.9999


def _solve(s, m, learned=0, mixed=0, coarse=0, tol=1e-8):
    g = m.copy()
    g.set_iter(20000)
    g.set_resid(tol)
    g.Iarray[42] = learned
    g.Iarray[43] = coarse
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


def test_training_gain_and_mixed():
    m = box_system(16, 16, 32, jitter=0.15, sigma_E=0.5, nu_range=(0.25, 0.4), seed=2)
    loads = _load_cases(m, 6, seed=3)
    with GpuSolver() as s:
        # earlier increments: plain FP64 SSOR-CG, recording (r, e) pairs
        s.learn_record(1, max_pairs=24)
        for b in loads[:3]:
            mm = m.copy()
            mm.B = b
            g, info, rec = _solve(s, mm)
            assert info["error"] == 0
        n_pairs = s.learn_record(0)
        assert n_pairs >= 10
        l0, l1 = s.learn_train(steps=40, lr=5e-3)
        assert np.isfinite(l1) and l1 < l0, (l0, l1)
        theta = s.learn_get_weights()
        assert theta is not None and theta.size == G.n_params()

        # held-out load cases: learned vs SSOR-CG and vs the unsmoothed coarse space
        for b in loads[3:5]:
            mm = m.copy()
            mm.B = b
            _, info_plain, _ = _solve(s, mm)
            _, info_unsm, _ = _solve(s, mm, learned=1, coarse=1)
            g, info, rec = _solve(s, mm, learned=1)
            assert info["error"] == 0 and rec["learned"] == 1 and rec["fallback"] == 0
            assert info["iter"] * 3 < info_plain["iter"], (info["iter"], info_plain["iter"])
            assert info["iter"] <= info_unsm["iter"], (info["iter"], info_unsm["iter"])
            assert Oracle(mm).rel_resid(g.X, mm.B) <= 1e-8
            g2, info2, rec2 = _solve(s, mm, learned=1, mixed=1)
            assert info2["error"] == 0 and abs(info2["iter"] - info["iter"]) <= 2
            assert Oracle(mm).rel_resid(g2.X, mm.B) <= 1e-8

        # a deliberately bad network (saturated smoothing weights) still converges
        bad = theta.copy()
        bad[-3 * G.WIDTH:] = 50.0 * np.random.default_rng(4).standard_normal(3 * G.WIDTH)
        s.learn_set_weights(bad)
        mm = m.copy()
        g, info, rec = _solve(s, mm, learned=1)
        assert info["error"] == 0
        assert Oracle(mm).rel_resid(g.X, mm.B) <= 1e-8


def test_fixed_weights_need_no_training_and_errors():
    """Iarray(44) = 1 / 2 (no smoothing / omega = 1/2) run without a trained network;
    the network's weights without training, and the two-level preconditioner around a
    preconditioner other than SSOR, are refused with 1001 as the reference refuses an
    inconsistent PRECOND."""
    from frontistr_b200.solver import HecmwSolverError
    m = box_system(8, 8, 16, jitter=0.1, seed=5)
    with GpuSolver() as s:
        _, info_plain, _ = _solve(s, m)
        for coarse in (1, 2):
            g, info, rec = _solve(s, m, learned=1, coarse=coarse)
            assert info["error"] == 0 and rec["learned"] == 1
            assert info["iter"] < info_plain["iter"]
            assert Oracle(m).rel_resid(g.X, m.B) <= 1e-8
        with pytest.raises(HecmwSolverError) as e:
            _solve(s, m, learned=1, coarse=0)
        assert e.value.code == 1001
        d = m.copy()
        d.set_precond(3)
        with pytest.raises(HecmwSolverError) as e:
            _solve(s, d, learned=1, coarse=2)
        assert e.value.code == 1001


def _renumbered_box(nx, ny, nz, seed):
    """A clamped HEX8 box loaded on its top face whose node numbers are a random
    permutation of the lexicographic ones (first-fit in node order then needs far more
    than the 8 parity colours)."""
    from frontistr_b200.mesh import mesh_system

    def idx(i, j, k):
        return (k * (ny + 1) + j) * (nx + 1) + i

    coords = np.array([(i, j, k) for k in range(nz + 1) for j in range(ny + 1) for i in range(nx + 1)], float)
    elems = np.array([[idx(i, j, k), idx(i + 1, j, k), idx(i + 1, j + 1, k), idx(i, j + 1, k),
                       idx(i, j, k + 1), idx(i + 1, j, k + 1), idx(i + 1, j + 1, k + 1), idx(i, j + 1, k + 1)]
                      for k in range(nz) for j in range(ny) for i in range(nx)])
    new = np.random.default_rng(seed).permutation(len(coords))  # old id -> new id
    c2 = np.empty_like(coords)
    c2[new] = coords
    fixed = [(int(new[idx(i, j, 0)]), d, 0.0) for j in range(ny + 1) for i in range(nx + 1) for d in (1, 2, 3)]
    cload = [(int(new[idx(i, j, nz)]), 2, -1.0) for j in range(ny + 1) for i in range(nx + 1)]
    return mesh_system(c2, new[elems], 361, 1000.0, 0.3, fixed=fixed, cload=cload)


@pytest.mark.parametrize("case", ["tet4", "renumbered_box"])
def test_learned_on_unstructured_numbering(case):
    """The smoother's colouring on numberings that are not lexicographic: the TET4
    cantilever of the reference's tests and a HEX8 box with randomly renumbered nodes.
    With omega = 1/2 (no training), in FP64 and with the BF16-stored smoother, the
    learned solve meets the FP64 true residual in fewer iterations than SSOR-CG."""
    from frontistr_b200.solver import smoother_schedule
    from test_oracle_golden import golden_system
    m = golden_system()[1] if case == "tet4" else _renumbered_box(10, 10, 20, seed=1)
    ci, _ = smoother_schedule(m)
    assert len(ci) - 1 <= 16
    with GpuSolver() as s:
        _, info_plain, _ = _solve(s, m)
        assert info_plain["error"] == 0
        for mixed in (0, 1):
            g, info, rec = _solve(s, m, learned=1, coarse=2, mixed=mixed)
            assert info["error"] == 0 and rec["learned"] == 1
            assert info["iter"] < info_plain["iter"], (info["iter"], info_plain["iter"])
            assert Oracle(m).rel_resid(g.X, m.B) <= 1e-8
