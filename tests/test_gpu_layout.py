"""The sliced layouts filled on the device from the resident profile
(fill_unified_kernel; count_parts_kernel + fill_reordered_kernel; fill_ordered_kernel)
against the host builders (HECMW33_HOST_LAYOUT=1: unified_rows, reordered_rows,
build_sell): solves through either give the same iterations and the same X bit for
bit -- the SpMV layout, the reference's RCM + multicolour SSOR schedule at several
ncolor_in, block ILU(0)'s level-ordered layouts, the learned preconditioner's first-fit
smoother, its network's graph and coarse space, and the 16-lane copy of A of the
multi-RHS solve, on a jittered box and on a box with randomly renumbered nodes."""
import numpy as np
import pytest

from frontistr_b200.mesh import box_system
from frontistr_b200.solver import GpuSolver
from test_gpu_learned import _renumbered_box
from test_gpu_multi import flags, load_cases

pytestmark = pytest.mark.gpu


def _system(name):
    if name == "jittered_box":
        return box_system(12, 10, 16, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=3)
    return _renumbered_box(8, 7, 12, seed=2)


def _layouts(monkeypatch, host):
    if host:
        monkeypatch.setenv("HECMW33_HOST_LAYOUT", "1")
    else:
        monkeypatch.delenv("HECMW33_HOST_LAYOUT", raising=False)


def _solve(m, monkeypatch, host, settings):
    _layouts(monkeypatch, host)
    g = m.copy()
    for k, v in settings:
        g.Iarray[k] = v
    with GpuSolver() as s:  # a new handle: the whole symbolic setup runs again
        info = s.solve(g)
    assert info["error"] == 0, info
    return info["iter"], g.X.copy()


@pytest.mark.parametrize("name", ["jittered_box", "renumbered_box"])
@pytest.mark.parametrize("settings", [
    [],                              # CG + SSOR, ncolor_in 10
    [(33, 2)],                       # ncolor_in 2
    [(33, 40)],                      # ncolor_in 40
    [(41, 1)],                       # BF16-stored SSOR values
    [(42, 1), (43, 2)],              # learned two-level preconditioner (first-fit smoother)
    [(2, 10)],                       # block ILU(0): level-ordered layouts of the matrix's pattern
], ids=["ssor", "ncolor2", "ncolor40", "bf16", "learned", "ilu0"])
def test_device_layouts_equal_host(name, settings, monkeypatch):
    m = _system(name)
    m.set_iter(20000)
    m.set_resid(1e-8)
    it_h, x_h = _solve(m, monkeypatch, True, settings)
    it_d, x_d = _solve(m, monkeypatch, False, settings)
    assert it_d == it_h
    assert np.array_equal(x_d, x_h)


def test_device_layout_multi_rhs_equals_host(monkeypatch):
    m = _system("jittered_box")
    B = load_cases(m, 3, seed=5)
    ia, ra = flags(m, 1)
    out = []
    for host in (True, False):
        _layouts(monkeypatch, host)
        with GpuSolver() as s:
            s.set_matrix(m)
            X = np.zeros_like(B)
            rec = s.solve_multi(B, X, ia, ra)
            out.append((list(rec["iter"]), X))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("name", ["jittered_box", "renumbered_box"])
def test_device_network_graph_equals_host(name, monkeypatch):
    """The learned preconditioner with its network (Iarray(44) = 0, fixed random
    weights): the edge list, raw ids and reverse edges built on the device
    (fill_edges_kernel, edge_reverse_kernel) and the coarse space's unified rows
    (fill_unified_csr_kernel) give the host-built solve bit for bit."""
    import gnn_reference as G
    theta = G.init_params(seed=1, scale_out=1.0).astype(np.float32)
    m = _system(name)
    m.set_iter(20000)
    m.set_resid(1e-8)
    out = []
    for host in (True, False):
        _layouts(monkeypatch, host)
        g = m.copy()
        g.Iarray[42] = 1
        g.Iarray[43] = 0
        with GpuSolver() as s:
            s.learn_set_weights(theta)
            info = s.solve(g)
            assert info["error"] == 0 and s.last_solve_info()["learned"] == 1
        out.append((info["iter"], g.X.copy()))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
