"""The allocation-free entry point hecmw33_gpu_rel_resid_noalloc.

It serves callers that cannot allocate GPU memory: their device memory is owned
in full by another allocator, or allocation is forbidden between their solves.
They hand over device arrays they already hold (the hecmwST_matrix layout) and
get ||b - A x|| / ||b|| back; the entry point's only scratch space is a static
array inside the library.

Checked through the C ABI against the existing entry points, twice in a row
(the second call must not see the first call's leftovers):
  * at the solution of a solve, against the true residual that
    hecmw33_gpu_solve reports (hecmw33_gpu_last_solve_info);
  * at a random x, against ||b - y|| / ||b|| with y from hecmw33_gpu_matvec.
Tolerance: the SpMV bar of the parity tests, 1e-14 of the row scale sum |A||x|,
carried to the norm: |delta resid| <= 1e-14 ||(|A||x|)|| / ||b|| (+1e-15 relative).

This file is named to be collected last, so that a run stopping at the first
failure has already run every other test.  It passes alone in a fresh process too:
the first call on the device sets up the scratch address itself.
"""
import ctypes

import numpy as np
import pytest

from frontistr_b200._lib import gpu_lib
from frontistr_b200.mesh import box_system
from frontistr_b200.solver import GpuSolver, last_error

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _noalloc(lib, n, d, x_dev, b_dev):
    res, err = ctypes.c_double(-1.0), ctypes.c_int(0)
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    lib.hecmw33_gpu_rel_resid_noalloc(ctypes.byref(ctypes.c_int(n)), p(d["indexL"]), p(d["itemL"]),
                                      p(d["indexU"]), p(d["itemU"]), p(d["D"]), p(d["AL"]), p(d["AU"]),
                                      p(x_dev), p(b_dev), ctypes.byref(res), ctypes.byref(err))
    return res.value, err.value


def test_rel_resid_noalloc_matches_existing_entry_points():
    torch = pytest.importorskip("torch")
    lib = gpu_lib()
    m = box_system(20, 20, 30, jitter=0.1, seed=4)
    m.set_iter(20000)
    rng = np.random.default_rng(9)
    x_rand = rng.standard_normal(3 * m.N)
    with GpuSolver() as s:
        g = m.copy()
        info = s.solve(g)
        assert info["error"] == 0
        ref_sol = s.last_solve_info()["true_resid"]
        y = s.matvec(x_rand)
    ref_rand = np.linalg.norm(m.B - y) / np.linalg.norm(m.B)

    d = {k: _dev(torch, getattr(m, k)) for k in ("indexL", "itemL", "indexU", "itemU", "D", "AL", "AU")}
    b_dev = _dev(torch, m.B)
    A_abs = abs(m.to_scipy())
    cases = []
    for x, ref in ((g.X, ref_sol), (x_rand, ref_rand)):
        bound = 1e-14 * np.linalg.norm(A_abs @ np.abs(x)) / np.linalg.norm(m.B) + 1e-15 * ref
        cases.append((_dev(torch, x), ref, bound))
    torch.cuda.synchronize()
    for call in range(2):
        for x_dev, ref, bound in cases:
            got, err = _noalloc(lib, m.N, d, x_dev, b_dev)
            assert err == 0, last_error()
            assert abs(got - ref) <= bound, (call, got, ref, bound)


def test_rel_resid_noalloc_rejects_sizes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    lib = gpu_lib()
    tiny = torch.zeros(16, dtype=torch.float64, device="cuda")
    d = {k: tiny for k in ("indexL", "itemL", "indexU", "itemU", "D", "AL", "AU")}
    got, err = _noalloc(lib, 2_097_153, d, tiny, tiny)
    assert err == 9101
    assert "2097152" in last_error()


def test_rel_resid_noalloc_rejects_a_decomposed_domain():
    """A domain of a decomposed mesh (external nodes N+1..NP in its items) is not a
    whole-mesh matrix: the kernel skips every item outside 1..N before reading X
    (which holds 3N doubles here) and the call returns 9101 without a residual."""
    torch = pytest.importorskip("torch")
    from frontistr_b200.domain import partition
    lib = gpu_lib()
    m = box_system(6, 5, 8, seed=2)
    dom = partition(m, 2)[0].matrix
    assert dom.NP > dom.N
    d = {k: _dev(torch, getattr(dom, k)) for k in ("indexL", "itemL", "indexU", "itemU", "D", "AL", "AU")}
    x_dev = _dev(torch, np.ones(3 * dom.N))
    b_dev = _dev(torch, dom.B[:3 * dom.N])
    torch.cuda.synchronize()
    got, err = _noalloc(lib, dom.N, d, x_dev, b_dev)
    assert err == 9101 and got == -1.0
    assert "outside 1..N" in last_error()
    # the whole mesh still gives a residual afterwards
    d = {k: _dev(torch, getattr(m, k)) for k in ("indexL", "itemL", "indexU", "itemU", "D", "AL", "AU")}
    got, err = _noalloc(lib, m.N, d, _dev(torch, np.zeros(3 * m.N)), _dev(torch, m.B))
    assert err == 0 and abs(got - 1.0) <= 1e-15
