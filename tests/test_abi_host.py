"""CPU-only checks of the C ABI library: it loads, exports every symbol that
include/hecmw33_gpu.h declares, and its host-side colour schedule (RCM +
multicolouring) is identical to the oracle's restatement of
hecmw_matrix_ordering_CM.f90 / _MC.f90.  No GPU compute is called here."""
import ctypes
import os
import re

import numpy as np
import pytest

from frontistr_b200 import _abi
from frontistr_b200._lib import gpu_lib
from frontistr_b200.matrix import HecMatrix
from frontistr_b200.mesh import box_system
from frontistr_b200.solver import HecmwSolverError, colour_schedule, last_error, smoother_schedule
from oracle_ctypes import Oracle
from test_oracle_golden import golden_system

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"HECMW33_API\s+[\w\s\*]+?\b(hecmw33_\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    lib = gpu_lib()
    names = declared_symbols()
    assert len(names) >= 10
    for n in names:
        assert hasattr(lib, n), n
    # and the Python declarations cover the header
    assert names == set(_abi.exported_names())


def oracle_schedule(m, ncolor_in):
    orc = Oracle(m)
    pc = orc.precond(1, ncolor_in=ncolor_in, coloured=1)
    ci, perm, _ = pc.ordering()
    return ci, perm


@pytest.mark.parametrize("case", ["tet4", "box1", "box_small", "box_flat"])
@pytest.mark.parametrize("ncolor_in", [10, 3, 50])
def test_colour_schedule_matches_oracle(case, ncolor_in):
    if case == "tet4":
        _, m = golden_system()
    elif case == "box1":
        m = box_system(16, 16, 64)
    elif case == "box_small":
        m = box_system(3, 4, 5)
    else:
        m = box_system(9, 7, 1)
    ci, perm = colour_schedule(m, ncolor_in)
    ci_o, perm_o = oracle_schedule(m, ncolor_in)
    assert np.array_equal(ci, ci_o)
    assert np.array_equal(perm, perm_o)
    # colours are independent sets (check_ordering, hecmw_precond_SSOR_33.F90:476-513)
    colour = np.empty(m.N, np.int64)
    for c in range(len(ci) - 1):
        colour[perm[ci[c]:ci[c + 1]] - 1] = c
    rows = np.repeat(np.arange(m.N), np.diff(m.indexU))
    cols = m.itemU[:m.NPU] - 1
    assert not np.any(colour[rows] == colour[cols])


def test_colour_schedule_rejects_bad_profile():
    m = box_system(2, 2, 2)
    bad = m.copy()
    bad.itemU[0] = bad.N + 5  # out of range
    with pytest.raises(HecmwSolverError) as e:
        colour_schedule(bad)
    assert e.value.code == 9101


def test_single_node_and_disconnected_profiles():
    # one node, no neighbours
    m = HecMatrix(1, 1, [0, 0], [0], [0, 0], [0], np.eye(3).ravel(), np.zeros(9), np.zeros(9))
    ci, perm = colour_schedule(m)
    assert list(ci) == [0, 1] and list(perm) == [1]
    # two disconnected 2x2x2 boxes side by side in one profile
    a = box_system(1, 1, 1)
    n = a.N
    indexL = np.concatenate([a.indexL, a.indexL[1:] + a.NPL])
    indexU = np.concatenate([a.indexU, a.indexU[1:] + a.NPU])
    itemL = np.concatenate([a.itemL[:a.NPL], a.itemL[:a.NPL] + n])
    itemU = np.concatenate([a.itemU[:a.NPU], a.itemU[:a.NPU] + n])
    D = np.concatenate([a.D, a.D])
    m2 = HecMatrix(2 * n, 2 * n, indexL, itemL, indexU, itemU, D, np.concatenate([a.AL, a.AL]),
                   np.concatenate([a.AU, a.AU]))
    ci, perm = colour_schedule(m2)
    ci_o, perm_o = oracle_schedule(m2, 10)
    assert np.array_equal(ci, ci_o) and np.array_equal(perm, perm_o)


def _neighbours(m):
    nb = [set() for _ in range(m.N)]
    for index, item in ((m.indexL, m.itemL), (m.indexU, m.itemU)):
        for i in range(m.N):
            for k in range(index[i], index[i + 1]):
                nb[i].add(int(item[k]) - 1)
    return nb


def _first_fit(nb, order):
    colour = {}
    for i in order:
        used = {colour[j] for j in nb[i] if j in colour and j != i}
        colour[i] = min(set(range(len(used) + 1)) - used)
    return 1 + max(colour.values())


@pytest.mark.parametrize("case", ["tet4", "box_small", "box_jitter", "box_renumbered"])
def test_smoother_schedule_is_a_greedy_colouring(case):
    """The learned preconditioner's smoother colours: a valid colouring (no two
    neighbours share a colour), rows by colour then node, and no more colours than
    first-fit in the node order (the library keeps the better of that and smallest-last
    order): 8 on a lexicographically numbered box, fewer than first-fit on a randomly
    renumbered one."""
    if case == "tet4":
        _, m = golden_system()
    elif case == "box_small":
        m = box_system(6, 5, 7)
    elif case == "box_jitter":
        m = box_system(5, 6, 4, jitter=0.2, seed=3)
    else:
        from test_gpu_learned import _renumbered_box
        m = _renumbered_box(6, 5, 7, seed=2)
    ci, perm = smoother_schedule(m)
    nc = len(ci) - 1
    colour = np.empty(m.N, np.int64)
    for c in range(nc):
        colour[perm[ci[c]:ci[c + 1]] - 1] = c
        assert np.all(np.diff(perm[ci[c]:ci[c + 1]]) > 0)  # node order inside a colour
    assert sorted(perm.tolist()) == list(range(1, m.N + 1))
    nb = _neighbours(m)
    for i in range(m.N):
        assert all(colour[j] != colour[i] for j in nb[i] if j != i)
    natural = _first_fit(nb, range(m.N))
    assert nc <= natural
    if case in ("box_small", "box_jitter"):
        assert nc == 8
    if case == "box_renumbered":
        assert nc < natural, (nc, natural)


def test_rel_resid_noalloc_rejects_null_pointers():
    """The allocation-free residual call checks its pointers on the host before any
    CUDA call: a null device array (or a null resid) returns 9101 with a message."""
    lib = gpu_lib()
    buf = (ctypes.c_double * 16)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    res, err = ctypes.c_double(-1.0), ctypes.c_int(0)
    n = ctypes.c_int(4)
    for hole in range(10):
        args = [p] * 9
        if hole < 9:
            args[hole] = None
        rp = None if hole == 9 else ctypes.byref(res)
        err.value = 0
        lib.hecmw33_gpu_rel_resid_noalloc(ctypes.byref(n), *args, rp, ctypes.byref(err))
        assert err.value == 9101, hole
        assert "null pointer" in last_error()
    assert res.value == -1.0
