"""Generators of hecmwST_matrix systems for the solver (the caller side of hecmw_solve).

Two entry points, both backed by libfistr_assemble.so (frontistr_b200/csrc/assemble.cpp):

* :func:`box_system` -- the structured HEX8 cantilever boxes (nx x ny x nz unit
  cubes, x-fastest lexicographic node numbering, FI 2x2x2 integration, face z=0
  clamped, -1.0 y-load on every top-face node), optionally with seeded interior
  node jitter and heterogeneous materials.
* :func:`mesh_system` -- any TET4 (341) / HEX8 (361) mesh with explicit fixed dofs
  and nodal loads, assembled like fistr1 (CLOAD first, then hecmw_mat_ass_bc).
"""
import ctypes

import numpy as np

from ._lib import assemble_lib
from .matrix import HecMatrix

_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)


def _ip(a):
    return a.ctypes.data_as(_i32p)


def _dp(a):
    return a.ctypes.data_as(_f64p)


def box_counts(nx, ny, nz):
    lib = assemble_lib()
    n, npl, npu = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    if lib.fistr_box_counts(nx, ny, nz, ctypes.byref(n), ctypes.byref(npl), ctypes.byref(npu)) != 0:
        raise ValueError("box too large for 32-bit indices")
    return n.value, npl.value, npu.value


def box_system(nx, ny, nz, h=1.0, E=210000.0, nu=0.3, load_y=-1.0, jitter=0.0,
               sigma_E=0.0, nu_range=None, seed=0, want_coords=False):
    """Assemble the clamped HEX8 box; returns a :class:`HecMatrix` with B set, X = 0."""
    lib = assemble_lib()
    n, npl, npu = box_counts(nx, ny, nz)
    m = HecMatrix.empty(n, npl, npu)
    numin, numax = (nu_range if nu_range is not None else (0.0, 0.0))
    params = np.array([h, E, nu, load_y, jitter, sigma_E, numin, numax], dtype=np.float64)
    coords = np.zeros(3 * n) if want_coords else None
    rc = lib.fistr_box_assemble(nx, ny, nz, _dp(params), ctypes.c_uint64(seed),
                                _ip(m.indexL), _ip(m.itemL), _ip(m.indexU), _ip(m.itemU),
                                _dp(m.D), _dp(m.AL), _dp(m.AU), _dp(m.B),
                                _dp(coords) if coords is not None else None)
    if rc != 0:
        raise RuntimeError("fistr_box_assemble failed: %d" % rc)
    if want_coords:
        m.coords = coords.reshape(-1, 3)
    return m


def mesh_system(coords, elements, etype, E, nu, fixed=(), cload=()):
    """Assemble a general mesh.

    coords: (n,3); elements: (ne, 4|8) 0-based node indices; E/nu: scalars or per element;
    fixed: iterable of (node0, dof1, value); cload: iterable of (node0, dof1, value).
    """
    lib = assemble_lib()
    coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
    conn = np.ascontiguousarray(elements, dtype=np.int32)
    n, ne = coords.shape[0], conn.shape[0]
    Ee = np.ascontiguousarray(np.broadcast_to(np.asarray(E, dtype=np.float64), (ne,)))
    nue = np.ascontiguousarray(np.broadcast_to(np.asarray(nu, dtype=np.float64), (ne,)))
    npl, npu = ctypes.c_int(), ctypes.c_int()
    if lib.fistr_mesh_profile_counts(n, ne, conn.shape[1], _ip(conn), ctypes.byref(npl),
                                     ctypes.byref(npu)) != 0:
        raise ValueError("element connectivity out of range")
    m = HecMatrix.empty(n, npl.value, npu.value)
    rc = lib.fistr_mesh_assemble(n, _dp(coords), ne, etype, _ip(conn), _dp(Ee), _dp(nue),
                                 _ip(m.indexL), _ip(m.itemL), _ip(m.indexU), _ip(m.itemU),
                                 _dp(m.D), _dp(m.AL), _dp(m.AU))
    if rc != 0:
        raise RuntimeError("fistr_mesh_assemble failed: %d" % rc)
    for node, dof, val in cload:
        m.B[3 * node + dof - 1] += val
    for node, dof, val in fixed:
        lib.fistr_mat_ass_bc(node + 1, dof, float(val), _ip(m.indexL), _ip(m.itemL),
                             _ip(m.indexU), _ip(m.itemU), _dp(m.D), _dp(m.AL), _dp(m.AU), _dp(m.B))
    m.coords = coords
    return m


def random_box_batch(nsys, edge_range=(8, 40), E_range=(1.0e3, 1.0e6), nu_range=(0.2, 0.45), seed=0):
    """nsys independent clamped HEX8 boxes: edge lengths (elements per axis) uniform
    in edge_range, E log-uniform in E_range, nu uniform in nu_range, and a random
    unit-norm traction on every node of the loaded face z = nz (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nsys):
        nx, ny, nz = (int(v) for v in rng.integers(edge_range[0], edge_range[1] + 1, size=3))
        E = float(np.exp(rng.uniform(np.log(E_range[0]), np.log(E_range[1]))))
        nu = float(rng.uniform(nu_range[0], nu_range[1]))
        m = box_system(nx, ny, nz, E=E, nu=nu)
        t = rng.standard_normal(3)
        t /= np.linalg.norm(t)
        top = np.unique(np.nonzero(m.B)[0] // 3)
        m.B[:] = 0.0
        for c in range(3):
            m.B[3 * top + c] = t[c]
        m.dims = (nx, ny, nz)
        out.append(m)
    return out
