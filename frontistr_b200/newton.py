"""Newton sequence of a compressible Neo-Hookean HEX8 block (the tangent systems that
the static nonlinear loop of fistr1 hands to hecmw_solve: fstr_Newton in
fistr1/src/analysis/static/fstr_solve_NonLinear.f90:32-200).

The block (nx x ny x nz elements of edge h, C10, D1; W = C10 (I1bar - 3) + (J - 1)^2 / D1)
is clamped on z = 0 and its top face z = nz h is moved by a prescribed displacement,
ramped in equal increments.  Every Newton iteration assembles the tangent K(u) and
residual R(u) = -f_int(u) on the host (libfistr_assemble.so), applies the
displacement conditions with hecmw_mat_ass_bc semantics (the prescribed increment
on the first iteration of an increment, 0 afterwards) and asks a solver for du."""
import numpy as np

from ._lib import assemble_lib
from .matrix import HecMatrix
from .mesh import _dp, _ip, box_counts


class NeoHookeBox:
    def __init__(self, nx, ny, nz, h=1.0, C10=1.0, D1=0.01):
        self.nx, self.ny, self.nz, self.h, self.C10, self.D1 = nx, ny, nz, h, C10, D1
        self.N, self.NPL, self.NPU = box_counts(nx, ny, nz)
        nx1, ny1 = nx + 1, ny + 1
        ix, iy = np.meshgrid(np.arange(nx1), np.arange(ny1), indexing="xy")
        face = (ix + nx1 * iy).ravel()
        self.bottom = face.astype(np.int32)                      # z = 0 (0-based node ids)
        self.top = (face + nx1 * ny1 * nz).astype(np.int32)      # z = nz h

    def tangent(self, U):
        """HecMatrix with D/AL/AU = K(U) and B = R(U) = -f_int(U); raises if an
        element has inverted (J <= 0)."""
        lib = assemble_lib()
        m = HecMatrix.empty(self.N, self.NPL, self.NPU)
        U = np.ascontiguousarray(U, dtype=np.float64)
        bad = lib.fistr_box_neohooke(self.nx, self.ny, self.nz, self.h, self.C10, self.D1, _dp(U),
                                     _ip(m.indexL), _ip(m.itemL), _ip(m.indexU), _ip(m.itemU),
                                     _dp(m.D), _dp(m.AL), _dp(m.AU), _dp(m.B))
        if bad:
            raise RuntimeError("%d elements inverted (J <= 0)" % bad)
        return m

    def constraints(self, top_uz):
        """(node1, dof, value) of the displacement conditions: bottom clamped, top face
        x, y held and z displaced by top_uz."""
        nodes, dofs, vals = [], [], []
        for n in self.bottom:
            for d in (1, 2, 3):
                nodes.append(n + 1), dofs.append(d), vals.append(0.0)
        for n in self.top:
            for d, v in ((1, 0.0), (2, 0.0), (3, top_uz)):
                nodes.append(n + 1), dofs.append(d), vals.append(v)
        return (np.array(nodes, np.int32), np.array(dofs, np.int32), np.array(vals))

    def apply_bc(self, m, nodes, dofs, values):
        lib = assemble_lib()
        lib.fistr_mat_ass_bc_list(len(nodes), _ip(nodes), _ip(dofs), _dp(np.ascontiguousarray(values)),
                                  _ip(m.indexL), _ip(m.itemL), _ip(m.indexU), _ip(m.itemU),
                                  _dp(m.D), _dp(m.AL), _dp(m.AU), _dp(m.B))


def newton_sequence(box, solve, top_uz, n_incr=12, max_newton=8, tol=1e-6):
    """Runs the ramped Newton sequence.  solve(increment, newton_iter, m) returns du for
    the tangent system m (hecmwST arrays, B = right-hand side, constraints applied).
    Yields one record per Newton iteration; the displacement is box.U afterwards."""
    U = np.zeros(3 * box.N)
    nodes, dofs, target = box.constraints(0.0)
    for inc in range(1, n_incr + 1):
        _, _, target = box.constraints(top_uz * inc / n_incr)
        r0 = None
        for it in range(1, max_newton + 1):
            m = box.tangent(U)
            free = np.ones(3 * box.N, bool)
            free[3 * (nodes - 1) + dofs - 1] = False
            rnorm = float(np.linalg.norm(m.B[free]))
            cur = U[3 * (nodes - 1) + dofs - 1]
            step = target - cur  # prescribed increment (0 once reached)
            if it > 1 and r0 is not None and rnorm <= tol * max(r0, 1e-300):
                yield dict(increment=inc, newton=it, residual=rnorm, converged=True)
                break
            if r0 is None:
                r0 = max(rnorm, float(np.linalg.norm(step)))
            box.apply_bc(m, nodes, dofs, step)
            du = solve(inc, it, m)
            U += du
            yield dict(increment=inc, newton=it, residual=rnorm, converged=False)
    box.U = U
