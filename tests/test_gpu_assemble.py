"""HEX8 assembly on the device (hecmw33_gpu_assemble_hex8) against the host
restatement (fistr_mesh_assemble + fistr_mat_ass_bc: STF_C3 2x2x2 Gauss, element-order
scatter of hecmw_mat_ass_elem, hecmw_mat_ass_bc in list order).

The device computes every element block with the host's operations in the host's
order and sums the blocks in element order, so the matrix and right-hand side must
be bitwise equal to the host's; the assembled system then solves like the host one.
"""
import numpy as np
import pytest

from frontistr_b200.mesh import mesh_system
from frontistr_b200.solver import GpuSolver
from oracle_ctypes import Oracle

pytestmark = pytest.mark.gpu


def box_mesh(nx, ny, nz, jitter=0.2, seed=0):
    """Nodes x fastest, elements in hex8n order; interior nodes jittered."""
    rng = np.random.default_rng(seed)
    ix, iy, iz = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    X = np.stack([ix, iy, iz], -1).transpose(2, 1, 0, 3).reshape(-1, 3).astype(np.float64)
    inner = np.all((X > 0) & (X < np.array([nx, ny, nz])), axis=1)
    X[inner] += rng.uniform(-jitter, jitter, size=(inner.sum(), 3))
    nid = lambda x, y, z: x + (nx + 1) * (y + (ny + 1) * z)
    el = []
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                el.append([nid(x, y, z), nid(x + 1, y, z), nid(x + 1, y + 1, z), nid(x, y + 1, z),
                           nid(x, y, z + 1), nid(x + 1, y, z + 1), nid(x + 1, y + 1, z + 1), nid(x, y + 1, z + 1)])
    return X, np.array(el, dtype=np.int32), nid


def problem(nx=6, ny=5, nz=7, seed=1):
    X, el, nid = box_mesh(nx, ny, nz, seed=seed)
    rng = np.random.default_rng(seed + 1)
    ne = len(el)
    E = 2.1e5 * np.exp(rng.standard_normal(ne))
    nu = rng.uniform(0.25, 0.4, ne)
    F = np.zeros(3 * len(X))
    top = [nid(x, y, nz) for y in range(ny + 1) for x in range(nx + 1)]
    for n in top:
        F[3 * n + 1] = -1.0
    fixed = [(nid(x, y, 0), d, 0.0) for y in range(ny + 1) for x in range(nx + 1) for d in (1, 2, 3)]
    # prescribed nonzero values, one dof constrained twice (the last value stays)
    fixed += [(nid(1, 1, nz), 3, -0.01), (nid(2, 1, nz), 3, -0.02), (nid(1, 1, nz), 3, -0.015)]
    return X, el, E, nu, F, fixed


def host_system(X, el, E, nu, F, fixed):
    cload = [(i // 3, i % 3 + 1, F[i]) for i in np.nonzero(F)[0]]
    return mesh_system(X, el, 361, E, nu, fixed=fixed, cload=cload)


def test_assembly_bitwise_equal_to_host():
    X, el, E, nu, F, fixed = problem()
    ref = host_system(X, el, E, nu, F, fixed)
    with GpuSolver() as s:
        npl, npu = s.assemble_hex8(X, el, E, nu, F=F, fixed=fixed)
        g = s.get_matrix()
    assert (npl, npu) == (ref.NPL, ref.NPU)
    for a in ("indexL", "indexU"):
        assert np.array_equal(getattr(g, a), getattr(ref, a))
    assert np.array_equal(g.itemL[:npl], ref.itemL[:npl]) and np.array_equal(g.itemU[:npu], ref.itemU[:npu])
    assert np.array_equal(g.D, ref.D)
    assert np.array_equal(g.AL[:9 * npl], ref.AL[:9 * npl])
    assert np.array_equal(g.AU[:9 * npu], ref.AU[:9 * npu])
    assert np.array_equal(g.B, ref.B)


def test_assembled_system_solves_like_host():
    X, el, E, nu, F, fixed = problem(8, 7, 9, seed=3)
    ref = host_system(X, el, E, nu, F, fixed)
    ref.set_iter(20000)
    orc = Oracle(ref).solve(coloured=1)
    with GpuSolver() as s:
        s.assemble_hex8(X, el, E, nu, F=F, fixed=fixed)
        x, rec = s.solve_assembled(ref.Iarray.copy(), ref.Rarray.copy())
    assert rec["error"] == 0 and orc["error"] == 0
    assert abs(rec["iter"] - orc["iter"]) <= 2
    assert np.linalg.norm(x - orc["X"]) <= 1e-8 * np.linalg.norm(orc["X"])


def test_reassembly_reuses_profile():
    """symbolic = 0 (a Newton iteration on the same mesh): new material values."""
    X, el, E, nu, F, fixed = problem(5, 4, 6, seed=5)
    with GpuSolver() as s:
        s.assemble_hex8(X, el, E, nu, F=F, fixed=fixed)
        s.assemble_hex8(X, el, 2.0 * E, nu, F=F, fixed=fixed, symbolic=False)
        g = s.get_matrix()
    ref = host_system(X, el, 2.0 * E, nu, F, fixed)
    assert np.array_equal(g.D, ref.D) and np.array_equal(g.AL[:9 * g.NPL], ref.AL[:9 * ref.NPL])
    assert np.array_equal(g.B, ref.B)


def box_grid(nx, ny, nz, h):
    X, el, nid = box_mesh(nx, ny, nz, jitter=0.0)
    return X * h, el, nid


@pytest.mark.parametrize("amp", [0.0, 0.02])
def test_neohooke_assembly_matches_host(amp):
    """Tangent and residual of the compressible Neo-Hookean block at a displacement
    field U against the host (fistr_box_neohooke + hecmw_mat_ass_bc), to rounding."""
    from frontistr_b200.newton import NeoHookeBox
    nx, ny, nz, h = 5, 4, 6, 0.5
    box = NeoHookeBox(nx, ny, nz, h=h, C10=1.0, D1=0.01)
    rng = np.random.default_rng(7)
    X, el, nid = box_grid(nx, ny, nz, h)
    U = amp * h * rng.standard_normal(3 * box.N)
    ref = box.tangent(U)
    nodes, dofs, vals = box.constraints(-0.05 * h)
    box.apply_bc(ref, nodes, dofs, vals)
    fixed = list(zip((nodes - 1).tolist(), dofs.tolist(), vals.tolist()))
    with GpuSolver() as s:
        npl, npu, inv = s.assemble_hex8_neohooke(X, el, 1.0, 0.01, U, fixed=fixed)
        g = s.get_matrix()
    assert inv == 0 and (npl, npu) == (ref.NPL, ref.NPU)
    assert np.array_equal(g.itemL[:npl], ref.itemL[:npl]) and np.array_equal(g.itemU[:npu], ref.itemU[:npu])
    scale = max(np.abs(ref.D).max(), np.abs(ref.AL[:9 * npl]).max())
    for a, n in (("D", 9 * g.N), ("AL", 9 * npl), ("AU", 9 * npu)):
        assert np.abs(getattr(g, a)[:n] - getattr(ref, a)[:n]).max() <= 1e-13 * scale, a
    bscale = max(np.abs(ref.B).max(), 1e-300)
    assert np.abs(g.B - ref.B).max() <= 1e-12 * bscale


def test_neohooke_inverted_elements_are_counted():
    nx, ny, nz, h = 2, 2, 2, 1.0
    X, el, nid = box_grid(nx, ny, nz, h)
    U = np.zeros(3 * len(X))
    c = nid(1, 1, 1)
    U[3 * c:3 * c + 3] = [2.5, 2.5, 2.5]  # the centre node pushed through its neighbours
    with GpuSolver() as s:
        _, _, inv = s.assemble_hex8_neohooke(X, el, 1.0, 0.01, U)
    assert inv == 4  # as the host counts them (fistr_box_neohooke)
