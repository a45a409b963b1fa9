"""Host side of the batched solves (no GPU): the block-diagonal stacking of
independent systems, the seeded box generator of the batched workload, and the
per-system independence the batched solve relies on (the oracle's solve of the
stacked matrix equals the per-system solves when it is block diagonal)."""
import numpy as np

from frontistr_b200.batch import stack_systems
from frontistr_b200.mesh import random_box_batch


def test_stack_is_block_diagonal():
    systems = random_box_batch(4, edge_range=(2, 4), seed=7)
    big, sys_ptr = stack_systems(systems)
    assert sys_ptr[0] == 0 and sys_ptr[-1] == big.N
    A = big.to_scipy().toarray()
    for s, m in enumerate(systems):
        a, e = 3 * sys_ptr[s], 3 * sys_ptr[s + 1]
        assert np.array_equal(A[a:e, a:e], m.to_scipy().toarray())
        assert np.count_nonzero(A[a:e, :a]) == 0 and np.count_nonzero(A[a:e, e:]) == 0
        assert np.array_equal(big.B[a:e], m.B)
    # hecmwST invariants of the stacked profile
    assert big.indexL[0] == 0 and big.indexU[0] == 0
    for i in range(big.N):
        cols = big.itemL[big.indexL[i]:big.indexL[i + 1]]
        assert np.all(np.diff(cols) > 0) and (len(cols) == 0 or cols[-1] < i + 1)


def test_random_box_batch_is_seeded_and_in_range():
    a = random_box_batch(6, edge_range=(3, 7), seed=11)
    b = random_box_batch(6, edge_range=(3, 7), seed=11)
    for ma, mb in zip(a, b):
        assert ma.dims == mb.dims and np.array_equal(ma.D, mb.D) and np.array_equal(ma.B, mb.B)
        assert all(3 <= d <= 7 for d in ma.dims)
        nx, ny, nz = ma.dims
        loaded = np.nonzero(np.any(ma.B.reshape(-1, 3) != 0, axis=1))[0]
        assert len(loaded) == (nx + 1) * (ny + 1)  # every node of the face z = nz
        t = ma.B.reshape(-1, 3)[loaded]
        assert np.allclose(np.linalg.norm(t, axis=1), 1.0) and np.allclose(t, t[0])


def test_block_diagonal_solve_splits(tmp_path):
    """CG on the stacked matrix with one shared recurrence differs from independent
    solves, but the exact solution splits: A_big^-1 b = [A_s^-1 b_s] (what every
    system of a batched solve converges to)."""
    import scipy.sparse.linalg as spla
    systems = random_box_batch(3, edge_range=(2, 3), seed=5)
    big, sys_ptr = stack_systems(systems)
    x = spla.spsolve(big.to_scipy().tocsc(), big.B)
    for s, m in enumerate(systems):
        xs = spla.spsolve(m.to_scipy().tocsc(), m.B)
        assert np.allclose(x[3 * sys_ptr[s]:3 * sys_ptr[s + 1]], xs, rtol=1e-10, atol=1e-14)
