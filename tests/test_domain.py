"""A decomposed mesh: hecmw_solve on each domain of an overlapping node-based
decomposition, with hecmw_update_R (halo exchange) and hecmw_allreduce_R1.

The reference's localised preconditioners make the iteration count depend on the
decomposition (SSOR and ILU(0) of each domain's internal block; the block diagonal
is unchanged), so the oracle here is its own domain-decomposed CG (o33_solve_dd) on
the same partition, and the gathered solution is also checked against the one-domain
solve of the whole mesh.

CPU: the partitioner's tables (internal rows complete, every export list the
neighbour's import list); one domain reproduces the one-domain oracle bit for bit;
2-4 domains converge to the whole-mesh solution; the same solve as two gloo processes
(torch.distributed, world size 2) gives the threads' bits.  GPU: each domain a
GpuSolver handle driven by its own thread on the one GPU (the domains exchange
through the host, no kernel waits on another) against the oracle: the same iteration
count within 2, solution within 1e-8 relative, the global true residual below the
tolerance, also with two outer preconditioner passes; the same as two processes with
a handle each, exchanging over torch.distributed (gloo); and the options a domain does
not run are refused (9101).
"""
import os
import socket
import sys
import threading

import numpy as np
import pytest
import torch.multiprocessing as mp

from frontistr_b200.domain import LocalExchange, gather_solution, partition
from frontistr_b200.mesh import box_system
from oracle_ctypes import Oracle, solve_dd, solve_dd_threads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _system(seed=3):
    m = box_system(6, 5, 12, jitter=0.2, sigma_E=1.0, nu_range=(0.25, 0.40), seed=seed)
    m.set_iter(20000)
    return m


def _domains(m, nd, precond, iterpremax=1):
    doms = partition(m, nd)
    for d in doms:
        d.matrix.set_precond(precond)
        d.matrix.set_iterpremax(iterpremax)
    return doms


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("nd", [2, 3, 4])
def test_partition_tables(nd):
    m = _system()
    doms = partition(m, nd)
    full = m.to_scipy().toarray()
    owned = np.zeros(m.N, np.int32)
    for d in doms:
        lm, g = d.matrix, d.global_ids
        owned[g[:d.N]] += 1
        # internal rows: complete, equal to the global rows at the local columns
        D = lm.D.reshape(-1, 3, 3)
        for i in range(d.N):
            gi = g[i]
            np.testing.assert_array_equal(D[i], full[3 * gi:3 * gi + 3, 3 * gi:3 * gi + 3])
            cols = list(lm.itemL[lm.indexL[i]:lm.indexL[i + 1]] - 1) + list(lm.itemU[lm.indexU[i]:lm.indexU[i + 1]] - 1)
            gcols = sorted(int(g[c]) for c in cols)
            nz = sorted(set(np.flatnonzero(np.any(full[3 * gi:3 * gi + 3].reshape(3, -1, 3) != 0, axis=(0, 2))))
                        - {int(gi)})
            assert set(nz) <= set(gcols)
        # every export list is the neighbour's import list from this domain
        c = d.comm
        for k, q in enumerate(c.neighbor_pe):
            exp = g[c.export_item[c.export_index[k]:c.export_index[k + 1]] - 1]
            cq = doms[q].comm
            kk = list(cq.neighbor_pe).index(d.comm.my_rank)
            imp = doms[q].global_ids[cq.import_item[cq.import_index[kk]:cq.import_index[kk + 1]] - 1]
            np.testing.assert_array_equal(exp, imp)
    assert np.all(owned == 1)


def test_oracle_one_domain_is_the_serial_solve():
    m = _system()
    ref = Oracle(m).solve()
    [out] = solve_dd_threads(partition(m, 1))
    assert out["error"] == ref["error"] == 0 and out["iter"] == ref["iter"]
    np.testing.assert_array_equal(out["X"], ref["X"])


@pytest.mark.parametrize("nd", [2, 3, 4])
@pytest.mark.parametrize("precond", [1, 3, 10, 11, 12])
def test_oracle_domains_converge_to_the_mesh_solution(nd, precond):
    m = _system()
    g = m.copy()
    g.set_precond(precond)
    ref = Oracle(g).solve()
    doms = _domains(m, nd, precond)
    out = solve_dd_threads(doms)
    assert all(o["error"] == 0 for o in out)
    assert len({o["iter"] for o in out}) == 1 and len({o["resid_true"] for o in out}) == 1
    X = gather_solution(doms, [o["X"] for o in out], m.N)
    assert _rel(X, ref["X"]) <= 1e-7
    assert Oracle(m).rel_resid(X, m.B) <= 1.0e-8
    if precond == 3:  # the block diagonal does not depend on the decomposition
        assert abs(out[0]["iter"] - ref["iter"]) <= 2
    # the halo of X is the owners' values (the final hecmw_update_R)
    for d, o in zip(doms, out):
        np.testing.assert_array_equal(o["X"].reshape(-1, 3)[d.N:], X.reshape(-1, 3)[d.global_ids[d.N:]])


@pytest.mark.parametrize("precond", [1, 10])
def test_oracle_domains_outer_preconditioner_passes(precond):
    """iterPREmax = 2: the second pass forms R - A Z, whose product updates the halo
    of Z (hecmw_precond.f90:166)."""
    m = _system()
    doms = _domains(m, 3, precond, iterpremax=2)
    out = solve_dd_threads(doms)
    assert all(o["error"] == 0 for o in out)
    X = gather_solution(doms, [o["X"] for o in out], m.N)
    assert Oracle(m).rel_resid(X, m.B) <= 1.0e-8
    one = solve_dd_threads(_domains(m, 3, precond, iterpremax=1))
    assert out[0]["iter"] < one[0]["iter"]


def _partition_loops(m, ndom):
    """The partition rule row by row (a slow restatement of domain.partition)."""
    from frontistr_b200.domain import slab_owner
    n = m.N
    owner = slab_owner(n, ndom)
    D0, AL0, AU0 = m.D.reshape(-1, 9), m.AL.reshape(-1, 9), m.AU.reshape(-1, 9)
    rows = []
    for i in range(n):
        lo, hi, ulo, uhi = m.indexL[i], m.indexL[i + 1], m.indexU[i], m.indexU[i + 1]
        rows.append((np.concatenate([m.itemL[lo:hi] - 1, [i], m.itemU[ulo:uhi] - 1]).astype(np.int64),
                     np.concatenate([AL0[lo:hi], D0[i:i + 1], AU0[ulo:uhi]])))
    members = [np.flatnonzero(owner == d) for d in range(ndom)]
    externals = []
    for d in range(ndom):
        ext = sorted({int(c) for g in members[d] for c in rows[g][0] if owner[c] != d},
                     key=lambda g: (int(owner[g]), g))
        externals.append(np.array(ext, dtype=np.int64))
    out = []
    for d in range(ndom):
        gids = np.concatenate([members[d], externals[d]]).astype(np.int64)
        loc = {int(g): k for k, g in enumerate(gids)}
        L, U, Dm = [], [], np.zeros((gids.size, 9))
        for k, g in enumerate(gids):
            c, v = rows[int(g)]
            lc = np.array([loc.get(int(x), -1) for x in c])
            keep = lc >= 0
            for col, val in sorted(zip(lc[keep], v[keep]), key=lambda t: t[0]):
                if col < k:
                    L.append((k, col, val))
                elif col == k:
                    Dm[k] = val
                else:
                    U.append((k, col, val))
        nb = sorted({int(owner[g]) for g in externals[d]} |
                    {q for q in range(ndom) if q != d and np.any(owner[externals[q]] == d)})
        imp = [[loc[int(g)] + 1 for g in externals[d] if owner[g] == q] for q in nb]
        exp = [[loc[int(g)] + 1 for g in externals[q] if owner[g] == d] for q in nb]
        out.append((gids, members[d].size, L, U, Dm, nb, imp, exp))
    return out


@pytest.mark.parametrize("nd", [2, 3, 4])
def test_partition_matches_the_row_by_row_rule(nd):
    m = _system(seed=5)
    fast = partition(m, nd)
    for dom, (gids, N, L, U, Dm, nb, imp, exp) in zip(fast, _partition_loops(m, nd)):
        lm, c = dom.matrix, dom.comm
        np.testing.assert_array_equal(dom.global_ids, gids)
        assert lm.N == N and lm.NP == gids.size
        np.testing.assert_array_equal(lm.D.reshape(-1, 9), Dm)
        for part, ind, item, A in ((L, lm.indexL, lm.itemL, lm.AL), (U, lm.indexU, lm.itemU, lm.AU)):
            assert ind[-1] == len(part)
            for j, (row, col, val) in enumerate(part):
                assert ind[row] <= j < ind[row + 1] and item[j] == col + 1
                np.testing.assert_array_equal(A.reshape(-1, 9)[j], val)
        assert list(c.neighbor_pe) == nb
        for k in range(len(nb)):
            assert list(c.import_item[c.import_index[k]:c.import_index[k + 1]]) == imp[k]
            assert list(c.export_item[c.export_index[k]:c.export_index[k + 1]]) == exp[k]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_rank(rank, world, port, out):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from datetime import timedelta
    from frontistr_b200.domain import TorchExchange, partition
    from oracle_ctypes import solve_dd
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        dom = _domains(_system(), world, 1)[rank]
        r = solve_dd(dom, TorchExchange(dom.comm))
        out[rank] = (r["error"], r["iter"], r["X"].tolist())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_oracle_domains_gloo_world2():
    """Two processes over torch.distributed (gloo): the same bits as two threads."""
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_gloo_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    doms = _domains(_system(), 2, 1)
    ref = solve_dd_threads(doms)
    for k in range(2):
        assert res[k][0] == ref[k]["error"] == 0 and res[k][1] == ref[k]["iter"]
        np.testing.assert_array_equal(np.array(res[k][2]), ref[k]["X"])


def _gpu_domains(doms, method_override=None):
    """Each domain solved by its own GpuSolver handle in its own thread."""
    from frontistr_b200.solver import GpuSolver
    ex = LocalExchange(doms)
    out = [None] * len(doms)
    errs = []

    def run(k):
        try:
            with GpuSolver() as s:
                m = doms[k].matrix.copy()
                if method_override is not None:
                    method_override(m)
                s.set_matrix(m)
                s.set_domain(doms[k].comm, ex.endpoint(k))
                info = s.solve_resident(m.B, m.X, m.Iarray, m.Rarray)
                out[k] = (info, m)
        except BaseException as e:  # surfaced below
            errs.append(e)
            ex.barrier.abort()

    ts = [threading.Thread(target=run, args=(k,)) for k in range(len(doms))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errs:
        raise errs[0]
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("nd,precond,iterpremax", [(2, 1, 1), (2, 3, 1), (2, 10, 1), (3, 1, 1), (3, 3, 1),
                                                   (3, 10, 1), (3, 1, 2), (2, 10, 2), (3, 11, 1), (2, 12, 1)])
def test_gpu_domains_match_oracle(nd, precond, iterpremax):
    m = _system(seed=7)
    doms = _domains(m, nd, precond, iterpremax)
    ref = solve_dd_threads(doms)
    out = _gpu_domains(doms)
    Xg = gather_solution(doms, [o[1].X for o in out], m.N)
    Xo = gather_solution(doms, [r["X"] for r in ref], m.N)
    for (info, lm), r in zip(out, ref):
        assert info["error"] == r["error"] == 0
        assert abs(info["iter"] - r["iter"]) <= 2, (info["iter"], r["iter"])
        assert lm.get_flag_converged() == 1
    assert _rel(Xg, Xo) <= 1e-8
    assert Oracle(m).rel_resid(Xg, m.B) <= 1.0e-8
    for d, (info, lm) in zip(doms, out):  # the halo of X holds the owners' values
        np.testing.assert_array_equal(lm.X.reshape(-1, 3)[d.N:], Xg.reshape(-1, 3)[d.global_ids[d.N:]])


@pytest.mark.gpu
def test_gpu_domain_refuses_other_options():
    from frontistr_b200.solver import HecmwSolverError
    m = _system()
    def mode1(a):
        a.Iarray[41] = 1

    for change in (lambda a: a.set_method(2), lambda a: a.set_scaling(1), mode1):
        doms = _domains(m, 2, 1)
        with pytest.raises(HecmwSolverError) as e:
            _gpu_domains(doms, change)
        assert e.value.code == 9101


def _gpu_rank(rank, world, port, out):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from datetime import timedelta
    from frontistr_b200.domain import TorchExchange
    from frontistr_b200.solver import GpuSolver
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        dom = _domains(_system(seed=7), world, 1)[rank]
        m = dom.matrix.copy()
        with GpuSolver() as s:
            s.set_matrix(m)
            s.set_domain(dom.comm, TorchExchange(dom.comm))
            info = s.solve_resident(m.B, m.X, m.Iarray, m.Rarray)
        out[rank] = (info["error"], info["iter"], m.X.tolist())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_gpu_domains_as_processes_over_gloo():
    """One process and handle per domain, the exchanges over torch.distributed (gloo,
    host buffers), as ranks of a distributed run; here both ranks share the one GPU
    (their kernels never wait on each other)."""
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        out = man.dict()
        mp.start_processes(_gpu_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    m = _system(seed=7)
    doms = _domains(m, 2, 1)
    ref = solve_dd_threads(doms)
    X = gather_solution(doms, [np.array(res[k][2]) for k in range(2)], m.N)
    Xo = gather_solution(doms, [r["X"] for r in ref], m.N)
    for k in range(2):
        assert res[k][0] == ref[k]["error"] == 0 and abs(res[k][1] - ref[k]["iter"]) <= 2
    assert _rel(X, Xo) <= 1e-8
    assert Oracle(m).rel_resid(X, m.B) <= 1.0e-8
