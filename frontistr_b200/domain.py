"""Node-based overlapping domain decomposition for the hecmw solver path.

A distributed FrontISTR run hands every rank one domain (hecmw1/src/common/hecmw_util_f.F90,
type hecmwST_local_mesh): its internal nodes numbered 1..N, then the external (halo)
nodes N+1..NP owned by neighbouring domains, and the communication table

    n_neighbor_pe, neighbor_pe(1:n)        the neighbouring domains
    import_index(0:n), import_item(:)      per neighbour, the local ids of the external
                                           nodes it owns (received)
    export_index(0:n), export_item(:)      per neighbour, the local ids of internal
                                           nodes it holds as external (sent)

The domain's hecmwST_matrix has NP rows; the rows of internal nodes are complete.
hecmw_update_R (hecmw1/src/solver/communication/hecmw_comm_f.F90:838-863, through
HECMW_SOLVE_SEND_RECV, hecmw_solver_SR.F90:36-179) sends, per neighbour, the values
at export_item and writes what it receives at import_item; hecmw_allreduce_R1 sums a
scalar over the domains.

This module builds such domains from one assembled system (the partitioner of the
distributed tests and benchmarks: hecmw_part1 itself is a separate tool) and gives
the two exchanges an implementation: `LocalExchange` for domains solved by threads of
one process, `TorchExchange` for one domain per process over torch.distributed.
"""
import threading

import numpy as np

from .matrix import HecMatrix


class CommTable:
    """The communication part of hecmwST_local_mesh (1-based items, 0-based ranks)."""

    def __init__(self, my_rank, neighbor_pe, import_index, import_item, export_index, export_item):
        self.my_rank = int(my_rank)
        self.neighbor_pe = np.ascontiguousarray(neighbor_pe, dtype=np.int32)
        self.import_index = np.ascontiguousarray(import_index, dtype=np.int32)
        self.import_item = np.ascontiguousarray(import_item, dtype=np.int32)
        self.export_index = np.ascontiguousarray(export_index, dtype=np.int32)
        self.export_item = np.ascontiguousarray(export_item, dtype=np.int32)

    @property
    def n_neighbor_pe(self):
        return int(self.neighbor_pe.size)

    def pack(self, x):
        """The send buffer of hecmw_solve_send_recv: x at export_item, 3 values each."""
        idx = self.export_item.astype(np.int64) - 1
        return np.ascontiguousarray(x.reshape(-1, 3)[idx].reshape(-1))

    def unpack(self, x, recv):
        """Received values into x at import_item (in place)."""
        idx = self.import_item.astype(np.int64) - 1
        x.reshape(-1, 3)[idx] = recv.reshape(-1, 3)


class Domain:
    """One domain: its matrix (N internal rows of NP), its communication table and
    the global node id of each local node."""

    def __init__(self, matrix, comm, global_ids):
        self.matrix = matrix
        self.comm = comm
        self.global_ids = np.ascontiguousarray(global_ids, dtype=np.int64)

    @property
    def N(self):
        return self.matrix.N

    @property
    def NP(self):
        return self.matrix.NP


def _global_csr(m):
    """The whole block matrix as CSR over nodes, each row in ascending column order
    (L, D, U): row pointer, 0-based columns, 9-value blocks."""
    n = m.N
    nl = np.diff(m.indexL[:n + 1]).astype(np.int64)
    nu = np.diff(m.indexU[:n + 1]).astype(np.int64)
    cnt = nl + 1 + nu
    ptr = np.zeros(n + 1, np.int64)
    np.cumsum(cnt, out=ptr[1:])
    rows = np.repeat(np.arange(n, dtype=np.int64), cnt)
    pos_in_row = np.arange(ptr[-1], dtype=np.int64) - ptr[rows]
    cols = np.empty(ptr[-1], np.int64)
    vals = np.empty((ptr[-1], 9))
    lsel = pos_in_row < nl[rows]
    dsel = pos_in_row == nl[rows]
    usel = pos_in_row > nl[rows]
    cols[lsel] = m.itemL[:m.indexL[n]].astype(np.int64) - 1
    vals[lsel] = m.AL.reshape(-1, 9)[:m.indexL[n]]
    cols[dsel] = np.arange(n)
    vals[dsel] = m.D.reshape(-1, 9)[:n]
    cols[usel] = m.itemU[:m.indexU[n]].astype(np.int64) - 1
    vals[usel] = m.AU.reshape(-1, 9)[:m.indexU[n]]
    return ptr, cols, vals


def slab_owner(n, ndom):
    """Domain of each node for contiguous ranges of node ids: on the lexicographically
    numbered boxes (x fastest) these are slabs across z."""
    return np.minimum((np.arange(n, dtype=np.int64) * ndom) // n, ndom - 1).astype(np.int32)


def partition(m, ndom, owner=None):
    """Split an assembled one-domain system (N == NP) into `ndom` overlapping domains.

    owner[i] is the domain of global node i (default: `slab_owner`).  Each domain's
    local nodes are its internal nodes (ascending global id) followed by the external
    nodes its internal rows reference (by owning domain, then global id).  Every row
    of a local node is the global row restricted to the local nodes: complete for the
    internal rows; for the external rows the values are those of the global matrix
    where the reference holds partial sums of the domain's elements -- the solve reads
    external rows nowhere (SpMV, inner products and every preconditioner apply run
    over the internal rows; hecmw_solver_las_33.F90:279, hecmw_precond_BILU_33.f90:98,130).
    B is the global right-hand side at the local nodes; X starts at zero."""
    n = m.N
    if m.NP != n:
        raise ValueError("partition: the input is one domain (N == NP)")
    owner = slab_owner(n, ndom) if owner is None else np.asarray(owner, dtype=np.int32)
    ptr, cols, vals = _global_csr(m)
    row_of = np.repeat(np.arange(n, dtype=np.int64), np.diff(ptr))
    members = [np.flatnonzero(owner == d).astype(np.int64) for d in range(ndom)]
    externals = []
    for d in range(ndom):
        mine = owner[row_of] == d
        ext = np.unique(cols[mine & (owner[cols] != d)])
        ext = ext[np.lexsort((ext, owner[ext]))]  # by owner, then global id
        externals.append(ext)
    domains = []
    for d in range(ndom):
        internal, ext = members[d], externals[d]
        gids = np.concatenate([internal, ext])
        N, NP = internal.size, gids.size
        loc = np.full(n, -1, np.int64)
        loc[gids] = np.arange(NP)
        # the local rows: the global rows of the local nodes, columns kept where local
        starts, ends = ptr[gids], ptr[gids + 1]
        lens = ends - starts
        sel = np.repeat(starts, lens) + (np.arange(lens.sum()) - np.repeat(np.cumsum(lens) - lens, lens))
        lrow = np.repeat(np.arange(NP, dtype=np.int64), lens)
        lcol = loc[cols[sel]]
        keep = lcol >= 0
        lrow, lcol, sel = lrow[keep], lcol[keep], sel[keep]
        order = np.lexsort((lcol, lrow))
        lrow, lcol, sel = lrow[order], lcol[order], sel[order]
        isL, isD, isU = lcol < lrow, lcol == lrow, lcol > lrow
        D = np.zeros((NP, 9))
        D[lrow[isD]] = vals[sel[isD]]
        indexL = np.zeros(NP + 1, np.int32)
        indexU = np.zeros(NP + 1, np.int32)
        np.cumsum(np.bincount(lrow[isL], minlength=NP), out=indexL[1:])
        np.cumsum(np.bincount(lrow[isU], minlength=NP), out=indexU[1:])
        itemL = (lcol[isL] + 1).astype(np.int32)
        itemU = (lcol[isU] + 1).astype(np.int32)
        AL = vals[sel[isL]]
        AU = vals[sel[isU]]
        if itemL.size == 0:  # keep the arrays non-empty (as HecMatrix.empty does)
            itemL, AL = np.zeros(1, np.int32), np.zeros((1, 9))
        if itemU.size == 0:
            itemU, AU = np.zeros(1, np.int32), np.zeros((1, 9))
        B = np.zeros(3 * NP)
        B.reshape(-1, 3)[:] = m.B.reshape(-1, 3)[gids]
        lm = HecMatrix(N, NP, indexL, itemL, indexU, itemU, D.reshape(-1), AL.reshape(-1), AU.reshape(-1), B=B)
        lm.Iarray, lm.Rarray = m.Iarray.copy(), m.Rarray.copy()
        # communication table: import = my external nodes by owner; export = my internal
        # nodes that a neighbour holds as external, in that neighbour's import order
        nbrs = sorted(set(int(q) for q in np.unique(owner[ext])) |
                      set(q for q in range(ndom) if q != d and np.any(owner[externals[q]] == d)))
        imp_index, imp_item, exp_index, exp_item = [0], [], [0], []
        for q in nbrs:
            imp = ext[owner[ext] == q]
            imp_item.extend((loc[imp] + 1).tolist())
            imp_index.append(len(imp_item))
            exq = externals[q]
            exp = exq[owner[exq] == d]  # q's import order from d
            exp_item.extend((loc[exp] + 1).tolist())
            exp_index.append(len(exp_item))
        comm = CommTable(d, nbrs, imp_index, imp_item, exp_index, exp_item)
        domains.append(Domain(lm, comm, gids))
    return domains


def gather_solution(domains, xs, n):
    """The global 3n vector from each domain's internal entries."""
    X = np.zeros(3 * n)
    for dom, x in zip(domains, xs):
        X.reshape(-1, 3)[dom.global_ids[:dom.N]] = np.asarray(x).reshape(-1, 3)[:dom.N]
    return X


class LocalExchange:
    """hecmw_update_R / hecmw_allreduce_R1 among the domains of one process, each
    driven by its own thread: the ranks meet at a barrier; a rank's buffer for
    neighbour q is taken by q.  Sums are formed in rank order, so every rank gets the
    same bits."""

    def __init__(self, domains, timeout=120.0):
        self.domains = domains
        self.n = len(domains)
        self.barrier = threading.Barrier(self.n, timeout=timeout)
        self.box = {}
        self.vals = [0.0] * self.n

    def endpoint(self, rank):
        return _LocalEndpoint(self, rank)


class _LocalEndpoint:
    def __init__(self, ex, rank):
        self.ex, self.rank = ex, rank
        self.comm = ex.domains[rank].comm

    def exchange(self, send):
        ex, c = self.ex, self.comm
        for k, q in enumerate(c.neighbor_pe):
            a, b = 3 * c.export_index[k], 3 * c.export_index[k + 1]
            ex.box[(self.rank, int(q))] = np.array(send[a:b], copy=True)
        ex.barrier.wait()
        recv = np.zeros(3 * int(c.import_index[-1]))
        for k, q in enumerate(c.neighbor_pe):
            a, b = 3 * c.import_index[k], 3 * c.import_index[k + 1]
            recv[a:b] = ex.box[(int(q), self.rank)]
        ex.barrier.wait()
        return recv

    def allreduce(self, v):
        ex = self.ex
        ex.vals[self.rank] = float(v)
        ex.barrier.wait()
        s = 0.0
        for x in ex.vals:
            s = s + x
        ex.barrier.wait()
        return s


class TorchExchange:
    """hecmw_update_R / hecmw_allreduce_R1 over torch.distributed (one domain per
    process): per neighbour an isend / irecv pair of float64 tensors (CPU tensors
    for gloo), and a float64 all_reduce."""

    def __init__(self, comm, device="cpu"):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.comm = comm
        self.device = device

    def exchange(self, send):
        torch, dist, c = self.torch, self.dist, self.comm
        send_t = torch.from_numpy(np.ascontiguousarray(send, dtype=np.float64)).to(self.device)
        recv_t = torch.zeros(3 * int(c.import_index[-1]), dtype=torch.float64, device=self.device)
        reqs = []
        for k, q in enumerate(c.neighbor_pe):
            a, b = 3 * int(c.export_index[k]), 3 * int(c.export_index[k + 1])
            if b > a:
                reqs.append(dist.isend(send_t[a:b].contiguous(), int(q)))
        for k, q in enumerate(c.neighbor_pe):
            a, b = 3 * int(c.import_index[k]), 3 * int(c.import_index[k + 1])
            if b > a:
                buf = torch.zeros(b - a, dtype=torch.float64, device=self.device)
                reqs.append((dist.irecv(buf, int(q)), buf, a, b))
        for r in reqs:
            if isinstance(r, tuple):
                r[0].wait()
                recv_t[r[2]:r[3]] = r[1]
            else:
                r.wait()
        return recv_t.cpu().numpy()

    def allreduce(self, v):
        t = self.torch.tensor([float(v)], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t)
        return float(t.item())
