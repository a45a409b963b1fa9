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


def _global_rows(m):
    """Per global row: (columns, 9-value blocks) in ascending column order, 0-based."""
    D = m.D.reshape(-1, 9)
    AL = m.AL.reshape(-1, 9)
    AU = m.AU.reshape(-1, 9)
    rows = []
    for i in range(m.N):
        lo, hi = m.indexL[i], m.indexL[i + 1]
        ulo, uhi = m.indexU[i], m.indexU[i + 1]
        cols = np.concatenate([m.itemL[lo:hi] - 1, [i], m.itemU[ulo:uhi] - 1]).astype(np.int64)
        vals = np.concatenate([AL[lo:hi], D[i:i + 1], AU[ulo:uhi]])
        rows.append((cols, vals))
    return rows


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
    rows = _global_rows(m)
    members = [np.flatnonzero(owner == d) for d in range(ndom)]
    local_of = []  # per domain: dict global id -> local id (0-based)
    externals = []
    for d in range(ndom):
        internal = members[d]
        ext = set()
        for g in internal:
            for c in rows[g][0]:
                if owner[c] != d:
                    ext.add(int(c))
        ext = sorted(ext, key=lambda g: (int(owner[g]), g))
        externals.append(np.array(ext, dtype=np.int64))
        gids = np.concatenate([internal, externals[d]]).astype(np.int64)
        local_of.append({int(g): k for k, g in enumerate(gids)})
    domains = []
    for d in range(ndom):
        internal, ext = members[d], externals[d]
        gids = np.concatenate([internal, ext]).astype(np.int64)
        loc = local_of[d]
        NP, N = gids.size, internal.size
        indexL, indexU, itemL, itemU, AL, AU = [0], [0], [], [], [], []
        D = np.zeros((NP, 9))
        for k, g in enumerate(gids):
            cols, vals = rows[int(g)]
            lcols = np.array([loc.get(int(c), -1) for c in cols], dtype=np.int64)
            keep = lcols >= 0
            lcols, lvals = lcols[keep], vals[keep]
            order = np.argsort(lcols, kind="stable")
            for lc, v in zip(lcols[order], lvals[order]):
                if lc < k:
                    itemL.append(lc + 1)
                    AL.append(v)
                elif lc == k:
                    D[k] = v
                else:
                    itemU.append(lc + 1)
                    AU.append(v)
            indexL.append(len(itemL))
            indexU.append(len(itemU))
        for items_, vals_ in ((itemL, AL), (itemU, AU)):
            if not items_:
                items_.append(0)
                vals_.append(np.zeros(9))
        B = np.zeros(3 * NP)
        B.reshape(-1, 3)[:] = m.B.reshape(-1, 3)[gids]
        lm = HecMatrix(N, NP, np.array(indexL, np.int32), np.array(itemL, np.int32),
                       np.array(indexU, np.int32), np.array(itemU, np.int32), D.reshape(-1),
                       np.array(AL, np.float64).reshape(-1), np.array(AU, np.float64).reshape(-1), B=B)
        lm.Iarray, lm.Rarray = m.Iarray.copy(), m.Rarray.copy()
        # communication table: import = my external nodes by owner; export = my internal
        # nodes that a neighbour holds as external, in that neighbour's import order
        nbrs = sorted(set(int(owner[g]) for g in ext) |
                      set(q for q in range(ndom) if q != d and np.any(owner[externals[q]] == d)))
        imp_index, imp_item, exp_index, exp_item = [0], [], [0], []
        for q in nbrs:
            imp = [g for g in ext if owner[g] == q]
            imp_item += [loc[int(g)] + 1 for g in imp]
            imp_index.append(len(imp_item))
            exp = [g for g in externals[q] if owner[g] == d]  # q's import order from d
            exp_item += [loc[int(g)] + 1 for g in exp]
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
