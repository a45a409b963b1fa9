"""Host-side mirror of FrontISTR's solver interface on top of the CUDA C ABI.

``hecmw_solve(hecMAT)`` follows hecmw_solve (hecmw1/src/solver/main/hecmw_solver.f90:9-88)
for METHOD=1-7 (CG, BiCGSTAB, GMRES, GPBiCG, GMRESR, GMRESREN, CR): it updates hecMAT.X and the converged / diverged flags in
hecMAT.Iarray(81)/(82), consumes the preconditioner flags 97/98 and returns the
iteration record.  Error behaviour follows hecmw_solve_error
(hecmw1/src/solver/init/hecmw_solve_error.f90:20-93): 1001 and 2001 abort the
reference (here: HecmwSolverError is raised), 2002 and 3001 are warnings, and
3002-3004 set the diverged flag.  There is no CPU fallback: every call goes to
libhecmw33_gpu.so.
"""
import ctypes

import numpy as np

from ._lib import gpu_lib
from .matrix import HecMatrix  # noqa: F401

FATAL = {1001, 2001, 9001, 9100, 9101, 9102, 9103, 9104}


class HecmwSolverError(RuntimeError):
    def __init__(self, code, message):
        super().__init__("HEC-MW-SOLVER-E-%d: %s" % (code, message))
        self.code = code


def _i(v):
    return ctypes.byref(ctypes.c_int(int(v)))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def last_error():
    lib = gpu_lib()
    buf = ctypes.create_string_buffer(4096)
    lib.hecmw33_gpu_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


class GpuSolver:
    """One solver handle (its own CUDA stream and device buffers)."""

    def __init__(self):
        self.lib = gpu_lib()
        h, err = ctypes.c_int(0), ctypes.c_int(0)
        self.lib.hecmw33_gpu_create(ctypes.byref(h), ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        self.handle = h
        self.N = None

    def close(self):
        if getattr(self, "handle", None) is not None:
            err = ctypes.c_int(0)
            self.lib.hecmw33_gpu_destroy(ctypes.byref(self.handle), ctypes.byref(err))
            self.handle = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, code, fatal_only=True):
        if code == 0:
            return
        if code in FATAL or not fatal_only:
            raise HecmwSolverError(code, last_error())

    # ---- matrix ------------------------------------------------------------
    def set_matrix(self, m, Iarray=None):
        err = ctypes.c_int(0)
        ia = None if Iarray is None else np.ascontiguousarray(Iarray, dtype=np.int32)
        self.lib.hecmw33_gpu_set_matrix(
            ctypes.byref(self.handle), _i(m.N), _i(m.NP), _i(m.NPL), _i(m.NPU),
            _ip(m.indexL), _ip(m.itemL), _ip(m.indexU), _ip(m.itemU), _dp(m.D), _dp(m.AL), _dp(m.AU),
            _ip(ia) if ia is not None else None, ctypes.byref(err))
        self._check(err.value)
        self.N = m.N

    def set_mpc(self, index, item, dof, val, const=None):
        """The mesh's MPCs (hecmwST_local_mesh%mpc: mpc_index(0:n), 1-based mpc_item,
        mpc_dof, mpc_val, mpc_const; the first term of an MPC is its slave) for the
        resident matrix: a solve with MPC_METHOD = Iarray(13) = 2 runs MPC-CG, whose
        products are T^T A T x (hecmw33_gpu_set_mpc)."""
        ix = np.ascontiguousarray(index, dtype=np.int32)
        it = np.ascontiguousarray(item, dtype=np.int32)
        df = np.ascontiguousarray(dof, dtype=np.int32)
        vl = np.ascontiguousarray(val, dtype=np.float64)
        cs = np.zeros(len(ix) - 1) if const is None else np.ascontiguousarray(const, dtype=np.float64)
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_set_mpc(ctypes.byref(self.handle), _i(len(ix) - 1), _ip(ix), _ip(it), _ip(df),
                                     _dp(vl), _dp(cs), ctypes.byref(err))
        self._check(err.value, fatal_only=False)

    def set_domain(self, comm, endpoint):
        """The communication table (domain.CommTable) of the resident domain matrix
        (N < NP) and its exchanges: endpoint.exchange(send) -> recv and
        endpoint.allreduce(v) (domain.LocalExchange / TorchExchange), called by the C
        solver at every hecmw_update_R / hecmw_allreduce_R1 (hecmw33_gpu_set_domain).
        An exception inside them turns the exchanged values into NaN, so that the CG
        stops at its next check; solve() then raises it."""
        from ._abi import ALLREDUCE_FN, EXCHANGE_FN
        n_send = 3 * int(comm.export_index[-1]) if comm.n_neighbor_pe else 0
        n_recv = 3 * int(comm.import_index[-1]) if comm.n_neighbor_pe else 0
        self._cb_error = None

        def exchange(_ctx, sp, rp):
            try:
                if self._cb_error is not None:
                    raise self._cb_error
                send = np.ctypeslib.as_array(sp, shape=(n_send,)).copy() if n_send else np.zeros(0)
                recv = np.asarray(endpoint.exchange(send), dtype=np.float64)
                if n_recv:
                    np.ctypeslib.as_array(rp, shape=(n_recv,))[:] = recv
            except BaseException as e:  # noqa: BLE001 -- surfaced by solve()
                self._cb_error = self._cb_error or e
                if n_recv:
                    np.ctypeslib.as_array(rp, shape=(n_recv,))[:] = np.nan

        def allreduce(_ctx, v):
            try:
                if self._cb_error is not None:
                    raise self._cb_error
                return float(endpoint.allreduce(v))
            except BaseException as e:  # noqa: BLE001
                self._cb_error = self._cb_error or e
                return float("nan")

        self._domain_cbs = (EXCHANGE_FN(exchange), ALLREDUCE_FN(allreduce))
        self._domain_arrays = (comm.neighbor_pe, comm.import_index, comm.import_item, comm.export_index,
                               comm.export_item)
        err = ctypes.c_int(0)
        empty = np.zeros(1, np.int32)
        self.lib.hecmw33_gpu_set_domain(
            ctypes.byref(self.handle), _i(comm.n_neighbor_pe), _ip(comm.neighbor_pe), _ip(comm.import_index),
            _ip(comm.import_item if comm.import_item.size else empty),
            _ip(comm.export_index), _ip(comm.export_item if comm.export_item.size else empty),
            self._domain_cbs[0], self._domain_cbs[1], None, ctypes.byref(err))
        self._check(err.value, fatal_only=False)

    def condition_estimate(self):
        """(n, emin, emax) of the last solve's Lanczos estimate (ESTCOND, Iarray(14));
        n = 0 when it was off."""
        n, lo, hi, err = ctypes.c_int(0), ctypes.c_double(0), ctypes.c_double(0), ctypes.c_int(0)
        self.lib.hecmw33_gpu_condition_estimate(ctypes.byref(self.handle), ctypes.byref(n), ctypes.byref(lo),
                                                ctypes.byref(hi), ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        return n.value, lo.value, hi.value

    def _raise_cb_error(self):
        e = getattr(self, "_cb_error", None)
        if e is not None:
            self._cb_error = None
            raise e

    def matvec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_matvec(ctypes.byref(self.handle), _dp(x), _dp(y), ctypes.byref(err))
        self._check(err.value)
        return y

    def precond_apply(self, r, Iarray, Rarray):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty_like(r)
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_precond_apply(ctypes.byref(self.handle), _dp(r), _dp(z), _ip(Iarray),
                                           _dp(Rarray), ctypes.byref(err))
        self._check(err.value)
        return z

    # ---- HEX8 assembly on the device -------------------------------------------
    def assemble_hex8(self, coords, elements, E, nu, F=None, fixed=(), symbolic=True):
        """Assembles a linear-elastic HEX8 mesh into the resident matrix and right-hand
        side (hecmw33_gpu_assemble_hex8).  coords (n,3); elements (ne,8) 0-based node
        indices in hex8n order; E, nu scalars or per element; F (3n) nodal loads;
        fixed: iterable of (node0, dof1, value) applied in order."""
        coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
        conn = np.ascontiguousarray(np.asarray(elements, dtype=np.int32) + 1)
        n, ne = coords.shape[0], conn.shape[0]
        Ee = np.ascontiguousarray(np.broadcast_to(np.asarray(E, dtype=np.float64), (ne,)))
        nue = np.ascontiguousarray(np.broadcast_to(np.asarray(nu, dtype=np.float64), (ne,)))
        fixed = list(fixed)
        bn = np.array([f[0] + 1 for f in fixed] or [0], dtype=np.int32)
        bd = np.array([f[1] for f in fixed] or [0], dtype=np.int32)
        bv = np.array([f[2] for f in fixed] or [0.0], dtype=np.float64)
        Fp = None if F is None else np.ascontiguousarray(F, dtype=np.float64)
        npl, npu, err = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        self.lib.hecmw33_gpu_assemble_hex8(
            ctypes.byref(self.handle), _i(n), _dp(coords), _i(ne), _ip(conn), _dp(Ee), _dp(nue),
            _dp(Fp) if Fp is not None else None, _i(len(fixed)), _ip(bn), _ip(bd), _dp(bv),
            _i(1 if symbolic else 0), ctypes.byref(npl), ctypes.byref(npu), ctypes.byref(err))
        self._check(err.value)
        self.N = n
        self.NPL, self.NPU = npl.value, npu.value
        return self.NPL, self.NPU

    def assemble_hex8_neohooke(self, coords, elements, C10, D1, U, F=None, fixed=(), symbolic=True):
        """Neo-Hookean tangent K(U) and right-hand side F - f_int(U), then the
        constraints (hecmw33_gpu_assemble_hex8_neohooke); returns (NPL, NPU, inverted)."""
        coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
        conn = np.ascontiguousarray(np.asarray(elements, dtype=np.int32) + 1)
        n, ne = coords.shape[0], conn.shape[0]
        U = np.ascontiguousarray(U, dtype=np.float64)
        fixed = list(fixed)
        bn = np.array([f[0] + 1 for f in fixed] or [0], dtype=np.int32)
        bd = np.array([f[1] for f in fixed] or [0], dtype=np.int32)
        bv = np.array([f[2] for f in fixed] or [0.0], dtype=np.float64)
        Fp = None if F is None else np.ascontiguousarray(F, dtype=np.float64)
        npl, npu, inv, err = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        c10, d1 = ctypes.c_double(C10), ctypes.c_double(D1)
        self.lib.hecmw33_gpu_assemble_hex8_neohooke(
            ctypes.byref(self.handle), _i(n), _dp(coords), _i(ne), _ip(conn), ctypes.byref(c10),
            ctypes.byref(d1), _dp(U), _dp(Fp) if Fp is not None else None, _i(len(fixed)), _ip(bn), _ip(bd),
            _dp(bv), _i(1 if symbolic else 0), ctypes.byref(npl), ctypes.byref(npu), ctypes.byref(inv),
            ctypes.byref(err))
        self._check(err.value)
        self.N = n
        self.NPL, self.NPU = npl.value, npu.value
        return self.NPL, self.NPU, inv.value

    def get_matrix(self):
        """The resident matrix and right-hand side as a HecMatrix."""
        from .matrix import HecMatrix
        m = HecMatrix.empty(self.N, self.NPL, self.NPU)
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_get_matrix(ctypes.byref(self.handle), _ip(m.indexL), _ip(m.itemL), _ip(m.indexU),
                                        _ip(m.itemU), _dp(m.D), _dp(m.AL), _dp(m.AU), _dp(m.B),
                                        ctypes.byref(err))
        self._check(err.value)
        return m

    def solve_assembled(self, Iarray, Rarray, X=None):
        """Solves the resident assembled system; returns (X, record)."""
        X = np.zeros(3 * self.N) if X is None else np.ascontiguousarray(X, dtype=np.float64).copy()
        err, it, res = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0)
        times = np.zeros(3)
        self.lib.hecmw33_gpu_solve_assembled(ctypes.byref(self.handle), _dp(X), _ip(Iarray), _dp(Rarray),
                                             ctypes.byref(it), ctypes.byref(res), _dp(times), ctypes.byref(err))
        self._check(err.value)
        return X, self._record(err.value, it, res, times)

    def colouring(self):
        n = self.N
        nc = ctypes.c_int(0)
        ci = np.zeros(n + 1, np.int32)
        perm = np.zeros(n, np.int32)
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_get_colouring(ctypes.byref(self.handle), ctypes.byref(nc), _ip(ci), _ip(perm),
                                           ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        return ci[:nc.value + 1].copy(), perm

    # ---- solves ------------------------------------------------------------
    def _record(self, err, it, res, times):
        return dict(error=err, iter=it.value, resid=res.value, t_setup=times[0], t_solve=times[1],
                    t_comm=times[2])

    def solve(self, m):
        """The drop-in hecmw_solve: matrix upload + solve; updates m.X and m.Iarray."""
        err, it, res = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0)
        times = np.zeros(3)
        self.lib.hecmw33_gpu_solve(
            ctypes.byref(self.handle), _i(m.N), _i(m.NP), _i(m.NPL), _i(m.NPU),
            _ip(m.indexL), _ip(m.itemL), _ip(m.indexU), _ip(m.itemU), _dp(m.D), _dp(m.AL), _dp(m.AU),
            _dp(m.B), _dp(m.X), _ip(m.Iarray), _dp(m.Rarray), ctypes.byref(it), ctypes.byref(res),
            _dp(times), ctypes.byref(err))
        self.N = m.N
        self._raise_cb_error()
        self._check(err.value)
        return self._record(err.value, it, res, times)

    def solve_resident(self, B, X, Iarray, Rarray):
        """Solve on the matrix already uploaded; X (host) is updated in place."""
        err, it, res = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0)
        times = np.zeros(3)
        self.lib.hecmw33_gpu_solve_resident(ctypes.byref(self.handle), _dp(B), _dp(X), _ip(Iarray),
                                            _dp(Rarray), ctypes.byref(it), ctypes.byref(res), _dp(times),
                                            ctypes.byref(err))
        self._raise_cb_error()
        self._check(err.value)
        return self._record(err.value, it, res, times)

    def solve_resident_device(self, dB_ptr, dX_ptr, Iarray, Rarray):
        """Solve with B and X in device memory (raw device pointers, e.g. tensor.data_ptr())."""
        err, it, res = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0)
        times = np.zeros(3)
        self.lib.hecmw33_gpu_solve_resident_device(ctypes.byref(self.handle), ctypes.c_void_p(dB_ptr),
                                                   ctypes.c_void_p(dX_ptr), _ip(Iarray), _dp(Rarray),
                                                   ctypes.byref(it), ctypes.byref(res), _dp(times),
                                                   ctypes.byref(err))
        self._check(err.value)
        return self._record(err.value, it, res, times)

    def solve_multi(self, B, X, Iarray, Rarray):
        """Several load cases on the resident matrix (hecmw33_gpu_solve_multi).

        B, X: host arrays of shape (nrhs, 3N) (row k = load case k, i.e. the
        column-major 3N x nrhs layout of the C call); X is updated in place.
        Returns per-case iter, resid, error and true_resid arrays and the times."""
        B = np.ascontiguousarray(B, dtype=np.float64)
        assert X.flags.c_contiguous and X.dtype == np.float64 and X.shape == B.shape
        nrhs = B.shape[0]
        it = np.zeros(nrhs, np.int32)
        res = np.zeros(nrhs)
        errs = np.zeros(nrhs, np.int32)
        tres = np.zeros(nrhs)
        times = np.zeros(3)
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_solve_multi(ctypes.byref(self.handle), _i(nrhs), _dp(B), _dp(X), _ip(Iarray),
                                         _dp(Rarray), _ip(it), _dp(res), _ip(errs), _dp(tres), _dp(times),
                                         ctypes.byref(err))
        self._check(err.value)
        return dict(error=int(err.value), iter=it, resid=res, errors=errs, true_resid=tres,
                    t_setup=float(times[0]), t_solve=float(times[1]))

    def solve_multi_device(self, nrhs, dB_ptr, dX_ptr, Iarray, Rarray):
        """As solve_multi with B and X in device memory (3N x nrhs column-major)."""
        it = np.zeros(nrhs, np.int32)
        res = np.zeros(nrhs)
        errs = np.zeros(nrhs, np.int32)
        tres = np.zeros(nrhs)
        times = np.zeros(3)
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_solve_multi_device(ctypes.byref(self.handle), _i(nrhs), ctypes.c_void_p(dB_ptr),
                                                ctypes.c_void_p(dX_ptr), _ip(Iarray), _dp(Rarray), _ip(it),
                                                _dp(res), _ip(errs), _dp(tres), _dp(times), ctypes.byref(err))
        self._check(err.value)
        return dict(error=int(err.value), iter=it, resid=res, errors=errs, true_resid=tres,
                    t_setup=float(times[0]), t_solve=float(times[1]))

    def last_solve_info(self):
        info = np.zeros(16, np.int32)
        dinfo = np.zeros(16)
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_last_solve_info(ctypes.byref(self.handle), _ip(info), _dp(dinfo), ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        return dict(iter=int(info[0]), kernels=int(info[1]), sweep_groups=int(info[2]),
                    kernels_per_iter=int(info[3]), nz_blocks=int(info[4]), spmv_slices=int(info[5]),
                    spmv_slots=int(info[6]), outer=int(info[7]), t_solve=float(dinfo[0]),
                    t_setup=float(dinfo[1]), spmv_bytes=float(dinfo[2]), iter_bytes=float(dinfo[3]),
                    device_bytes=float(dinfo[4]), true_resid=float(dinfo[5]), learned=int(info[8]),
                    fallback=int(info[9]), pairs=int(info[10]))

    # ---- learned preconditioner (hecmw33_gpu_learn_*) -------------------------
    def learn_record(self, enable=1, max_pairs=0):
        n, err = ctypes.c_int(0), ctypes.c_int(0)
        self.lib.hecmw33_gpu_learn_record(ctypes.byref(self.handle), _i(enable), _i(max_pairs), ctypes.byref(n),
                                          ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        return n.value

    def learn_train(self, steps=100, lr=1e-3):
        loss = np.zeros(2)
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_learn_train(ctypes.byref(self.handle), _i(steps), ctypes.byref(ctypes.c_double(lr)),
                                         _dp(loss), ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        return float(loss[0]), float(loss[1])

    def learn_get_weights(self):
        n, err = ctypes.c_int(0), ctypes.c_int(0)
        self.lib.hecmw33_gpu_learn_weights(ctypes.byref(self.handle), _i(0), None, ctypes.byref(n), ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        if n.value <= 0:
            return None
        th = np.zeros(n.value, np.float32)
        self.lib.hecmw33_gpu_learn_weights(ctypes.byref(self.handle), _i(0),
                                           th.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), ctypes.byref(n),
                                           ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        return th

    def learn_set_weights(self, theta):
        th = np.ascontiguousarray(theta, dtype=np.float32)
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_learn_weights(ctypes.byref(self.handle), _i(1),
                                           th.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                           ctypes.byref(ctypes.c_int(th.size)), ctypes.byref(err))
        self._check(err.value, fatal_only=False)

    def learn_eval(self, theta, R, E):
        th = np.ascontiguousarray(theta, dtype=np.float32)
        R = np.ascontiguousarray(R, dtype=np.float64)
        E = np.ascontiguousarray(E, dtype=np.float64)
        Z = np.zeros_like(R)
        grad = np.zeros(th.size, np.float32)
        loss = ctypes.c_double(0)
        err = ctypes.c_int(0)
        fp = ctypes.POINTER(ctypes.c_float)
        self.lib.hecmw33_gpu_learn_eval(ctypes.byref(self.handle), th.ctypes.data_as(fp), _dp(R), _dp(E), _dp(Z),
                                        ctypes.byref(loss), grad.ctypes.data_as(fp), ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        return Z, loss.value, grad

    def time_spmv(self, reps=20):
        ms = ctypes.c_double(0)
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_time_spmv(ctypes.byref(self.handle), _i(reps), ctypes.byref(ms), ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        return ms.value

    def time_precond(self, reps=20, lowp=0, smoother=False):
        """(ms per application, algorithmic bytes per application) of the resident
        preconditioner, one pass z = M^-1 r, timed with device events; smoother=True
        times the learned preconditioner's SSOR smoother (first-fit colour order)."""
        ms, nbytes = ctypes.c_double(0), ctypes.c_double(0)
        err = ctypes.c_int(0)
        flags = (1 if lowp else 0) | (2 if smoother else 0)
        self.lib.hecmw33_gpu_time_precond(ctypes.byref(self.handle), _i(reps), _i(flags), ctypes.byref(ms),
                                          ctypes.byref(nbytes), ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        return ms.value, nbytes.value


_default = None


_dumper = None


def hecmw_solve(hecMAT, solver=None, dumper=None):
    """hecmw_solve(hecMESH, hecMAT) for a whole mesh (N == NP): updates hecMAT.X and
    flags.  hecMAT.mpc (the mesh's MPC table, HecMatrix.mpc) goes to the solver
    (GpuSolver.set_mpc), so that MPC_METHOD = Iarray(13) = 2 runs MPC-CG.  A domain of a
    decomposed mesh is solved through GpuSolver.set_domain.

    With Iarray(31) = DUMPTYPE (1 MM, 2 CSR, 3 BSR) the matrix and right-hand side
    are dumped before the solve and the solution after it, as hecmw_solve_iterative
    does (hecmw_solver_Iterative.f90:90,160); a zero right-hand side returns before
    that (hecmw_solver.f90:32-37).  `dumper` (frontistr_b200.dump.Dumper) sets the
    directory and rank of the files; by default one process-wide Dumper in ".".
    """
    global _default, _dumper
    if solver is None:
        if _default is None:
            _default = GpuSolver()
        solver = _default
    if dumper is None:
        from .dump import Dumper
        if _dumper is None:
            _dumper = Dumper()
        dumper = _dumper
    mpc = getattr(hecMAT, "mpc", None)

    def run():
        if mpc is None:
            return solver.solve(hecMAT)
        solver.set_matrix(hecMAT, hecMAT.Iarray)
        solver.set_mpc(*mpc)
        return solver.solve_resident(hecMAT.B, hecMAT.X, hecMAT.Iarray, hecMAT.Rarray)

    b = hecMAT.B[:3 * hecMAT.NP]
    consts = 0.0 if mpc is None else float(np.dot(mpc[4], mpc[4]))
    if float(np.dot(b, b)) + consts == 0.0:
        return run()
    dumper.dump(hecMAT)
    info = run()
    dumper.dump_solution(hecMAT)
    return info


def colour_schedule(m, ncolor_in=10):
    """Host-only SSOR colour schedule (RCM + multicolouring) of a HecMatrix profile."""
    lib = gpu_lib()
    n = m.N
    nc = ctypes.c_int(0)
    ci = np.zeros(n + 1, np.int32)
    perm = np.zeros(n, np.int32)
    err = ctypes.c_int(0)
    lib.hecmw33_gpu_colour_schedule(_i(n), _ip(m.indexL), _ip(m.itemL), _ip(m.indexU), _ip(m.itemU),
                                    _i(ncolor_in), ctypes.byref(nc), _ip(ci), _ip(perm), ctypes.byref(err))
    if err.value:
        raise HecmwSolverError(err.value, last_error())
    return ci[:nc.value + 1].copy(), perm


def smoother_schedule(m):
    """Host-only colour schedule of the learned preconditioner's SSOR smoother
    (first-fit colours in node order): (colorindex, perm), as colour_schedule."""
    lib = gpu_lib()
    n = m.N
    nc = ctypes.c_int(0)
    ci = np.zeros(n + 1, np.int32)
    perm = np.zeros(n, np.int32)
    err = ctypes.c_int(0)
    lib.hecmw33_gpu_smoother_schedule(_i(n), _ip(m.indexL), _ip(m.itemL), _ip(m.indexU), _ip(m.itemU),
                                      ctypes.byref(nc), _ip(ci), _ip(perm), ctypes.byref(err))
    if err.value:
        raise HecmwSolverError(err.value, last_error())
    return ci[:nc.value + 1].copy(), perm


def coarse_aggregates(m, max_aggregates=0):
    """Host-only aggregates of the node graph of a HecMatrix profile (the coarse space of
    the learned two-level preconditioner): (number of aggregates, 0-based id per node)."""
    lib = gpu_lib()
    n = m.N
    na = ctypes.c_int(0)
    agg = np.zeros(n, np.int32)
    err = ctypes.c_int(0)
    lib.hecmw33_gpu_coarse_aggregates(_i(n), _ip(m.indexL), _ip(m.itemL), _ip(m.indexU), _ip(m.itemU),
                                      _i(max_aggregates), ctypes.byref(na), _ip(agg), ctypes.byref(err))
    if err.value:
        raise HecmwSolverError(err.value, last_error())
    return na.value, agg
