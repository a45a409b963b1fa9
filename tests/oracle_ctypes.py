"""ctypes bindings of the CPU oracle (oracle/hecmw33_oracle.c) for the tests.

The oracle is test infrastructure: the checker for the CUDA solver, and the
timed CPU baseline in bench.py.  It is never on the product path.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "libhecmw33_oracle.so")

_i32p = ctypes.POINTER(ctypes.c_int)
_f64p = ctypes.POINTER(ctypes.c_double)


class O33Matrix(ctypes.Structure):
    _fields_ = [("N", ctypes.c_int), ("NP", ctypes.c_int), ("NPL", ctypes.c_int),
                ("NPU", ctypes.c_int), ("indexL", _i32p), ("itemL", _i32p), ("indexU", _i32p),
                ("itemU", _i32p), ("D", _f64p), ("AL", _f64p), ("AU", _f64p), ("usejad", ctypes.c_int),
                ("n_mpc", ctypes.c_int), ("mpc_index", _i32p), ("mpc_item", _i32p), ("mpc_dof", _i32p),
                ("mpc_val", _f64p), ("mpc_const", _f64p), ("mpc_matvec", ctypes.c_int)]


UPDATE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, _f64p)
ALLREDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_void_p, ctypes.c_double)


class O33Comm(ctypes.Structure):
    _fields_ = [("ctx", ctypes.c_void_p), ("update", UPDATE_FN), ("allreduce", ALLREDUCE_FN)]


_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        L.o33_matvec.argtypes = [ctypes.POINTER(O33Matrix), _f64p, _f64p]
        L.o33_matresid.argtypes = [ctypes.POINTER(O33Matrix), _f64p, _f64p, _f64p]
        L.o33_matvec_jad.argtypes = [ctypes.POINTER(O33Matrix), _f64p, _f64p]
        L.o33_rel_resid_L2.argtypes = [ctypes.POINTER(O33Matrix), _f64p, _f64p]
        L.o33_rel_resid_L2.restype = ctypes.c_double
        L.o33_dot.argtypes = [ctypes.c_int, _f64p, _f64p]
        L.o33_dot.restype = ctypes.c_double
        L.o33_ordering_rcm.argtypes = [ctypes.c_int, _i32p, _i32p, _i32p, _i32p, _i32p, _i32p]
        L.o33_ordering_mc.argtypes = [ctypes.c_int, _i32p, _i32p, _i32p, _i32p, _i32p, ctypes.c_int,
                                      _i32p, _i32p, _i32p]
        L.o33_ordering_mc.restype = ctypes.c_int
        L.o33_precond_setup.argtypes = [ctypes.POINTER(O33Matrix), ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_int, _i32p]
        L.o33_precond_setup.restype = ctypes.c_void_p
        L.o33_precond_free.argtypes = [ctypes.c_void_p]
        L.o33_precond_sweep.argtypes = [ctypes.c_void_p, _f64p]
        L.o33_precond_apply.argtypes = [ctypes.c_void_p, ctypes.POINTER(O33Matrix), ctypes.c_int,
                                        _f64p, _f64p, _f64p]
        L.o33_precond_ncolor.argtypes = [ctypes.c_void_p]
        L.o33_precond_ncolor.restype = ctypes.c_int
        L.o33_precond_ordering.argtypes = [ctypes.c_void_p, _i32p, _i32p, _i32p]
        L.o33_precond_bilu_pattern.argtypes = [ctypes.c_void_p, _i32p, _i32p, _i32p, _i32p]
        L.o33_precond_bilu_pattern.restype = ctypes.c_int
        L.o33_solve.argtypes = [ctypes.POINTER(O33Matrix), _f64p, _f64p, _i32p, _f64p, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_void_p), _i32p, _f64p, _f64p]
        L.o33_solve.restype = ctypes.c_int
        L.o33_cg.argtypes = [ctypes.POINTER(O33Matrix), ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                             ctypes.c_double, _f64p, _f64p, _i32p, _f64p, _f64p]
        L.o33_cg.restype = ctypes.c_int
        L.o33_cg_lanczos.argtypes = [ctypes.POINTER(O33Matrix), ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_double, _f64p, _f64p, _i32p, _f64p, _f64p]
        L.o33_cg_lanczos.restype = ctypes.c_int
        L.o33_gmres_hess.argtypes = [ctypes.POINTER(O33Matrix), ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_double, ctypes.c_int, _f64p, _f64p, _i32p, _f64p, _f64p, _i32p]
        L.o33_gmres_hess.restype = ctypes.c_int
        L.o33_cg_fixed_iters.argtypes = [ctypes.POINTER(O33Matrix), ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_int, _f64p, _f64p]
        L.o33_cg_fixed_iters.restype = ctypes.c_double
        L.o33_max_threads.restype = ctypes.c_int
        L.o33_solve_dd.argtypes = [ctypes.POINTER(O33Matrix), _f64p, _f64p, _i32p, _f64p,
                                   ctypes.POINTER(O33Comm), _i32p, _f64p, _f64p]
        L.o33_solve_dd.restype = ctypes.c_int
        _lib = L
    return _lib


def _ip(a):
    return a.ctypes.data_as(_i32p)


def _dp(a):
    return a.ctypes.data_as(_f64p)


class Oracle:
    """Holds an o33_matrix view of a HecMatrix (arrays are kept alive here)."""

    def __init__(self, m):
        self.m = m
        self.mat = O33Matrix(m.N, m.NP, m.NPL, m.NPU, _ip(m.indexL), _ip(m.itemL), _ip(m.indexU),
                             _ip(m.itemU), _dp(m.D), _dp(m.AL), _dp(m.AU))
        mpc = getattr(m, "mpc", None)  # (index, item, dof, val, const) of the mesh's MPCs
        if mpc is not None:
            self._mpc = tuple(np.ascontiguousarray(a, dtype=t) for a, t in
                              zip(mpc, (np.int32, np.int32, np.int32, np.float64, np.float64)))
            ix, it, dof, val, const = self._mpc
            self.mat.n_mpc = len(ix) - 1
            self.mat.mpc_index, self.mat.mpc_item, self.mat.mpc_dof = _ip(ix), _ip(it), _ip(dof)
            self.mat.mpc_val, self.mat.mpc_const = _dp(val), _dp(const)
        self.L = lib()

    def matvec(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(3 * self.m.NP)
        self.L.o33_matvec(ctypes.byref(self.mat), _dp(x), _dp(y))
        return y

    def matvec_jad(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(3 * self.m.NP)
        self.L.o33_matvec_jad(ctypes.byref(self.mat), _dp(x), _dp(y))
        return y

    def rel_resid(self, x, b):
        x = np.ascontiguousarray(x, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        return self.L.o33_rel_resid_L2(ctypes.byref(self.mat), _dp(x), _dp(b))

    def rcm(self):
        m = self.m
        perm = np.zeros(m.N, np.int32)
        iperm = np.zeros(m.N, np.int32)
        self.L.o33_ordering_rcm(m.N, _ip(m.indexL), _ip(m.itemL), _ip(m.indexU), _ip(m.itemU),
                                _ip(perm), _ip(iperm))
        return perm, iperm

    def precond(self, kind, ncolor_in=10, sigma_diag=1.0, coloured=1):
        err = ctypes.c_int(0)
        p = self.L.o33_precond_setup(ctypes.byref(self.mat), kind, ncolor_in, sigma_diag, coloured,
                                     ctypes.byref(err))
        return OraclePrecond(self, p, err.value)

    def solve(self, B=None, X=None, Iarray=None, Rarray=None, coloured=1):
        m = self.m
        B = np.ascontiguousarray(m.B if B is None else B, dtype=np.float64)
        X = np.zeros(3 * m.NP) if X is None else np.ascontiguousarray(X, dtype=np.float64).copy()
        Ia = (m.Iarray if Iarray is None else Iarray).astype(np.int32).copy()
        Ra = (m.Rarray if Rarray is None else Rarray).astype(np.float64).copy()
        it = ctypes.c_int(0)
        res = ctypes.c_double(0)
        rtrue = ctypes.c_double(0)
        err = self.L.o33_solve(ctypes.byref(self.mat), _dp(B), _dp(X), _ip(Ia), _dp(Ra), coloured,
                               None, ctypes.byref(it), ctypes.byref(res), ctypes.byref(rtrue))
        return dict(X=X, error=err, iter=it.value, resid=res.value, resid_true=rtrue.value,
                    Iarray=Ia, Rarray=Ra)


class OraclePrecond:
    def __init__(self, orc, handle, err):
        self.orc, self.h, self.error = orc, handle, err

    def __del__(self):
        if getattr(self, "h", None):
            self.orc.L.o33_precond_free(self.h)
            self.h = None

    def sweep(self, zp):
        zp = np.ascontiguousarray(zp, dtype=np.float64).copy()
        self.orc.L.o33_precond_sweep(self.h, _dp(zp))
        return zp

    def apply(self, r, iterpremax=1):
        m = self.orc.m
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros(3 * m.NP)
        zp = np.zeros(3 * m.NP)
        self.orc.L.o33_precond_apply(self.h, ctypes.byref(self.orc.mat), iterpremax, _dp(r), _dp(z),
                                     _dp(zp))
        return z

    def bilu_pattern(self):
        """(indexL, itemL, indexU, itemU) of a block ILU(p) factor."""
        m = self.orc.m
        self.orc.L.o33_precond_bilu_pattern(self.h, None, None, None, None)
        inL = np.zeros(m.NP + 1, np.int32)
        inU = np.zeros(m.NP + 1, np.int32)
        tot = self.orc.L.o33_precond_bilu_pattern(self.h, None, None, None, None)
        iaL = np.zeros(tot + 1, np.int32)
        iaU = np.zeros(tot + 1, np.int32)
        self.orc.L.o33_precond_bilu_pattern(self.h, _ip(inL), _ip(iaL), _ip(inU), _ip(iaU))
        return inL, iaL[:inL[-1]], inU, iaU[:inU[-1]]

    def ordering(self):
        n = self.orc.m.N
        nc = self.orc.L.o33_precond_ncolor(self.h)
        ci = np.zeros(nc + 1, np.int32)
        perm = np.zeros(n, np.int32)
        iperm = np.zeros(n, np.int32)
        self.orc.L.o33_precond_ordering(self.h, _ip(ci), _ip(perm), _ip(iperm))
        return ci, perm, iperm

    def cg_lanczos(self, B, maxit=20000, tol=1e-8, iterpremax=1):
        """CG that also returns ALPHA and BETA per iteration (ESTCOND's data)."""
        orc = self.orc
        m = orc.m
        B = np.ascontiguousarray(B, dtype=np.float64)
        X = np.zeros(3 * m.NP)
        it = ctypes.c_int(0)
        res = ctypes.c_double(0)
        ab = np.zeros(2 * maxit)
        err = orc.L.o33_cg_lanczos(ctypes.byref(orc.mat), self.h, iterpremax, maxit, tol, _dp(B), _dp(X),
                                   ctypes.byref(it), ctypes.byref(res), _dp(ab))
        n = min(it.value, maxit)
        return dict(X=X, error=err, iter=it.value, alpha=ab[0:2 * n:2].copy(), beta=ab[1:2 * n:2].copy())

    def gmres_hess(self, B, nrest, maxit=20000, tol=1e-8, iterpremax=1):
        """GMRES(nrest) with this preconditioner; also the final Hessenberg (column-major,
        leading dimension nrest + 7) and the last step index I."""
        orc = self.orc
        m = orc.m
        B = np.ascontiguousarray(B, dtype=np.float64)
        X = np.zeros(3 * m.NP)
        it, res, I = ctypes.c_int(0), ctypes.c_double(0), ctypes.c_int(0)
        ld = nrest + 7
        H = np.zeros(ld * ld)
        err = orc.L.o33_gmres_hess(ctypes.byref(orc.mat), self.h, iterpremax, maxit, tol, nrest, _dp(B), _dp(X),
                                   ctypes.byref(it), ctypes.byref(res), _dp(H), ctypes.byref(I))
        return dict(X=X, error=err, iter=it.value, I=I.value, H=H.reshape(ld, ld).T.copy(), ld=ld)

    def cg(self, B, maxit=20000, tol=1e-8, iterpremax=1, X=None, hist=False, on=None):
        """CG with this preconditioner; `on` (an Oracle) selects another matrix."""
        orc = self.orc if on is None else on
        m = orc.m
        B = np.ascontiguousarray(B, dtype=np.float64)
        X = np.zeros(3 * m.NP) if X is None else np.ascontiguousarray(X, dtype=np.float64).copy()
        it = ctypes.c_int(0)
        res = ctypes.c_double(0)
        h = np.zeros(maxit) if hist else None
        err = orc.L.o33_cg(ctypes.byref(orc.mat), self.h, iterpremax, maxit, tol, _dp(B),
                                _dp(X), ctypes.byref(it), ctypes.byref(res),
                                _dp(h) if hist else None)
        out = dict(X=X, error=err, iter=it.value, resid=res.value)
        if hist:
            out["hist"] = h[:it.value]
        return out


def solve_dd(domain, endpoint, Iarray=None, Rarray=None):
    """o33_solve_dd on one domain; `endpoint` supplies exchange(send) -> recv and
    allreduce(v) (frontistr_b200.domain).  Every domain of the decomposition must
    call this at the same time (threads or processes)."""
    m, c = domain.matrix, domain.comm
    L = lib()
    mat = O33Matrix(m.N, m.NP, m.NPL, m.NPU, _ip(m.indexL), _ip(m.itemL), _ip(m.indexU),
                    _ip(m.itemU), _dp(m.D), _dp(m.AL), _dp(m.AU))
    n3p = 3 * m.NP

    def update(_ctx, xp):
        x = np.ctypeslib.as_array(xp, shape=(n3p,))
        c.unpack(x, endpoint.exchange(c.pack(x)))

    def allreduce(_ctx, v):
        return endpoint.allreduce(v)

    cb_u, cb_a = UPDATE_FN(update), ALLREDUCE_FN(allreduce)
    comm = O33Comm(None, cb_u, cb_a)
    B = np.ascontiguousarray(m.B, dtype=np.float64)
    X = np.zeros(n3p)
    Ia = (m.Iarray if Iarray is None else Iarray).astype(np.int32).copy()
    Ra = (m.Rarray if Rarray is None else Rarray).astype(np.float64).copy()
    it = ctypes.c_int(0)
    res = ctypes.c_double(0)
    rtrue = ctypes.c_double(0)
    err = L.o33_solve_dd(ctypes.byref(mat), _dp(B), _dp(X), _ip(Ia), _dp(Ra), ctypes.byref(comm),
                         ctypes.byref(it), ctypes.byref(res), ctypes.byref(rtrue))
    return dict(X=X, error=err, iter=it.value, resid=res.value, resid_true=rtrue.value, Iarray=Ia)


def solve_dd_threads(domains, Iarray=None, Rarray=None):
    """o33_solve_dd on every domain, one thread each, exchanging in process."""
    import threading
    from frontistr_b200.domain import LocalExchange
    ex = LocalExchange(domains)
    out = [None] * len(domains)
    errs = []

    def run(k):
        try:
            out[k] = solve_dd(domains[k], ex.endpoint(k), Iarray, Rarray)
        except BaseException as e:  # surfaced below
            errs.append(e)
            ex.barrier.abort()

    ts = [threading.Thread(target=run, args=(k,)) for k in range(len(domains))]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errs:
        raise errs[0]
    return out
