"""Batched solves: many independent hecmwST systems in one persistent GPU launch.

``stack_systems`` joins systems into one block-diagonal hecmwST matrix with the
system offsets ``sys_ptr``; :class:`BatchSolver` wraps the hecmw33_gpu_batch_* calls
of include/hecmw33_gpu.h.  Each system is solved as hecmw_solve would solve it
alone (hecmw1/src/solver/main/hecmw_solver.f90:9-88 with hecmw_solve_CG and the
SSOR_33 / DIAG_33 preconditioners in the reference's ordering); the reference has no
batched call, so the per-system results are checked against per-system solves.
"""
import ctypes

import numpy as np

from ._lib import gpu_lib
from .matrix import HecMatrix
from .solver import FATAL, HecmwSolverError, _dp, _i, _ip, last_error


def stack_systems(systems):
    """Block-diagonal HecMatrix of the given systems and the node offsets sys_ptr."""
    ns = [m.N for m in systems]
    sys_ptr = np.zeros(len(systems) + 1, np.int32)
    sys_ptr[1:] = np.cumsum(ns)
    N = int(sys_ptr[-1])
    indexL = np.zeros(N + 1, np.int32)
    indexU = np.zeros(N + 1, np.int32)
    itemL, itemU, D, AL, AU, B, X = [], [], [], [], [], [], []
    offL = offU = 0
    for s, m in enumerate(systems):
        a = int(sys_ptr[s])
        indexL[a + 1:a + m.N + 1] = m.indexL[1:m.N + 1] + offL
        indexU[a + 1:a + m.N + 1] = m.indexU[1:m.N + 1] + offU
        itemL.append(m.itemL[:m.NPL] + a)
        itemU.append(m.itemU[:m.NPU] + a)
        D.append(m.D[:9 * m.N])
        AL.append(m.AL[:9 * m.NPL])
        AU.append(m.AU[:9 * m.NPU])
        B.append(m.B[:3 * m.N])
        X.append(m.X[:3 * m.N])
        offL += m.NPL
        offU += m.NPU
    out = HecMatrix(N, N, indexL, np.concatenate(itemL), indexU, np.concatenate(itemU),
                    np.concatenate(D), np.concatenate(AL), np.concatenate(AU),
                    np.concatenate(B), np.concatenate(X))
    out.Iarray, out.Rarray = systems[0].Iarray.copy(), systems[0].Rarray.copy()
    return out, sys_ptr


class BatchSolver:
    """One batch handle (its own stream, device buffers and launch schedule)."""

    def __init__(self):
        self.lib = gpu_lib()
        h, err = ctypes.c_int(0), ctypes.c_int(0)
        self.lib.hecmw33_gpu_batch_create(ctypes.byref(h), ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        self.handle = h
        self.nsys = 0

    def close(self):
        if getattr(self, "handle", None) is not None:
            err = ctypes.c_int(0)
            self.lib.hecmw33_gpu_batch_destroy(ctypes.byref(self.handle), ctypes.byref(err))
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

    def _check_solve(self, code):
        # per-system codes (2001 zero diagonal, 3001-3004) are results, not failures
        if code not in (2001, 3001, 3002, 3003, 3004):
            self._check(code)

    def set_matrix(self, m, sys_ptr, Iarray=None, Rarray=None):
        sys_ptr = np.ascontiguousarray(sys_ptr, dtype=np.int32)
        ia = np.ascontiguousarray(m.Iarray if Iarray is None else Iarray, dtype=np.int32)
        ra = np.ascontiguousarray(m.Rarray if Rarray is None else Rarray, dtype=np.float64)
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_batch_set_matrix(
            ctypes.byref(self.handle), _i(len(sys_ptr) - 1), _ip(sys_ptr), _i(m.N), _i(m.NP), _i(m.NPL),
            _i(m.NPU), _ip(m.indexL), _ip(m.itemL), _ip(m.indexU), _ip(m.itemU), _dp(m.D), _dp(m.AL),
            _dp(m.AU), _ip(ia), _dp(ra), ctypes.byref(err))
        self._check(err.value)
        self.nsys = len(sys_ptr) - 1

    def _out(self):
        n = self.nsys
        return (np.zeros(n, np.int32), np.zeros(n), np.zeros(n, np.int32), np.zeros(n), np.zeros(3))

    def solve(self, B, X, Iarray, Rarray):
        """Host B/X (3N); X is updated in place.  Returns per-system arrays."""
        it, res, errs, tres, times = self._out()
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_batch_solve(ctypes.byref(self.handle), _dp(B), _dp(X), _ip(Iarray), _dp(Rarray),
                                         _ip(it), _dp(res), _ip(errs), _dp(tres), _dp(times), ctypes.byref(err))
        self._check_solve(err.value)
        return dict(error=int(err.value), iter=it, resid=res, errors=errs, true_resid=tres,
                    t_setup=float(times[0]), t_solve=float(times[1]))

    def solve_device(self, dB_ptr, dX_ptr, Iarray, Rarray):
        it, res, errs, tres, times = self._out()
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_batch_solve_device(ctypes.byref(self.handle), ctypes.c_void_p(dB_ptr),
                                                ctypes.c_void_p(dX_ptr), _ip(Iarray), _dp(Rarray), _ip(it),
                                                _dp(res), _ip(errs), _dp(tres), _dp(times), ctypes.byref(err))
        self._check_solve(err.value)
        return dict(error=int(err.value), iter=it, resid=res, errors=errs, true_resid=tres,
                    t_setup=float(times[0]), t_solve=float(times[1]))

    def autotune(self, B, X, Iarray, Rarray):
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_batch_autotune(ctypes.byref(self.handle), _dp(B), _dp(X), _ip(Iarray), _dp(Rarray),
                                            ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        return self.info()

    def info(self):
        info = np.zeros(16, np.int32)
        dinfo = np.zeros(16)
        err = ctypes.c_int(0)
        self.lib.hecmw33_gpu_batch_info(ctypes.byref(self.handle), _ip(info), _dp(dinfo), ctypes.byref(err))
        self._check(err.value, fatal_only=False)
        return dict(lanes=int(info[0]), cluster=int(info[1]), big=int(info[2]), small=int(info[3]),
                    grid=int(info[4]), tuned=int(info[5]), nsys=int(info[6]), kernels_per_solve=int(info[7]),
                    total_iter=int(info[8]), max_iter=int(info[9]), t_solve=float(dinfo[0]),
                    t_setup=float(dinfo[1]), big_frac=float(dinfo[2]), device_bytes=float(dinfo[3]))
