"""Python mirror of the hecmwST_matrix fields that the 3x3 solve path uses.

Layout (hecmw1/src/common/hecmw_util_f.F90:458-470, NDOF = 3):
  indexL/indexU  int32[NP+1], index[0] = 0
  itemL/itemU    int32, 1-based node ids, ascending within each row
  D float64[9*NP], AL float64[9*NPL], AU float64[9*NPU]  (row-major 3x3 blocks)
  B, X           float64[3*NP]
  Iarray int32[100], Rarray float64[100] with the index map of
  hecmw1/src/solver/matrix/hecmw_matrix_misc.F90:107-150 (stored 0-based here:
  Iarray[k-1] is Fortran Iarray(k)).

The defaults are those of hecmw_mat_init (hecmw_matrix_misc.F90:171-212).
"""
import numpy as np

# Fortran Iarray / Rarray indices (1-based), hecmw_matrix_misc.F90:107-150
IDX_I_ITER = 1
IDX_I_METHOD = 2
IDX_I_PRECOND = 3
IDX_I_NSET = 4
IDX_I_ITERPREMAX = 5
IDX_I_NREST = 6
IDX_I_SCALING = 7
IDX_I_METHOD2 = 8
IDX_I_MPC_METHOD = 13
IDX_I_ESTCOND = 14
IDX_I_ITERLOG = 21
IDX_I_TIMELOG = 22
IDX_I_DUMP = 31
IDX_I_DUMP_EXIT = 32
IDX_I_USEJAD = 33
IDX_I_NCOLOR_IN = 34
IDX_I_MAXRECYCLE_PRECOND = 35
IDX_I_FLAG_CONVERGED = 81
IDX_I_FLAG_DIVERGED = 82
IDX_I_NRECYCLE_PRECOND = 96
IDX_I_FLAG_NUMFACT = 97
IDX_I_FLAG_SYMBFACT = 98
IDX_I_SOLVER_TYPE = 99
IDX_R_RESID = 1
IDX_R_SIGMA_DIAG = 2
IDX_R_SIGMA = 3

# hecmw1/src/solver/init/hecmw_solve_error.f90:9-16
HECMW_SOLVER_ERROR_INCONS_PC = 1001
HECMW_SOLVER_ERROR_ZERO_DIAG = 2001
HECMW_SOLVER_ERROR_ZERO_RHS = 2002
HECMW_SOLVER_ERROR_NOCONV_MAXIT = 3001
HECMW_SOLVER_ERROR_DIVERGE_MAT = 3002
HECMW_SOLVER_ERROR_DIVERGE_PC = 3003
HECMW_SOLVER_ERROR_DIVERGE_NAN = 3004


def default_iarray_rarray():
    """Iarray/Rarray as left by hecmw_mat_init."""
    ia = np.zeros(100, dtype=np.int32)
    ra = np.zeros(100, dtype=np.float64)
    ia[IDX_I_ITER - 1] = 100
    ia[IDX_I_METHOD - 1] = 1
    ia[IDX_I_PRECOND - 1] = 1
    ia[IDX_I_NSET - 1] = 0
    ia[IDX_I_ITERPREMAX - 1] = 1
    ia[IDX_I_NREST - 1] = 10
    ia[IDX_I_SCALING - 1] = 0
    ia[IDX_I_NCOLOR_IN - 1] = 10
    ia[IDX_I_MAXRECYCLE_PRECOND - 1] = 3
    ia[IDX_I_NRECYCLE_PRECOND - 1] = 0
    ia[IDX_I_FLAG_NUMFACT - 1] = 1
    ia[IDX_I_FLAG_SYMBFACT - 1] = 1
    ia[IDX_I_SOLVER_TYPE - 1] = 1
    ra[IDX_R_RESID - 1] = 1.0e-8
    ra[IDX_R_SIGMA_DIAG - 1] = 1.0
    ra[IDX_R_SIGMA - 1] = 0.0
    ra[3] = 0.10  # THRESH
    ra[4] = 0.10  # FILTER
    ra[10] = 1.0e4  # PENALTY
    return ia, ra


class HecMatrix:
    """hecmwST_matrix for NDOF = 3: N internal of NP nodes (N == NP for a whole mesh;
    N < NP for a domain of a decomposed mesh, frontistr_b200.domain)."""

    NDOF = 3

    def __init__(self, N, NP, indexL, itemL, indexU, itemU, D, AL, AU, B=None, X=None):
        self.N, self.NP = int(N), int(NP)
        self.indexL = np.ascontiguousarray(indexL, dtype=np.int32)
        self.itemL = np.ascontiguousarray(itemL, dtype=np.int32)
        self.indexU = np.ascontiguousarray(indexU, dtype=np.int32)
        self.itemU = np.ascontiguousarray(itemU, dtype=np.int32)
        self.D = np.ascontiguousarray(D, dtype=np.float64)
        self.AL = np.ascontiguousarray(AL, dtype=np.float64)
        self.AU = np.ascontiguousarray(AU, dtype=np.float64)
        self.B = np.zeros(3 * self.NP) if B is None else np.ascontiguousarray(B, dtype=np.float64)
        self.X = np.zeros(3 * self.NP) if X is None else np.ascontiguousarray(X, dtype=np.float64)
        self.Iarray, self.Rarray = default_iarray_rarray()
        self.coords = None
        self.mpc = None  # (mpc_index, mpc_item, mpc_dof, mpc_val, mpc_const) of the mesh, if any

    @classmethod
    def empty(cls, n, npl, npu):
        return cls(n, n, np.zeros(n + 1, np.int32), np.zeros(max(npl, 1), np.int32),
                   np.zeros(n + 1, np.int32), np.zeros(max(npu, 1), np.int32),
                   np.zeros(9 * n), np.zeros(9 * max(npl, 1)), np.zeros(9 * max(npu, 1)))

    @property
    def NPL(self):
        return int(self.indexL[self.NP])

    @property
    def NPU(self):
        return int(self.indexU[self.NP])

    @property
    def NZ(self):
        return self.N + self.NPL + self.NPU

    # ---- hecmw_mat_get/set_* mirrors used by the solver path -----------------
    def set_iter(self, v): self.Iarray[IDX_I_ITER - 1] = v
    def set_method(self, v): self.Iarray[IDX_I_METHOD - 1] = v
    def set_precond(self, v): self.Iarray[IDX_I_PRECOND - 1] = v

    def set_iterpremax(self, v):
        self.Iarray[IDX_I_ITERPREMAX - 1] = min(max(int(v), 0), 4)

    def set_ncolor_in(self, v): self.Iarray[IDX_I_NCOLOR_IN - 1] = v
    def set_scaling(self, v): self.Iarray[IDX_I_SCALING - 1] = v
    def set_resid(self, v): self.Rarray[IDX_R_RESID - 1] = v
    def set_sigma_diag(self, v): self.Rarray[IDX_R_SIGMA_DIAG - 1] = v
    def get_flag_converged(self): return int(self.Iarray[IDX_I_FLAG_CONVERGED - 1])
    def get_flag_diverged(self): return int(self.Iarray[IDX_I_FLAG_DIVERGED - 1])

    def copy(self):
        m = HecMatrix(self.N, self.NP, self.indexL.copy(), self.itemL.copy(), self.indexU.copy(),
                      self.itemU.copy(), self.D.copy(), self.AL.copy(), self.AU.copy(),
                      self.B.copy(), self.X.copy())
        m.Iarray, m.Rarray = self.Iarray.copy(), self.Rarray.copy()
        m.coords = self.coords
        m.mpc = getattr(self, "mpc", None)
        return m

    def to_scipy(self):
        """Assembled scalar CSR (scipy) of the full 3N x 3N matrix; for checks only."""
        import scipy.sparse as sp
        N = self.N
        rows, cols, vals = [], [], []
        r3 = np.repeat(np.arange(3), 3)
        c3 = np.tile(np.arange(3), 3)
        ib = np.arange(N)
        rows.append((3 * ib[:, None] + r3).ravel())
        cols.append((3 * ib[:, None] + c3).ravel())
        vals.append(self.D[:9 * N])
        for index, item, A in ((self.indexL, self.itemL, self.AL), (self.indexU, self.itemU, self.AU)):
            cnt = np.diff(index[:N + 1])
            rb = np.repeat(np.arange(N), cnt)
            cb = item[:index[N]] - 1
            rows.append((3 * rb[:, None] + r3).ravel())
            cols.append((3 * cb[:, None] + c3).ravel())
            vals.append(A[:9 * index[N]])
        return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                             shape=(3 * N, 3 * N))
