/*
 * hecmw33_oracle.h -- CPU restatement of FrontISTR's 3x3-block CG solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * CUDA solver in frontistr_b200/.  Only tests/, __graft_entry__.smoke() and
 * the CPU-baseline leg of bench.py may load it.  It is never part of the
 * product path.
 *
 * Every function restates the cited reference Fortran line by line, keeping
 * the reference's summation order, so that its results can be compared with
 * the reference's own outputs (the golden vectors of tests/solver/CG) and
 * with the GPU solver.
 *
 * Matrix layout (hecmwST_matrix, hecmw1/src/common/hecmw_util_f.F90:458-470):
 *   indexL/indexU : NP+1 entries, index[0] = 0
 *   itemL/itemU   : 1-based node ids, sorted ascending within each row
 *   D  : 9*NP  row-major 3x3 blocks  (r1c1, r1c2, r1c3, r2c1, ...)
 *   AL : 9*NPL, AU : 9*NPU
 * Vectors have 3*NP entries.  Iarray/Rarray follow the index map of
 * hecmw1/src/solver/matrix/hecmw_matrix_misc.F90:107-150 (1-based there,
 * so Iarray[k-1] here holds Fortran Iarray(k)).
 */
#ifndef HECMW33_ORACLE_H
#define HECMW33_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int N, NP, NPL, NPU;
  const int *indexL, *itemL, *indexU, *itemU;
  const double *D, *AL, *AU;
  /* USEJAD (Iarray(33)): products in the jagged-diagonal order of
   * hecmw1/src/solver/las/hecmw_jadm_33.f90 (o33_solve sets it from Iarray) */
  int usejad;
  /* the mesh's MPCs (hecmwST_local_mesh%mpc: mpc_index(0:n_mpc), 1-based items, DOFs,
   * coefficients, constants); mpc_matvec: products are T^T A T x
   * (hecmw_TtmatTvec_33; o33_solve sets it for MPC_METHOD = Iarray(13) = 2) */
  int n_mpc;
  const int *mpc_index, *mpc_item, *mpc_dof;
  const double *mpc_val, *mpc_const;
  int mpc_matvec;
} o33_matrix;

/* ---- kernels of hecmw1/src/solver/las/hecmw_solver_las_33.F90 ---- */
void o33_matvec(const o33_matrix *A, const double *x, double *y);
/* hecmw_JAD_MATVEC_33: y_i = D_i x_i plus the row's off-diagonal blocks summed from
 * zero (L then U, in index order) */
void o33_matvec_jad(const o33_matrix *A, const double *x, double *y);
void o33_matresid(const o33_matrix *A, const double *x, const double *b, double *r);
double o33_rel_resid_L2(const o33_matrix *A, const double *x, const double *b);

/* ---- hecmw1/src/solver/communication/hecmw_solver_misc.F90 ---- */
double o33_dot(int n, const double *x, const double *y);

/* ---- orderings (hecmw1/src/solver/matrix/hecmw_matrix_ordering_CM.f90, _MC.f90) ----
 * perm[new-1] = old (1-based), iperm[old-1] = new (1-based). */
void o33_ordering_rcm(int N, const int *indexL, const int *itemL,
                      const int *indexU, const int *itemU, int *perm, int *iperm);
/* colorindex must hold N+1 entries; returns NColor */
int o33_ordering_mc(int N, const int *indexL, const int *itemL,
                    const int *indexU, const int *itemU, const int *perm_cur,
                    int ncolor_in, int *colorindex, int *perm, int *iperm);

/* ---- preconditioners ---- */
typedef struct o33_precond o33_precond;
/* kind: 1,2 = SSOR, 3 = DIAG, 10 = BILU(0).
 * ssor_coloured: 1 = RCM + multicolour ordering (the reference's OpenMP
 * (>1 thread) and OpenACC path), 0 = natural order, one colour (1 thread). */
o33_precond *o33_precond_setup(const o33_matrix *A, int kind, int ncolor_in,
                               double sigma_diag, int ssor_coloured, int *ierr);
void o33_precond_free(o33_precond *P);
/* one sweep of the preconditioner, in place on zp (3*NP) */
void o33_precond_sweep(const o33_precond *P, double *zp);
/* hecmw_precond_apply: z = M^-1 r with iterPREmax outer passes */
void o33_precond_apply(const o33_precond *P, const o33_matrix *A, int iterpremax,
                       const double *r, double *z, double *zp);
/* SSOR ordering queries */
int o33_precond_ncolor(const o33_precond *P);
/* block ILU(p) factor pattern (indexL/U of NP+1, 1-based items); with NULL arrays,
 * only the total block count.  -1 for other preconditioners. */
int o33_precond_bilu_pattern(const o33_precond *P, int *inL, int *iaL, int *inU, int *iaU);
void o33_precond_ordering(const o33_precond *P, int *colorindex, int *perm, int *iperm);

/* ---- hecmw_solve (hecmw1/src/solver/main/hecmw_solver.f90:9-88) restricted to
 * METHOD=1 (CG), 2 (BiCGSTAB), 3 (GMRES), 4 (GPBiCG) or 7 (CR), the last four also as
 * the METHOD2 fallback of a diverged CG,
 * PRECOND in {1,2,3,10}.  X holds x0 on entry and the solution on
 * return.  Iarray flags 81/82/96/97/98 are updated as the reference does.
 * Returns the solver error code (0, 2001, 2002, 3001..3004, 1001).  The
 * preconditioner may be kept between calls through *cache (NULL to disable);
 * the recycle policy of hecmw_mat_recycle_precond_setting decides reuse. */
int o33_solve(const o33_matrix *A, const double *B, double *X, int *Iarray,
              double *Rarray, int ssor_coloured, o33_precond **cache,
              int *iter_out, double *resid_out, double *resid_true_out);

/* CG iterations only (hecmw_solve_CG), given a ready preconditioner.
 * resid_hist (optional, length >= maxit) receives RESID per iteration. */
int o33_cg(const o33_matrix *A, const o33_precond *P, int iterpremax, int maxit,
           double tol, const double *B, double *X, int *iter_out, double *resid_out,
           double *resid_hist);

/* BiCGSTAB iterations only (hecmw_solve_BiCGSTAB), given a ready preconditioner. */
int o33_bicgstab(const o33_matrix *A, const o33_precond *P, int iterpremax, int maxit,
                 double tol, const double *B, double *X, int *iter_out, double *resid_out);

/* GMRES(nrest) iterations only (hecmw_solve_GMRES), given a ready preconditioner. */
int o33_gmres(const o33_matrix *A, const o33_precond *P, int iterpremax, int maxit, double tol,
              int nrest, const double *B, double *X, int *iter_out, double *resid_out);

/* o33_cg that also returns ALPHA and BETA of every iteration (ab[2k], ab[2k+1]; BETA
 * of the first iteration 0): the data of ESTCOND's Lanczos estimate
 * (hecmw_solver_CG.f90:256-264). */
int o33_cg_lanczos(const o33_matrix *A, const o33_precond *P, int iterpremax, int maxit, double tol,
                   const double *B, double *X, int *iter_out, double *resid_out, double *ab);

/* o33_gmres that also returns the Hessenberg as the solve leaves it (NREST+7 squared
 * doubles, column-major, the rotated leading block) and the last step index I: the
 * data of ESTCOND's estimate (hecmw_solver_GMRES.f90:290-291, 416-417). */
int o33_gmres_hess(const o33_matrix *A, const o33_precond *P, int iterpremax, int maxit, double tol, int nrest,
                   const double *B, double *X, int *iter_out, double *resid_out, double *H_out, int *I_out);

/* Conjugate residual iterations only (hecmw_solve_CR), given a ready preconditioner. */
int o33_cr(const o33_matrix *A, const o33_precond *P, int iterpremax, int maxit, double tol,
           const double *B, double *X, int *iter_out, double *resid_out);

/* GPBiCG iterations only (hecmw_solve_GPBiCG), given a ready preconditioner. */
int o33_gpbicg(const o33_matrix *A, const o33_precond *P, int iterpremax, int maxit, double tol,
               const double *B, double *X, int *iter_out, double *resid_out);

/* GMRESR (ren = 0; nbfgs quasi-Newton pairs) or GMRESREN (ren = 1) iterations only
 * (hecmw_solve_GMRESR / hecmw_solve_GMRESREN), given a ready preconditioner. */
int o33_gmresr(const o33_matrix *A, const o33_precond *P, int iterpremax, int maxit, double tol, int nrest,
               int nbfgs, int ren, const double *B, double *X, int *iter_out, double *resid_out);

/* ---- domain decomposition (hecmw1/src/solver/communication) ----
 * One domain of an overlapping node-based decomposition: rows 0..N-1 are its
 * internal nodes, N..NP-1 the external (halo) nodes owned by neighbours.
 * update: hecmw_update_R (hecmw_comm_f.F90:838-863) -- fills the external entries
 *   3N..3NP-1 of a 3NP vector from their owners, in place;
 * allreduce: hecmw_allreduce_R1 with hecmw_sum (:494-528) -- the sum of v over the
 *   domains.  Both are called by every domain at the same points. */
typedef struct {
  void *ctx;
  void (*update)(void *ctx, double *x);
  double (*allreduce)(void *ctx, double v);
} o33_comm;

/* hecmw_solve_CG on one domain: matvec / matresid after hecmw_update_R of their
 * input, inner products over the internal entries and allreduced, the final update
 * of X (hecmw_solver_CG.f90:77-288, hecmw_solver_las_33.F90:231). */
int o33_cg_dd(const o33_matrix *A, const o33_precond *P, int iterpremax, int maxit, double tol,
              const double *B, double *X, int *iter_out, double *resid_out, const o33_comm *comm);

/* hecmw_solve -> hecmw_solve_iterative for METHOD = 1 on one domain: allreduced
 * zero-RHS and zero-diagonal checks, a new local preconditioner (kind as o33_solve;
 * only internal rows, as the reference's), CG, the sigma_diag retry of a diverged
 * ILU, the allreduced true residual and the flags.  Other METHODs: 9101. */
int o33_solve_dd(const o33_matrix *A, const double *B, double *X, int *Iarray, double *Rarray,
                 const o33_comm *comm, int *iter_out, double *resid_out, double *resid_true_out);

/* run exactly n CG iterations (no convergence exit) and return elapsed seconds;
 * used for the bounded CPU-baseline sample. */
double o33_cg_fixed_iters(const o33_matrix *A, const o33_precond *P, int iterpremax,
                          int n, const double *B, double *X);

int o33_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
