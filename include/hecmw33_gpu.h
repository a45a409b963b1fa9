/*
 * hecmw33_gpu.h -- C ABI of the B200 (sm_100a) 3x3-block CG solver, a drop-in for
 * FrontISTR's hecmw_solve on a hecmwST_matrix with NDOF = 3 and METHOD = 1 (CG),
 * 2 (BiCGSTAB, hecmw1/src/solver/iterative/hecmw_solver_BiCGSTAB.f90:16), 3 (GMRES,
 * hecmw1/src/solver/iterative/hecmw_solver_GMRES.f90), 4 (GPBiCG,
 * hecmw1/src/solver/iterative/hecmw_solver_GPBiCG.f90), 5 (GMRESR with NBFGS = Iarray(60)
 * quasi-Newton pairs, hecmw1/src/solver/iterative/hecmw_solver_GMRESR.f90), 6 (GMRESREN,
 * hecmw1/src/solver/iterative/hecmw_solver_GMRESREN.f90) or 7 (CR,
 * hecmw1/src/solver/iterative/hecmw_solver_CR.f90).
 *
 * Reference interfaces replaced (paths inside the FrontISTR tree):
 *   hecmw_solve(hecMESH, hecMAT)          hecmw1/src/solver/main/hecmw_solver.f90:9
 *   hecmw_solve_iterative(hecMESH, hecMAT) hecmw1/src/solver/iterative/hecmw_solver_Iterative.f90:13
 *   hecmw_solve_CG(hecMESH, hecMAT, ITER, RESID, error, Tset, Tsol, Tcomm)
 *                                          hecmw1/src/solver/iterative/hecmw_solver_CG.f90:19-20
 *   hecmw_matvec / hecmw_matvec_33         hecmw1/src/solver/las/hecmw_solver_las.f90:42,
 *                                          hecmw1/src/solver/las/hecmw_solver_las_33.F90:34
 *   hecmw_precond_setup / _apply           hecmw1/src/solver/precond/hecmw_precond.f90:30,86
 *   (C-side plugin precedent: hecmw_ML_wrapper_setup/apply/clear,
 *    hecmw1/src/solver/precond/ml/hecmw_ML_wrapper.c:320,546,571)
 *
 * Conventions (all arguments by pointer, callable from Fortran through iso_c_binding
 * with bind(C, name=...), as frontistr_b200/fortran/hecmw_solver_gpu33.f90 does):
 *   - Matrix arrays use the hecmwST_matrix layout: indexL/indexU have NP+1 entries
 *     (index[0] = 0); itemL/itemU hold 1-based node ids sorted ascending per row;
 *     D has 9*NP, AL 9*NPL, AU 9*NPU doubles of row-major 3x3 blocks.
 *   - Vectors B and X have 3*NP doubles.  Iarray[100]/Rarray[100] are hecMAT%Iarray
 *     /Rarray (Iarray[k-1] is Fortran Iarray(k)); map in
 *     hecmw1/src/solver/matrix/hecmw_matrix_misc.F90:107-150.
 *   - Host pointers are borrowed for the duration of the call only.  Device buffers
 *     belong to the handle.  One host thread per handle; every call is synchronous.
 *   - One domain per handle.  N < NP is a domain of a decomposed mesh (internal nodes
 *     1..N, external nodes N+1..NP): hecmw33_gpu_set_domain gives its communication
 *     table and the caller's exchange / allreduce; such a domain runs CG (METHOD = 1)
 *     in FP64 with SCALING=NO (9101 otherwise).  The whole-mesh entries (multi-RHS
 *     solves, matvec, precond_apply, get_matrix) refuse a domain handle (9101); an
 *     assembly on the device makes the handle one whole mesh again.
 *   - Iarray(7) = 1 (SCALING=YES, hecmw_solver_scaling_33.f90:20-208): the CG runs on
 *     S A S, S b with S = diag(1/sqrt|D_kk|) and X is multiplied by S after it; the
 *     caller's arrays are not written.  FP64 CG only (Iarray(42) = 0 or 1): 9101 for
 *     Iarray(42) = 2, 3 and for the multi-RHS solves.
 *   - Options of this library in the SOLVER_OPT block of Iarray/Rarray (41-50,
 *     hecmw_matrix_misc.F90:137-147), unused by the reference's CG:
 *       Iarray(42) = 0  FP64 CG (the drop-in, default)
 *                  = 1  mixed precision, low-precision preconditioner: FP64 CG whose
 *                       preconditioner sweeps read BF16-stored factors (FP32 diagonal
 *                       LU) and compute in FP64; matrix, vectors, dots and residuals
 *                       stay FP64, so the convergence test is the reference's
 *                  = 2  mixed precision, restarted refinement: inner FP32 CG (FP32
 *                       matrix and preconditioner copies, FP64 dot products) from zero
 *                       to Rarray(42) relative (0 -> 1e-4), FP64 correction and true
 *                       residual
 *                  = 3  mixed precision, reliable updates: FP32 CG whose solution and
 *                       residual are folded into FP64 (x64 += x32, r = b - A x in FP64)
 *                       each time the FP32 residual has fallen by Rarray(42) (0 -> 0.1)
 *       Rarray(42)      inner tolerance (mode 2) / refinement factor (mode 3)
 *       Iarray(43) = 1  learned two-level preconditioner around SSOR (see
 *                       hecmw33_gpu_learn_*; Iarray(44) its coarse smoothing weights)
 *   - *ierr receives 0 or an error code: the reference's codes (1001, 2001, 2002,
 *     3001-3004; hecmw1/src/solver/init/hecmw_solve_error.f90:9-16) or the
 *     HECMW33_ERR_* codes below.  1001 and 2001 are fatal in the reference
 *     (hecmw_abort); 2002 and 3001 are warnings; 3002-3004 set the diverged flag.
 */
#ifndef HECMW33_GPU_H
#define HECMW33_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define HECMW33_API __attribute__((visibility("default")))
#else
#define HECMW33_API
#endif

/* reference error codes (hecmw_solve_error.f90:9-16) */
#define HECMW33_ERR_INCONS_PC 1001
#define HECMW33_ERR_ZERO_DIAG 2001
#define HECMW33_ERR_ZERO_RHS 2002
#define HECMW33_ERR_NOCONV_MAXIT 3001
#define HECMW33_ERR_DIVERGE_MAT 3002
#define HECMW33_ERR_DIVERGE_PC 3003
#define HECMW33_ERR_DIVERGE_NAN 3004
/* codes of this library (no counterpart in the reference) */
#define HECMW33_ERR_ILU_ZERO_PIVOT 9001 /* the reference stops the program here */
#define HECMW33_ERR_CUDA 9100           /* CUDA runtime error; see hecmw33_gpu_last_error */
#define HECMW33_ERR_BAD_INPUT 9101      /* inconsistent sizes, indices out of range, unsupported options */
#define HECMW33_ERR_BAD_HANDLE 9102
#define HECMW33_ERR_TIMEOUT 9103        /* a bounded device-side wait gave up */
#define HECMW33_ERR_NO_MATRIX 9104      /* solve/matvec before set_matrix */

/* The two communications of a decomposed domain, supplied by the caller (MPI through
 * hecmw_solve_send_recv / hecmw_allreduce_R1 in FrontISTR; torch.distributed in the
 * Python mirror).  Every domain calls them at the same points of the solve.
 *   exchange: hecmw_update_R (hecmw1/src/solver/communication/hecmw_comm_f.F90:838-863)
 *     -- send[] holds 3 values per export item (in export_item order, i.e. grouped by
 *     neighbour as export_index says); the function sends each neighbour its part and
 *     fills recv[] with 3 values per import item (import_item order).
 *   allreduce: hecmw_allreduce_R1 with hecmw_sum (:494-528) -- the sum of value over
 *     the domains (every domain must get the same bits). */
typedef void (*hecmw33_exchange_fn)(void *ctx, const double *send, double *recv);
typedef double (*hecmw33_allreduce_fn)(void *ctx, double value);

/* Create a solver handle bound to the current CUDA device (its own stream).
 * Counterpart of the integer id table of hecmw1/src/solver/matrix/hecmw_mat_id.f90:21-72. */
HECMW33_API void hecmw33_gpu_create(int *handle, int *ierr);

/* Release every device buffer of the handle (hecmw_precond_clear + deallocation). */
HECMW33_API void hecmw33_gpu_destroy(const int *handle, int *ierr);

/* Upload the matrix.  Symbolic setup (device layout, SSOR ordering) runs when the
 * handle has no matrix, when N/NP/NPL/NPU change, or when Iarray(98) != 0
 * (hecMAT%Iarray(98): symbolic factorisation flag); otherwise only the values are
 * copied and the device layout is reused.  Iarray may be NULL (= symbolic setup).
 * Does not build the preconditioner (hecmw33_gpu_solve does, per flags 97/98). */
HECMW33_API void hecmw33_gpu_set_matrix(const int *handle, const int *N, const int *NP,
                                        const int *NPL, const int *NPU, const int *indexL,
                                        const int *itemL, const int *indexU, const int *itemU,
                                        const double *D, const double *AL, const double *AU,
                                        const int *Iarray, int *ierr);

/* The MPCs of the mesh (hecmwST_local_mesh%mpc, hecmw1/src/common/hecmw_util_f.F90:98-103):
 * mpc_index(0:n_mpc), then per term the 1-based node mpc_item, its DOF mpc_dof and the
 * coefficient mpc_val (the first term of an MPC is its slave); mpc_const(n_mpc) (may
 * be NULL) enters the zero-RHS check.  MPCs with a DOF above 3 are left out, as
 * hecmw_Tvec_33 does.  With MPC_METHOD = Iarray(13) = 2 the solve is MPC-CG
 * (hecmw_solver_Iterative.f90:79-84): CG (METHOD = 1, FP64, SCALING=NO) whose products
 * are T^T A T x (hecmw_TtmatTvec_33, hecmw_solver_las_33.F90:572-586), the true
 * residual included.  Kept across value updates; a matrix of another N drops them;
 * n_mpc = 0 clears them.  One whole (one-domain) mesh. */
HECMW33_API void hecmw33_gpu_set_mpc(const int *handle, const int *n_mpc, const int *mpc_index, const int *mpc_item,
                                     const int *mpc_dof, const double *mpc_val, const double *mpc_const,
                                     int *ierr);

/* The communication table of the handle's domain (hecmwST_local_mesh:
 * n_neighbor_pe, neighbor_pe, import_index(0:n), import_item, export_index(0:n),
 * export_item; items are 1-based local node ids, imports in N+1..NP, exports in 1..N)
 * and the caller's exchange / allreduce (ctx is passed back to them).  Call after
 * hecmw33_gpu_set_matrix with N < NP; a domain without this call has no neighbours
 * (hecmw_update_R returns at once, hecmw_solver_SR's n_neighbor_pe == 0) and sums
 * over itself.  Replaces the hecMESH argument of hecmw_solve
 * (hecmw1/src/solver/main/hecmw_solver.f90:9) for the communication it carries. */
HECMW33_API void hecmw33_gpu_set_domain(const int *handle, const int *n_neighbor_pe, const int *neighbor_pe,
                                        const int *import_index, const int *import_item,
                                        const int *export_index, const int *export_item,
                                        hecmw33_exchange_fn exchange, hecmw33_allreduce_fn allreduce,
                                        void *ctx, int *ierr);

/* Iarray(21) = ITERLOG = 1 (hecmw_solver_CG.f90:251-253): the CG and BiCGSTAB record RESID
 * of every iteration and print the reference's "ITER RESID" lines ('(i7, 1pe16.6)') on
 * stdout when the solve returns; GMRES, GPBiCG, CR, GMRESR and GMRESREN print each
 * iteration's line in their reference's format as they go.  Solves in precision modes 2
 * and 3 (Iarray(42)) and with the learned preconditioner (Iarray(43)) have no reference
 * counterpart and print no history lines.
 * Iarray(14) = ESTCOND > 0 (hecmw_solver_CG.f90:256-264, 299-301): the CG records ALPHA
 * and BETA; every ESTCOND iterations and at the end of a solve without error the
 * extreme eigenvalues of the Lanczos tridiagonal are printed on stdout as
 * "emin=..., emax=..., emax/emin=..." (hecmw_estimate_condition.F90:14-99).  GMRES
 * prints the extreme singular values of its rotated Hessenberg block the same way
 * (hecmw_solver_GMRES.f90:290-291, 416-417).  This call returns the size of the last
 * estimate's matrix (0 when off) and that estimate. */
HECMW33_API void hecmw33_gpu_condition_estimate(const int *handle, int *n, double *emin, double *emax, int *ierr);

/* hecmw_solve (hecmw_solver.f90:9-88) for METHOD = 1-7 on the resident matrix:
 * zero-RHS check, zero-diagonal check, preconditioner recycle policy
 * (hecmw_matrix_misc.F90:858-877), preconditioner setup (PRECOND 1,2 = SSOR with the
 * reference's RCM + multicolour ordering, 3 = DIAG, 10 / 11 / 12 = block ILU(0) / ILU(1) /
 * ILU(2)), CG (or
 * BiCGSTAB, GMRES(Iarray(6)), GPBiCG, GMRESR, GMRESREN, CR) to Rarray(1), the METHOD2 = 2-7
 * fallback of a diverged CG (GMRESR and GMRESREN clear the preconditioner when they return,
 * as hecmw_precond_clear does, so the next solve sets it up again)
 * (hecmw_solver_Iterative.f90:138-142), true relative residual, converged/diverged
 * flags Iarray(81)/(82).
 * B, X: host arrays of 3*NP (X: initial guess in, solution out).
 * iter, resid: ITER and RESID as hecmw_solve_CG returns them.
 * times[3]: set-up, solve and communication seconds (Tset, Tsol, Tcomm = 0). */
HECMW33_API void hecmw33_gpu_solve_resident(const int *handle, const double *B, double *X,
                                            int *Iarray, double *Rarray, int *iter,
                                            double *resid, double *times, int *ierr);

/* As hecmw33_gpu_solve_resident, with B and X in device memory (3*NP doubles each,
 * on the handle's device).  Used when the caller keeps its vectors in HBM. */
HECMW33_API void hecmw33_gpu_solve_resident_device(const int *handle, const double *dB,
                                                   double *dX, int *Iarray, double *Rarray,
                                                   int *iter, double *resid, double *times,
                                                   int *ierr);

/* The drop-in for hecmw_solve(hecMESH, hecMAT): set_matrix + solve_resident. */
HECMW33_API void hecmw33_gpu_solve(const int *handle, const int *N, const int *NP,
                                   const int *NPL, const int *NPU, const int *indexL,
                                   const int *itemL, const int *indexU, const int *itemU,
                                   const double *D, const double *AL, const double *AU,
                                   const double *B, double *X, int *Iarray, double *Rarray,
                                   int *iter, double *resid, double *times, int *ierr);

/* Several load cases on the resident matrix: hecmw_solve once per column of B
 * (hecmw_solver.f90:9-88 per right-hand side), with the checks, the recycle policy and
 * the preconditioner setup done once.  Every right-hand side runs its own CG
 * recurrence (hecmw_solver_CG.f90:19-289: own RHO/ALPHA/BETA, breakdown codes, 50-
 * iteration true-residual refresh, convergence and ITER), while the matrix and
 * preconditioner values are read once per iteration for up to 16 of them (SpMM and
 * 16-vector sweeps); more than 16 are taken 16 at a time.
 * B, X: host arrays of 3*NP x nrhs, column-major (column k = load case k; X: initial
 * guesses in, solutions out).  iter[k], resid[k], error[k]: ITER, RESID and the
 * hecmw_solve_CG code of case k (2002 for a zero column, whose solution is 0);
 * true_resid[k] (may be NULL): ||b - A x|| / ||b|| after the solve.
 * Iarray(81) = 1 when every case reached Rarray(1); Iarray(82) = 1 when one diverged.
 * ierr: the first non-zero code of a case other than 2002, or 0.
 * Iarray(43) = 1 (no counterpart in the reference): every case runs the learned
 * two-level preconditioner's flexible CG instead (see hecmw33_gpu_learn_record; FP64
 * smoother and recurrences, Iarray(44) as for one solve, iterPREmax 1), with Ac^-1 read
 * once per iteration for all cases; a coarse matrix that is not positive definite
 * leaves every case on SSOR-CG.  Precision modes (Iarray(42)) do not apply here. */
HECMW33_API void hecmw33_gpu_solve_multi(const int *handle, const int *nrhs, const double *B,
                                         double *X, int *Iarray, double *Rarray, int *iter,
                                         double *resid, int *error, double *true_resid,
                                         double *times, int *ierr);

/* As hecmw33_gpu_solve_multi, with B and X in device memory (3*NP x nrhs doubles). */
HECMW33_API void hecmw33_gpu_solve_multi_device(const int *handle, const int *nrhs,
                                                const double *dB, double *dX, int *Iarray,
                                                double *Rarray, int *iter, double *resid,
                                                int *error, double *true_resid, double *times,
                                                int *ierr);

/* y = A x on the resident matrix (hecmw_matvec_33), host vectors of 3*NP. */
HECMW33_API void hecmw33_gpu_matvec(const int *handle, const double *X, double *Y, int *ierr);

/* z = M^-1 r (hecmw_precond_apply, hecmw_precond.f90:86-172): builds the preconditioner
 * selected by Iarray/Rarray if needed (same recycle rules as solve), then applies
 * Iarray(5) = iterPREmax passes.  Host vectors of 3*NP. */
HECMW33_API void hecmw33_gpu_precond_apply(const int *handle, const double *R, double *Z,
                                           int *Iarray, double *Rarray, int *ierr);

/* The SSOR colour schedule of the current preconditioner: *ncolor, colorindex[0..ncolor]
 * (COLORindex) and perm[0..N-1] (new -> old, 1-based), as hecmw_precond_SSOR_33_setup
 * builds them (hecmw_precond_SSOR_33.F90:93-128).  colorindex needs N+1 entries. */
HECMW33_API void hecmw33_gpu_get_colouring(const int *handle, int *ncolor, int *colorindex,
                                           int *perm, int *ierr);

/* Host-only (no GPU needed): the SSOR colour schedule that hecmw33_gpu_solve would
 * build for this profile with Iarray(34) = ncolor_in: RCM (hecmw_matrix_ordering_CM.f90)
 * followed by multicolouring (hecmw_matrix_ordering_MC.f90).  Outputs as
 * hecmw33_gpu_get_colouring (colorindex needs N+1 entries, perm N, 1-based ids). */
HECMW33_API void hecmw33_gpu_colour_schedule(const int *N, const int *indexL, const int *itemL,
                                             const int *indexU, const int *itemU,
                                             const int *ncolor_in, int *ncolor, int *colorindex,
                                             int *perm, int *ierr);

/* Host-only (no GPU needed; no counterpart in the reference): the colour schedule of
 * the learned preconditioner's SSOR smoother (Iarray(43) = 1): first-fit colours (each
 * node takes the smallest colour that none of its already coloured neighbours has) in
 * the node order and in smallest-last order, whichever needs fewer (8 colours on a
 * lexicographically numbered structured hexahedral mesh); rows ordered by colour and by
 * node inside a colour.  Outputs as hecmw33_gpu_colour_schedule (colorindex needs N+1
 * entries, perm N, 1-based ids). */
HECMW33_API void hecmw33_gpu_smoother_schedule(const int *N, const int *indexL, const int *itemL,
                                               const int *indexU, const int *itemU, int *ncolor,
                                               int *colorindex, int *perm, int *ierr);

/* Host-only (no GPU needed; no counterpart in the reference): the aggregates of the
 * node graph on which the learned two-level preconditioner (Iarray(43) = 1) builds its
 * coarse space.  Greedy passes (a node whose closed neighbourhood is free roots an
 * aggregate of it; the rest join a neighbour's), the first always, then repeated on the
 * aggregate graph while more than *max_aggregates remain (<= 0: the library default,
 * 2000, or HECMW33_COARSE_AGG) and a pass at least halves the count.  agg[0..N-1]
 * receives 0-based aggregate ids, *n_agg their number. */
HECMW33_API void hecmw33_gpu_coarse_aggregates(const int *N, const int *indexL, const int *itemL,
                                               const int *indexU, const int *itemU, const int *max_aggregates,
                                               int *n_agg, int *agg, int *ierr);

/* ---- learned preconditioner (no counterpart in the reference) -------------------
 * Selected by Iarray(43) = 1 (with SSOR, PRECOND 1/2, iterPREmax 1, a whole mesh): a
 * two-level preconditioner in flexible CG (BETA = z.(r - r_old)/RHO_old), the
 * symmetric two-grid cycle
 *     zs = SSOR(r);  zc = zs + P Ac^-1 P^T (r - A zs);  z = zc + SSOR(r - A zc),
 * Ac = P^T A P, on aggregates of the node graph (hecmw33_gpu_coarse_aggregates).  The
 * smoother SSOR is the solve's (same blocks, same SIGMA_DIAG) on its own layouts in
 * first-fit colour order (hecmw33_gpu_smoother_schedule): not bound to the reference's
 * schedule, it needs far fewer colour launches per sweep.  The
 * prolongator is a smoothed aggregation P = (I - Omega D^-1 A) P0 (P0: the aggregates'
 * translations, zero on constrained DOFs; D: the diagonal blocks) whose per-DOF
 * smoothing weights Omega = sigmoid(out) come from a 3-layer message-passing network
 * over the matrix graph (width 32, edge features the scaled 3x3 blocks, BF16 weights,
 * FP32 accumulation), run once per matrix.  Ac is formed on the device and inverted
 * there (FP64, blocked Gauss-Jordan); a coarse correction is P^T r, one dense GEMV and
 * P y.  Iarray(44) picks the smoothing weights: 0 the network's (default), 1 none
 * (Omega = 0: plain aggregation), 2 one half everywhere (the untrained network).  The
 * correction is switched off on the device -- SSOR-CG takes over, restarted -- when
 * RHO <= 0 or the residual falls by less than 20 % over 25 iterations, and from the
 * start when Ac is not positive definite.  Works in FP64 (Iarray(42) = 0) and with
 * the BF16-stored SSOR of precision mode 1 (whose residuals inside the cycle use an
 * FP32 copy of A).  Training data are (r, e) pairs recorded from earlier FP64 SSOR-CG
 * solves on the same handle (earlier Newton or load increments): r_k = b - A x_k and
 * e_k = x* - x_k at iterations 1, 2, 4, 8, ...
 *
 * enable: 1 record pairs during the following FP64 solves, 0 stop, -1 forget them;
 * max_pairs (optional, >0): keep the newest max_pairs pairs; *npairs: pairs held. */
HECMW33_API void hecmw33_gpu_learn_record(const int *handle, const int *enable, const int *max_pairs,
                                          int *npairs, int *ierr);

/* Trains the network on the recorded pairs with the handle's GPU kernels (forward,
 * backward, Adam; FP32 master weights).  Each pair is first smoothed by one step of
 * the smoother (e' = e - SSOR(r), r' = A e': the error the coarse space has to
 * capture); the loss
 * is the mean share of a pair's error energy outside the coarse space,
 * (e'^T r' - (P^T r')^T Ac^-1 P^T r') / (e'^T r'), with Ac rebuilt and inverted at
 * every step.  loss[0]/loss[1]: mean loss before the first and after the last of
 * `steps` steps (learning rate lr). */
HECMW33_API void hecmw33_gpu_learn_train(const int *handle, const int *steps, const double *lr, double *loss,
                                         int *ierr);

/* mode 0: copy the FP32 weights out (theta may be NULL; *n receives the count, or
 * minus the count when there are no weights yet); mode 1: load *n weights (the count
 * must match) and reset the optimiser.  Used to save and restore trained networks. */
HECMW33_API void hecmw33_gpu_learn_weights(const int *handle, const int *mode, float *theta, int *n, int *ierr);

/* One evaluation of the network for checking: with weights theta (FP32) and one pair,
 * residual R and error E (host, 3*NP, R = A E, kept in FP32 as recorded pairs are),
 * returns the network's smoothing weights Omega (Z, 3*NP), the loss of that pair as
 * hecmw33_gpu_learn_train defines it but without the SSOR smoothing,
 * (E^T R - (P^T R)^T Ac^-1 P^T R) / (E^T R), and its gradient with respect to theta
 * (grad, may be NULL): network in FP32, coarse algebra in FP64 on the GPU.  Needs the
 * SSOR preconditioner already built. */
HECMW33_API void hecmw33_gpu_learn_eval(const int *handle, const float *theta, const double *R, const double *E,
                                        double *Z, double *loss, float *grad, int *ierr);

/* Record of the last solve on this handle, the counterpart of the reference's
 * TIMELOG summary and matvec bandwidth model (hecmw_solver_Iterative.f90:170-254):
 *   info[0] iterations, info[1] kernels launched by the last solve (prologue +
 *   iterations + epilogue), info[2] preconditioner sweep groups (colours or levels,
 *   forward + backward), info[3] kernels per iteration, info[4] NZ (blocks),
 *   info[5] SpMV slices, info[6] padded SpMV slots, info[7] outer refinement
 *   steps (1 for the FP64 solve);
 *   dinfo[0] solve seconds (device events), dinfo[1] setup seconds,
 *   dinfo[2] algorithmic SpMV bytes (reference model: 72 NZ + 4 (NPL+NPU)
 *   + 8 (N+1) + 24 N + 24 NP), dinfo[3] algorithmic bytes of one FP64 iteration,
 *   dinfo[4] device bytes held by the handle, dinfo[5] final FP64 true relative
 *   residual ||b - A x|| / ||b||;
 *   info[8] learned preconditioner used (1/0), info[9] iteration at which its
 *   SSOR-CG fallback took over (0 = none), info[10] training pairs held.
 *   info/dinfo need 16 entries each. */
HECMW33_API void hecmw33_gpu_last_solve_info(const int *handle, int *info, double *dinfo, int *ierr);

/* Times `reps` back-to-back launches of the plain SpMV y = A x on the resident
 * matrix (x taken from the last solve) with device events on the handle's stream;
 * *ms_per_launch receives the average.  For bandwidth measurements. */
HECMW33_API void hecmw33_gpu_time_spmv(const int *handle, const int *reps, double *ms_per_launch,
                                       int *ierr);

/* Times `reps` back-to-back applications of the resident preconditioner, one pass
 * z = M^-1 r (hecmw_precond_apply with iterPREmax = 1, hecmw_precond.f90:86-172; for
 * SSOR the forward and backward colour sweeps of hecmw_precond_SSOR_33.F90:302-405, for
 * ILU(p) the level-scheduled sweeps of hecmw_precond_BILU_33.f90), on the last solve's
 * residual, with device events on the handle's stream.  *lowp bit 0 times the
 * BF16-stored factors of precision mode 1; bit 1 times the learned preconditioner's
 * smoother (the same SSOR on its own layouts in first-fit colour order, Iarray(43) = 1)
 * instead of the solve's SSOR.  *ms_per_apply receives the average;
 * *bytes_per_apply (may be NULL) the algorithmic bytes of one application:
 * 76 B per off-diagonal block (22 B with *lowp), the diagonal LU read by both sweeps
 * (72 B per node each, 36 B with *lowp), both triangles' row pointers and 96 B of
 * vector traffic per node.  Needs a solve (or a preconditioner setup) first. */
HECMW33_API void hecmw33_gpu_time_precond(const int *handle, const int *reps, const int *lowp,
                                          double *ms_per_apply, double *bytes_per_apply, int *ierr);

/* No counterpart in the reference.  For callers that cannot allocate GPU memory
 * (their device memory is owned in full by another allocator, or allocation is
 * forbidden between their solves): the relative residual ||b - A x|| / ||b|| of
 * hecmw_rel_resid_L2_33 for a matrix, x and b that the caller already holds in
 * device memory, in the hecmwST_matrix layout (d_indexL/d_indexU: N+1 ints,
 * 1-based items, row-major 3x3 blocks, vectors of 3N doubles).  No handle, no
 * device or pinned allocation: the scratch space is a static 131 kB array in the
 * library, held by every GPU that loads it.  N is limited to 2,097,152 block rows
 * (larger N: HECMW33_ERR_BAD_INPUT, nothing runs).
 * Whole-mesh matrices only (N == NP): every itemL / itemU entry must lie in 1..N.  A
 * domain of a decomposed mesh (external nodes N+1..NP) is rejected: the kernel checks
 * every item before it reads X, skips one outside 1..N, and the call then returns
 * HECMW33_ERR_BAD_INPUT without a residual.  Null pointers are rejected with
 * HECMW33_ERR_BAD_INPUT before anything runs.
 * *resid is a host double; the call returns when it is written.  The work is ordered
 * on the legacy default stream (stream 0): arrays produced on a non-blocking stream
 * must be complete (that stream synchronised) before the call.  Calls share the
 * scratch array: calls that overlap on the GPU race and must be serialised.  The
 * first call on a device looks up the array's address there and keeps it for the
 * process; make it before any stream capture, and do not cudaDeviceReset between
 * calls. */
HECMW33_API void hecmw33_gpu_rel_resid_noalloc(const int *N, const int *d_indexL, const int *d_itemL,
                                               const int *d_indexU, const int *d_itemU,
                                               const double *d_D, const double *d_AL,
                                               const double *d_AU, const double *d_X,
                                               const double *d_B, double *resid, int *ierr);

/* ---- batched solves ------------------------------------------------------------
 * Many independent systems solved together, each as hecmw_solve would solve it alone
 * (hecmw_solver.f90:9-88, hecmw_solve_CG in hecmw_solver_CG.f90:19-289, SSOR_33 in its
 * own RCM + multicolour order or DIAG_33).  The systems are the diagonal blocks of one
 * hecmwST matrix: system s owns the nodes sys_ptr[s] .. sys_ptr[s+1]-1 (0-based,
 * sys_ptr[0] = 0, sys_ptr[nsys] = N) and no block couples two systems.  One solve is
 * one CUDA-graph launch of a persistent kernel; its launch schedule (lanes per sweep
 * row, cluster size of the teams that take the largest systems, their share) comes
 * from hecmw33_gpu_batch_autotune or a JSON-lines cache of earlier tunings
 * (HECMW33_AUTOTUNE_CACHE, default $HOME/.cache/frontistr_b200_autotune.jsonl).
 * No single call of the reference takes a batch: the reference solves the systems
 * one hecmw_solve at a time. */
HECMW33_API void hecmw33_gpu_batch_create(int *handle, int *ierr);
HECMW33_API void hecmw33_gpu_batch_destroy(const int *handle, int *ierr);

/* Uploads the block-diagonal matrix and builds the per-system preconditioners
 * (Iarray(3) PRECOND 1, 2 = SSOR or 3 = DIAG; Iarray(34) ncolor_in; Rarray(2)
 * sigma_diag).  Structure kept when nsys, sys_ptr, N, NPL, NPU, PRECOND and ncolor_in
 * are unchanged and Iarray(98) == 0 (values only). */
HECMW33_API void hecmw33_gpu_batch_set_matrix(const int *handle, const int *nsys, const int *sys_ptr,
                                              const int *N, const int *NP, const int *NPL,
                                              const int *NPU, const int *indexL, const int *itemL,
                                              const int *indexU, const int *itemU, const double *D,
                                              const double *AL, const double *AU, const int *Iarray,
                                              const double *Rarray, int *ierr);

/* Solves every system: B, X host arrays of 3*N (system s at 3*sys_ptr[s]); Iarray(1)
 * MAXIT, Rarray(1) tolerance, Iarray(5) iterPREmax 0 or 1, for every system.
 * iter[s], resid[s], error[s]: ITER, RESID and the hecmw_solve_CG code of system s
 * (2002 zero right-hand side, 2001 zero diagonal: not solved); true_resid[s] (may be
 * NULL): ||b - A x|| / ||b|| of system s.  Iarray(81) = 1 when every system reached
 * the tolerance, Iarray(82) = 1 when one diverged.  ierr: the first non-zero system
 * code other than 2002, or 0.  times: set-up, device solve time, 0. */
HECMW33_API void hecmw33_gpu_batch_solve(const int *handle, const double *B, double *X, int *Iarray,
                                         double *Rarray, int *iter, double *resid, int *error,
                                         double *true_resid, double *times, int *ierr);

/* As hecmw33_gpu_batch_solve with B and X in device memory. */
HECMW33_API void hecmw33_gpu_batch_solve_device(const int *handle, const double *dB, double *dX,
                                                int *Iarray, double *Rarray, int *iter,
                                                double *resid, int *error, double *true_resid,
                                                double *times, int *ierr);

/* Times candidate launch schedules by solving from B/X (X is not modified), keeps the
 * fastest for this handle and appends it to the cache. */
HECMW33_API void hecmw33_gpu_batch_autotune(const int *handle, const double *B, const double *X,
                                            const int *Iarray, const double *Rarray, int *ierr);

/* info[16]: lanes, cluster size, systems taken by teams, by single CTAs, grid (CTAs),
 * tuned (1/0), nsys, kernels per solve, total and largest iteration count of the last
 * solve.  dinfo[16]: last device solve seconds, last set-up seconds, team share,
 * device bytes held. */
HECMW33_API void hecmw33_gpu_batch_info(const int *handle, int *info, double *dinfo, int *ierr);

/* ---- HEX8 assembly on the device (the caller side of hecmw_solve) -------------
 * Linear-elastic HEX8 stiffness (fistr1/src/lib/static_LIB_3d.f90:50-208, STF_C3 with
 * full 2x2x2 Gauss, FORM361=FI; isotropic D of fistr1/src/lib/physics/ElasticLinear.f90)
 * assembled into the handle's resident matrix in element order
 * (hecmw1/src/solver/matrix/hecmw_mat_ass.f90:32-135), with the profile of
 * hecmw_mat_con.f90:21-107, nodal loads F and the constraints of hecmw_mat_ass_bc
 * (hecmw_mat_ass.f90:328-463) applied in list order.  coords: 3*n_node; conn:
 * 8*n_elem 1-based node ids in hex8n order; E, nu: per element; F: 3*n_node nodal
 * loads (NULL = none); bc_node (1-based), bc_dof (1..3), bc_value: n_bc constraints.
 * symbolic = 0 reuses the profile of the previous call on the same mesh (Newton
 * iterations).  NPL, NPU (may be NULL) receive the profile sizes.  Afterwards the
 * matrix and right-hand side are resident: hecmw33_gpu_solve_assembled solves them,
 * hecmw33_gpu_get_matrix copies them out.  No counterpart in hecmw_solve's interface:
 * the reference assembles on the host before calling it. */
HECMW33_API void hecmw33_gpu_assemble_hex8(const int *handle, const int *n_node, const double *coords,
                                           const int *n_elem, const int *conn, const double *E,
                                           const double *nu, const double *F, const int *n_bc,
                                           const int *bc_node, const int *bc_dof, const double *bc_value,
                                           const int *symbolic, int *NPL, int *NPU, int *ierr);

/* As hecmw33_gpu_assemble_hex8 for a compressible Neo-Hookean material
 * (fistr1/src/lib/physics/Hyperelastic.f90:286-381, W = C10 (I1bar - 3) + (J - 1)^2 / D1),
 * total Lagrangian: the tangent K(U) (material + geometric) at nodal displacements U
 * (3*n_node) and the right-hand side F - f_int(U), then the constraints.  Blocks agree
 * with the host restatement to rounding (J^-2/3 comes from CUDA's pow).  n_inverted
 * (may be NULL) receives the number of elements with J <= 0 at a Gauss point. */
HECMW33_API void hecmw33_gpu_assemble_hex8_neohooke(const int *handle, const int *n_node,
                                                    const double *coords, const int *n_elem,
                                                    const int *conn, const double *C10, const double *D1,
                                                    const double *U, const double *F, const int *n_bc,
                                                    const int *bc_node, const int *bc_dof,
                                                    const double *bc_value, const int *symbolic, int *NPL,
                                                    int *NPU, int *n_inverted, int *ierr);

/* Copies the resident matrix (hecmwST arrays, sizes as hecmw33_gpu_assemble_hex8
 * reports) and right-hand side to host arrays; any pointer may be NULL. */
HECMW33_API void hecmw33_gpu_get_matrix(const int *handle, int *indexL, int *itemL, int *indexU,
                                        int *itemU, double *D, double *AL, double *AU, double *B,
                                        int *ierr);

/* hecmw33_gpu_solve_resident on the resident right-hand side of the last assembly:
 * X (host, 3*N) initial guess in, solution out. */
HECMW33_API void hecmw33_gpu_solve_assembled(const int *handle, double *X, int *Iarray, double *Rarray,
                                             int *iter, double *resid, double *times, int *ierr);

/* Copies the message of the last error of the calling thread into buf; returns its length. */
HECMW33_API int hecmw33_gpu_last_error(char *buf, int len);

#ifdef __cplusplus
}
#endif
#endif /* HECMW33_GPU_H */
