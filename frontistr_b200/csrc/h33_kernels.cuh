// h33_kernels.cuh -- device kernels of the B200 3x3-block CG solver.
//
// Layout (see SellView): one warp per slice of 32 block rows, one lane per block
// row.  A slice's blocks are stored slot by slot; within a slot the 32 lanes'
// entries e are contiguous, so every value load of a warp is a fully coalesced
// 256-byte (double) / 128-byte (float) transaction streamed from HBM.
//
// The CG scalars live in a device CgState; reductions are deterministic: every
// CTA writes one partial, the last CTA to arrive (ticket counter) sums the
// partials in a fixed order and runs the "finisher" that applies the
// hecmw_solve_CG decisions (hecmw_solver_CG.f90:164-279).
#pragma once

#include "h33_common.cuh"

namespace h33 {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide deterministic sum; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  v = 0.0;
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = lane < nw ? sh[lane] : 0.0;
    v = warp_sum(v);
  }
  return v;
}

// Publishes this CTA's partial at partials[part]; the last of `total` arriving
// CTAs (across launches, counted on *ticket) sums partials[0..total) in a fixed
// order and calls fin(sum) on thread 0, then re-arms the ticket.
template <class Fin>
__device__ __forceinline__ void reduce_finish(double v, double *partials, int part, int total,
                                              unsigned int *ticket, Fin fin) {
  __shared__ double sh[32];
  __shared__ int is_last;
  v = block_sum(v, sh);
  if (threadIdx.x == 0) {
    partials[part] = v;
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == unsigned(total) - 1u);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double s = 0.0;
  for (int i = threadIdx.x; i < total; i += blockDim.x) s += __ldcg(&partials[i]);
  s = block_sum(s, sh);
  if (threadIdx.x == 0) {
    fin(s);
    *ticket = 0u;
  }
}

// ---- CG decisions (hecmw_solver_CG.f90) ------------------------------------
__device__ __forceinline__ void set_loop(cudaGraphConditionalHandle h, int use_cond, int go) {
  if (use_cond) cudaGraphSetConditional(h, go ? 1u : 0u);
}

// RHO = {r}{z} and its breakdown tests (:179-194), BETA (:202-207)
__device__ __forceinline__ void fin_rho(CgState *st, double rho) {
  st->rho = rho;
  if (rho == 0.0) {
    st->done = 1;
    return;
  } else if (st->iter > 1 && rho * st->rho1 <= 0) {
    st->n_indef++;
    if (st->n_indef >= 3) {
      st->error = HECMW33_ERR_DIVERGE_PC;
      st->done = 1;
      return;
    }
  } else if (rho != rho) {
    st->error = HECMW33_ERR_DIVERGE_NAN;
    st->done = 1;
    return;
  }
  st->beta = st->iter == 1 ? 0.0 : rho / st->rho1;
}

// C1 = {p}{q} and ALPHA (:221-234)
__device__ __forceinline__ void fin_pq(CgState *st, double c1) {
  st->pq = c1;
  if (c1 <= 0) {
    st->error = HECMW33_ERR_DIVERGE_MAT;
    st->done = 1;
  } else if (c1 != c1) {
    st->error = HECMW33_ERR_DIVERGE_NAN;
    st->done = 1;
  } else {
    st->alpha = st->rho / c1;
  }
}

// DNRM2 after r -= alpha q (:248-250): a residual at or below TOL asks for a recompute
__device__ __forceinline__ void fin_rr(CgState *st, double rr) {
  st->rr = rr;
  st->resid = sqrt(rr / st->bnrm2);
  st->recompute = st->resid <= st->tol ? 1 : 0;
}

// End of one iteration: MAXIT test (:275) and the loop condition.  Only this
// function sets the condition back to 1; iter_begin_kernel clears it first, so an
// iteration whose control never ran ends the loop instead of repeating forever.
__device__ __forceinline__ void loop_ctl(CgState *st, cudaGraphConditionalHandle h, int use_cond) {
  if (!st->done && st->guard > st->maxit + 1) {
    st->error = HECMW33_ERR_TIMEOUT;
    st->done = 1;
  }
  if (!st->done) {
    if (st->iter == st->maxit) {
      st->error = HECMW33_ERR_NOCONV_MAXIT;
      st->done = 1;
      st->iter = st->maxit + 1;  // a completed Fortran DO loop leaves ITER = MAXIT+1
    } else {
      st->rho1 = st->rho;
      st->iter++;
    }
  }
  set_loop(h, use_cond, !st->done);
}

// ---- 3x3 helpers -----------------------------------------------------------
// Forward/backward substitution with a reciprocal-pivot LU block stored SoA:
// entry e of position `row` at alu[e*stride + row] (hecmw_precond_SSOR_33.F90:332-338).
template <class T>
__device__ __forceinline__ void lu_solve(const T *__restrict__ alu, int stride, int row, double &x1,
                                         double &x2, double &x3) {
  const double a0 = alu[0 * stride + row], a1 = alu[1 * stride + row], a2 = alu[2 * stride + row];
  const double a3 = alu[3 * stride + row], a4 = alu[4 * stride + row], a5 = alu[5 * stride + row];
  const double a6 = alu[6 * stride + row], a7 = alu[7 * stride + row], a8 = alu[8 * stride + row];
  x2 = x2 - a3 * x1;
  x3 = x3 - a6 * x1 - a7 * x2;
  x3 = a8 * x3;
  x2 = a4 * (x2 - a5 * x3);
  x1 = a0 * (x1 - a2 * x3 - a1 * x2);
}

template <class T>
__device__ __forceinline__ T ld_stream(const T *p) {
  return __ldcs(p);
}

// y(row) = sum over the row's blocks of A_blk * x(col), ascending columns.
// SIGN = +1 accumulates, -1 subtracts (forward sweep).  BACKWARD walks the
// slots in descending order (the reference's backward-sweep order).
template <class T, bool BACKWARD>
__device__ __forceinline__ void row_gemv(const SellView<T> &A, int s, int lane, int len,
                                         const double *__restrict__ x, double &y0, double &y1,
                                         double &y2) {
  const int slot0 = A.slot0[s];
#pragma unroll 2
  for (int kk = 0; kk < len; kk++) {
    const int k = BACKWARD ? len - 1 - kk : kk;
    const int sl = slot0 + k;
    const int c = __ldg(&A.col[sl * 32 + lane]);
    const T *v = A.val + sl * 288 + lane;
    const double x0 = __ldg(&x[3 * c]), x1 = __ldg(&x[3 * c + 1]), x2 = __ldg(&x[3 * c + 2]);
    const double v0 = ld_stream(v), v1 = ld_stream(v + 32), v2 = ld_stream(v + 64);
    const double v3 = ld_stream(v + 96), v4 = ld_stream(v + 128), v5 = ld_stream(v + 160);
    const double v6 = ld_stream(v + 192), v7 = ld_stream(v + 224), v8 = ld_stream(v + 256);
    y0 = fma(v2, x2, fma(v1, x1, fma(v0, x0, y0)));
    y1 = fma(v5, x2, fma(v4, x1, fma(v3, x0, y1)));
    y2 = fma(v8, x2, fma(v7, x1, fma(v6, x0, y2)));
  }
}

// ---- kernels ---------------------------------------------------------------

// Scatter raw hecmwST blocks (D|AL|AU, 9 doubles each) into a sliced layout.
template <class T>
__global__ void pack_sell_kernel(T *__restrict__ val, const int *__restrict__ src, int nslots,
                                 const double *__restrict__ raw) {
  const int total = nslots * 32;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int b = src[t];
    const int slot = t >> 5, lane = t & 31;
    T *dst = val + slot * 288 + lane;
#pragma unroll
    for (int e = 0; e < 9; e++) dst[e * 32] = b >= 0 ? T(raw[9 * size_t(b) + e]) : T(0);
  }
}

// ALU for position `pos` from the diagonal block of node perm[pos]: sigma-scaled
// diagonal, in-place LU with reciprocal pivots (hecmw_precond_SSOR_33.F90:157-208).
// With lu_done != 0 the raw blocks are already factorised (block ILU(0)).
template <class T>
__global__ void alu_kernel(const double *__restrict__ blocks, const int *__restrict__ perm, int n,
                           double sigma, int lu_done, T *__restrict__ alu, int *__restrict__ err) {
  for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < n; pos += gridDim.x * blockDim.x) {
    const int node = perm ? perm[pos] : pos;
    double a[3][3];
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) a[r][c] = blocks[9 * size_t(node) + 3 * r + c];
    if (!lu_done) {
      a[0][0] *= sigma;
      a[1][1] *= sigma;
      a[2][2] *= sigma;
      for (int k = 0; k < 3; k++) {
        if (a[k][k] == 0.0) atomicOr(err, 1);
        a[k][k] = 1.0 / a[k][k];
        for (int i = k + 1; i < 3; i++) {
          a[i][k] = a[i][k] * a[k][k];
          double pw[3];
          for (int j = k + 1; j < 3; j++) pw[j] = a[i][j] - a[i][k] * a[k][j];
          for (int j = k + 1; j < 3; j++) a[i][j] = pw[j];
        }
      }
    }
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) alu[(3 * r + c) * size_t(n) + pos] = T(a[r][c]);
  }
}

// y = A x (MODE 0), r = b - A x (MODE 1); MODE 2: q = A p with the {p}{q} partial
// and the ALPHA finisher.
template <class T, int MODE>
__global__ void __launch_bounds__(kThreads) spmv_kernel(SellView<T> A, const double *__restrict__ x,
                                                        double *__restrict__ y,
                                                        const double *__restrict__ b, CgState *st,
                                                        double *partials) {
  if (MODE == 2 && st->done) return;
  const int lane = threadIdx.x & 31;
  const int warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double dot = 0.0;
  for (int s = warp0; s < A.nslices; s += nwarps) {
    const bool active = lane < A.nrows[s];
    const int row = A.row0[s] + lane;
    const int len = active ? A.rowlen[s * 32 + lane] : 0;
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    row_gemv<T, false>(A, s, lane, len, x, y0, y1, y2);
    if (active) {
      if (MODE == 1) {
        y0 = b[3 * row] - y0;
        y1 = b[3 * row + 1] - y1;
        y2 = b[3 * row + 2] - y2;
      }
      y[3 * row] = y0;
      y[3 * row + 1] = y1;
      y[3 * row + 2] = y2;
      if (MODE == 2) dot += x[3 * row] * y0 + x[3 * row + 1] * y1 + x[3 * row + 2] * y2;
    }
  }
  if (MODE == 2) reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[1], [&](double v) { fin_pq(st, v); });
}

// Forward sweep over the slices [sbeg, send) of one colour / level:
// z(node) = LU^-1 ( r(node) - sum_lower A z(col) )   (hecmw_precond_SSOR_33.F90:309-345)
template <class T>
__global__ void __launch_bounds__(kThreads) sweep_fwd_kernel(SellView<T> L, const int *__restrict__ perm,
                                                             const T *__restrict__ alu, int npos,
                                                             const double *__restrict__ r,
                                                             double *__restrict__ z, int sbeg,
                                                             int send, const CgState *st) {
  if (st && st->done) return;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int s = sbeg + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); s < send; s += nwarps) {
    if (lane >= L.nrows[s]) continue;
    const int row = L.row0[s] + lane;
    const int node = perm[row];
    const int len = L.rowlen[s * 32 + lane];
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    row_gemv<T, false>(L, s, lane, len, z, a0, a1, a2);
    double x1 = r[3 * node] - a0, x2 = r[3 * node + 1] - a1, x3 = r[3 * node + 2] - a2;
    lu_solve(alu, npos, row, x1, x2, x3);
    z[3 * node] = x1;
    z[3 * node + 1] = x2;
    z[3 * node + 2] = x3;
  }
}

// Backward sweep over [sbeg, send): z(node) -= LU^-1 ( sum_upper A z(col) )
// (hecmw_precond_SSOR_33.F90:353-405).  FUSE_RHO accumulates {r}{z} of the
// finished rows; the last launch's last CTA runs the RHO finisher.
template <class T, bool FUSE_RHO>
__global__ void __launch_bounds__(kThreads) sweep_bwd_kernel(SellView<T> U, const int *__restrict__ perm,
                                                             const T *__restrict__ alu, int npos,
                                                             const double *__restrict__ r,
                                                             double *__restrict__ z, int sbeg,
                                                             int send, CgState *st, double *partials,
                                                             int part_base, int part_total) {
  if (st && st->done) return;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double dot = 0.0;
  for (int s = sbeg + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); s < send; s += nwarps) {
    if (lane >= U.nrows[s]) continue;
    const int row = U.row0[s] + lane;
    const int node = perm[row];
    const int len = U.rowlen[s * 32 + lane];
    double x1 = 0.0, x2 = 0.0, x3 = 0.0;
    row_gemv<T, true>(U, s, lane, len, z, x1, x2, x3);
    lu_solve(alu, npos, row, x1, x2, x3);
    const double z0 = z[3 * node] - x1, z1 = z[3 * node + 1] - x2, z2 = z[3 * node + 2] - x3;
    z[3 * node] = z0;
    z[3 * node + 1] = z1;
    z[3 * node + 2] = z2;
    if (FUSE_RHO) dot += r[3 * node] * z0 + r[3 * node + 1] * z1 + r[3 * node + 2] * z2;
  }
  if (FUSE_RHO)
    reduce_finish(dot, partials, part_base + blockIdx.x, part_total, &st->ticket[0],
                  [&](double v) { fin_rho(st, v); });
}

// Block-diagonal preconditioner z = ALU^-1 r (hecmw_precond_DIAG_33.F90:116-136),
// optionally with the fused {r}{z} partial.
template <class T, bool FUSE_RHO>
__global__ void __launch_bounds__(kThreads) diag_kernel(const T *__restrict__ alu, int n,
                                                        const double *__restrict__ r,
                                                        double *__restrict__ z, CgState *st,
                                                        double *partials) {
  if (st && st->done) return;
  double dot = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double x1 = r[3 * i], x2 = r[3 * i + 1], x3 = r[3 * i + 2];
    lu_solve(alu, n, i, x1, x2, x3);
    z[3 * i] = x1;
    z[3 * i + 1] = x2;
    z[3 * i + 2] = x3;
    if (FUSE_RHO) dot += r[3 * i] * x1 + r[3 * i + 1] * x2 + r[3 * i + 2] * x3;
  }
  if (FUSE_RHO) reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[0], [&](double v) { fin_rho(st, v); });
}

// {p} = {z} (first iteration) or {z} + BETA {p}  (hecmw_solver_CG.f90:202-207)
__global__ void __launch_bounds__(kThreads) update_p_kernel(const double *__restrict__ z,
                                                            double *__restrict__ p, int n3,
                                                            const CgState *st) {
  if (st->done) return;
  const bool first = st->iter == 1;
  const double beta = st->beta;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
    p[i] = first ? z[i] : z[i] + beta * p[i];
}

// {x} += ALPHA {p}; {r} -= ALPHA {q} with the DNRM2 partial, except on every
// 50th iteration where r is recomputed from b - A x instead (:240-246).
__global__ void __launch_bounds__(kThreads) update_xr_kernel(double *__restrict__ x,
                                                             const double *__restrict__ p,
                                                             double *__restrict__ r,
                                                             const double *__restrict__ q, int n3,
                                                             CgState *st, double *partials) {
  if (st->done) return;
  const double alpha = st->alpha;
  const bool refresh = (st->iter % kIterRecomputeR) == 0;
  double dot = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    x[i] = alpha * p[i] + x[i];
    if (!refresh) {
      const double ri = -alpha * q[i] + r[i];
      r[i] = ri;
      dot += ri * ri;
    }
  }
  if (!refresh) reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[2], [&](double v) { fin_rr(st, v); });
}

// End of an iteration: when a true residual is due (every 50th iteration, or
// RESID <= TOL, :242-274) r = b - A x and RESID are recomputed; then the loop
// control.  Exactly one thread runs loop_ctl per iteration.
template <class T>
__global__ void __launch_bounds__(kThreads) resid_ctl_kernel(SellView<T> A, const double *__restrict__ x,
                                                             double *__restrict__ r,
                                                             const double *__restrict__ b, CgState *st,
                                                             double *partials,
                                                             cudaGraphConditionalHandle h, int use_cond) {
  const bool need = !st->done && ((st->iter % kIterRecomputeR) == 0 || st->recompute);
  if (!need) {
    if (blockIdx.x == 0 && threadIdx.x == 0) loop_ctl(st, h, use_cond);
    return;
  }
  const int lane = threadIdx.x & 31;
  const int warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double dot = 0.0;
  for (int s = warp0; s < A.nslices; s += nwarps) {
    const bool active = lane < A.nrows[s];
    const int row = A.row0[s] + lane;
    const int len = active ? A.rowlen[s * 32 + lane] : 0;
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    row_gemv<T, false>(A, s, lane, len, x, y0, y1, y2);
    if (active) {
      y0 = b[3 * row] - y0;
      y1 = b[3 * row + 1] - y1;
      y2 = b[3 * row + 2] - y2;
      r[3 * row] = y0;
      r[3 * row + 1] = y1;
      r[3 * row + 2] = y2;
      dot += y0 * y0 + y1 * y1 + y2 * y2;
    }
  }
  reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[3], [&](double v) {
    st->rr = v;
    st->resid = sqrt(v / st->bnrm2);
    if (st->resid <= st->tol) {
      st->done = 1;
      st->converged = 1;
    }
    loop_ctl(st, h, use_cond);
  });
}

// Generic dot with a selectable finisher:
//   WHICH 0: BNRM2 at the start of a solve (also decides whether the loop runs)
//   WHICH 1: RHO (unfused preconditioner paths)
//   WHICH 2: plain result into st->rr_true
template <int WHICH>
__global__ void __launch_bounds__(kThreads) dot_kernel(const double *__restrict__ a,
                                                       const double *__restrict__ b, int n3,
                                                       CgState *st, double *partials,
                                                       cudaGraphConditionalHandle h, int use_cond) {
  if (WHICH == 1 && st->done) return;
  double dot = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) dot += a[i] * b[i];
  reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[4 + WHICH], [&](double v) {
    if (WHICH == 0) {
      st->bnrm2 = v;
      if (v == 0.0) {
        st->zero_rhs = 1;
        st->done = 1;
      }
      if (st->maxit <= 0) st->done = 1;
      set_loop(h, use_cond, !st->done);
    } else if (WHICH == 1) {
      fin_rho(st, v);
    } else {
      st->rr_true = v;
    }
  });
}

// First kernel of every loop body: fail-safe loop condition and body counter.
__global__ void iter_begin_kernel(CgState *st, cudaGraphConditionalHandle h, int use_cond) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  st->guard++;
  set_loop(h, use_cond, 0);
}

__global__ void cg_init_kernel(CgState *st, const CgParams *prm) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  st->rho = st->rho1 = st->alpha = st->beta = st->pq = st->rr = 0.0;
  st->bnrm2 = 0.0;
  st->resid = 0.0;
  st->rr_true = 0.0;
  st->tol = prm->tol;
  st->maxit = prm->maxit;
  st->iter = 1;
  st->done = 0;
  st->error = 0;
  st->n_indef = 0;
  st->recompute = 0;
  st->converged = 0;
  st->zero_rhs = 0;
  st->guard = 0;
  for (int i = 0; i < 8; i++) st->ticket[i] = 0u;
}

// Vector helpers for the unfused preconditioner paths (iterPREmax != 1).
__global__ void copy_kernel(const double *__restrict__ a, double *__restrict__ b, int n, const CgState *st) {
  if (st && st->done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}
__global__ void add_kernel(const double *__restrict__ a, double *__restrict__ b, int n, const CgState *st) {
  if (st && st->done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = b[i] + a[i];
}
__global__ void zero_kernel(double *__restrict__ b, int n, const CgState *st) {
  if (st && st->done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = 0.0;
}

}  // namespace h33
