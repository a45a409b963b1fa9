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

#include <cooperative_groups.h>
#include <cuda_bf16.h>

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

// As reduce_finish for two values at once (partials[part] and partials[total + part]).
template <class Fin>
__device__ __forceinline__ void reduce_finish2(double v1, double v2, double *partials, int part, int total,
                                               unsigned int *ticket, Fin fin) {
  __shared__ double sh[32];
  __shared__ int is_last;
  v1 = block_sum(v1, sh);
  v2 = block_sum(v2, sh);
  if (threadIdx.x == 0) {
    partials[part] = v1;
    partials[total + part] = v2;
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == unsigned(total) - 1u);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double s1 = 0.0, s2 = 0.0;
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    s1 += __ldcg(&partials[i]);
    s2 += __ldcg(&partials[total + i]);
  }
  s1 = block_sum(s1, sh);
  s2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    fin(s1, s2);
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
    if (st->lanczos && st->iter <= st->lanczos_cap) {
      st->lanczos[2 * (st->iter - 1)] = st->alpha;
      st->lanczos[2 * (st->iter - 1) + 1] = st->beta;
      st->lanczos_n = st->iter;
    }
  }
}

// DNRM2 after r -= alpha q (:248-250): a residual at or below TOL asks for a recompute
// ITERLOG: this iteration's RESID into the history
__device__ __forceinline__ void record_resid(CgState *st) {
  if (st->rhist && st->iter >= 1 && st->iter <= st->rhist_cap) {
    st->rhist[st->iter - 1] = st->resid;
    st->rhist_n = st->iter;
  }
}

__device__ __forceinline__ void fin_rr(CgState *st, double rr) {
  st->rr = rr;
  st->resid = sqrt(rr / st->bnrm2);
  record_resid(st);
  if (st->reliable) {
    // FP32 recursive residual: ask for an FP64 reliable update when it has fallen
    // by ru_delta since the last one, or reached the tolerance
    if (st->resid <= st->ru_delta * st->ru_mark || st->resid <= st->tol) st->ru_pending = 1;
    st->recompute = 0;
    return;
  }
  if (st->inner) {
    // inner solve of the refinement: the recursive residual decides; the outer
    // FP64 loop recomputes the true residual itself
    if (st->resid <= st->tol) {
      st->done = 1;
      st->converged = 1;
    }
    st->recompute = 0;
    return;
  }
  st->recompute = st->resid <= st->tol ? 1 : 0;
}

// Flexible CG: RHO = z.r, DELTA = z.r_old, BETA = (RHO - DELTA) / RHO_old (the
// Polak-Ribiere form that keeps CG convergent with a preconditioner that changes
// from one iteration to the next).  A non-positive RHO while the network is active
// means the learned step points away from the error: the network is switched off
// (SSOR-CG fallback) and the recurrence restarts.
__device__ __forceinline__ void fin_rho_flex(CgState *st, double rho, double delta) {
  st->rho = rho;
  if (rho == 0.0) {
    st->done = 1;
    return;
  }
  if (rho != rho) {
    st->error = HECMW33_ERR_DIVERGE_NAN;
    st->done = 1;
    return;
  }
  if (rho < 0.0 && st->use_gnn) {
    st->use_gnn = 0;
    st->fallback = st->iter;
    st->restart = 1;
  } else if (st->iter > 1 && !st->restart && rho * st->rho1 <= 0) {
    st->n_indef++;
    if (st->n_indef >= 3) {
      st->error = HECMW33_ERR_DIVERGE_PC;
      st->done = 1;
      return;
    }
  }
  st->beta = (st->iter == 1 || st->restart) ? 0.0 : (rho - delta) / st->rho1;
  st->restart = 0;
}

// End of one iteration: MAXIT test (:275) and the loop condition.  Only this
// function sets the condition back to 1; iter_begin_kernel clears it first, so an
// iteration whose control never ran ends the loop instead of repeating forever.
__device__ __forceinline__ void loop_ctl(CgState *st, cudaGraphConditionalHandle h, int use_cond) {
  if (!st->done && st->guard > st->maxit + 1) {
    st->error = HECMW33_ERR_TIMEOUT;
    st->done = 1;
  }
  // learned preconditioner: less than 20 % residual reduction over 25 iterations
  // counts as stagnation and hands over to SSOR-CG (restarted)
  if (!st->done && st->use_gnn && (st->iter % 25) == 0) {
    if (st->iter > 25 && st->resid > 0.8 * st->resid_mark) {
      st->use_gnn = 0;
      st->fallback = st->iter;
      st->restart = 1;
    }
    st->resid_mark = st->resid;
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
template <class TA, class R>
__device__ __forceinline__ void lu_solve(const TA *__restrict__ alu, int stride, int row, R &x1, R &x2,
                                         R &x3) {
  const R a0 = R(alu[0 * stride + row]), a1 = R(alu[1 * stride + row]), a2 = R(alu[2 * stride + row]);
  const R a3 = R(alu[3 * stride + row]), a4 = R(alu[4 * stride + row]), a5 = R(alu[5 * stride + row]);
  const R a6 = R(alu[6 * stride + row]), a7 = R(alu[7 * stride + row]), a8 = R(alu[8 * stride + row]);
  x2 = x2 - a3 * x1;
  x3 = x3 - a6 * x1 - a7 * x2;
  x3 = a8 * x3;
  x2 = a4 * (x2 - a5 * x3);
  x1 = a0 * (x1 - a2 * x3 - a1 * x2);
}

// Streaming (evict-first) load of a stored matrix value, widened to the working
// precision R.  Values may be stored in FP64, FP32 or BF16.
template <class R, class T>
__device__ __forceinline__ R ld_val(const T *p) {
  return R(__ldcs(p));
}
template <>
__device__ __forceinline__ double ld_val<double, __nv_bfloat16>(const __nv_bfloat16 *p) {
  const unsigned short u = __ldcs(reinterpret_cast<const unsigned short *>(p));
  return double(__uint_as_float(unsigned(u) << 16));
}
template <>
__device__ __forceinline__ float ld_val<float, __nv_bfloat16>(const __nv_bfloat16 *p) {
  const unsigned short u = __ldcs(reinterpret_cast<const unsigned short *>(p));
  return __uint_as_float(unsigned(u) << 16);
}

// Partial sums of one row of a sliced layout whose rows are spread over K lanes
// (SellLayout: block k of a row sits in slot k/K at lane offset k%K): this lane
// accumulates blocks sub, sub+K, sub+2K, ... of the row in the working precision
// R (matrix values, vectors and accumulators alike).  BACKWARD walks them in
// descending order (the reference's backward-sweep order when K == 1).  XL2 reads x
// through L2 (coherent with writes made earlier in the same launch by other CTAs)
// instead of the read-only path.
template <class R, class TV, int K, bool BACKWARD, bool XL2 = false>
__device__ __forceinline__ void row_gemv(const SellView<TV> &A, int s, int lane, int rowlen,
                                         const R *__restrict__ x, R &y0, R &y1, R &y2) {
  const int sub = lane & (K - 1);
  const int nb = rowlen > sub ? (rowlen - sub + K - 1) / K : 0;
  const int slot0 = A.slot0[s];
#pragma unroll 4
  for (int kk = 0; kk < nb; kk++) {
    const int k = BACKWARD ? nb - 1 - kk : kk;
    const int sl = slot0 + k;
    const int c = __ldg(&A.col[sl * 32 + lane]);
    const TV *v = A.val + sl * 288 + lane;
    const R x0 = XL2 ? __ldcg(&x[3 * c]) : __ldg(&x[3 * c]);
    const R x1 = XL2 ? __ldcg(&x[3 * c + 1]) : __ldg(&x[3 * c + 1]);
    const R x2 = XL2 ? __ldcg(&x[3 * c + 2]) : __ldg(&x[3 * c + 2]);
    const R v0 = ld_val<R>(v), v1 = ld_val<R>(v + 32), v2 = ld_val<R>(v + 64);
    const R v3 = ld_val<R>(v + 96), v4 = ld_val<R>(v + 128), v5 = ld_val<R>(v + 160);
    const R v6 = ld_val<R>(v + 192), v7 = ld_val<R>(v + 224), v8 = ld_val<R>(v + 256);
    y0 = fma(v2, x2, fma(v1, x1, fma(v0, x0, y0)));
    y1 = fma(v5, x2, fma(v4, x1, fma(v3, x0, y1)));
    y2 = fma(v8, x2, fma(v7, x1, fma(v6, x0, y2)));
  }
  // combine the K lanes of the row (aligned groups of K lanes)
#pragma unroll
  for (int o = K / 2; o > 0; o >>= 1) {
    y0 += __shfl_xor_sync(0xffffffffu, y0, o);
    y1 += __shfl_xor_sync(0xffffffffu, y1, o);
    y2 += __shfl_xor_sync(0xffffffffu, y2, o);
  }
}

// row_gemv for a uniform layout: every row of the slice owns nslots slots starting
// at slot0, padded with zero blocks (column 0), so the loop needs no row length.
// Padding adds exact zeros; the real blocks are summed in row_gemv's order.
template <class R, class TV, int K, bool BACKWARD>
__device__ __forceinline__ void row_gemv_u(const SellView<TV> &A, int slot0, int nslots, int lane,
                                           const R *__restrict__ x, R &y0, R &y1, R &y2) {
#pragma unroll 4
  for (int kk = 0; kk < nslots; kk++) {
    const int sl = slot0 + (BACKWARD ? nslots - 1 - kk : kk);
    const int c = __ldg(&A.col[sl * 32 + lane]);
    const TV *v = A.val + sl * 288 + lane;
    const R x0 = __ldg(&x[3 * c]), x1 = __ldg(&x[3 * c + 1]), x2 = __ldg(&x[3 * c + 2]);
    const R v0 = ld_val<R>(v), v1 = ld_val<R>(v + 32), v2 = ld_val<R>(v + 64);
    const R v3 = ld_val<R>(v + 96), v4 = ld_val<R>(v + 128), v5 = ld_val<R>(v + 160);
    const R v6 = ld_val<R>(v + 192), v7 = ld_val<R>(v + 224), v8 = ld_val<R>(v + 256);
    y0 = fma(v2, x2, fma(v1, x1, fma(v0, x0, y0)));
    y1 = fma(v5, x2, fma(v4, x1, fma(v3, x0, y1)));
    y2 = fma(v8, x2, fma(v7, x1, fma(v6, x0, y2)));
  }
#pragma unroll
  for (int o = K / 2; o > 0; o >>= 1) {
    y0 += __shfl_xor_sync(0xffffffffu, y0, o);
    y1 += __shfl_xor_sync(0xffffffffu, y1, o);
    y2 += __shfl_xor_sync(0xffffffffu, y2, o);
  }
}

// Launch parameters of one colour of a uniform layout: rows [row0, row1) in slices of
// 32/K rows, slice j of the colour starting at slot slot0 + j*len.
// One colour of a run-table layout: rows [row0, row1), 32/K rows per slice; run r
// covers the colour's slices slice[r] .. slice[r+1]-1 (relative to its first slice),
// starting at slot slot[r] with len[r] slots per slice.
constexpr int kMaxRuns = 24;
struct RunShape {
  int row0, row1, nruns;
  int slice[kMaxRuns + 1];
  int slot[kMaxRuns];
  int len[kMaxRuns];
};

// ---- kernels ---------------------------------------------------------------

// Scatter raw hecmwST blocks (D|AL|AU, 9 doubles each) into a sliced layout.
template <class T>
__global__ void pack_sell_kernel(T *__restrict__ val, const int *__restrict__ src, int nslots,
                                 const double *__restrict__ raw) {
  pdl_entry();
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
  pdl_entry();
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
// TV: the stored values (R by default; FP32 for the residuals inside the learned
// preconditioner of precision mode 1).
template <class R, int MODE, class TV = R>
__global__ void __launch_bounds__(kThreads) spmv_kernel(SellView<TV> A, const R *__restrict__ x,
                                                        R *__restrict__ y, const R *__restrict__ b,
                                                        CgState *st, double *partials) {
  pdl_entry();
  if (MODE == 2 && st->done) return;
  const int lane = threadIdx.x & 31;
  const int warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double dot = 0.0;
  for (int s = warp0; s < A.nslices; s += nwarps) {
    const bool active = lane < A.nrows[s];
    const int row = A.row0[s] + lane;
    const int len = active ? A.rowlen[s * 32 + lane] : 0;
    R y0 = 0, y1 = 0, y2 = 0;
    row_gemv<R, TV, 1, false>(A, s, lane, len, x, y0, y1, y2);
    if (active) {
      if (MODE == 1) {
        y0 = b[3 * row] - y0;
        y1 = b[3 * row + 1] - y1;
        y2 = b[3 * row + 2] - y2;
      }
      y[3 * row] = y0;
      y[3 * row + 1] = y1;
      y[3 * row + 2] = y2;
      if (MODE == 2)
        dot += double(x[3 * row]) * double(y0) + double(x[3 * row + 1]) * double(y1) +
               double(x[3 * row + 2]) * double(y2);
    }
  }
  if (MODE == 2) reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[1], [&](double v) { fin_pq(st, v); });
}

// Start of a node-order level launch.  pre & 1: the launch was made with programmatic
// stream serialisation -- let the next level launch as soon as all CTAs of this one
// run, and wait for the previous level only after the static work; that work brings
// into L2 this warp's slices' values (pre & 2) and columns (pre & 4) and its rows'
// diagonal LU entries (pre & 8).  Nothing before the wait reads what an earlier
// launch wrote.
template <class TV, class TA, int K>
__device__ __forceinline__ void level_prologue(const SellView<TV> &A, const TA *alu, int npos, int sbeg, int send,
                                               int pre) {
  if (pre & 1) asm volatile("griddepcontrol.launch_dependents;" :::);
  if (pre & 14) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int s = sbeg + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); s < send; s += nwarps) {
      const int nslots = A.len[s];
      if (lane == 0 && nslots > 0 && (pre & 6)) {
        const int slot0 = A.slot0[s];
        if (pre & 2)
          asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(A.val + size_t(slot0) * 288),
                       "r"(unsigned(nslots) * 288u * unsigned(sizeof(TV)))
                       : "memory");
        if (pre & 4)
          asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(A.col + size_t(slot0) * 32),
                       "r"(unsigned(nslots) * 128u)
                       : "memory");
      }
      const int roff = lane / K;
      if ((pre & 8) && (lane & (K - 1)) == 0 && roff < A.nrows[s]) {
        const int row = A.row0[s] + roff;
#pragma unroll
        for (int e = 0; e < 9; e++) asm volatile("prefetch.global.L2 [%0];" ::"l"(alu + size_t(e) * npos + row));
      }
    }
  }
  if (pre & 1) asm volatile("griddepcontrol.wait;" ::: "memory");
  else pdl_entry();
}

// Node-order sweeps (the ILU(0) level schedules, whose forward and backward orders
// differ).  Forward sweep over the slices [sbeg, send) of one level, each row spread
// over K lanes:  z(node) = LU^-1 ( r(node) - sum_lower A z(col) )
// (hecmw_precond_SSOR_33.F90:309-345)
template <class R, class TV, class TA, int K>
__global__ void __launch_bounds__(kThreads) sweep_fwd_kernel(SellView<TV> L, const int *__restrict__ perm,
                                                             const TA *__restrict__ alu, int npos,
                                                             const R *__restrict__ r, R *__restrict__ z,
                                                             int sbeg, int send, const CgState *st, int pre) {
  level_prologue<TV, TA, K>(L, alu, npos, sbeg, send, pre);
  if (st && st->done) return;
  const int lane = threadIdx.x & 31;
  const int roff = lane / K;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int s = sbeg + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); s < send; s += nwarps) {
    const bool active = roff < L.nrows[s];
    const int row = L.row0[s] + roff;
    const int len = active ? L.rowlen[s * 32 + roff] : 0;
    R a0 = 0, a1 = 0, a2 = 0;
    row_gemv<R, TV, K, false>(L, s, lane, len, z, a0, a1, a2);
    if (active && (lane & (K - 1)) == 0) {
      const int node = perm[row];
      R x1 = r[3 * node] - a0, x2 = r[3 * node + 1] - a1, x3 = r[3 * node + 2] - a2;
      lu_solve(alu, npos, row, x1, x2, x3);
      z[3 * node] = x1;
      z[3 * node + 1] = x2;
      z[3 * node + 2] = x3;
    }
  }
}

// Backward sweep over [sbeg, send), rows spread over K lanes:
// z(node) -= LU^-1 ( sum_upper A z(col) )   (hecmw_precond_SSOR_33.F90:353-405).
// FUSE_RHO accumulates {r}{z} of the finished rows; the last launch's last CTA
// runs the RHO finisher.
template <class R, class TV, class TA, int K, bool FUSE_RHO>
__global__ void __launch_bounds__(kThreads) sweep_bwd_kernel(SellView<TV> U, const int *__restrict__ perm,
                                                             const TA *__restrict__ alu, int npos,
                                                             const R *__restrict__ r, R *__restrict__ z,
                                                             int sbeg, int send, CgState *st,
                                                             double *partials, int part_base,
                                                             int part_total, int pre) {
  level_prologue<TV, TA, K>(U, alu, npos, sbeg, send, pre);
  if (st && st->done) return;
  const int lane = threadIdx.x & 31;
  const int roff = lane / K;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double dot = 0.0;
  for (int s = sbeg + ((blockIdx.x * blockDim.x + threadIdx.x) >> 5); s < send; s += nwarps) {
    const bool active = roff < U.nrows[s];
    const int row = U.row0[s] + roff;
    const int len = active ? U.rowlen[s * 32 + roff] : 0;
    R x1 = 0, x2 = 0, x3 = 0;
    row_gemv<R, TV, K, true>(U, s, lane, len, z, x1, x2, x3);
    if (active && (lane & (K - 1)) == 0) {
      const int node = perm[row];
      lu_solve(alu, npos, row, x1, x2, x3);
      const R z0 = z[3 * node] - x1, z1 = z[3 * node + 1] - x2, z2 = z[3 * node + 2] - x3;
      z[3 * node] = z0;
      z[3 * node + 1] = z1;
      z[3 * node + 2] = z2;
      if (FUSE_RHO)
        dot += double(r[3 * node]) * double(z0) + double(r[3 * node + 1]) * double(z1) +
               double(r[3 * node + 2]) * double(z2);
    }
  }
  if (FUSE_RHO)
    reduce_finish(dot, partials, part_base + blockIdx.x, part_total, &st->ticket[0],
                  [&](double v) { fin_rho(st, v); });
}

// ---- sweeps on the run-table colour layout (multicolour SSOR) --------------
// The rows of a colour are ordered by slot count, so its slices form a few runs of
// equal slot count (RunShape, a kernel parameter): a slice's rows, first slot and slot
// count follow from its index without a load.  The intermediate zpos is in
// colour-position order (columns of the layout are positions).

// Gather of one slice: this lane's blocks of slots slot0 .. slot0+nslots-1 (in
// reverse for BACKWARD), then the sum over the row's K lanes.
// XL2: x was written during this launch (by other CTAs): read it through L2, never
// the read-only path.
template <class R, class TV, int K, bool BACKWARD, bool XL2 = false>
__device__ __forceinline__ void slice_gemv_u(const SellView<TV> &A, int slot0, int nslots, int lane,
                                             const R *__restrict__ x, R &y0, R &y1, R &y2) {
#pragma unroll 4
  for (int kk = 0; kk < nslots; kk++) {
    const int sl = slot0 + (BACKWARD ? nslots - 1 - kk : kk);
    const int c = __ldg(&A.col[sl * 32 + lane]);
    const TV *v = A.val + sl * 288 + lane;
    const R x0 = XL2 ? __ldcg(&x[3 * c]) : __ldg(&x[3 * c]);
    const R x1 = XL2 ? __ldcg(&x[3 * c + 1]) : __ldg(&x[3 * c + 1]);
    const R x2 = XL2 ? __ldcg(&x[3 * c + 2]) : __ldg(&x[3 * c + 2]);
    const R v0 = ld_val<R>(v), v1 = ld_val<R>(v + 32), v2 = ld_val<R>(v + 64);
    const R v3 = ld_val<R>(v + 96), v4 = ld_val<R>(v + 128), v5 = ld_val<R>(v + 160);
    const R v6 = ld_val<R>(v + 192), v7 = ld_val<R>(v + 224), v8 = ld_val<R>(v + 256);
    y0 = fma(v2, x2, fma(v1, x1, fma(v0, x0, y0)));
    y1 = fma(v5, x2, fma(v4, x1, fma(v3, x0, y1)));
    y2 = fma(v8, x2, fma(v7, x1, fma(v6, x0, y2)));
  }
#pragma unroll
  for (int o = K / 2; o > 0; o >>= 1) {
    y0 += __shfl_xor_sync(0xffffffffu, y0, o);
    y1 += __shfl_xor_sync(0xffffffffu, y1, o);
    y2 += __shfl_xor_sync(0xffffffffu, y2, o);
  }
}

// L2 prefetch of slots [slot0, slot0 + nslots) of a layout (values and columns), by
// one lane (cp.async.bulk.prefetch.L2: nothing returns to the SM, nothing waits).
template <class TV>
__device__ __forceinline__ void l2_prefetch_slots(const SellView<TV> &A, int slot0, int nslots, bool vals = true,
                                                  bool cols = true) {
  if (nslots <= 0) return;
  if (vals)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(A.val + size_t(slot0) * 288),
                 "r"(unsigned(nslots) * 288u * unsigned(sizeof(TV)))
                 : "memory");
  if (cols)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(A.col + size_t(slot0) * 32),
                 "r"(unsigned(nslots) * 128u)
                 : "memory");
}

// First slot and slot count of slice t (relative to the colour's first slice).
template <class Shape>
__device__ __forceinline__ void run_slots(const Shape &sh, int t, int &slot0, int &nslots) {
  int r = 0;
  while (r + 1 < sh.nruns && sh.slice[r + 1] <= t) r++;
  nslots = sh.len[r];
  slot0 = sh.slot[r] + (t - sh.slice[r]) * nslots;
}

// Start of a colour launch.  pre & 1: the launch was made with programmatic stream
// serialisation -- let the next colour launch as soon as all CTAs of this one run,
// and wait for the previous colour only after the static work; that static work
// brings into L2 this warp's slices' values (pre & 2), columns (pre & 4) and
// diagonal LU entries (pre & 8).  Nothing before the wait reads what an earlier
// launch wrote.
template <class TV, class TA, int K>
__device__ __forceinline__ void colour_prologue(const SellView<TV> &A, const TA *alu, int npos, int nslices,
                                                const RunShape &sh, int pre) {
  if (pre & 1) asm volatile("griddepcontrol.launch_dependents;" :::);
  if (pre & 14) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nslices; t += nwarps) {
      int slot0, nslots;
      run_slots(sh, t, slot0, nslots);
      if (lane == 0) l2_prefetch_slots(A, slot0, nslots, (pre & 2) != 0, (pre & 4) != 0);
      const int row = sh.row0 + t * (32 / K);
      if ((pre & 8) && lane >= 1 && lane <= 9 && row < sh.row1)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(alu + size_t(lane - 1) * npos + row));
    }
  }
  if (pre & 1) asm volatile("griddepcontrol.wait;" ::: "memory");
  else pdl_entry();
}

// Forward sweep of one colour: zpos(pos) = LU^-1 ( r(perm(pos)) - sum_lower A zpos(col) )
// (hecmw_precond_SSOR_33.F90:309-345).
template <class R, class TV, class TA, int K>
__global__ void __launch_bounds__(kThreads) sweep_fwd_uni_kernel(SellView<TV> L, const int *__restrict__ perm,
                                                                 const TA *__restrict__ alu, int npos,
                                                                 const R *__restrict__ r, R *__restrict__ zpos,
                                                                 int nslices, RunShape sh, const CgState *st,
                                                                 int pre) {
  colour_prologue<TV, TA, K>(L, alu, npos, nslices, sh, pre);
  if (st && st->done) return;
  const int lane = threadIdx.x & 31;
  const int roff = lane / K;
  const bool leader = (lane & (K - 1)) == 0;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nslices; t += nwarps) {
    int slot0, nslots;
    run_slots(sh, t, slot0, nslots);
    const int row = sh.row0 + t * (32 / K) + roff;
    const bool act = row < sh.row1 && leader;
    R r0 = R(0), r1 = R(0), r2 = R(0);
    if (act) {
      const int node = perm[row];
      r0 = r[3 * node];
      r1 = r[3 * node + 1];
      r2 = r[3 * node + 2];
    }
    R y0 = R(0), y1 = R(0), y2 = R(0);
    slice_gemv_u<R, TV, K, false>(L, slot0, nslots, lane, zpos, y0, y1, y2);
    if (act) {
      R x1 = r0 - y0, x2 = r1 - y1, x3 = r2 - y2;
      lu_solve(alu, npos, row, x1, x2, x3);
      zpos[3 * row] = x1;
      zpos[3 * row + 1] = x2;
      zpos[3 * row + 2] = x3;
    }
  }
}

// Backward sweep of one colour: zpos(pos) -= LU^-1 ( sum_upper A zpos(col) ), the
// finished rows also written to z in node order; FUSE_RHO accumulates {r}{z} and the
// last launch's last CTA runs the RHO finisher (hecmw_precond_SSOR_33.F90:353-405).
// DPOS: dpos receives the row's correction LU^-1 (...) = y - z (y the forward value),
// in colour-position order, for lower_resid_kernel.  A compile-time choice: the extra
// store changes how the compiler contracts z = c - x, so the kernel without it keeps
// the drop-in's arithmetic bit for bit.
template <class R, class TV, class TA, int K, bool FUSE_RHO, bool DPOS = false>
__global__ void __launch_bounds__(kThreads) sweep_bwd_uni_kernel(SellView<TV> U, const int *__restrict__ perm,
                                                                 const TA *__restrict__ alu, int npos,
                                                                 const R *__restrict__ r, R *__restrict__ z,
                                                                 R *__restrict__ zpos, int nslices, RunShape sh,
                                                                 CgState *st, double *partials, int part_base,
                                                                 int part_total, int pre, R *__restrict__ dpos) {
  colour_prologue<TV, TA, K>(U, alu, npos, nslices, sh, pre);
  if (st && st->done) return;
  const int lane = threadIdx.x & 31;
  const int roff = lane / K;
  const bool leader = (lane & (K - 1)) == 0;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double dot = 0.0;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < nslices; t += nwarps) {
    int slot0, nslots;
    run_slots(sh, t, slot0, nslots);
    const int row = sh.row0 + t * (32 / K) + roff;
    const bool act = row < sh.row1 && leader;
    int node = 0;
    R c0 = R(0), c1 = R(0), c2 = R(0);
    if (act) {  // this row's node and current value (written by the forward sweep)
      node = perm[row];
      c0 = zpos[3 * row];
      c1 = zpos[3 * row + 1];
      c2 = zpos[3 * row + 2];
    }
    R x1 = R(0), x2 = R(0), x3 = R(0);
    slice_gemv_u<R, TV, K, true>(U, slot0, nslots, lane, zpos, x1, x2, x3);
    if (act) {
      lu_solve(alu, npos, row, x1, x2, x3);
      const R z0 = c0 - x1, z1 = c1 - x2, z2 = c2 - x3;
      zpos[3 * row] = z0;
      zpos[3 * row + 1] = z1;
      zpos[3 * row + 2] = z2;
      z[3 * node] = z0;
      z[3 * node + 1] = z1;
      z[3 * node + 2] = z2;
      if constexpr (DPOS) {
        dpos[3 * row] = x1;
        dpos[3 * row + 1] = x2;
        dpos[3 * row + 2] = x3;
      }
      if (FUSE_RHO)
        dot += double(r[3 * node]) * double(z0) + double(r[3 * node + 1]) * double(z1) +
               double(r[3 * node + 2]) * double(z2);
    }
  }
  if (FUSE_RHO)
    reduce_finish(dot, partials, part_base + blockIdx.x, part_total, &st->ticket[0],
                  [&](double v) { fin_rho(st, v); });
}

// w = r - A z for z = SSOR(r) from a zero start with unit SIGMA_DIAG, without A: the
// forward sweep solves (D + L) y = r, the backward (D + U) z = D y, so
// r - A z = (D + L) y - L z - (D + U) z = L (y - z), and the backward sweep wrote
// d = y - z (dpos).  One pass over the lower layout (all colours), warp per slice;
// w in node order.
template <class R, class TV, int K>
__global__ void __launch_bounds__(kThreads) lower_resid_kernel(SellView<TV> L, const int *__restrict__ perm,
                                                               const R *__restrict__ dpos, R *__restrict__ w,
                                                               const CgState *st) {
  pdl_entry();
  if (st && st->done) return;
  const int lane = threadIdx.x & 31;
  const int roff = lane / K;
  const bool leader = (lane & (K - 1)) == 0;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < L.nslices; s += nwarps) {
    const bool act = roff < L.nrows[s] && leader;
    R y0 = R(0), y1 = R(0), y2 = R(0);
    slice_gemv_u<R, TV, K, false>(L, L.slot0[s], L.len[s], lane, dpos, y0, y1, y2);
    if (act) {
      const int node = perm[L.row0[s] + roff];
      w[3 * node] = y0;
      w[3 * node + 1] = y1;
      w[3 * node + 2] = y2;
    }
  }
}

// ---- symmetric diagonal scaling (SCALING=YES, hecmw_solver_scaling_33.f90) ----
// s_(3i+a) = 1 / sqrt(|D_i(a,a)|) (:47-51).
static __global__ void scale_vector_kernel(const double *__restrict__ D, int n, double *__restrict__ s) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n; i += gridDim.x * blockDim.x) {
    const int node = i / 3, a = i - 3 * node;
    s[i] = 1.0 / sqrt(fabs(D[9 * size_t(node) + 4 * a]));
  }
}

// out = in with entry (a,b) of each block (row r, column c) multiplied by s_(3r+a)
// and then s_(3c+b), in that order (:55-110).
static __global__ void scale_blocks_kernel(const double *__restrict__ in, double *__restrict__ out,
                                           const int *__restrict__ brow, const int *__restrict__ bcol,
                                           const double *__restrict__ s, int64_t nblocks) {
  pdl_entry();
  const int64_t total = 9 * nblocks;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < total;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t k = i / 9;
    const int e = int(i - 9 * k), a = e / 3, b = e - 3 * a;
    out[i] = in[i] * s[3 * size_t(brow[k]) + a] * s[3 * size_t(bcol[k]) + b];
  }
}

// y = y * s elementwise (B scaled forward :112-116, X scaled back :144-147).
static __global__ void mul_vec_kernel(double *__restrict__ y, const double *__restrict__ s, int n) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = y[i] * s[i];
}

// Block-diagonal preconditioner z = ALU^-1 r (hecmw_precond_DIAG_33.F90:116-136),
// optionally with the fused {r}{z} partial.
template <class R, class TA, bool FUSE_RHO>
__global__ void __launch_bounds__(kThreads) diag_kernel(const TA *__restrict__ alu, int n,
                                                        const R *__restrict__ r, R *__restrict__ z,
                                                        CgState *st, double *partials) {
  pdl_entry();
  if (st && st->done) return;
  double dot = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    R x1 = r[3 * i], x2 = r[3 * i + 1], x3 = r[3 * i + 2];
    lu_solve(alu, n, i, x1, x2, x3);
    z[3 * i] = x1;
    z[3 * i + 1] = x2;
    z[3 * i + 2] = x3;
    if (FUSE_RHO)
      dot += double(r[3 * i]) * double(x1) + double(r[3 * i + 1]) * double(x2) +
             double(r[3 * i + 2]) * double(x3);
  }
  if (FUSE_RHO) reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[0], [&](double v) { fin_rho(st, v); });
}

// RHO and DELTA of flexible CG in one pass, with the fin_rho_flex decisions.
template <class R>
__global__ void __launch_bounds__(kThreads) fcg_rho_kernel(const R *__restrict__ z, const R *__restrict__ r,
                                                           const R *__restrict__ r_old, int n3, CgState *st,
                                                           double *partials) {
  pdl_entry();
  if (st->done) return;
  double a = 0.0, b = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    const double zi = double(z[i]);
    a += zi * double(r[i]);
    b += zi * double(r_old[i]);
  }
  reduce_finish2(a, b, partials, blockIdx.x, gridDim.x, &st->ticket[0],
                 [&](double rho, double delta) { fin_rho_flex(st, rho, delta); });
}

// Flexible CG update: r_old = r, then as update_xr_kernel.
template <class R>
__global__ void __launch_bounds__(kThreads) update_xr_flex_kernel(R *__restrict__ x, const R *__restrict__ p,
                                                                  R *__restrict__ r, R *__restrict__ r_old,
                                                                  const R *__restrict__ q, int n3, CgState *st,
                                                                  double *partials) {
  pdl_entry();
  if (st->done) return;
  const R alpha = R(st->alpha);
  const bool refresh = !st->inner && (st->iter % st->nrecompute) == 0;
  double dot = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    x[i] = alpha * p[i] + x[i];
    const R ri = r[i];
    r_old[i] = ri;
    if (!refresh) {
      const R rn = -alpha * q[i] + ri;
      r[i] = rn;
      dot += double(rn) * double(rn);
    }
  }
  if (!refresh) reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[2], [&](double v) { fin_rr(st, v); });
}

// gamma = sqrt(mean(zs^2)), the learned preconditioner's scale (skipped when off)
template <class R>
__global__ void __launch_bounds__(kThreads) gamma_kernel(const R *__restrict__ zs, int n3, CgState *st,
                                                         double *partials) {
  pdl_entry();
  if (st->done || !st->use_gnn) return;
  double a = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
    a += double(zs[i]) * double(zs[i]);
  reduce_finish(a, partials, blockIdx.x, gridDim.x, &st->ticket[7], [&](double v) {
    const double g2 = v / double(n3);
    st->gamma = g2 > 0.0 ? float(sqrt(g2)) : 1.0f;
  });
}

// {p} = {z} (first iteration) or {z} + BETA {p}  (hecmw_solver_CG.f90:202-207)
template <class R>
__global__ void __launch_bounds__(kThreads) update_p_kernel(const R *__restrict__ z, R *__restrict__ p,
                                                            int n3, const CgState *st) {
  pdl_entry();
  if (st->done) return;
  const bool first = st->iter == 1;
  const R beta = R(st->beta);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
    p[i] = first ? z[i] : z[i] + beta * p[i];
}

// {x} += ALPHA {p}; {r} -= ALPHA {q} with the DNRM2 partial, except on every
// 50th iteration where r is recomputed from b - A x instead (:240-246).
template <class R>
__global__ void __launch_bounds__(kThreads) update_xr_kernel(R *__restrict__ x, const R *__restrict__ p,
                                                             R *__restrict__ r, const R *__restrict__ q,
                                                             int n3, CgState *st, double *partials) {
  pdl_entry();
  if (st->done) return;
  const R alpha = R(st->alpha);
  const bool refresh = !st->inner && (st->iter % st->nrecompute) == 0;
  double dot = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    x[i] = alpha * p[i] + x[i];
    if (!refresh) {
      const R ri = -alpha * q[i] + r[i];
      r[i] = ri;
      dot += double(ri) * double(ri);
    }
  }
  if (!refresh) reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[2], [&](double v) { fin_rr(st, v); });
}

// End of an iteration: when a true residual is due (every 50th iteration, or
// RESID <= TOL, :242-274) r = b - A x and RESID are recomputed; then the loop
// control.  Exactly one thread runs loop_ctl per iteration.
template <class R>
__global__ void __launch_bounds__(kThreads) resid_ctl_kernel(SellView<R> A, const R *__restrict__ x,
                                                             R *__restrict__ r, const R *__restrict__ b,
                                                             CgState *st, double *partials,
                                                             cudaGraphConditionalHandle h, int use_cond) {
  pdl_entry();
  const bool need = !st->done && ((!st->inner && (st->iter % st->nrecompute) == 0) || st->recompute);
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
    R y0 = 0, y1 = 0, y2 = 0;
    row_gemv<R, R, 1, false>(A, s, lane, len, x, y0, y1, y2);
    if (active) {
      y0 = b[3 * row] - y0;
      y1 = b[3 * row + 1] - y1;
      y2 = b[3 * row + 2] - y2;
      r[3 * row] = y0;
      r[3 * row + 1] = y1;
      r[3 * row + 2] = y2;
      dot += double(y0) * double(y0) + double(y1) * double(y1) + double(y2) * double(y2);
    }
  }
  reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[3], [&](double v) {
    st->rr = v;
    st->resid = sqrt(v / st->bnrm2);
    if (!st->inner && (st->iter % st->nrecompute) == 0) record_resid(st);  // the iteration's RESID
    if (st->resid <= st->tol) {
      st->done = 1;
      st->converged = 1;
    }
    loop_ctl(st, h, use_cond);
  });
}

// ---- mixed precision with reliable updates --------------------------------
// Start: r32 = float(r64) (r64 = b - A x64 computed by the FP64 SpMV), x32 = 0,
// ru_mark = ||r64|| / ||b||; a start already within the tolerance ends the loop.
static __global__ void __launch_bounds__(kThreads) ru_init_kernel(const double *__restrict__ r64, float *__restrict__ r32,
                                                           float *__restrict__ x32, int n3, CgState *st,
                                                           double *partials, cudaGraphConditionalHandle h,
                                                           int use_cond) {
  pdl_entry();
  double dot = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    const double v = r64[i];
    r32[i] = float(v);
    x32[i] = 0.0f;
    dot += v * v;
  }
  reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[6], [&](double v) {
    if (st->bnrm2 > 0.0) {
      st->ru_mark = sqrt(v / st->bnrm2);
      st->resid = st->ru_mark;
      if (st->ru_mark <= st->tol) {
        st->done = 1;
        st->converged = 1;
      }
    }
    set_loop(h, use_cond, !st->done);
  });
}

// Reliable update, part 1 (only when pending): x64 += x32, x32 = 0.
static __global__ void __launch_bounds__(kThreads) ru_update_x_kernel(double *__restrict__ x64, float *__restrict__ x32,
                                                               int n3, const CgState *st) {
  pdl_entry();
  if (st->done || !st->ru_pending) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    x64[i] = x64[i] + double(x32[i]);
    x32[i] = 0.0f;
  }
}

// Reliable update, part 2 and the end of the iteration: when pending, the FP64 true
// residual r64 = b - A x64 replaces the FP32 one (r32 = float(r64)) and decides
// convergence on ||r64|| / ||b||; then the loop control.
static __global__ void __launch_bounds__(kThreads) ru_resid_kernel(SellView<double> A, const double *__restrict__ x64,
                                                            double *__restrict__ r64, const double *__restrict__ b64,
                                                            float *__restrict__ r32, CgState *st, double *partials,
                                                            cudaGraphConditionalHandle h, int use_cond) {
  pdl_entry();
  const bool need = !st->done && st->ru_pending;
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
    row_gemv<double, double, 1, false>(A, s, lane, len, x64, y0, y1, y2);
    if (active) {
      y0 = b64[3 * row] - y0;
      y1 = b64[3 * row + 1] - y1;
      y2 = b64[3 * row + 2] - y2;
      r64[3 * row] = y0;
      r64[3 * row + 1] = y1;
      r64[3 * row + 2] = y2;
      r32[3 * row] = float(y0);
      r32[3 * row + 1] = float(y1);
      r32[3 * row + 2] = float(y2);
      dot += y0 * y0 + y1 * y1 + y2 * y2;
    }
  }
  reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[3], [&](double v) {
    st->rr = v;
    st->resid = sqrt(v / st->bnrm2);
    st->ru_pending = 0;
    st->ru_count++;
    st->ru_mark = st->resid;
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
template <class R, int WHICH>
__global__ void __launch_bounds__(kThreads) dot_kernel(const R *__restrict__ a, const R *__restrict__ b,
                                                       int n3, CgState *st, double *partials,
                                                       cudaGraphConditionalHandle h, int use_cond) {
  pdl_entry();
  if (WHICH == 1 && st->done) return;
  double dot = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
    dot += double(a[i]) * double(b[i]);
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
static __global__ void iter_begin_kernel(CgState *st, cudaGraphConditionalHandle h, int use_cond) {
  pdl_entry();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  st->guard++;
  set_loop(h, use_cond, 0);
}

static __global__ void cg_init_kernel(CgState *st, const CgParams *prm) {
  pdl_entry();
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
  st->inner = prm->inner;
  st->flexible = prm->flexible;
  st->use_gnn = prm->use_gnn;
  st->restart = 0;
  st->fallback = 0;
  st->omega = st->c2 = 0.0;
  st->nrecompute = prm->method == 2 ? kIterRecomputeRBicg : kIterRecomputeR;
  st->resid_mark = 1.0;
  st->gamma = 1.0f;
  st->reliable = prm->reliable;
  st->ru_pending = 0;
  st->ru_count = 0;
  st->ru_delta = prm->ru_delta;
  st->ru_mark = 1.0;
  st->lanczos = prm->lanczos;
  st->lanczos_cap = prm->lanczos_cap;
  st->lanczos_n = 0;
  st->rhist = prm->rhist;
  st->rhist_cap = prm->rhist_cap;
  st->rhist_n = 0;
  for (int i = 0; i < 8; i++) st->ticket[i] = 0u;
}

// Vector helpers for the unfused preconditioner paths (iterPREmax != 1) and the
// precision conversions of the mixed-precision refinement.
template <class R>
__global__ void copy_kernel(const R *__restrict__ a, R *__restrict__ b, int n, const CgState *st) {
  pdl_entry();
  if (st && st->done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = a[i];
}
template <class R>
__global__ void add_kernel(const R *__restrict__ a, R *__restrict__ b, int n, const CgState *st) {
  pdl_entry();
  if (st && st->done) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = b[i] + a[i];
}
// b = float(a) (inner right-hand side from the FP64 residual)
static __global__ void narrow_kernel(const double *__restrict__ a, float *__restrict__ b, int n) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) b[i] = float(a[i]);
}
// x += double(d) (FP64 correction of the outer refinement)
static __global__ void widen_add_kernel(const float *__restrict__ d, double *__restrict__ x, int n) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = x[i] + double(d[i]);
}
// b = R(a) for value arrays (FP32 copies of the matrix / preconditioner values)
template <class R>
__global__ void convert_kernel(const double *__restrict__ a, R *__restrict__ b, size_t n) {
  pdl_entry();
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    b[i] = R(a[i]);
}
// BF16 copies of stored values (round to nearest even)
static __global__ void convert_bf16_kernel(const double *__restrict__ a, __nv_bfloat16 *__restrict__ b, size_t n) {
  pdl_entry();
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    b[i] = __float2bfloat16_rn(float(a[i]));
}

}  // namespace h33
