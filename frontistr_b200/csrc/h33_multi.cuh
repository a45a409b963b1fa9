// h33_multi.cuh -- multi-right-hand-side CG: up to 16 load cases on one matrix.
//
// Every right-hand side runs its own hecmw_solve_CG recurrence (its own RHO, ALPHA,
// BETA, breakdown tests, 50-iteration true-residual refresh and convergence), but
// the matrix and preconditioner values are streamed once per iteration for all of
// them: the SpMV becomes an SpMM and the SSOR / ILU(0) sweeps solve 16 vectors at
// once.  A half-warp covers one block row and lane l of it carries right-hand side
// l, so each 3x3 block is read once (a broadcast to the 16 lanes) and the vector
// gathers are 128-byte coalesced.
//
// Vector layout ("node-major, RHS-minor"): entry c of node i for right-hand side l
// is v[i*48 + c*16 + l].  Right-hand sides beyond nrhs are padding lanes that start
// as converged.
#pragma once

#include "h33_coarse.cuh"
#include "h33_kernels.cuh"

namespace h33 {

constexpr int kMaxRhs = 16;
constexpr int kMrLanes = 16;  // lanes per row of the SpMM's copy of A
constexpr int kRhsStride = 3 * kMaxRhs;  // doubles per node

// Loop control shared by all right-hand sides.
struct MultiCtl {
  int all_done;
  int guard;
  int nrhs;
  int fault;  // a bounded wait of the tiled SpMM ran out (reported as an error)
  unsigned int ticket[8];
};

// Deterministic per-RHS reduction: this CTA's 16 sums go to partials[cta*16 + l];
// the last CTA to arrive sums the partials of every CTA in a fixed order and runs
// fin(l, sum) on threads 0..15, then re-arms the ticket.  v is this thread's
// partial for RHS (threadIdx.x & 15).
template <class Fin>
__device__ __forceinline__ void mr_reduce_finish(double v, double *partials, int part, int total,
                                                 unsigned int *ticket, Fin fin) {
  __shared__ double sh[kThreads / 16][kMaxRhs];
  __shared__ int is_last;
  const int l = threadIdx.x & 15, hw = threadIdx.x >> 4;
  sh[hw][l] = v;
  __syncthreads();
  if (threadIdx.x < kMaxRhs) {
    double s = 0.0;
    for (int k = 0; k < kThreads / 16; k++) s += sh[k][threadIdx.x];
    partials[size_t(part) * kMaxRhs + threadIdx.x] = s;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == unsigned(total) - 1u);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  // 16 threads per RHS sum strided subsets, then thread l combines its 16 subsets
  double s = 0.0;
  for (int i = hw; i < total; i += kThreads / 16) s += __ldcg(&partials[size_t(i) * kMaxRhs + l]);
  __syncthreads();
  sh[hw][l] = s;
  __syncthreads();
  if (threadIdx.x < kMaxRhs) {
    double t = 0.0;
    for (int k = 0; k < kThreads / 16; k++) t += sh[k][threadIdx.x];
    fin(int(threadIdx.x), t);
  }
  __syncthreads();
  if (threadIdx.x == 0) *ticket = 0u;
}

// Sum of A(row, :) x over the blocks of one row of a sliced layout with K lanes per
// row (block k at slot slot0 + k/K, lane roff*K + k%K), for this lane's RHS.  The
// row is taken 16 blocks at a time: lane j of the half-warp loads block j's column
// index and its nine entries (all issued at once), then every lane receives them by
// shuffles, so inside a chunk only the x gathers touch memory.  hmask: this
// half-warp's lanes.
template <int K>
__device__ __forceinline__ void mr_row(const SellView<double> &A, int s, int roff, int len, int l,
                                       unsigned hmask, const double *__restrict__ x, double &y0, double &y1,
                                       double &y2) {
  const int slot0 = A.slot0[s];
  for (int k0 = 0; k0 < len; k0 += 16) {
    const int kn = min(16, len - k0);
    int myc = 0;
    double mv[9];
#pragma unroll
    for (int e = 0; e < 9; e++) mv[e] = 0.0;
    if (l < kn) {
      const int k = k0 + l;
      const int sl = slot0 + k / K, lp = roff * K + (k & (K - 1));
      myc = __ldg(&A.col[sl * 32 + lp]);
      const double *v = A.val + sl * 288 + lp;
#pragma unroll
      for (int e = 0; e < 9; e++) mv[e] = __ldg(v + 32 * e);
    }
#pragma unroll 4
    for (int kk = 0; kk < kn; kk++) {
      const int c = __shfl_sync(hmask, myc, kk, 16);
      const double *xc = x + size_t(c) * kRhsStride + l;
      const double x0 = xc[0], x1 = xc[16], x2 = xc[32];
      double v[9];
#pragma unroll
      for (int e = 0; e < 9; e++) v[e] = __shfl_sync(hmask, mv[e], kk, 16);
      y0 = fma(v[2], x2, fma(v[1], x1, fma(v[0], x0, y0)));
      y1 = fma(v[5], x2, fma(v[4], x1, fma(v[3], x0, y1)));
      y2 = fma(v[8], x2, fma(v[7], x1, fma(v[6], x0, y2)));
    }
  }
}

// Half-warp t of a group of slices [sb, se) with 32/K rows per slice -> (slice, row offset).
template <int K>
__device__ __forceinline__ bool mr_locate(const SellView<double> &A, int sb, int se, int t, int &s, int &roff) {
  constexpr int rps = 32 / K;
  s = sb + t / rps;
  roff = t % rps;
  return s < se && roff < A.nrows[s];
}

// y = A x (MODE 0); y = b - A x (MODE 1); MODE 2: q = A p with the per-RHS {p}{q}
// and ALPHA; MODE 3: r = b - A x with the per-RHS DNRM2 for the RHS whose true
// residual is due, then the per-RHS end-of-iteration control (resid_ctl_kernel's
// logic for every RHS).  A has K lanes per row (32/K rows per slice): with K = 16 the
// half-warp's 16 blocks of one chunk of its row sit in one slot, so each of the nine
// value loads and the column load is one contiguous 128-byte segment.
template <int MODE, int K>
__global__ void __launch_bounds__(kThreads) mr_spmv_kernel(SellView<double> A, const double *__restrict__ x,
                                                           double *__restrict__ y, const double *__restrict__ b,
                                                           CgState *st, MultiCtl *ctl, double *partials) {
  pdl_entry();
  if (MODE >= 2 && ctl->all_done) return;
  const int l = threadIdx.x & 15;
  bool mine = true;  // this lane's RHS takes part
  if (MODE == 2) mine = !st[l].done;
  if (MODE == 3) {
    mine = !st[l].done && ((st[l].iter % kIterRecomputeR) == 0 || st[l].recompute);
    // no true residual due for any RHS: only the end-of-iteration control runs
    const int any = __syncthreads_or(mine ? 1 : 0);
    if (!any) {
      if (blockIdx.x == 0 && threadIdx.x < kMaxRhs) loop_ctl(&st[threadIdx.x], 0, 0);
      return;
    }
  }
  const int hw0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 4;
  const int nhw = (gridDim.x * blockDim.x) >> 4;
  constexpr int rps = 32 / K;  // rows per slice
  const int nrows_total = A.nslices * rps;
  const unsigned hmask = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
  double dot = 0.0;
  for (int t = hw0; t < nrows_total; t += nhw) {
    const int s = t / rps, roff = t % rps;
    if (roff >= A.nrows[s]) continue;
    const int row = A.row0[s] + roff;
    const int len = A.rowlen[s * 32 + roff];
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    mr_row<K>(A, s, roff, len, l, hmask, x, y0, y1, y2);
    const size_t o = size_t(row) * kRhsStride + l;
    if (MODE == 1 || MODE == 3) {
      y0 = b[o] - y0;
      y1 = b[o + 16] - y1;
      y2 = b[o + 32] - y2;
    }
    if ((MODE == 2 || MODE == 3) && !mine) continue;  // the other RHS keep their vectors
    y[o] = y0;
    y[o + 16] = y1;
    y[o + 32] = y2;
    if (MODE == 2) dot += x[o] * y0 + x[o + 16] * y1 + x[o + 32] * y2;
    if (MODE == 3) dot += y0 * y0 + y1 * y1 + y2 * y2;
  }
  if (MODE == 2)
    mr_reduce_finish(dot, partials, blockIdx.x, gridDim.x, &ctl->ticket[1], [&](int k, double v) {
      if (!st[k].done) fin_pq(&st[k], v);
    });
  if (MODE == 3)
    mr_reduce_finish(dot, partials, blockIdx.x, gridDim.x, &ctl->ticket[3], [&](int k, double v) {
      CgState *s = &st[k];
      const bool need = !s->done && ((s->iter % kIterRecomputeR) == 0 || s->recompute);
      if (need) {
        s->rr = v;
        s->resid = sqrt(v / s->bnrm2);
        if (s->resid <= s->tol) {
          s->done = 1;
          s->converged = 1;
        }
      }
      loop_ctl(s, 0, 0);  // the loop decision over all RHS is mr_ctl_kernel's
    });
}

// ---- tiled SpMM: p staged in shared memory by the bulk-copy engine ------------
// A tile is 16 consecutive block rows (half a slice of the SpMV layout).  The host
// lists each tile's distinct columns (tile_cols[tile_ptr[t] ..]) and, for every block,
// the column's place in that list (lidx, same layout as col).  Warp 0 copies the
// 384-byte rows p[c][0..47] of the tile's columns into shared memory with
// cp.async.bulk on an mbarrier; the half-warps then read p from shared memory.  Each
// p row crosses L2 once per tile instead of once per block that uses it.

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Waits for the mbarrier phase `parity`; bounded by two seconds of the global
// timer (try_wait itself suspends for a bounded time), returns false when it ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity) {
  const uint32_t a = smem_addr(mbar);
  uint64_t t0, t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 > 2000000000ull) return false;
  }
}

__global__ void __launch_bounds__(kThreads) mr_spmm_tiled_kernel(SellView<double> A, const int *__restrict__ tile_ptr,
                                                                 const int *__restrict__ tile_cols,
                                                                 const uint16_t *__restrict__ lidx, int ntiles,
                                                                 const double *__restrict__ x, double *__restrict__ y,
                                                                 CgState *st, MultiCtl *ctl, double *partials) {
  pdl_entry();
  extern __shared__ __align__(128) double xs[];
  __shared__ __align__(8) uint64_t mbar;
  if (ctl->all_done) return;
  const int l = threadIdx.x & 15, hw = threadIdx.x >> 4;
  const bool mine = !st[l].done;
  const unsigned hmask = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  uint32_t parity = 0;
  double dot = 0.0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int c0 = tile_ptr[t], nc = tile_ptr[t + 1] - c0;
    if (threadIdx.x < 32) {
      // the previous tile's reads of xs are complete (barrier below); order them
      // before the copy engine's writes
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      if (threadIdx.x == 0)
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&mbar)),
                     "r"(uint32_t(nc) * 384u)
                     : "memory");
      __syncwarp();
      for (int i = threadIdx.x; i < nc; i += 32) {
        const double *src = x + size_t(tile_cols[c0 + i]) * kRhsStride;
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], 384, [%2];" ::"r"(
                smem_addr(xs + size_t(i) * kRhsStride)),
            "l"(src), "r"(smem_addr(&mbar))
            : "memory");
      }
    }
    const bool ok = mbar_wait(&mbar, parity);
    parity ^= 1u;
    if (!ok) {
      if (threadIdx.x == 0) atomicExch(&ctl->fault, 1);
      mbar_wait(&mbar, parity ^ 1u);  // the copies of this tile, once more (bounded)
    } else {
      const int s = t >> 1, roff = 16 * (t & 1) + hw;
      if (roff < A.nrows[s]) {
        const int row = A.row0[s] + roff;
        const int len = A.rowlen[s * 32 + roff];
        const int slot0 = A.slot0[s];
        double y0 = 0.0, y1 = 0.0, y2 = 0.0;
        for (int k0 = 0; k0 < len; k0 += 16) {
          const int kn = min(16, len - k0);
          int myi = 0;
          double mv[9];
#pragma unroll
          for (int e = 0; e < 9; e++) mv[e] = 0.0;
          if (l < kn) {
            const int sl = slot0 + k0 + l;
            myi = lidx[sl * 32 + roff];
            const double *v = A.val + sl * 288 + roff;
#pragma unroll
            for (int e = 0; e < 9; e++) mv[e] = __ldg(v + 32 * e);
          }
#pragma unroll 4
          for (int kk = 0; kk < kn; kk++) {
            const int li = __shfl_sync(hmask, myi, kk, 16);
            const double *xc = xs + li * kRhsStride + l;
            const double x0 = xc[0], x1 = xc[16], x2 = xc[32];
            double v[9];
#pragma unroll
            for (int e = 0; e < 9; e++) v[e] = __shfl_sync(hmask, mv[e], kk, 16);
            y0 = fma(v[2], x2, fma(v[1], x1, fma(v[0], x0, y0)));
            y1 = fma(v[5], x2, fma(v[4], x1, fma(v[3], x0, y1)));
            y2 = fma(v[8], x2, fma(v[7], x1, fma(v[6], x0, y2)));
          }
        }
        if (mine) {
          const size_t o = size_t(row) * kRhsStride + l;
          y[o] = y0;
          y[o + 16] = y1;
          y[o + 32] = y2;
          dot += x[o] * y0 + x[o + 16] * y1 + x[o + 32] * y2;
        }
      }
    }
    __syncthreads();  // every half-warp is done with xs before the next tile's copies
  }
  if (threadIdx.x == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(&mbar)) : "memory");
  mr_reduce_finish(dot, partials, blockIdx.x, gridDim.x, &ctl->ticket[1], [&](int k, double v) {
    if (!st[k].done) fin_pq(&st[k], v);
  });
}

// Forward sweep over the slices [sb, se) of one colour / level, 16 RHS at once.
// POS: columns are colour positions and the intermediate lives in zpos (colour
// order), as in sweep_fwd_kernel; otherwise node order throughout.
template <int K, bool POS>
__global__ void __launch_bounds__(kThreads) mr_sweep_fwd_kernel(SellView<double> L, const int *__restrict__ perm,
                                                                const double *__restrict__ alu, int npos,
                                                                const double *__restrict__ r, double *__restrict__ z,
                                                                double *__restrict__ zpos, int sb, int se,
                                                                const MultiCtl *ctl) {
  pdl_entry();
  if (ctl && ctl->all_done) return;
  const int l = threadIdx.x & 15;
  const int nhw = (gridDim.x * blockDim.x) >> 4;
  const int total = (se - sb) * (32 / K);
  const unsigned hmask = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; t < total; t += nhw) {
    int s, roff;
    if (!mr_locate<K>(L, sb, se, t, s, roff)) continue;
    const int row = L.row0[s] + roff;
    const int len = L.rowlen[s * 32 + roff];
    const int node = perm[row];
    const size_t o = size_t(node) * kRhsStride + l;
    const double r0 = r[o], r1 = r[o + 16], r2 = r[o + 32];
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    mr_row<K>(L, s, roff, len, l, hmask, POS ? zpos : z, a0, a1, a2);
    double x1 = r0 - a0, x2 = r1 - a1, x3 = r2 - a2;
    lu_solve(alu, npos, row, x1, x2, x3);
    double *out = (POS ? zpos + size_t(row) * kRhsStride + l : z + o);
    out[0] = x1;
    out[16] = x2;
    out[32] = x3;
  }
}

// Backward sweep; FUSE_RHO: per-RHS {r}{z} of the finished rows and, in the last
// launch's last CTA, the RHO finisher of every RHS.  POS: updates zpos and writes the
// finished rows to z in node order.
// DPOS (POS layouts): dpos receives each row's correction y - z per RHS, in position
// order, for mr_lower_resid_kernel (a compile-time choice, as in sweep_bwd_uni_kernel).
template <int K, bool FUSE_RHO, bool POS, bool DPOS = false>
__global__ void __launch_bounds__(kThreads) mr_sweep_bwd_kernel(SellView<double> U, const int *__restrict__ perm,
                                                                const double *__restrict__ alu, int npos,
                                                                const double *__restrict__ r, double *__restrict__ z,
                                                                double *__restrict__ zpos, int sb, int se, CgState *st,
                                                                MultiCtl *ctl, double *partials, int part_base,
                                                                int part_total, double *__restrict__ dpos) {
  pdl_entry();
  if (ctl && ctl->all_done) return;
  const int l = threadIdx.x & 15;
  const int nhw = (gridDim.x * blockDim.x) >> 4;
  const int total = (se - sb) * (32 / K);
  const unsigned hmask = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
  double dot = 0.0;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; t < total; t += nhw) {
    int s, roff;
    if (!mr_locate<K>(U, sb, se, t, s, roff)) continue;
    const int row = U.row0[s] + roff;
    const int len = U.rowlen[s * 32 + roff];
    const int node = perm[row];
    const size_t o = size_t(node) * kRhsStride + l;
    const size_t op = POS ? size_t(row) * kRhsStride + l : o;
    const double *zc = POS ? zpos : z;
    const double c0 = zc[op], c1 = zc[op + 16], c2 = zc[op + 32];
    double x1 = 0.0, x2 = 0.0, x3 = 0.0;
    mr_row<K>(U, s, roff, len, l, hmask, POS ? zpos : z, x1, x2, x3);
    lu_solve(alu, npos, row, x1, x2, x3);
    const double z0 = c0 - x1, z1 = c1 - x2, z2 = c2 - x3;
    if (POS) {
      zpos[op] = z0;
      zpos[op + 16] = z1;
      zpos[op + 32] = z2;
    }
    z[o] = z0;
    z[o + 16] = z1;
    z[o + 32] = z2;
    if constexpr (DPOS) {
      dpos[op] = x1;
      dpos[op + 16] = x2;
      dpos[op + 32] = x3;
    }
    if (FUSE_RHO) dot += r[o] * z0 + r[o + 16] * z1 + r[o + 32] * z2;
  }
  if (FUSE_RHO)
    mr_reduce_finish(dot, partials, part_base + blockIdx.x, part_total, &ctl->ticket[0], [&](int k, double v) {
      if (!st[k].done) fin_rho(&st[k], v);
    });
}

// w = r - A z per RHS after z = SSOR(r) with dpos (unit SIGMA_DIAG): L (y - z) over the
// smoother's lower layout (all colours, a half-warp per row), w in node order.
template <int K>
__global__ void __launch_bounds__(kThreads) mr_lower_resid_kernel(SellView<double> L, const int *__restrict__ perm,
                                                                  const double *__restrict__ dpos,
                                                                  double *__restrict__ w, const MultiCtl *ctl) {
  pdl_entry();
  if (ctl && ctl->all_done) return;
  const int l = threadIdx.x & 15;
  const int nhw = (gridDim.x * blockDim.x) >> 4;
  const int total = L.nslices * (32 / K);
  const unsigned hmask = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; t < total; t += nhw) {
    int s, roff;
    if (!mr_locate<K>(L, 0, L.nslices, t, s, roff)) continue;
    const int row = L.row0[s] + roff;
    const int len = L.rowlen[s * 32 + roff];
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    mr_row<K>(L, s, roff, len, l, hmask, dpos, y0, y1, y2);
    const size_t o = size_t(perm[row]) * kRhsStride + l;
    w[o] = y0;
    w[o + 16] = y1;
    w[o + 32] = y2;
  }
}

// Block-diagonal preconditioner for 16 RHS (optionally with the fused RHO).
template <bool FUSE_RHO>
__global__ void __launch_bounds__(kThreads) mr_diag_kernel(const double *__restrict__ alu, int n,
                                                           const double *__restrict__ r, double *__restrict__ z,
                                                           CgState *st, MultiCtl *ctl, double *partials) {
  pdl_entry();
  if (ctl && ctl->all_done) return;
  const int l = threadIdx.x & 15;
  const int nhw = (gridDim.x * blockDim.x) >> 4;
  double dot = 0.0;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; i < n; i += nhw) {
    const size_t o = size_t(i) * kRhsStride + l;
    double x1 = r[o], x2 = r[o + 16], x3 = r[o + 32];
    lu_solve(alu, n, i, x1, x2, x3);
    z[o] = x1;
    z[o + 16] = x2;
    z[o + 32] = x3;
    if (FUSE_RHO) dot += r[o] * x1 + r[o + 16] * x2 + r[o + 32] * x3;
  }
  if (FUSE_RHO)
    mr_reduce_finish(dot, partials, blockIdx.x, gridDim.x, &ctl->ticket[0], [&](int k, double v) {
      if (!st[k].done) fin_rho(&st[k], v);
    });
}

// Per-RHS dot over all nodes: WHICH 0 = BNRM2 at the start, 1 = RHO (unfused
// preconditioner paths), 2 = plain result into rr_true (final true residual).
template <int WHICH>
__global__ void __launch_bounds__(kThreads) mr_dot_kernel(const double *__restrict__ a, const double *__restrict__ b,
                                                          int n, CgState *st, MultiCtl *ctl, double *partials) {
  pdl_entry();
  if (WHICH == 1 && ctl->all_done) return;
  const int l = threadIdx.x & 15;
  const int nhw = (gridDim.x * blockDim.x) >> 4;
  double dot = 0.0;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; i < n; i += nhw) {
    const size_t o = size_t(i) * kRhsStride + l;
    dot += a[o] * b[o] + a[o + 16] * b[o + 16] + a[o + 32] * b[o + 32];
  }
  mr_reduce_finish(dot, partials, blockIdx.x, gridDim.x, &ctl->ticket[4 + WHICH], [&](int k, double v) {
    CgState *s = &st[k];
    if (WHICH == 0) {
      s->bnrm2 = v;
      if (k >= ctl->nrhs) {
        s->done = 1;  // padding lane
      } else if (v == 0.0) {
        s->zero_rhs = 1;
        s->done = 1;
      }
      if (s->maxit <= 0) s->done = 1;
    } else if (WHICH == 1) {
      if (!s->done) fin_rho(s, v);
    } else {
      s->rr_true = v;
    }
  });
}

// {p} = {z} or {z} + BETA {p} for the RHS still iterating.
__global__ void __launch_bounds__(kThreads) mr_update_p_kernel(const double *__restrict__ z, double *__restrict__ p,
                                                               int n, const CgState *st, const MultiCtl *ctl) {
  pdl_entry();
  if (ctl->all_done) return;
  const int l = threadIdx.x & 15;
  if (st[l].done) return;  // no barrier below: lanes of finished RHS simply leave
  const bool first = st[l].iter == 1;
  const double beta = st[l].beta;
  const int nhw = (gridDim.x * blockDim.x) >> 4;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; i < n; i += nhw) {
    const size_t o = size_t(i) * kRhsStride + l;
#pragma unroll
    for (int c = 0; c < 3; c++) p[o + 16 * c] = first ? z[o + 16 * c] : z[o + 16 * c] + beta * p[o + 16 * c];
  }
}

// {x} += ALPHA {p}; {r} -= ALPHA {q} with the per-RHS DNRM2 (not on refresh iterations).
__global__ void __launch_bounds__(kThreads) mr_update_xr_kernel(double *__restrict__ x, const double *__restrict__ p,
                                                                double *__restrict__ r, const double *__restrict__ q,
                                                                int n, CgState *st, MultiCtl *ctl, double *partials) {
  pdl_entry();
  if (ctl->all_done) return;
  const int l = threadIdx.x & 15;
  const bool act = !st[l].done;
  const double alpha = st[l].alpha;
  const bool refresh = (st[l].iter % kIterRecomputeR) == 0;
  const int nhw = (gridDim.x * blockDim.x) >> 4;
  double dot = 0.0;
  if (act) {
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; i < n; i += nhw) {
      const size_t o = size_t(i) * kRhsStride + l;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        x[o + 16 * c] = alpha * p[o + 16 * c] + x[o + 16 * c];
        if (!refresh) {
          const double ri = -alpha * q[o + 16 * c] + r[o + 16 * c];
          r[o + 16 * c] = ri;
          dot += ri * ri;
        }
      }
    }
  }
  mr_reduce_finish(dot, partials, blockIdx.x, gridDim.x, &ctl->ticket[2], [&](int k, double v) {
    CgState *s = &st[k];
    if (!s->done && (s->iter % kIterRecomputeR) != 0) fin_rr(s, v);
  });
}

__global__ void mr_init_kernel(CgState *st, MultiCtl *ctl, const CgParams *prm, int nrhs) {
  pdl_entry();
  const int k = threadIdx.x;
  if (blockIdx.x != 0) return;
  if (k < kMaxRhs) {
    CgState *s = &st[k];
    s->rho = s->rho1 = s->alpha = s->beta = s->pq = s->rr = 0.0;
    s->bnrm2 = s->resid = s->rr_true = 0.0;
    s->tol = prm->tol;
    s->maxit = prm->maxit;
    s->iter = 1;
    s->done = s->error = s->n_indef = s->recompute = s->converged = s->zero_rhs = 0;
    s->guard = 0;
    s->inner = 0;
    s->flexible = prm->flexible;
    s->use_gnn = prm->use_gnn;
    s->restart = s->fallback = 0;
    s->resid_mark = 1.0;
    s->gamma = 1.0f;
    s->reliable = s->ru_pending = s->ru_count = 0;
    s->ru_delta = 0.0;
    s->ru_mark = 1.0;
    s->lanczos = nullptr;  // no condition estimate or residual history for several load cases
    s->lanczos_cap = s->lanczos_n = 0;
    s->rhist = nullptr;
    s->rhist_cap = s->rhist_n = 0;
    for (int i = 0; i < 8; i++) s->ticket[i] = 0u;
  }
  if (k == 0) {
    ctl->all_done = 0;
    ctl->guard = 0;
    ctl->nrhs = nrhs;
    ctl->fault = 0;
    for (int i = 0; i < 8; i++) ctl->ticket[i] = 0u;
  }
}

// Start of a loop body: body counter of every RHS still iterating, fail-safe condition.
__global__ void mr_iter_begin_kernel(CgState *st, MultiCtl *ctl, cudaGraphConditionalHandle h, int use_cond) {
  pdl_entry();
  if (blockIdx.x != 0) return;
  const int k = threadIdx.x;
  if (k < kMaxRhs && !st[k].done) st[k].guard++;
  if (k == 0) {
    ctl->guard++;
    set_loop(h, use_cond, 0);
  }
}

// Loop decision after the control of every RHS: continue while one still iterates
// (and the body count stays within the fail-safe bound).
__global__ void mr_ctl_kernel(const CgState *st, MultiCtl *ctl, cudaGraphConditionalHandle h, int use_cond) {
  pdl_entry();
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int any = 0, maxit = 0;
  for (int k = 0; k < kMaxRhs; k++) {
    any |= !st[k].done;
    maxit = max(maxit, st[k].maxit);
  }
  if (ctl->guard > maxit + 1) any = 0;
  ctl->all_done = !any;
  set_loop(h, use_cond, any);
}

// ---- the learned two-level preconditioner for 16 RHS ---------------------------
// The single-RHS cycle (zs = SSOR(r); zc = zs + P Ac^-1 P^T (r - A zs); z = zc +
// SSOR(r - A zc)) in flexible CG, with the smoother's sweeps and A streamed once for
// all RHS, and Ac^-1 (FP32 copy) read once per iteration for all of them (a GEMM with
// 16 columns instead of 16 GEMVs).  Coarse vectors are RHS-minor: bc[(3a+c)*16 + l].
// A RHS whose correction was switched off (st.use_gnn = 0: the stagnation fallback of
// loop_ctl, or a non-positive RHO) gets zc = zs and w = 0, so the post-smoothing adds
// exactly nothing and z = zs = SSOR(r): SSOR-CG, as the single solve's fallback.

// Deterministic per-RHS reduction of two values (as mr_reduce_finish); partials hold
// 32 doubles per CTA.
template <class Fin>
__device__ __forceinline__ void mr_reduce_finish2(double va, double vb, double *partials, int part, int total,
                                                  unsigned int *ticket, Fin fin) {
  __shared__ double sha[kThreads / 16][kMaxRhs], shb[kThreads / 16][kMaxRhs];
  __shared__ int is_last;
  const int l = threadIdx.x & 15, hw = threadIdx.x >> 4;
  sha[hw][l] = va;
  shb[hw][l] = vb;
  __syncthreads();
  if (threadIdx.x < kMaxRhs) {
    double a = 0.0, b = 0.0;
    for (int k = 0; k < kThreads / 16; k++) {
      a += sha[k][threadIdx.x];
      b += shb[k][threadIdx.x];
    }
    partials[size_t(part) * 2 * kMaxRhs + threadIdx.x] = a;
    partials[size_t(part) * 2 * kMaxRhs + kMaxRhs + threadIdx.x] = b;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int t = atomicAdd(ticket, 1u);
    is_last = (t == unsigned(total) - 1u);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double a = 0.0, b = 0.0;
  for (int i = hw; i < total; i += kThreads / 16) {
    a += __ldcg(&partials[size_t(i) * 2 * kMaxRhs + l]);
    b += __ldcg(&partials[size_t(i) * 2 * kMaxRhs + kMaxRhs + l]);
  }
  __syncthreads();
  sha[hw][l] = a;
  shb[hw][l] = b;
  __syncthreads();
  if (threadIdx.x < kMaxRhs) {
    double ta = 0.0, tb = 0.0;
    for (int k = 0; k < kThreads / 16; k++) {
      ta += sha[k][threadIdx.x];
      tb += shb[k][threadIdx.x];
    }
    fin(int(threadIdx.x), ta, tb);
  }
  __syncthreads();
  if (threadIdx.x == 0) *ticket = 0u;
}

// z = z + (zs + P y): the two-grid cycle's post-smoothing plus its coarse-corrected
// part, the prolongation done here so that zc never goes through memory (P y is added
// only for a RHS whose correction is on, in the order of
// mr_coarse_resid_kernel's (A P) y); stored back into z.  Then RHO = {z}{r} and DELTA
// = {z}{r_old} per RHS in the same pass and fin_rho_flex.
__global__ void __launch_bounds__(kThreads) mr_fcg_rho_kernel(double *__restrict__ z,
                                                              const double *__restrict__ zs, CoarseApply c,
                                                              const double *__restrict__ y,
                                                              const double *__restrict__ r,
                                                              const double *__restrict__ r_old, int n, CgState *st,
                                                              MultiCtl *ctl, double *partials) {
  pdl_entry();
  if (ctl->all_done) return;
  const int l = threadIdx.x & 15;
  const int nhw = (gridDim.x * blockDim.x) >> 4;
  const bool on = st[l].use_gnn;
  double a = 0.0, b = 0.0;
  if (!st[l].done) {
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; i < n; i += nhw) {
      const size_t o = size_t(i) * kRhsStride + l;
      // the streamed operands first, so that their loads overlap the P y gathers
      double zv[3], zsv[3], rv[3], rov[3];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        zv[d] = z[o + 16 * d];
        zsv[d] = zs[o + 16 * d];
        rv[d] = r[o + 16 * d];
        rov[d] = r_old[o + 16 * d];
      }
      double py[3] = {0.0, 0.0, 0.0};
      if (on) {
        for (int k = c.pptr[i]; k < c.pptr[i + 1]; k++) {
          const float *pb = c.p + 9 * size_t(k);
          const size_t bo = size_t(3 * c.pagg[k]) * kMaxRhs + l;
          const double y0 = y[bo], y1 = y[bo + 16], y2 = y[bo + 32];
#pragma unroll
          for (int d = 0; d < 3; d++)
            py[d] += double(pb[3 * d]) * y0 + double(pb[3 * d + 1]) * y1 + double(pb[3 * d + 2]) * y2;
        }
      }
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const double zi = zv[d] + (zsv[d] + py[d]);
        z[o + 16 * d] = zi;
        a += zi * rv[d];
        b += zi * rov[d];
      }
    }
  }
  mr_reduce_finish2(a, b, partials, blockIdx.x, gridDim.x, &ctl->ticket[0], [&](int k, double rho, double delta) {
    if (!st[k].done) fin_rho_flex(&st[k], rho, delta);
  });
}

// Flexible CG update per RHS: r_old = r, x += ALPHA p, r -= ALPHA q with the DNRM2
// (every 50th iteration r is recomputed from b - A x instead).
__global__ void __launch_bounds__(kThreads) mr_update_xr_flex_kernel(double *__restrict__ x,
                                                                     const double *__restrict__ p,
                                                                     double *__restrict__ r,
                                                                     double *__restrict__ r_old,
                                                                     const double *__restrict__ q, int n, CgState *st,
                                                                     MultiCtl *ctl, double *partials) {
  pdl_entry();
  if (ctl->all_done) return;
  const int l = threadIdx.x & 15;
  const bool act = !st[l].done;
  const double alpha = st[l].alpha;
  const bool refresh = (st[l].iter % kIterRecomputeR) == 0;
  const int nhw = (gridDim.x * blockDim.x) >> 4;
  double dot = 0.0;
  if (act) {
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; i < n; i += nhw) {
      const size_t o = size_t(i) * kRhsStride + l;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        x[o + 16 * c] = alpha * p[o + 16 * c] + x[o + 16 * c];
        const double ri = r[o + 16 * c];
        r_old[o + 16 * c] = ri;
        if (!refresh) {
          const double rn = -alpha * q[o + 16 * c] + ri;
          r[o + 16 * c] = rn;
          dot += rn * rn;
        }
      }
    }
  }
  mr_reduce_finish(dot, partials, blockIdx.x, gridDim.x, &ctl->ticket[2], [&](int k, double v) {
    CgState *s = &st[k];
    if (!s->done && (s->iter % kIterRecomputeR) != 0) fin_rr(s, v);
  });
}

// bc = P^T w for 16 RHS: a CTA per aggregate, 16 groups of 16 lanes (lane = RHS) over
// the aggregate's restriction entries, group partial sums added in group order.
__global__ void __launch_bounds__(kThreads) mr_coarse_restrict_kernel(CoarseApply c, const double *__restrict__ w,
                                                                      double *__restrict__ bc, const MultiCtl *ctl) {
  pdl_entry();
  if (ctl->all_done) return;
  __shared__ double sh[kThreads / 16][3][kMaxRhs];
  const int l = threadIdx.x & 15, g = threadIdx.x >> 4;
  for (int a = blockIdx.x; a < c.nagg; a += gridDim.x) {
    double acc[3] = {0.0, 0.0, 0.0};
    for (int e = c.rptr[a] + g; e < c.rptr[a + 1]; e += kThreads / 16) {
      const size_t o = size_t(c.rnode[e]) * kRhsStride + l;
      const float *pb = c.p + 9 * size_t(c.rpos[e]);
      const double w0 = w[o], w1 = w[o + 16], w2 = w[o + 32];
#pragma unroll
      for (int k = 0; k < 3; k++)  // (P^T w)_k = sum_d P(d, k) w_d
        acc[k] += double(pb[k]) * w0 + double(pb[3 + k]) * w1 + double(pb[6 + k]) * w2;
    }
#pragma unroll
    for (int k = 0; k < 3; k++) sh[g][k][l] = acc[k];
    __syncthreads();
    if (threadIdx.x < 3 * kMaxRhs) {
      const int k = threadIdx.x >> 4, ll = threadIdx.x & 15;
      double s = 0.0;
      for (int gg = 0; gg < kThreads / 16; gg++) s += sh[gg][k][ll];
      bc[size_t(3 * a + k) * kMaxRhs + ll] = s;
    }
    __syncthreads();
  }
}

// y = Ac^-1 bc for 16 RHS (FP32 copy of Ac^-1, FP64 sums).  A CTA takes 16 rows:
// each step stages a 16 x 128 tile of Ac^-1 and the matching 128 x 16 rows of bc in
// shared memory, and every thread accumulates a 4-row x 4-RHS tile over the columns
// k = s (mod 16) of its slice s; the 16 slices are then added in a fixed order (pairs
// in the warp, then the 8 warps in order), so y does not depend on the grid.  The next
// step's tiles are loaded into registers while the current one is multiplied.  Ac^-1
// is read once per launch and bc once per CTA.
constexpr int kMrGemmRows = 16;
constexpr int kMrGemmChunk = 128;
constexpr int kMrGemmSlices = kThreads / kMrGemmRows;
constexpr int kMrGemmAPer = kMrGemmRows * kMrGemmChunk / kThreads;        // floats of Ac^-1 per thread and step
constexpr int kMrGemmBPer = kMrGemmChunk * (kMaxRhs / 2) / kThreads;      // double2 of bc per thread and step
static_assert(kMrGemmSlices == 16 && kMaxRhs == 16, "4 x 4 thread tiles of a 16 x 16 output block");
static_assert(kMrGemmAPer * kThreads == kMrGemmRows * kMrGemmChunk && kMrGemmBPer * kThreads == kMrGemmChunk * 8,
              "whole tiles per thread");
__global__ void __launch_bounds__(kThreads, 3) mr_coarse_gemm_kernel(int nc, const float *__restrict__ ainv,
                                                                     const double *__restrict__ bc,
                                                                     double *__restrict__ y, const MultiCtl *ctl) {
  pdl_entry();
  if (ctl->all_done) return;
  // row stride 129: the 8 (row, slice) pairs a load of a warp touches sit in 8 banks
  __shared__ float as[kMrGemmRows][kMrGemmChunk + 1];
  // row stride 18 doubles (144 bytes): the two slices of a warp read adjacent rows in
  // disjoint banks
  __shared__ __align__(16) double bs[kMrGemmChunk][kMaxRhs + 2];
  __shared__ double red[kWarpsPerCta][kMrGemmRows][kMaxRhs];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int s = t >> 4, rg = (t >> 2) & 3, q = t & 3;
  float ra[kMrGemmAPer];
  double2 rb[kMrGemmBPer];
  auto fetch = [&](int r0, int k0) {
    const int kn = min(kMrGemmChunk, nc - k0);
#pragma unroll
    for (int m = 0; m < kMrGemmAPer; m++) {
      const int e = t + kThreads * m, r = e / kMrGemmChunk, k = e % kMrGemmChunk;
      ra[m] = (r0 + r < nc && k < kn) ? __ldcs(ainv + size_t(r0 + r) * nc + k0 + k) : 0.0f;
    }
#pragma unroll
    for (int m = 0; m < kMrGemmBPer; m++) {
      const int e = t + kThreads * m, k = e / (kMaxRhs / 2), c2 = e % (kMaxRhs / 2);
      rb[m] = k < kn ? reinterpret_cast<const double2 *>(bc + size_t(k0 + k) * kMaxRhs)[c2] : make_double2(0.0, 0.0);
    }
  };
  for (int r0 = blockIdx.x * kMrGemmRows; r0 < nc; r0 += gridDim.x * kMrGemmRows) {
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int c = 0; c < 4; c++) acc[i][c] = 0.0;
    fetch(r0, 0);
    for (int k0 = 0; k0 < nc; k0 += kMrGemmChunk) {
      __syncthreads();  // the previous step's reads of as and bs are done
#pragma unroll
      for (int m = 0; m < kMrGemmAPer; m++) {
        const int e = t + kThreads * m;
        as[e / kMrGemmChunk][e % kMrGemmChunk] = ra[m];
      }
#pragma unroll
      for (int m = 0; m < kMrGemmBPer; m++) {
        const int e = t + kThreads * m;
        *reinterpret_cast<double2 *>(&bs[e / (kMaxRhs / 2)][2 * (e % (kMaxRhs / 2))]) = rb[m];
      }
      __syncthreads();
      if (k0 + kMrGemmChunk < nc) fetch(r0, k0 + kMrGemmChunk);
#pragma unroll 2
      for (int j = 0; j < kMrGemmChunk / kMrGemmSlices; j++) {
        const int k = s + kMrGemmSlices * j;
        const double2 b01 = *reinterpret_cast<const double2 *>(&bs[k][4 * q]);
        const double2 b23 = *reinterpret_cast<const double2 *>(&bs[k][4 * q + 2]);
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const double a = double(as[4 * rg + i][k]);
          acc[i][0] += a * b01.x;
          acc[i][1] += a * b01.y;
          acc[i][2] += a * b23.x;
          acc[i][3] += a * b23.y;
        }
      }
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int c = 0; c < 4; c++) {
        const double v = acc[i][c] + __shfl_xor_sync(0xffffffffu, acc[i][c], 16);
        if (lane < 16) red[warp][4 * rg + i][4 * q + c] = v;
      }
    __syncthreads();
    {
      const int row = t >> 4, l = t & 15;
      double v = 0.0;
#pragma unroll
      for (int w = 0; w < kWarpsPerCta; w++) v += red[w][row][l];
      if (r0 + row < nc) y[size_t(r0 + row) * kMaxRhs + l] = v;
    }
  }
}

// w -= (A P) y per RHS (a half-warp per node, lane = RHS), the residual after the
// coarse correction; a RHS whose correction is off gets w = 0 (its cycle is the plain
// smoother).  The correction zs + P y itself is formed in mr_fcg_rho_kernel.
__global__ void __launch_bounds__(kThreads) mr_coarse_resid_kernel(CoarseApply c, const double *__restrict__ y,
                                                                   double *__restrict__ w, const CgState *st,
                                                                   const MultiCtl *ctl) {
  pdl_entry();
  if (ctl->all_done) return;
  const int l = threadIdx.x & 15;
  const bool on = !st[l].done && st[l].use_gnn;
  const int nhw = (gridDim.x * blockDim.x) >> 4;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 4; i < c.n; i += nhw) {
    const size_t o = size_t(i) * kRhsStride + l;
    if (!on) {
#pragma unroll
      for (int d = 0; d < 3; d++) w[o + 16 * d] = 0.0;
      continue;
    }
    double wv[3], q[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < 3; d++) wv[d] = w[o + 16 * d];  // overlaps the (A P) y gathers
    {
      for (int k = c.qptr[i]; k < c.qptr[i + 1]; k++) {
        const float *qb = c.q + 9 * size_t(k);
        const size_t b = size_t(3 * c.qagg[k]) * kMaxRhs + l;
        const double y0 = y[b], y1 = y[b + 16], y2 = y[b + 32];
#pragma unroll
        for (int d = 0; d < 3; d++)
          q[d] += double(qb[3 * d]) * y0 + double(qb[3 * d + 1]) * y1 + double(qb[3 * d + 2]) * y2;
      }
    }
#pragma unroll
    for (int d = 0; d < 3; d++) w[o + 16 * d] = wv[d] - q[d];
  }
}

// Column-major host layout (n3 x nrhs) <-> node-major RHS-minor layout.
__global__ void mr_pack_kernel(const double *__restrict__ src, double *__restrict__ dst, int n, int nrhs) {
  pdl_entry();
  const size_t total = size_t(n) * kRhsStride;
  for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    const int l = int(t % kMaxRhs);
    const int c = int((t / kMaxRhs) % 3);
    const size_t i = t / kRhsStride;
    dst[t] = l < nrhs ? src[size_t(l) * 3 * n + 3 * i + c] : 0.0;
  }
}
__global__ void mr_unpack_kernel(const double *__restrict__ src, double *__restrict__ dst, int n, int nrhs) {
  pdl_entry();
  const size_t total = size_t(n) * 3 * nrhs;
  for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x) {
    const int l = int(t / (3 * size_t(n)));
    const size_t j = t % (3 * size_t(n));
    dst[t] = src[(j / 3) * kRhsStride + (j % 3) * kMaxRhs + l];
  }
}
// Zero-RHS lanes leave x = 0 (hecmw_solver.f90:32-37).
__global__ void mr_zero_x_kernel(double *__restrict__ x, int n, const CgState *st) {
  pdl_entry();
  const size_t total = size_t(n) * kRhsStride;
  for (size_t t = blockIdx.x * size_t(blockDim.x) + threadIdx.x; t < total; t += size_t(gridDim.x) * blockDim.x)
    if (st[t % kMaxRhs].zero_rhs) x[t] = 0.0;
}

}  // namespace h33
