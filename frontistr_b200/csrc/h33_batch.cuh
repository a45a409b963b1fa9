// h33_batch.cuh -- many independent systems in one persistent launch.
//
// The systems are the diagonal blocks of one hecmwST matrix (system s owns the nodes
// node0[s] .. node0[s] + n[s] - 1).  Every system runs the drop-in's CG
// (hecmw_solver_CG.f90:19-289: RHO / ALPHA / BETA, breakdown codes, 50-iteration
// true-residual refresh, recompute on convergence, MAXIT) with the SSOR sweeps in its
// own RCM + multicolour order (hecmw_precond_SSOR_33.F90), or DIAG.
//
// Work is taken from two queues by persistent CTAs launched in thread-block clusters:
//  * big systems (first queue): a whole cluster (team of C CTAs on C SMs) solves one
//    system; the phases of an iteration (colours of the sweeps, SpMV, vector updates)
//    are separated by hardware cluster barriers, dot products are reduced through
//    distributed shared memory, and every CTA keeps an identical replica of the CG
//    scalars in its shared memory (each computes the same decisions from the same
//    sums in the same order, so no scalar round-trips through global memory and all
//    CTAs of a team take the same branches);
//  * small systems (second queue): each CTA solves one system alone (CTA barriers).
// Queues are ordered by decreasing estimated work (longest-first scheduling), so
// the big systems start first and the small ones fill the gaps.  All vector reads
// of data written during the launch go through L2 (__ldcg), never the read-only path.
// No CTA ever waits on another outside its own cluster, and every loop is bounded by
// MAXIT (plus the fail-safe body counter of loop_ctl).
#pragma once

#include <cooperative_groups.h>

#include "h33_kernels.cuh"

namespace h33 {

namespace cgrp = cooperative_groups;

struct BatchSys {
  int n;       // nodes
  int node0;   // first node (vector offset / 3)
  int a0, a1;  // SpMV slices
  int g0, g1;  // colour groups in the sweep tables (lo/up share them)
  int skip;    // 1: not solved (zero diagonal, reported by the host)
  int pad;
};

// Per-system result.
struct BatchOut {
  int iter, error, converged, zero_rhs;
  double resid, true_resid, bnrm2;
  int guard, team;
};

struct BatchArgs {
  SellView<double> A, lo, up;
  const int *lo_gs, *up_gs;  // group g -> slices [gs[g], gs[g+1])
  const int *perm;           // position -> node (global)
  const double *alu;         // SoA, stride npos
  int npos;
  int kind;                  // 1 SSOR, 3 DIAG
  int iterpremax;            // 0 or 1
  const BatchSys *sys;
  const int *big, *small;    // queue entries (system ids)
  int nbig, nsmall;
  int *queue;                // [0] big, [1] small
  const double *b;
  double *x, *r, *z, *p, *q;
  BatchOut *out;
  double tol;
  int maxit;
};

// A team: C CTAs of one cluster (cluster != 0) or one CTA.
struct Team {
  int rank, size;
  bool cluster;
  int warp, nwarps;   // warp index within the team, warps in the team
  int tid, nthreads;  // thread index within the team, threads in the team
  int slot;           // rotating reduction slot
};

__device__ __forceinline__ void team_sync(const Team &t) {
  if (t.cluster) cgrp::this_cluster().sync();
  else __syncthreads();
}

// Deterministic team sum (the same value in every thread of every CTA of the team):
// warp sums, the CTA's sum in warp order, then the CTAs' sums in rank order read
// from each CTA's shared memory.
__device__ __forceinline__ double team_sum(Team &t, double v, double *s_warp, double *s_red, double *s_out) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) s_warp[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double c = 0.0;
    for (int k = 0; k < kWarpsPerCta; k++) c += s_warp[k];
    s_red[t.slot] = c;
  }
  if (t.cluster) {
    cgrp::cluster_group cl = cgrp::this_cluster();
    cl.sync();
    if (threadIdx.x == 0) {
      double tot = 0.0;
      for (int k = 0; k < t.size; k++) tot += *cl.map_shared_rank(&s_red[t.slot], k);
      *s_out = tot;
    }
  } else {
    __syncthreads();
    if (threadIdx.x == 0) *s_out = s_red[t.slot];
  }
  __syncthreads();
  const double tot = *s_out;
  t.slot = (t.slot + 1) & 3;  // a slot is rewritten only after later cluster barriers
  __syncthreads();            // s_out may be rewritten by the next sum
  return tot;
}

// r = b - A x over the system's slices (one lane per row); returns this thread's
// partial of |r|^2 (WITH_RR) or of |b|^2 (WITH_BB).
template <bool WITH_RR, bool WITH_BB>
__device__ __forceinline__ double team_resid(const BatchArgs &a, const BatchSys &sy, const Team &t, const double *x,
                                             double *r) {
  const int lane = threadIdx.x & 31;
  double acc = 0.0;
  for (int s = sy.a0 + t.warp; s < sy.a1; s += t.nwarps) {
    const bool active = lane < a.A.nrows[s];
    const int row = a.A.row0[s] + lane;
    const int len = active ? a.A.rowlen[s * 32 + lane] : 0;
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    row_gemv<double, double, 1, false, true>(a.A, s, lane, len, x, y0, y1, y2);
    if (active) {
      const double b0 = a.b[3 * row], b1 = a.b[3 * row + 1], b2 = a.b[3 * row + 2];
      y0 = b0 - y0;
      y1 = b1 - y1;
      y2 = b2 - y2;
      r[3 * row] = y0;
      r[3 * row + 1] = y1;
      r[3 * row + 2] = y2;
      if (WITH_RR) acc += y0 * y0 + y1 * y1 + y2 * y2;
      if (WITH_BB) acc += b0 * b0 + b1 * b1 + b2 * b2;
    }
  }
  return acc;
}

// q = A p with this thread's partial of {p}{q}.
__device__ __forceinline__ double team_spmv_pq(const BatchArgs &a, const BatchSys &sy, const Team &t) {
  const int lane = threadIdx.x & 31;
  double acc = 0.0;
  for (int s = sy.a0 + t.warp; s < sy.a1; s += t.nwarps) {
    const bool active = lane < a.A.nrows[s];
    const int row = a.A.row0[s] + lane;
    const int len = active ? a.A.rowlen[s * 32 + lane] : 0;
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    row_gemv<double, double, 1, false, true>(a.A, s, lane, len, a.p, y0, y1, y2);
    if (active) {
      a.q[3 * row] = y0;
      a.q[3 * row + 1] = y1;
      a.q[3 * row + 2] = y2;
      acc += __ldcg(&a.p[3 * row]) * y0 + __ldcg(&a.p[3 * row + 1]) * y1 + __ldcg(&a.p[3 * row + 2]) * y2;
    }
  }
  return acc;
}

// One colour of the forward sweep (rows over K lanes); with FUSE the finished rows'
// {r}{z} (the DIAG case, which has no backward sweep).
template <int K, bool FUSE>
__device__ __forceinline__ double team_fwd(const BatchArgs &a, const Team &t, int sb, int se) {
  const int lane = threadIdx.x & 31, roff = lane / K;
  double acc = 0.0;
  for (int s = sb + t.warp; s < se; s += t.nwarps) {
    const bool active = roff < a.lo.nrows[s];
    const int row = a.lo.row0[s] + roff;
    const int len = active ? a.lo.rowlen[s * 32 + roff] : 0;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    row_gemv<double, double, K, false, true>(a.lo, s, lane, len, a.z, a0, a1, a2);
    if (active && (lane & (K - 1)) == 0) {
      const int node = a.perm[row];
      const double r0 = __ldcg(&a.r[3 * node]), r1 = __ldcg(&a.r[3 * node + 1]), r2 = __ldcg(&a.r[3 * node + 2]);
      double x1 = r0 - a0, x2 = r1 - a1, x3 = r2 - a2;
      lu_solve(a.alu, a.npos, row, x1, x2, x3);
      a.z[3 * node] = x1;
      a.z[3 * node + 1] = x2;
      a.z[3 * node + 2] = x3;
      if (FUSE) acc += r0 * x1 + r1 * x2 + r2 * x3;
    }
  }
  return acc;
}

// One colour of the backward sweep with the finished rows' {r}{z}.
template <int K>
__device__ __forceinline__ double team_bwd(const BatchArgs &a, const Team &t, int sb, int se) {
  const int lane = threadIdx.x & 31, roff = lane / K;
  double acc = 0.0;
  for (int s = sb + t.warp; s < se; s += t.nwarps) {
    const bool active = roff < a.up.nrows[s];
    const int row = a.up.row0[s] + roff;
    const int len = active ? a.up.rowlen[s * 32 + roff] : 0;
    double x1 = 0.0, x2 = 0.0, x3 = 0.0;
    row_gemv<double, double, K, true, true>(a.up, s, lane, len, a.z, x1, x2, x3);
    if (active && (lane & (K - 1)) == 0) {
      const int node = a.perm[row];
      lu_solve(a.alu, a.npos, row, x1, x2, x3);
      const double z0 = __ldcg(&a.z[3 * node]) - x1, z1 = __ldcg(&a.z[3 * node + 1]) - x2,
                   z2 = __ldcg(&a.z[3 * node + 2]) - x3;
      a.z[3 * node] = z0;
      a.z[3 * node + 1] = z1;
      a.z[3 * node + 2] = z2;
      acc += __ldcg(&a.r[3 * node]) * z0 + __ldcg(&a.r[3 * node + 1]) * z1 + __ldcg(&a.r[3 * node + 2]) * z2;
    }
  }
  return acc;
}

// The CG of one system by one team.
template <int K>
__device__ void team_solve(const BatchArgs &a, int id, Team &t, CgState &st, double *s_warp, double *s_red,
                           double *s_out) {
  const BatchSys sy = a.sys[id];
  const int lo3 = 3 * sy.node0, n3 = 3 * sy.n;
  if (threadIdx.x == 0) {
    st.rho = st.rho1 = st.alpha = st.beta = st.pq = st.rr = 0.0;
    st.bnrm2 = st.resid = st.rr_true = 0.0;
    st.tol = a.tol;
    st.maxit = a.maxit;
    st.iter = 1;
    st.done = st.error = st.n_indef = st.recompute = st.converged = st.zero_rhs = 0;
    st.guard = 0;
    st.inner = st.flexible = st.use_gnn = st.restart = st.fallback = 0;
    st.reliable = 0;
    st.lanczos = nullptr;  // no condition estimate or residual history in a batch
    st.lanczos_cap = st.lanczos_n = 0;
    st.rhist = nullptr;
    st.rhist_cap = st.rhist_n = 0;
  }
  __syncthreads();
  // prologue: r = b - A x and BNRM2 in one pass
  const double bb = team_sum(t, team_resid<false, true>(a, sy, t, a.x, a.r), s_warp, s_red, s_out);
  if (threadIdx.x == 0) {
    st.bnrm2 = bb;
    if (bb == 0.0) {
      st.zero_rhs = 1;
      st.done = 1;
    }
    if (st.maxit <= 0) st.done = 1;
  }
  __syncthreads();
  if (st.zero_rhs) {
    for (int i = t.tid; i < n3; i += t.nthreads) a.x[lo3 + i] = 0.0;  // hecmw_solver.f90:32-37
  }
  team_sync(t);  // r and x of the prologue visible to the team
  while (!st.done) {
    if (threadIdx.x == 0) st.guard++;
    // z = M^-1 r with RHO fused into the last pass
    double rho_part = 0.0;
    if (a.iterpremax <= 0) {
      for (int i = t.tid; i < n3; i += t.nthreads) {
        const double ri = __ldcg(&a.r[lo3 + i]);
        a.z[lo3 + i] = ri;
        rho_part += ri * ri;
      }
    } else if (a.kind == 3) {
      for (int g = sy.g0; g < sy.g1; g++) rho_part += team_fwd<K, true>(a, t, a.lo_gs[g], a.lo_gs[g + 1]);
    } else {
      for (int g = sy.g0; g < sy.g1; g++) {
        team_fwd<K, false>(a, t, a.lo_gs[g], a.lo_gs[g + 1]);
        team_sync(t);
      }
      for (int g = sy.g1 - 1; g >= sy.g0; g--) {
        rho_part += team_bwd<K>(a, t, a.up_gs[g], a.up_gs[g + 1]);
        if (g > sy.g0) team_sync(t);
      }
    }
    const double rho = team_sum(t, rho_part, s_warp, s_red, s_out);  // includes a team barrier
    if (threadIdx.x == 0) fin_rho(&st, rho);
    __syncthreads();
    if (st.done) break;
    // {p} = {z} + BETA {p}
    {
      const bool first = st.iter == 1;
      const double beta = st.beta;
      for (int i = t.tid; i < n3; i += t.nthreads) {
        const double zi = __ldcg(&a.z[lo3 + i]);
        a.p[lo3 + i] = first ? zi : zi + beta * __ldcg(&a.p[lo3 + i]);
      }
    }
    team_sync(t);
    const double pq = team_sum(t, team_spmv_pq(a, sy, t), s_warp, s_red, s_out);
    if (threadIdx.x == 0) fin_pq(&st, pq);
    __syncthreads();
    if (st.done) break;
    // {x} += ALPHA {p}; {r} -= ALPHA {q} (unless the true residual is due)
    const bool refresh = (st.iter % kIterRecomputeR) == 0;
    {
      const double alpha = st.alpha;
      double rr_part = 0.0;
      for (int i = t.tid; i < n3; i += t.nthreads) {
        a.x[lo3 + i] = alpha * __ldcg(&a.p[lo3 + i]) + __ldcg(&a.x[lo3 + i]);
        if (!refresh) {
          const double ri = -alpha * __ldcg(&a.q[lo3 + i]) + __ldcg(&a.r[lo3 + i]);
          a.r[lo3 + i] = ri;
          rr_part += ri * ri;
        }
      }
      if (!refresh) {
        const double rr = team_sum(t, rr_part, s_warp, s_red, s_out);
        if (threadIdx.x == 0) fin_rr(&st, rr);
        __syncthreads();
      }
    }
    if (refresh || st.recompute) {
      team_sync(t);  // x complete before r = b - A x
      const double rr = team_sum(t, team_resid<true, false>(a, sy, t, a.x, a.r), s_warp, s_red, s_out);
      if (threadIdx.x == 0) {
        st.rr = rr;
        st.resid = sqrt(rr / st.bnrm2);
        if (st.resid <= st.tol) {
          st.done = 1;
          st.converged = 1;
        }
      }
    }
    if (threadIdx.x == 0) loop_ctl(&st, 0, 0);
    __syncthreads();
    team_sync(t);  // r, x of this iteration visible before the next sweeps
  }
  // final true residual ||b - A x|| / ||b|| (hecmw_rel_resid_L2_33), q as scratch
  team_sync(t);
  const double rt = team_sum(t, team_resid<true, false>(a, sy, t, a.x, a.q), s_warp, s_red, s_out);
  if (t.rank == 0 && threadIdx.x == 0) {
    BatchOut o;
    o.iter = st.zero_rhs ? 0 : st.iter;
    o.error = st.zero_rhs ? HECMW33_ERR_ZERO_RHS : st.error;
    o.zero_rhs = st.zero_rhs;
    o.resid = st.zero_rhs ? 0.0 : st.resid;
    o.bnrm2 = st.bnrm2;
    o.true_resid = st.bnrm2 > 0.0 ? sqrt(rt / st.bnrm2) : 0.0;
    o.converged = st.zero_rhs || o.true_resid < st.tol;
    o.guard = st.guard;
    o.team = t.size;
    a.out[id] = o;
  }
  team_sync(t);
}

// The arguments live in device memory (written before each launch), so one captured
// graph serves every solve of the same launch shape.
template <int K>
__global__ void __launch_bounds__(kThreads, 4) batch_cg_kernel(const BatchArgs *__restrict__ args) {
  __shared__ BatchArgs a;
  __shared__ CgState st;
  __shared__ double s_warp[kWarpsPerCta];
  __shared__ double s_red[4];
  __shared__ double s_out;
  __shared__ int s_item;
  if (threadIdx.x == 0) a = *args;
  __syncthreads();
  cgrp::cluster_group cl = cgrp::this_cluster();
  Team t;
  // phase 1: big systems, one cluster per system
  t.rank = int(cl.block_rank());
  t.size = int(cl.num_blocks());
  t.cluster = t.size > 1;
  t.warp = t.rank * kWarpsPerCta + (threadIdx.x >> 5);
  t.nwarps = t.size * kWarpsPerCta;
  t.tid = t.rank * kThreads + threadIdx.x;
  t.nthreads = t.size * kThreads;
  t.slot = 0;
  for (;;) {
    if (t.rank == 0 && threadIdx.x == 0) s_item = atomicAdd(&a.queue[0], 1);
    cl.sync();
    const int item = *cl.map_shared_rank(&s_item, 0);
    cl.sync();  // every CTA has read the item before rank 0 draws the next one
    if (item >= a.nbig) break;
    team_solve<K>(a, a.big[item], t, st, s_warp, s_red, &s_out);
  }
  // phase 2: small systems, one CTA per system
  t.rank = 0;
  t.size = 1;
  t.cluster = false;
  t.warp = threadIdx.x >> 5;
  t.nwarps = kWarpsPerCta;
  t.tid = threadIdx.x;
  t.nthreads = kThreads;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(&a.queue[1], 1);
    __syncthreads();
    const int item = s_item;
    __syncthreads();
    if (item >= a.nsmall) break;
    team_solve<K>(a, a.small[item], t, st, s_warp, s_red, &s_out);
  }
  // every CTA of a cluster stays until the others are done with its shared memory
  cl.sync();
}

}  // namespace h33
