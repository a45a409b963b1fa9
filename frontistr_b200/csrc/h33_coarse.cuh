// h33_coarse.cuh -- the coarse space of the learned two-level preconditioner.
//
// No counterpart in the reference solver.  After SSOR, the flexible CG adds a coarse
// correction:  z = SSOR(r) + P Ac^-1 P^T r,  Ac = P^T A P,  on aggregates of the node
// graph (h33_setup.cpp aggregate_nodes).  The prolongator is a smoothed aggregation
//   P = (I - Omega D^-1 A) P0,
// P0 the piecewise-constant translations of each aggregate (zero on DOFs whose row of
// A has no off-diagonal entry: the constrained ones), D the diagonal blocks, and
// Omega = diag(omega) per DOF from the network (h33_gnn.cuh): omega = sigmoid(out).
// Row i of P has one 3x3 block per aggregate of i's closed neighbourhood:
//   P(i,b) = [b == agg(i)] M_i - diag(omega_i) T0(i,b),
//   T0(i,b) = D_i^-1 sum_{j in N[i], agg(j) = b} A_ij M_j      (M = DOF mask)
// The coarse matrix is dense (3 x aggregates square, a few thousand) and inverted
// once per matrix; an application is then one gather (P^T r), one dense GEMV and one
// scatter (P y).  Every sum runs in a fixed order (warp shuffles in lane order, no
// atomics), so a coarse operator and its application are deterministic.
#pragma once

#include "h33_common.cuh"

namespace h33 {

struct CoarseView {
  int n, nagg, nc;                 // fine nodes, aggregates, coarse DOFs (3 nagg)
  const int *agg;                  // n
  const int *pptr, *pagg;          // P pattern (n + 1, nnzp)
  const int *rptr, *rnode, *rpos;  // restriction gather (nagg + 1, nnzp, nnzp)
  const int *qptr, *qagg;          // A P pattern (n + 1, nnzq)
  const int *cptr, *cagg;          // Ac pattern (nagg + 1, nnzc)
  const int *uptr, *ucol, *usrc;   // unified rows of A (L, D, U; raw block ids)
  float *mask;                     // 3n: 1 where the DOF's row couples, else 0
  double *t0, *p;                  // 9 nnzp each
  double *q;                       // 9 nnzq: A P
  double *ac;                      // nc x nc, row-major: Ac, then Ac^-1
};

// FP32 copies of P, A P and Ac^-1 for the application inside a solve (the training
// and the operator build keep FP64): the correction only shapes the preconditioner,
// and the copies halve the bytes an application streams.
struct CoarseApply {
  int n, nagg, nc;
  const int *pptr, *pagg, *qptr, *qagg, *rptr, *rnode, *rpos;
  const float *p, *q, *ainv;
};

__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// mask[3i+d] = 1 when row 3i+d of A has a nonzero off-diagonal entry (warp per node,
// lane k over block k of the row).
__global__ void __launch_bounds__(kThreads) coarse_mask_kernel(CoarseView c, const double *__restrict__ raw) {
  pdl_entry();
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < c.n; i += nwarps) {
    bool cpl[3] = {false, false, false};
    for (int k = c.uptr[i] + lane; k < c.uptr[i + 1]; k += 32) {
      const double *a = raw + 9 * size_t(c.usrc[k]);
      const bool diag = c.ucol[k] == i;
      for (int d = 0; d < 3; d++)
        for (int e = 0; e < 3; e++)
          if (!(diag && d == e) && a[3 * d + e] != 0.0) cpl[d] = true;
    }
    for (int d = 0; d < 3; d++) {
      const bool any = __any_sync(0xffffffffu, cpl[d]);
      if (lane == 0) c.mask[3 * i + d] = any ? 1.0f : 0.0f;
    }
  }
}

// The network's static input per node: [1, (aggregates of the closed neighbourhood
// - 1) / 7, share of the neighbours outside the node's aggregate, DOF mask (3)].
__global__ void coarse_features_kernel(CoarseView c, float *__restrict__ x) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c.n; i += gridDim.x * blockDim.x) {
    int nb = 0, out = 0;
    for (int k = c.uptr[i]; k < c.uptr[i + 1]; k++) {
      const int j = c.ucol[k];
      if (j == i) continue;
      nb++;
      out += c.agg[j] != c.agg[i];
    }
    float *xi = x + 6 * size_t(i);
    xi[0] = 1.0f;
    xi[1] = float(c.pptr[i + 1] - c.pptr[i] - 1) / 7.0f;
    xi[2] = nb ? float(out) / float(nb) : 0.0f;
    for (int d = 0; d < 3; d++) xi[3 + d] = c.mask[3 * i + d];
  }
}

// sum of a[k] b[k], k < n (one CTA; lane-order partial sums, fixed tree)
__global__ void coarse_dot_kernel(int n, const double *__restrict__ a, const double *__restrict__ b,
                                  double *__restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) s += a[k] * b[k];
  s = warp_sum_d(s);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    s = warp_sum_d(s);
    if (threadIdx.x == 0) *out = s;
  }
}

// T0(i,b) = D_i^-1 sum_{j in N[i], agg(j) = b} A_ij M_j   (warp per node: per entry b
// of the node's pattern, lane k sums block k of the row, then a warp sum; lane 0
// writes the entry).  A singular D_i (no such block in an assembled stiffness) leaves
// the node's T0 at zero.
__global__ void __launch_bounds__(kThreads) coarse_t0_kernel(CoarseView c, const double *__restrict__ raw) {
  pdl_entry();
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < c.n; i += nwarps) {
    const int k0 = c.uptr[i], k1 = c.uptr[i + 1];
    // D_i^-1 by the adjugate (every lane; lane 0 uses it)
    const double *D = raw + 9 * size_t(i);
    const double c00 = D[4] * D[8] - D[5] * D[7], c01 = D[5] * D[6] - D[3] * D[8], c02 = D[3] * D[7] - D[4] * D[6];
    const double det = D[0] * c00 + D[1] * c01 + D[2] * c02;
    double inv[9];
    if (det != 0.0) {
      const double id = 1.0 / det;
      inv[0] = c00 * id;
      inv[1] = (D[2] * D[7] - D[1] * D[8]) * id;
      inv[2] = (D[1] * D[5] - D[2] * D[4]) * id;
      inv[3] = c01 * id;
      inv[4] = (D[0] * D[8] - D[2] * D[6]) * id;
      inv[5] = (D[2] * D[3] - D[0] * D[5]) * id;
      inv[6] = c02 * id;
      inv[7] = (D[1] * D[6] - D[0] * D[7]) * id;
      inv[8] = (D[0] * D[4] - D[1] * D[3]) * id;
    } else {
      for (int e = 0; e < 9; e++) inv[e] = 0.0;
    }
    for (int q = c.pptr[i]; q < c.pptr[i + 1]; q++) {
      const int b = c.pagg[q];
      double t[9];
      for (int e = 0; e < 9; e++) t[e] = 0.0;
      for (int k = k0 + lane; k < k1; k += 32) {
        const int j = c.ucol[k];
        if (c.agg[j] != b) continue;
        const double *a = raw + 9 * size_t(c.usrc[k]);
        const double m[3] = {double(c.mask[3 * j]), double(c.mask[3 * j + 1]), double(c.mask[3 * j + 2])};
        for (int d = 0; d < 3; d++)
          for (int e = 0; e < 3; e++) t[3 * d + e] += a[3 * d + e] * m[e];
      }
      for (int e = 0; e < 9; e++) t[e] = warp_sum_d(t[e]);
      if (lane == 0) {
        double *o = c.t0 + 9 * size_t(q);
        for (int d = 0; d < 3; d++)
          for (int e = 0; e < 3; e++)
            o[3 * d + e] = inv[3 * d] * t[e] + inv[3 * d + 1] * t[3 + e] + inv[3 * d + 2] * t[6 + e];
      }
    }
  }
}

// P(i,b) = [b == agg(i)] M_i - diag(omega_i) T0(i,b)   (thread per node)
__global__ void coarse_p_kernel(CoarseView c, const float *__restrict__ omega) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c.n; i += gridDim.x * blockDim.x) {
    const int ai = c.agg[i];
    const double w0 = omega ? double(omega[3 * i]) : 0.0, w1 = omega ? double(omega[3 * i + 1]) : 0.0,
                 w2 = omega ? double(omega[3 * i + 2]) : 0.0;
    const double w[3] = {w0, w1, w2};
    for (int q = c.pptr[i]; q < c.pptr[i + 1]; q++) {
      const double *t = c.t0 + 9 * size_t(q);
      double *p = c.p + 9 * size_t(q);
      for (int d = 0; d < 3; d++)
        for (int e = 0; e < 3; e++)
          p[3 * d + e] = (c.pagg[q] == ai && d == e ? double(c.mask[3 * i + d]) : 0.0) - w[d] * t[3 * d + e];
    }
  }
}

// Q(i,b) = sum_{j in N[i]} A_ij P(j,b) for b in row i's two-ring pattern (warp per
// node; lane k takes block k of the row, then a lane-order warp sum per entry).
__global__ void __launch_bounds__(kThreads) coarse_ap_kernel(CoarseView c, const double *__restrict__ raw) {
  pdl_entry();
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < c.n; i += nwarps) {
    const int k0 = c.uptr[i], k1 = c.uptr[i + 1];
    for (int qq = c.qptr[i]; qq < c.qptr[i + 1]; qq++) {
      const int b = c.qagg[qq];
      double acc[9];
      for (int e = 0; e < 9; e++) acc[e] = 0.0;
      for (int k = k0 + lane; k < k1; k += 32) {
        const int j = c.ucol[k];
        int q = c.pptr[j];
        const int qe = c.pptr[j + 1];
        while (q < qe && c.pagg[q] != b) q++;
        if (q == qe) continue;
        const double *a = raw + 9 * size_t(c.usrc[k]);
        const double *p = c.p + 9 * size_t(q);
        for (int d = 0; d < 3; d++)
          for (int e = 0; e < 3; e++) acc[3 * d + e] += a[3 * d] * p[e] + a[3 * d + 1] * p[3 + e] + a[3 * d + 2] * p[6 + e];
      }
      for (int e = 0; e < 9; e++) {
        const double v = warp_sum_d(acc[e]);
        if (lane == 0) c.q[9 * size_t(qq) + e] = v;
      }
    }
  }
}

// Ac(a,b) = sum_{i in restriction of a} P(i,a)^T Q(i,b)   (warp per aggregate a and
// coarse block b of its pattern; lanes over the restriction's nodes in ascending
// order, then a lane-order warp sum).  Ac is dense, zero outside the pattern.
__global__ void __launch_bounds__(kThreads) coarse_ac_kernel(CoarseView c) {
  pdl_entry();
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int nblk = c.cptr[c.nagg];
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nblk; w += nwarps) {
    int a = 0;
    {  // row of pattern entry w (binary search in cptr)
      int lo = 0, hi = c.nagg;
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (c.cptr[mid] <= w) lo = mid;
        else hi = mid;
      }
      a = lo;
    }
    const int b = c.cagg[w];
    double acc[9];
    for (int e = 0; e < 9; e++) acc[e] = 0.0;
    for (int t = c.rptr[a] + lane; t < c.rptr[a + 1]; t += 32) {
      const int i = c.rnode[t];
      int qq = c.qptr[i];
      const int qe = c.qptr[i + 1];
      while (qq < qe && c.qagg[qq] != b) qq++;
      if (qq == qe) continue;
      const double *p = c.p + 9 * size_t(c.rpos[t]);
      const double *qv = c.q + 9 * size_t(qq);
      for (int d = 0; d < 3; d++)
        for (int e = 0; e < 3; e++) acc[3 * d + e] += p[d] * qv[e] + p[3 + d] * qv[3 + e] + p[6 + d] * qv[6 + e];
    }
    for (int d = 0; d < 3; d++)
      for (int e = 0; e < 3; e++) {
        const double v = warp_sum_d(acc[3 * d + e]);
        if (lane == 0) c.ac[size_t(3 * a + d) * c.nc + 3 * b + e] = v;
      }
  }
}

// A coarse DOF whose basis vector is zero (every DOF of that direction in the
// aggregate constrained) has a zero row and column in Ac (p^T A p = 0 only for p = 0,
// A being SPD): its diagonal is set to 1, so that Ac stays invertible and the DOF's
// correction, from a zero restriction, stays zero.
__global__ void coarse_zero_diag_kernel(double *__restrict__ ac, int nc) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nc; k += gridDim.x * blockDim.x)
    if (ac[size_t(k) * nc + k] == 0.0) ac[size_t(k) * nc + k] = 1.0;
}

// ---- in-place inversion of the SPD coarse matrix: blocked Gauss-Jordan ----------
// For each block K of kGjBlock pivots (no pivoting: Ac is SPD), with A = M_KK,
// B = M_Kj, C = M_iK, E = M_ij (i, j not in K), Gauss-Jordan makes
//   M_KK = A^-1,  M_Kj = A^-1 B,  M_iK = -C A^-1,  M_ij = E - C A^-1 B.
// For symmetric A the matrix stays symmetric, except that the blocks between pivoted
// and not yet pivoted indices are antisymmetric (M_ab = -M_ba^T for a pivoted, b not).
// Only the lower triangle is kept up to date (half the update work); an upper entry
// is read from its mirror with that sign:
//   gj_diag:   Dinv = A^-1, A read from the lower triangle     (one CTA)
//   gj_col:    C_i from the lower triangle (row K for i before K, sign -1), G_i = C_i Dinv,
//              B_j = s_j C_j (s_j = -1 before K, +1 after: the old row panel), the new
//              column panel -G into the lower triangle (row K for i before K), M_KK = Dinv
//   gj_update: M_ij -= G_i B_j for i >= j outside K
// and after the last block (all pivoted, symmetric again) gj_mirror copies the lower
// triangle onto the upper.  Then M holds Ac^-1.
constexpr int kGjBlock = 64;

// Dinv = M_KK^-1 by unblocked Gauss-Jordan in shared memory (one CTA of 1024
// threads; thread t owns row t / 16, columns t % 16 + 16 v).  A pivot that is not
// positive sets *err (the coarse operator is then not used).
__global__ void __launch_bounds__(1024) gj_diag_kernel(double *__restrict__ M, int n, int k0, int nb,
                                                       double *__restrict__ dinv, int *err) {
  __shared__ double s[kGjBlock][kGjBlock + 1];
  const int i = threadIdx.x >> 4, jl = threadIdx.x & 15;
#pragma unroll
  for (int v = 0; v < 4; v++) {
    const int j = jl + 16 * v;
    const int a = max(i, j), b = min(i, j);  // the lower-triangle copy
    s[i][j] = (i < nb && j < nb) ? M[size_t(k0 + a) * n + k0 + b] : 0.0;
  }
  __syncthreads();
  for (int k = 0; k < nb; k++) {
    // row and column k are not written before the barrier below, so every thread
    // reads the same pivot
    const double piv = s[k][k];
    if (!(piv > 0.0)) {
      if (threadIdx.x == 0) atomicOr(err, 1);
      return;  // uniform
    }
    const double d = 1.0 / piv;
    if (i != k) {
      const double sik = s[i][k];
#pragma unroll
      for (int v = 0; v < 4; v++) {
        const int j = jl + 16 * v;
        if (j != k) s[i][j] -= sik * s[k][j] * d;
      }
    }
    __syncthreads();
    const int t = threadIdx.x;
    if (t < nb && t != k) {
      s[k][t] *= d;
      s[t][k] *= -d;
    }
    if (t == 0) s[k][k] = d;
    __syncthreads();
  }
#pragma unroll
  for (int v = 0; v < 4; v++) {
    const int j = jl + 16 * v;
    if (i < nb && j < nb) dinv[i * nb + j] = s[i][j];
  }
}

// Warp per row i.  Rows of K: M(i, k0 + s) = Dinv(i - k0, s) for s <= i - k0, G = B = 0.
// Other rows: lane l holds C(i, l) and C(i, l + 32) (after K: M(i, k0 + t); before K:
// -M(k0 + t, i)), broadcast by shuffles; lane l computes G(i, l) and G(i, l + 32).
// G and B are stored transposed (GT[t * n + i], BT[t * n + j]) so that the update
// kernel's panel loads run along i and j.
__global__ void __launch_bounds__(256) gj_col_kernel(double *__restrict__ M, int n, int k0, int nb,
                                                     const double *__restrict__ dinv, double *__restrict__ GT,
                                                     double *__restrict__ BT) {
  __shared__ double D[kGjBlock][kGjBlock];
  for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) D[t / nb][t % nb] = dinv[t];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
    if (i >= k0 && i < k0 + nb) {
      for (int s = lane; s <= i - k0; s += 32) M[size_t(i) * n + k0 + s] = D[i - k0][s];
      for (int s = lane; s < nb; s += 32) {
        GT[size_t(s) * n + i] = 0.0;
        BT[size_t(s) * n + i] = 0.0;
      }
      continue;
    }
    const bool before = i < k0;
    double c0 = 0.0, c1 = 0.0;
    if (before) {
      if (lane < nb) c0 = -M[size_t(k0 + lane) * n + i];
      if (lane + 32 < nb) c1 = -M[size_t(k0 + lane + 32) * n + i];
    } else {
      const double *row = M + size_t(i) * n + k0;
      if (lane < nb) c0 = row[lane];
      if (lane + 32 < nb) c1 = row[lane + 32];
    }
    double g0 = 0.0, g1 = 0.0;
    const int s1 = min(lane + 32, kGjBlock - 1);
    for (int t = 0; t < nb; t++) {
      const double ct = __shfl_sync(0xffffffffu, t < 32 ? c0 : c1, t & 31);
      g0 += ct * D[t][lane];
      g1 += ct * D[t][s1];
    }
    const double sg = before ? -1.0 : 1.0;
    if (lane < nb) {
      GT[size_t(lane) * n + i] = g0;
      BT[size_t(lane) * n + i] = sg * c0;
      if (before) M[size_t(k0 + lane) * n + i] = -g0;
      else M[size_t(i) * n + k0 + lane] = -g0;
    }
    if (lane + 32 < nb) {
      GT[size_t(lane + 32) * n + i] = g1;
      BT[size_t(lane + 32) * n + i] = sg * c1;
      if (before) M[size_t(k0 + lane + 32) * n + i] = -g1;
      else M[size_t(i) * n + k0 + lane + 32] = -g1;
    }
  }
}

// M(i, j) -= G(i, :) B(j, :) for i >= j outside K.  Tiles of 128 rows x 64 columns
// (tiles wholly above the diagonal leave at once), 256 threads with 8 x 4 outputs
// each, two CTAs per SM: the tile's values are loaded into the accumulators first,
// then both panels of the whole pivot block go to shared memory at once (contiguous
// loads along i and j, conflict-free stores), one barrier, nb rank-1 steps.
constexpr int kGjTileI = 128, kGjTileJ = 64;
constexpr int kGjGs = kGjTileI + 4, kGjBs = kGjTileJ + 4;  // padded panel rows (doubles)
constexpr size_t kGjUpdateSmem = sizeof(double) * size_t(kGjBlock) * (kGjGs + kGjBs);
__global__ void __launch_bounds__(256, 2) gj_update_kernel(double *__restrict__ M, int n, int k0, int nb,
                                                           const double *__restrict__ GT,
                                                           const double *__restrict__ BT) {
  extern __shared__ __align__(16) double gj_smem[];
  double *Gs = gj_smem;                     // Gs[k][i] = G(i0 + i, k)
  double *Bs = gj_smem + kGjBlock * kGjGs;  // Bs[k][j] = B(j0 + j, k)
  const int i0 = blockIdx.y * kGjTileI, j0 = blockIdx.x * kGjTileJ;
  // nothing to update: the tile lies above the diagonal, or inside the pivot rows or
  // columns
  if (i0 + kGjTileI <= j0 || (i0 >= k0 && i0 + kGjTileI <= k0 + nb) || (j0 >= k0 && j0 + kGjTileJ <= k0 + nb))
    return;
  const int tr = threadIdx.x >> 4, tc = threadIdx.x & 15;
  double acc[8][4];
#pragma unroll
  for (int u = 0; u < 8; u++) {
    const int i = i0 + tr * 8 + u;
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const int j = j0 + tc * 4 + v;
      acc[u][v] = (i < n && j <= i) ? M[size_t(i) * n + j] : 0.0;
    }
  }
  for (int e = threadIdx.x; e < kGjBlock * kGjTileI; e += blockDim.x) {
    const int k = e / kGjTileI, i = e % kGjTileI;
    Gs[k * kGjGs + i] = (i0 + i < n && k < nb) ? GT[size_t(k) * n + i0 + i] : 0.0;
  }
  for (int e = threadIdx.x; e < kGjBlock * kGjTileJ; e += blockDim.x) {
    const int k = e / kGjTileJ, j = e % kGjTileJ;
    Bs[k * kGjBs + j] = (j0 + j < n && k < nb) ? BT[size_t(k) * n + j0 + j] : 0.0;
  }
  __syncthreads();
#pragma unroll 4
  for (int k = 0; k < nb; k++) {
    const double *gk = Gs + k * kGjGs + tr * 8;
    const double *bk = Bs + k * kGjBs + tc * 4;
    const double2 a01 = *reinterpret_cast<const double2 *>(gk);
    const double2 a23 = *reinterpret_cast<const double2 *>(gk + 2);
    const double2 a45 = *reinterpret_cast<const double2 *>(gk + 4);
    const double2 a67 = *reinterpret_cast<const double2 *>(gk + 6);
    const double2 b01 = *reinterpret_cast<const double2 *>(bk);
    const double2 b23 = *reinterpret_cast<const double2 *>(bk + 2);
    const double a[8] = {a01.x, a01.y, a23.x, a23.y, a45.x, a45.y, a67.x, a67.y};
    const double b[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
    for (int u = 0; u < 8; u++)
#pragma unroll
      for (int v = 0; v < 4; v++) acc[u][v] = fma(-a[u], b[v], acc[u][v]);
  }
#pragma unroll
  for (int u = 0; u < 8; u++) {
    const int i = i0 + tr * 8 + u;
    if (i >= n || (i >= k0 && i < k0 + nb)) continue;
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const int j = j0 + tc * 4 + v;
      if (j > i || (j >= k0 && j < k0 + nb)) continue;
      M[size_t(i) * n + j] = acc[u][v];
    }
  }
}

// M(j, i) = M(i, j) for i > j: 32 x 32 tiles of the lower triangle through shared
// memory, written transposed (both sides contiguous).
__global__ void __launch_bounds__(256) gj_mirror_kernel(double *__restrict__ M, int n) {
  __shared__ double t[32][33];
  const int bi = blockIdx.y, bj = blockIdx.x;
  if (bj > bi) return;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int r = ty; r < 32; r += 8) {
    const int i = bi * 32 + r, j = bj * 32 + tx;
    t[r][tx] = (i < n && j < n) ? M[size_t(i) * n + j] : 0.0;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int j = bj * 32 + r, i = bi * 32 + tx;  // write M(j, i) = M(i, j) for i > j
    if (i < n && j < n && i > j) M[size_t(j) * n + i] = t[tx][r];
  }
}

// ---- application ------------------------------------------------------------
// bc = P^T r   (warp per aggregate; lanes over its restriction entries in order)
template <class R>
__global__ void __launch_bounds__(kThreads) coarse_restrict_kernel(CoarseView c, const R *__restrict__ r,
                                                                   double *__restrict__ bc, const CgState *st) {
  pdl_entry();
  if (st && (st->done || !st->use_gnn)) return;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < c.nagg; a += nwarps) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int t = c.rptr[a] + lane; t < c.rptr[a + 1]; t += 32) {
      const int i = c.rnode[t];
      const double *p = c.p + 9 * size_t(c.rpos[t]);
      const double r0 = double(r[3 * i]), r1 = double(r[3 * i + 1]), r2 = double(r[3 * i + 2]);
      s0 += p[0] * r0 + p[3] * r1 + p[6] * r2;
      s1 += p[1] * r0 + p[4] * r1 + p[7] * r2;
      s2 += p[2] * r0 + p[5] * r1 + p[8] * r2;
    }
    s0 = warp_sum_d(s0);
    s1 = warp_sum_d(s1);
    s2 = warp_sum_d(s2);
    if (lane == 0) {
      bc[3 * a] = s0;
      bc[3 * a + 1] = s1;
      bc[3 * a + 2] = s2;
    }
  }
}

// y = Ainv bc   (warp per coarse row, FP64)
__global__ void __launch_bounds__(kThreads) coarse_gemv_kernel(int nc, const double *__restrict__ ainv,
                                                               const double *__restrict__ bc, double *__restrict__ y,
                                                               const CgState *st) {
  pdl_entry();
  if (st && (st->done || !st->use_gnn)) return;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nc; row += nwarps) {
    const double *a = ainv + size_t(row) * nc;
    double s = 0.0;
    for (int k = lane; k < nc; k += 32) s += __ldcs(a + k) * bc[k];
    s = warp_sum_d(s);
    if (lane == 0) y[row] = s;
  }
}

// z = zs + P y (thread per node); z = zs once the correction is off.  With t0y given,
// also t0y = T0 y and v = P y (training).
template <class R>
__global__ void coarse_prolong_kernel(CoarseView c, const double *__restrict__ y, const R *__restrict__ zs,
                                      R *__restrict__ z, double *__restrict__ v, double *__restrict__ t0y,
                                      const CgState *st) {
  pdl_entry();
  if (st && st->done) return;
  const bool on = !st || st->use_gnn;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c.n; i += gridDim.x * blockDim.x) {
    double a[3] = {0.0, 0.0, 0.0}, t[3] = {0.0, 0.0, 0.0};
    if (on)
      for (int q = c.pptr[i]; q < c.pptr[i + 1]; q++) {
        const double *p = c.p + 9 * size_t(q);
        const int b = c.pagg[q];
        const double y0 = y[3 * b], y1 = y[3 * b + 1], y2 = y[3 * b + 2];
        for (int d = 0; d < 3; d++) a[d] += p[3 * d] * y0 + p[3 * d + 1] * y1 + p[3 * d + 2] * y2;
        if (t0y) {
          const double *tq = c.t0 + 9 * size_t(q);
          for (int d = 0; d < 3; d++) t[d] += tq[3 * d] * y0 + tq[3 * d + 1] * y1 + tq[3 * d + 2] * y2;
        }
      }
    for (int d = 0; d < 3; d++) {
      if (z) z[3 * i + d] = R(double(zs[3 * i + d]) + a[d]);
      if (v) v[3 * i + d] = a[d];
      if (t0y) t0y[3 * i + d] = t[d];
    }
  }
}

// bc = P^T r with the FP32 copy of P: one CTA per aggregate (an aggregate's
// restriction gathers ~1,000 nodes on the 9x9x9 aggregates); per-thread sums in
// entry order, then a fixed-order CTA sum.
template <class R>
__global__ void __launch_bounds__(256) coarse_restrict32_kernel(CoarseApply c, const R *__restrict__ r,
                                                                double *__restrict__ bc, const CgState *st) {
  pdl_entry();
  if (st && (st->done || !st->use_gnn)) return;
  __shared__ double sh[3][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int a = blockIdx.x; a < c.nagg; a += gridDim.x) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int t = c.rptr[a] + threadIdx.x; t < c.rptr[a + 1]; t += blockDim.x) {
      const int i = c.rnode[t];
      const float *p = c.p + 9 * size_t(c.rpos[t]);
      const double r0 = double(r[3 * i]), r1 = double(r[3 * i + 1]), r2 = double(r[3 * i + 2]);
      s0 += double(p[0]) * r0 + double(p[3]) * r1 + double(p[6]) * r2;
      s1 += double(p[1]) * r0 + double(p[4]) * r1 + double(p[7]) * r2;
      s2 += double(p[2]) * r0 + double(p[5]) * r1 + double(p[8]) * r2;
    }
    s0 = warp_sum_d(s0);
    s1 = warp_sum_d(s1);
    s2 = warp_sum_d(s2);
    if (lane == 0) {
      sh[0][warp] = s0;
      sh[1][warp] = s1;
      sh[2][warp] = s2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
      double v = 0.0;
      for (int w = 0; w < int(blockDim.x >> 5); w++) v += sh[threadIdx.x][w];
      bc[3 * a + threadIdx.x] = v;
    }
    __syncthreads();
  }
}

// y = Ainv bc with the FP32 copy of Ac^-1, FP64 accumulation (warp per coarse row)
__global__ void __launch_bounds__(kThreads) coarse_gemv32_kernel(int nc, const float *__restrict__ ainv,
                                                                 const double *__restrict__ bc, double *__restrict__ y,
                                                                 const CgState *st) {
  pdl_entry();
  if (st && (st->done || !st->use_gnn)) return;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nc; row += nwarps) {
    const float *a = ainv + size_t(row) * nc;
    double s = 0.0;
    for (int k = lane; k < nc; k += 32) s += double(__ldcs(a + k)) * bc[k];
    s = warp_sum_d(s);
    if (lane == 0) y[row] = s;
  }
}

// The coarse correction inside the two-grid cycle: zc = zs + P y and, in place,
// w = w - (A P) y with the stored A P (the residual after the correction without a
// full SpMV: a row of A P has a few blocks, a row of A 27), FP32 copies.  With the
// correction off zc = zs and w is left alone.
template <class R>
__global__ void coarse_prolong_resid32_kernel(CoarseApply c, const double *__restrict__ y, const R *__restrict__ zs,
                                              R *__restrict__ zc, R *__restrict__ w, const CgState *st) {
  pdl_entry();
  if (st && st->done) return;
  const bool on = !st || st->use_gnn;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c.n; i += gridDim.x * blockDim.x) {
    double a[3] = {0.0, 0.0, 0.0}, q[3] = {0.0, 0.0, 0.0};
    if (on) {
      for (int k = c.pptr[i]; k < c.pptr[i + 1]; k++) {
        const float *p = c.p + 9 * size_t(k);
        const int b = c.pagg[k];
        const double y0 = y[3 * b], y1 = y[3 * b + 1], y2 = y[3 * b + 2];
        for (int d = 0; d < 3; d++)
          a[d] += double(p[3 * d]) * y0 + double(p[3 * d + 1]) * y1 + double(p[3 * d + 2]) * y2;
      }
      for (int k = c.qptr[i]; k < c.qptr[i + 1]; k++) {
        const float *qb = c.q + 9 * size_t(k);
        const int b = c.qagg[k];
        const double y0 = y[3 * b], y1 = y[3 * b + 1], y2 = y[3 * b + 2];
        for (int d = 0; d < 3; d++)
          q[d] += double(qb[3 * d]) * y0 + double(qb[3 * d + 1]) * y1 + double(qb[3 * d + 2]) * y2;
      }
    }
    for (int d = 0; d < 3; d++) {
      zc[3 * i + d] = R(double(zs[3 * i + d]) + a[d]);
      if (on) w[3 * i + d] = R(double(w[3 * i + d]) - q[d]);
    }
  }
}

// z = zs + P y with the FP32 copy of P (the additive form); z = zs once off.
template <class R>
__global__ void coarse_prolong32_kernel(CoarseApply c, const double *__restrict__ y, const R *__restrict__ zs,
                                        R *__restrict__ z, const CgState *st) {
  pdl_entry();
  if (st && st->done) return;
  const bool on = !st || st->use_gnn;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < c.n; i += gridDim.x * blockDim.x) {
    double a[3] = {0.0, 0.0, 0.0};
    if (on)
      for (int k = c.pptr[i]; k < c.pptr[i + 1]; k++) {
        const float *p = c.p + 9 * size_t(k);
        const int b = c.pagg[k];
        const double y0 = y[3 * b], y1 = y[3 * b + 1], y2 = y[3 * b + 2];
        for (int d = 0; d < 3; d++)
          a[d] += double(p[3 * d]) * y0 + double(p[3 * d + 1]) * y1 + double(p[3 * d + 2]) * y2;
      }
    for (int d = 0; d < 3; d++) z[3 * i + d] = R(double(zs[3 * i + d]) + a[d]);
  }
}

// End of the symmetric two-grid application: z = zc + z (z the post-smoothing SSOR
// step), or z = zs once the correction is off (SSOR-CG).
template <class R>
__global__ void coarse_post_kernel(const R *__restrict__ zc, const R *__restrict__ zs, R *__restrict__ z, int n3,
                                   const CgState *st) {
  pdl_entry();
  if (st && st->done) return;
  const bool on = !st || st->use_gnn;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n3; k += gridDim.x * blockDim.x)
    z[k] = on ? z[k] + zc[k] : zs[k];
}

// ---- training -----------------------------------------------------------------
// out = double(a) (- b when given): a recorded FP32 pair vector widened, optionally
// less an FP64 vector.
__global__ void coarse_widen_kernel(const float *__restrict__ a, const double *__restrict__ b, double *__restrict__ out,
                                    int n) {
  pdl_entry();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    out[k] = double(a[k]) - (b ? b[k] : 0.0);
}

// Loss of one recorded pair (r = A e): the energy of e outside the coarse space,
//   L = (e^T r - bc^T y) / (e^T r),   y = Ac^-1 P^T r,
// whose gradient in P is -2 (r - A P y) y^T / (e^T r), so in omega (dP/domega = -T0):
//   dL/domega_(i,d) = 2 g_(i,d) (T0 y)_(i,d) / (e^T r),   g = r - A P y.
// Accumulated into dout through omega = sigmoid(out): domega * omega (1 - omega).
template <class RT>
__global__ void coarse_grad_kernel(int n3, const RT *__restrict__ r, const double *__restrict__ apy,
                                   const double *__restrict__ t0y, const float *__restrict__ omega, double coef,
                                   float *__restrict__ dout) {
  pdl_entry();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n3; k += gridDim.x * blockDim.x) {
    const double g = double(r[k]) - apy[k];
    const double w = double(omega[k]);
    dout[k] += float(2.0 * coef * g * t0y[k] * w * (1.0 - w));
  }
}

}  // namespace h33
