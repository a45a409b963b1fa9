// h33_gmres.cuh -- GMRES(m) on the device (hecmw_solver_GMRES.f90:174-411), METHOD = 3.
//
// Right-preconditioned restarted GMRES with modified Gram-Schmidt and Givens
// rotations, in the reference's order.  The Krylov basis V (m+1 vectors of 3N) and
// the small Hessenberg system stay on the device: H is an (m+7) x (m+7) column-major
// matrix as the reference's H(NRK,NRK), with the rotations in its columns CS = m+1 and
// SN = m+2; s is the rotated right-hand side; the dots write straight into H.  The
// host drives the loop (one read of RESID per iteration) because the restart logic
// branches on it.
#pragma once

#include "h33_kernels.cuh"

namespace h33 {

struct GmresDev {
  double *H;    // (ld x ld), column-major, 1-based (k, i) at H[(i-1)*ld + (k-1)]
  double *s;    // rotated right-hand side, 1-based
  double *y;    // solution of the triangular system, 1-based
  double *val;  // last {w}{w}
  double *coef; // 1 / H(I+1, I)
  double *resid;
  int *breakdown;
  int ld;
};

__device__ __forceinline__ double &Hat(const GmresDev &g, int k, int i) { return g.H[size_t(i - 1) * g.ld + (k - 1)]; }

// H(K, I) = {w}{v_K}
static __global__ void __launch_bounds__(kThreads) gmres_dot_kernel(const double *__restrict__ w,
                                                                   const double *__restrict__ v, int n3,
                                                                   GmresDev g, int K, int I, CgState *st,
                                                                   double *partials) {
  pdl_entry();
  double dot = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) dot += w[i] * v[i];
  reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[4], [&](double x) { Hat(g, K, I) = x; });
}

// {w} = -H(K, I) {v_K} + {w}  (hecmw_axpy_R, :226)
static __global__ void __launch_bounds__(kThreads) gmres_orth_kernel(double *__restrict__ w,
                                                                    const double *__restrict__ v, int n3,
                                                                    GmresDev g, int K, int I) {
  pdl_entry();
  const double c = -Hat(g, K, I);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) w[i] = c * v[i] + w[i];
}

// val = {w}{w}; a zero value is the reference's exit of the inner loop (:231);
// otherwise H(I+1, I) = sqrt(val) and coef = 1 / H(I+1, I)
static __global__ void __launch_bounds__(kThreads) gmres_norm_kernel(const double *__restrict__ w, int n3,
                                                                    GmresDev g, int I, CgState *st,
                                                                    double *partials) {
  pdl_entry();
  double dot = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) dot += w[i] * w[i];
  reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[4], [&](double x) {
    *g.val = x;
    if (x == 0.0) {
      *g.breakdown = 1;
    } else {
      Hat(g, I + 1, I) = sqrt(x);
      *g.coef = 1.0 / Hat(g, I + 1, I);
    }
  });
}

// {v_{I+1}} = coef {w} (hecmw_axpby_R with beta = 0, :235), unless the loop broke down
static __global__ void __launch_bounds__(kThreads) gmres_scale_kernel(const double *__restrict__ w,
                                                                     double *__restrict__ v, int n3, GmresDev g) {
  pdl_entry();
  if (*g.breakdown) return;
  const double c = *g.coef;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) v[i] = c * w[i];
}

// Givens rotations of column I and of s, RESID = |s(I+1)| / sqrt(BNRM2) (:242-285)
static __global__ void gmres_givens_kernel(GmresDev g, int I, int CS, int SN, double bnrm2) {
  pdl_entry();
  if (threadIdx.x != 0 || blockIdx.x != 0 || *g.breakdown) return;
  for (int k = 1; k <= I - 1; k++) {
    const double vcs = Hat(g, k, CS), vsn = Hat(g, k, SN);
    const double dt = vcs * Hat(g, k, I) + vsn * Hat(g, k + 1, I);
    Hat(g, k + 1, I) = vcs * Hat(g, k + 1, I) - vsn * Hat(g, k, I);
    Hat(g, k, I) = dt;
  }
  const double aa = Hat(g, I, I), bb = Hat(g, I + 1, I);
  double r0 = bb;
  if (fabs(aa) > fabs(bb)) r0 = aa;
  const double scale = fabs(aa) + fabs(bb);
  double rr;
  if (scale != 0.0) {
    const double qa = aa / scale, qb = bb / scale;
    rr = scale * sqrt(qa * qa + qb * qb);
    rr = copysign(1.0, r0) * rr;
    Hat(g, I, CS) = aa / rr;
    Hat(g, I, SN) = bb / rr;
  } else {
    Hat(g, I, CS) = 1.0;
    Hat(g, I, SN) = 0.0;
    rr = 0.0;
  }
  (void)rr;
  const double vcs = Hat(g, I, CS), vsn = Hat(g, I, SN);
  double dt = vcs * Hat(g, I, I) + vsn * Hat(g, I + 1, I);
  Hat(g, I + 1, I) = vcs * Hat(g, I + 1, I) - vsn * Hat(g, I, I);
  Hat(g, I, I) = dt;
  dt = vcs * g.s[I] + vsn * g.s[I + 1];
  g.s[I + 1] = vcs * g.s[I + 1] - vsn * g.s[I];
  g.s[I] = dt;
  *g.resid = fabs(g.s[I + 1]) / sqrt(bnrm2);
}

// [H]{y} = {s} for the leading irow x irow upper triangle (:296-306)
static __global__ void gmres_trisolve_kernel(GmresDev g, int irow, double *ss) {
  pdl_entry();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int ik = 1; ik <= irow; ik++) ss[ik] = g.s[ik];
  g.y[irow] = ss[irow] / Hat(g, irow, irow);
  for (int kk = irow - 1; kk >= 1; kk--) {
    for (int jj = irow; jj >= kk + 1; jj--) ss[kk] = ss[kk] - Hat(g, kk, jj) * g.y[jj];
    g.y[kk] = ss[kk] / Hat(g, kk, kk);
  }
}

// {v_1} = (1 / |r|) {r} (hecmw_axpby_R with beta = 0, :190)
static __global__ void __launch_bounds__(kThreads) gmres_start_kernel(const double *__restrict__ r,
                                                                     double *__restrict__ v, int n3, double coef) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) v[i] = coef * r[i];
}

// {x} = 1.0 {zq} + {x} (:319)
static __global__ void __launch_bounds__(kThreads) gmres_update_x_kernel(const double *__restrict__ zq,
                                                                        double *__restrict__ x, int n3) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) x[i] = 1.0 * zq[i] + x[i];
}

// {av} = sum_jj y(jj) {v_jj}, accumulated as the reference's axpy sequence (:309-315)
static __global__ void __launch_bounds__(kThreads) gmres_combine_kernel(const double *__restrict__ V, size_t stride,
                                                                       int irow, GmresDev g, int n3,
                                                                       double *__restrict__ av) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    double a = 0.0;
    for (int jj = 1; jj <= irow; jj++) a = g.y[jj] * V[size_t(jj - 1) * stride + i] + a;
    av[i] = a;
  }
}

}  // namespace h33
