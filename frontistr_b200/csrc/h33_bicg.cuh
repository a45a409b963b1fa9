// h33_bicg.cuh -- BiCGSTAB on the device (hecmw_solver_BiCGSTAB.f90:161-271),
// METHOD = 2 of hecmw_solve_iterative and the METHOD2 fallback of a diverged CG.
//
// One iteration, in the reference's order:
//   RHO = {r}{r_tld};  BETA = (RHO/RHO1)(ALPHA/OMEGA);  {p} = {r} + BETA({p} - OMEGA{v})
//   {p_tld} = M^-1 {p};  {v} = A {p_tld};  ALPHA = RHO / {r_tld}{v}
//   {s} = {r} - ALPHA {v};  {s_tld} = M^-1 {s};  {t} = A {s_tld}
//   OMEGA = {t}{s} / {t}{t};  {x} += ALPHA {p_tld};  {x} += OMEGA {s_tld}
//   {r} = {s} - OMEGA {t} (or b - A x every 100th iteration);  RESID = |r| / |b|
// The reference has no breakdown tests in this loop: a zero denominator runs on to
// MAXIT (3001) as there.  Reductions and the end-of-iteration control are those of
// the CG (reduce_finish, fin_rr, resid_ctl_kernel with st->nrecompute = 100).
#pragma once

#include "h33_kernels.cuh"

namespace h33 {

// RHO = {r}{r_tld} (:168) and BETA (:177), the latter from the second iteration on.
template <class R>
__global__ void __launch_bounds__(kThreads) bicg_rho_kernel(const R *__restrict__ r, const R *__restrict__ rt,
                                                            int n3, CgState *st, double *partials) {
  pdl_entry();
  if (st->done) return;
  double dot = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
    dot += double(r[i]) * double(rt[i]);
  reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[0], [&](double v) {
    st->rho = v;
    if (st->iter > 1) st->beta = (v / st->rho1) * (st->alpha / st->omega);
  });
}

// {p} = {r} (first iteration) or {p} = -OMEGA {v} + {p}; {p} = {r} + BETA {p}
// (hecmw_axpy_R then hecmw_xpay_R, :178-181).
template <class R>
__global__ void __launch_bounds__(kThreads) bicg_p_kernel(const R *__restrict__ r, R *__restrict__ p,
                                                          const R *__restrict__ v, int n3, const CgState *st) {
  pdl_entry();
  if (st->done) return;
  const bool first = st->iter == 1;
  const R beta = R(st->beta), momega = R(-st->omega);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    if (first) {
      p[i] = r[i];
    } else {
      const R pi = momega * v[i] + p[i];
      p[i] = r[i] + beta * pi;
    }
  }
}

// y = A x with one or two dots against the result:
//   MODE 0: {v} = A {p_tld}, C2 = {r_tld}{v}, ALPHA = RHO / C2 (:196-202)
//   MODE 1: {t} = A {s_tld}, {t}{s} and {t}{t}, OMEGA = {t}{s} / {t}{t} (:220-234)
template <class R, int MODE>
__global__ void __launch_bounds__(kThreads) bicg_spmv_kernel(SellView<R> A, const R *__restrict__ x,
                                                             R *__restrict__ y, const R *__restrict__ w,
                                                             CgState *st, double *partials) {
  pdl_entry();
  if (st->done) return;
  const int lane = threadIdx.x & 31;
  const int warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double d1 = 0.0, d2 = 0.0;
  for (int s = warp0; s < A.nslices; s += nwarps) {
    const bool active = lane < A.nrows[s];
    const int row = A.row0[s] + lane;
    const int len = active ? A.rowlen[s * 32 + lane] : 0;
    R y0 = 0, y1 = 0, y2 = 0;
    row_gemv<R, R, 1, false>(A, s, lane, len, x, y0, y1, y2);
    if (active) {
      y[3 * row] = y0;
      y[3 * row + 1] = y1;
      y[3 * row + 2] = y2;
      d1 += double(w[3 * row]) * double(y0) + double(w[3 * row + 1]) * double(y1) +
            double(w[3 * row + 2]) * double(y2);
      if (MODE == 1) d2 += double(y0) * double(y0) + double(y1) * double(y1) + double(y2) * double(y2);
    }
  }
  if (MODE == 0) {
    reduce_finish(d1, partials, blockIdx.x, gridDim.x, &st->ticket[1], [&](double v) {
      st->c2 = v;
      st->alpha = st->rho / v;
    });
  } else {
    reduce_finish2(d1, d2, partials, blockIdx.x, gridDim.x, &st->ticket[1],
                   [&](double ts, double tt) { st->omega = ts / tt; });
  }
}

// {s} = -ALPHA {v} + {r} (hecmw_axpyz_R, :206)
template <class R>
__global__ void __launch_bounds__(kThreads) bicg_s_kernel(R *__restrict__ s, const R *__restrict__ r,
                                                          const R *__restrict__ v, int n3, const CgState *st) {
  pdl_entry();
  if (st->done) return;
  const R malpha = R(-st->alpha);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x)
    s[i] = malpha * v[i] + r[i];
}

// {x} = ALPHA {p_tld} + {x}; {x} = OMEGA {s_tld} + {x} (:241-242); {r} = -OMEGA {t} + {s}
// with the DNRM2 partial (:244-253), except on every 100th iteration where
// resid_ctl_kernel recomputes r = b - A x instead.
template <class R>
__global__ void __launch_bounds__(kThreads) bicg_update_kernel(R *__restrict__ x, const R *__restrict__ pt,
                                                               const R *__restrict__ stl, R *__restrict__ r,
                                                               const R *__restrict__ s, const R *__restrict__ t,
                                                               int n3, CgState *st, double *partials) {
  pdl_entry();
  if (st->done) return;
  const R alpha = R(st->alpha), omega = R(st->omega), momega = R(-st->omega);
  const bool refresh = (st->iter % st->nrecompute) == 0;
  double dot = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    const R xi = alpha * pt[i] + x[i];
    x[i] = omega * stl[i] + xi;
    if (!refresh) {
      const R ri = momega * t[i] + s[i];
      r[i] = ri;
      dot += double(ri) * double(ri);
    }
  }
  if (!refresh) reduce_finish(dot, partials, blockIdx.x, gridDim.x, &st->ticket[2], [&](double v) { fin_rr(st, v); });
}

}  // namespace h33
