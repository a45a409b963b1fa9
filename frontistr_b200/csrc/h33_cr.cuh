// h33_cr.cuh -- preconditioned conjugate residual (hecmw_solver_CR.f90:108-296), METHOD = 7.
// The host drives the loop (its decisions need three reductions per iteration); these
// are its vector updates.
#pragma once

#include "h33_kernels.cuh"

namespace h33 {

// {x} = ALPHA {p} + {x}; {rt} = -ALPHA {ap} + {rt}; {z} = -ALPHA {map} + {z} (:210-212)
static __global__ void __launch_bounds__(kThreads) cr_update_kernel(double *__restrict__ x,
                                                                   const double *__restrict__ p,
                                                                   double *__restrict__ rt,
                                                                   const double *__restrict__ ap,
                                                                   double *__restrict__ z,
                                                                   const double *__restrict__ map, int n3,
                                                                   double alpha) {
  pdl_entry();
  const double malpha = -alpha;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    x[i] = alpha * p[i] + x[i];
    rt[i] = malpha * ap[i] + rt[i];
    z[i] = malpha * map[i] + z[i];
  }
}

// {p} = {z} + BETA {p}; {ap} = {az} + BETA {ap} (hecmw_xpay_R, :292-293)
static __global__ void __launch_bounds__(kThreads) cr_direction_kernel(double *__restrict__ p,
                                                                      const double *__restrict__ z,
                                                                      double *__restrict__ ap,
                                                                      const double *__restrict__ az, int n3,
                                                                      double beta) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += gridDim.x * blockDim.x) {
    p[i] = z[i] + beta * p[i];
    ap[i] = az[i] + beta * ap[i];
  }
}

}  // namespace h33
