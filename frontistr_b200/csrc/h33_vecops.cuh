// h33_vecops.cuh -- the vector operations of hecmw_solver_misc.F90 as device kernels,
// for the host-driven Krylov methods (GPBiCG): each one pass over n values, the
// operands in the reference's order.
#pragma once

#include "h33_common.cuh"

namespace h33 {

// hecmw_axpy_R: y = a x + y (hecmw_solver_misc.F90:137-166)
static __global__ void __launch_bounds__(kThreads) vec_axpy_kernel(double *__restrict__ y, double a,
                                                                  const double *__restrict__ x, int n) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = a * x[i] + y[i];
}

// hecmw_xpay_R: y = x + a y (:173-201)
static __global__ void __launch_bounds__(kThreads) vec_xpay_kernel(double *__restrict__ y, double a,
                                                                  const double *__restrict__ x, int n) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = x[i] + a * y[i];
}

// hecmw_axpyz_R: z = a x + y (:263-291)
static __global__ void __launch_bounds__(kThreads) vec_axpyz_kernel(double *__restrict__ z, double a,
                                                                   const double *__restrict__ x,
                                                                   const double *__restrict__ y, int n) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) z[i] = a * x[i] + y[i];
}

// hecmw_axpby_R: y = a x (b == 0) or a x + b y (:208-256)
static __global__ void __launch_bounds__(kThreads) vec_axpby_kernel(double *__restrict__ y, double a, double b,
                                                                   const double *__restrict__ x, int n) {
  pdl_entry();
  if (b == 0.0) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = a * x[i];
  } else {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
      y[i] = a * x[i] + b * y[i];
  }
}

}  // namespace h33
