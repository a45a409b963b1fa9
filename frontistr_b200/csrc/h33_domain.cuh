// h33_domain.cuh -- one domain of an overlapping node-based decomposition.
//
// A distributed run gives each rank the rows of its N internal nodes over NP local
// nodes (internal, then external).  Every preconditioner of the path works on the
// internal rows and columns only (SSOR drops columns > N, hecmw_precond_SSOR_33.F90:130-155;
// the block ILU(0) and DIAG apply run over rows 1..N with the external entries of ZP
// kept at zero, hecmw_precond.f90:120-126, hecmw_precond_BILU_33.f90:98,130), so the
// solver keeps the internal block A_II in its usual layouts and the blocks of internal
// rows at external columns (A_IE) in a small CSR list that the kernels below apply
// after the SpMV of A_II, in the reference's order (external columns are the largest
// ids of a row, summed last; hecmw_solver_las_33.F90:279-308).  The external values of
// the vector being multiplied are in xe (3 per external node, in local order
// N+1..NP), filled by hecmw_update_R's exchange (pack / unpack here, the transfer by
// the caller's exchange function).
#pragma once

#include "h33_common.cuh"

namespace h33 {

// y(row) += sum over the row's external blocks A x_e, for every interface row.
static __global__ void __launch_bounds__(kThreads) interface_spmv_kernel(const int *__restrict__ irow,
                                                                        const int *__restrict__ iptr,
                                                                        const int *__restrict__ icol,
                                                                        const double *__restrict__ ival, int nrows,
                                                                        const double *__restrict__ xe,
                                                                        double *__restrict__ y) {
  pdl_entry();
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nrows; t += gridDim.x * blockDim.x) {
    const int row = irow[t];
    double y0 = y[3 * row], y1 = y[3 * row + 1], y2 = y[3 * row + 2];
    for (int j = iptr[t]; j < iptr[t + 1]; j++) {
      const int c = icol[j];
      const double x0 = xe[3 * c], x1 = xe[3 * c + 1], x2 = xe[3 * c + 2];
      const double *a = ival + 9 * size_t(j);
      y0 = fma(a[2], x2, fma(a[1], x1, fma(a[0], x0, y0)));
      y1 = fma(a[5], x2, fma(a[4], x1, fma(a[3], x0, y1)));
      y2 = fma(a[8], x2, fma(a[7], x1, fma(a[6], x0, y2)));
    }
    y[3 * row] = y0;
    y[3 * row + 1] = y1;
    y[3 * row + 2] = y2;
  }
}

// send(3k + c) = v(3 idx(k) + c): the export values of hecmw_solve_send_recv
// (hecmw_solver_SR.F90:97-112), idx 0-based internal nodes.
static __global__ void __launch_bounds__(kThreads) halo_pack_kernel(const double *__restrict__ v,
                                                                   const int *__restrict__ idx, int n,
                                                                   double *__restrict__ send) {
  pdl_entry();
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * n; t += gridDim.x * blockDim.x) {
    const int k = t / 3, c = t - 3 * k;
    send[t] = v[3 * idx[k] + c];
  }
}

// xe(3 idx(k) + c) = recv(3k + c): the received values at the import items
// (:146-161), idx 0-based external positions (local id - N - 1).
static __global__ void __launch_bounds__(kThreads) halo_unpack_kernel(const double *__restrict__ recv,
                                                                     const int *__restrict__ idx, int n,
                                                                     double *__restrict__ xe) {
  pdl_entry();
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * n; t += gridDim.x * blockDim.x) {
    const int k = t / 3, c = t - 3 * k;
    xe[3 * idx[k] + c] = recv[t];
  }
}

// MPC-CG (MPC_METHOD = 2, hecmw_solver_Iterative.f90:79-84): every product is
// T^T A T x (hecmw_TtmatTvec_33, hecmw_solver_las_33.F90:572-586).  An MPC is a slave
// DOF (its first term) and masters with coefficients: T x sets the slave to
// -sum val_j x(master_j) (hecmw_Tvec_33, :442-497); T^T y zeroes the slave and adds
// -val_j y(slave) to every master (hecmw_Ttvec_33, :504-565, an atomic scatter as the
// reference's).  DOF indices are 0-based (3 (node-1) + dof-1); y starts as a copy of x.
static __global__ void __launch_bounds__(kThreads) mpc_tvec_kernel(const int *__restrict__ slave,
                                                                  const int *__restrict__ ptr,
                                                                  const int *__restrict__ idx,
                                                                  const double *__restrict__ val, int n_mpc,
                                                                  const double *__restrict__ x,
                                                                  double *__restrict__ y) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_mpc; i += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int j = ptr[i]; j < ptr[i + 1]; j++) s = s - val[j] * x[idx[j]];
    y[slave[i]] = s;
  }
}

static __global__ void __launch_bounds__(kThreads) mpc_ttvec_kernel(const int *__restrict__ slave,
                                                                   const int *__restrict__ ptr,
                                                                   const int *__restrict__ idx,
                                                                   const double *__restrict__ val, int n_mpc,
                                                                   const double *__restrict__ x,
                                                                   double *__restrict__ y) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_mpc; i += gridDim.x * blockDim.x) {
    const double xs = x[slave[i]];
    y[slave[i]] = 0.0;
    for (int j = ptr[i]; j < ptr[i + 1]; j++) atomicAdd(&y[idx[j]], -val[j] * xs);
  }
}

}  // namespace h33
