// h33_common.cuh -- shared host/device definitions of the B200 3x3-block solver.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "hecmw33_gpu.h"

namespace h33 {

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may start while its predecessor drains; it waits here until the
// predecessor grid has completed and its writes are visible, then lets its own
// successor start launching.  Without the launch attribute both are no-ops.  Every
// kernel of the solver calls this first, before it reads anything.
__device__ __forceinline__ void pdl_entry() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" :::);
}

// Slice height of the sliced block-ELL layout: one warp lane per block row.
constexpr int kSlice = 32;
// Threads per CTA for the sliced kernels (8 slices per CTA).
constexpr int kThreads = 256;
constexpr int kWarpsPerCta = kThreads / 32;

// True-residual refresh period of hecmw_solve_CG (hecmw_solver_CG.f90:67).
constexpr int kIterRecomputeR = 50;       // hecmw_solver_CG.f90 N_ITER_RECOMPUTE_R
constexpr int kIterRecomputeRBicg = 100;  // hecmw_solver_BiCGSTAB.f90:65

struct Failure : std::runtime_error {
  int code;
  Failure(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define H33_CUDA(call)                                                                     \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      throw ::h33::Failure(HECMW33_ERR_CUDA, std::string(#call) + ": " +                   \
                                                 cudaGetErrorString(e_) + " at " __FILE__); \
  } while (0)

// Owning device array (cudaMalloc'd).
template <class T>
struct DevArray {
  T *p = nullptr;
  size_t n = 0;
  DevArray() = default;
  DevArray(const DevArray &) = delete;
  DevArray &operator=(const DevArray &) = delete;
  DevArray(DevArray &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevArray &operator=(DevArray &&o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DevArray() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    if (count == n && p) return;
    release();
    if (count == 0) return;
    H33_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void upload(const T *h, size_t count, cudaStream_t s) {
    alloc(count);
    if (count) H33_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void upload(const std::vector<T> &v, cudaStream_t s) { upload(v.data(), v.size(), s); }
  void zero(cudaStream_t s) {
    if (n) H33_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  size_t bytes() const { return n * sizeof(T); }
};

// Device-side view of a sliced block-ELL matrix (3x3 blocks).
//   slice s covers rows [row0[s], row0[s] + nrows[s]) (nrows <= 32), lane l -> row row0[s]+l
//   its blocks occupy slots [slot0[s], slot0[s] + len[s]); rowlen[s*32 + l] <= len[s]
//   col[slot*32 + l]          : block column (0-based node index)
//   val[(slot*9 + e)*32 + l]  : entry e (row-major r*3+c) of that block
template <class T>
struct SellView {
  int nslices;
  const int *row0, *nrows, *slot0, *len, *rowlen, *col;
  const T *val;
};

// Device-resident state of one CG solve (scalars of hecmw_solve_CG).
struct CgState {
  double rho, rho1, alpha, beta, pq, rr, bnrm2, resid, tol;
  double rr_true;
  int iter, maxit, done, error, n_indef, recompute, converged, zero_rhs;
  int guard;  // body executions of this solve (fail-safe bound on the device loop)
  int inner;  // inner solve of the mixed-precision refinement: no true-residual refresh
  // flexible CG with the learned preconditioner
  int flexible;   // BETA = z.(r - r_old) / RHO_old
  int use_gnn;    // the network is applied after SSOR (cleared by the fallback)
  int restart;    // next BETA is 0 (after a fallback)
  int fallback;   // iteration at which the SSOR-CG fallback took over (0 = never)
  double resid_mark;
  float gamma;    // RMS of the SSOR output, the network's input/output scale
  // mixed precision with reliable updates: FP32 CG whose solution and residual are
  // folded into FP64 each time the FP32 residual falls by ru_delta
  int reliable, ru_pending, ru_count;
  double ru_delta, ru_mark;
  // BiCGSTAB (hecmw_solver_BiCGSTAB.f90): OMEGA and C2 = {r_tld}{v}; the true
  // residual refresh period (50 for CG, 100 for BiCGSTAB)
  double omega, c2;
  int nrecompute;
  // ESTCOND (Iarray(14)): ALPHA and BETA of every iteration, for the Lanczos
  // condition estimate of hecmw_solver_CG.f90:256-264 (null when off)
  double *lanczos;
  int lanczos_cap, lanczos_n;
  // ITERLOG (Iarray(21) = 1): RESID of every iteration as hecmw_solve_CG prints it
  // (hecmw_solver_CG.f90:251-253; null when off)
  double *rhist;
  int rhist_cap, rhist_n;
  unsigned int ticket[8];
};

// Solve parameters copied to the device before each graph launch.
struct CgParams {
  double tol;
  int maxit;
  int iterpremax;
  int inner;  // 1: stop on the recursive residual (the outer FP64 loop checks the true one)
  int flexible;  // 1: flexible CG (BETA of Polak-Ribiere form)
  int use_gnn;   // 1: learned preconditioner active at the start of the solve
  int reliable;  // 1: FP32 CG with FP64 reliable updates
  double ru_delta;
  int method;    // hecmw METHOD: 1 CG, 2 BiCGSTAB
  double *lanczos;  // ESTCOND: 2 x maxit doubles (ALPHA, BETA per iteration) or null
  int lanczos_cap;
  double *rhist;    // ITERLOG: maxit doubles (RESID per iteration) or null
  int rhist_cap;
};

}  // namespace h33
