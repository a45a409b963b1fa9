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

// Slice height of the sliced block-ELL layout: one warp lane per block row.
constexpr int kSlice = 32;
// Threads per CTA for the sliced kernels (8 slices per CTA).
constexpr int kThreads = 256;
constexpr int kWarpsPerCta = kThreads / 32;

// True-residual refresh period of hecmw_solve_CG (hecmw_solver_CG.f90:67).
constexpr int kIterRecomputeR = 50;

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
  unsigned int ticket[8];
};

// Solve parameters copied to the device before each graph launch.
struct CgParams {
  double tol;
  int maxit;
  int iterpremax;
};

}  // namespace h33
