// hecmw33_noalloc.cu -- a relative-residual entry point that allocates no memory.
//
// Some callers cannot call cudaMalloc: programs whose GPU memory is owned in full by
// another allocator (a pool that reserved the HBM up front, such as a framework's
// caching allocator or a solver stack that sizes its arrays to the device), and
// latency-critical loops that forbid allocation between solves.  They already hold
// the matrix and the vectors on the device and only need the answer.  This entry
// point takes their device pointers in the hecmwST_matrix layout and computes
// ||b - A x|| / ||b|| (the quantity of hecmw_rel_resid_L2_33) without creating a
// handle and without any device or pinned allocation: its only scratch memory is
// the file-scope array below, which every GPU that loads this library holds until
// the process exits.
//
// Limits and sharing rules:
//   * at most kMaxRows block rows (one CTA of 256 rows per partial sum pair);
//     larger N is rejected with HECMW33_ERR_BAD_INPUT before anything runs;
//   * one whole-mesh matrix only (N == NP, no external nodes): every itemL / itemU
//     must lie in 1..N, since X and B hold 3N doubles.  A domain of a decomposed mesh
//     (items up to NP > N) needs a halo exchange and a sum over ranks that this call
//     does not make.  The kernel checks every item before it reads X; an item outside
//     1..N is skipped and the call returns HECMW33_ERR_BAD_INPUT with no residual;
//   * null pointers (resid, ierr or any device array) are rejected before any launch;
//   * the memset, the kernel and the copy of the result run on the legacy default
//     stream (stream 0), which does not order against non-blocking streams: a caller
//     whose arrays come from such a stream synchronises it before the call;
//   * all calls share the scratch array and it keeps the last call's contents, so
//     the arrival counter is cleared at the start of every call; calls that overlap
//     on the GPU (from several host threads, or on several devices' streams sharing
//     one context) race on it and must be serialised by the caller;
//   * the first call on a device looks up the array's device address there
//     (cudaGetSymbolAddress with that device current) and keeps it for the life of
//     the process; make that first call before any stream capture.  cudaDeviceReset
//     between calls is not supported: the module may load again at another address.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "hecmw33_gpu.h"

namespace h33 {
void set_last_error(const std::string &msg);  // message for hecmw33_gpu_last_error
}

namespace {

constexpr int kRowsPerCta = 256;
constexpr int kMaxParts = 8192;                     // CTAs, i.e. partial-sum pairs
constexpr int kMaxRows = kMaxParts * kRowsPerCta;  // 2,097,152 block rows
// layout: [0, kMaxParts) r.r partials, [kMaxParts, 2 kMaxParts) b.b partials,
// [2 kMaxParts] result, [2 kMaxParts + 1] arrival counter (as unsigned int),
// [2 kMaxParts + 2] count of items outside 1..N (as unsigned int)
constexpr int kResult = 2 * kMaxParts;
constexpr int kCounter = kResult + 1;
constexpr int kBadItems = kResult + 2;
constexpr int kScratchDoubles = 2 * kMaxParts + 8;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_scratch_ptr[kMaxDevices] = {nullptr};

__device__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ double block_sum(double v, double *sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  v = 0.0;
  if (warp == 0) {
    v = lane < int(blockDim.x >> 5) ? sh[lane] : 0.0;
    v = warp_sum(v);
  }
  return v;
}

// One thread per block row: r_i = b_i - (D_i x_i + sum_L A x + sum_U A x), with the
// hecmwST arrays as given (1-based items); per-CTA partials of r.r and b.b in the
// scratch array; the last CTA sums them in a fixed order and stores the result.
// An item outside 1..N is counted in the scratch array and its block skipped, so X
// is never read outside its 3N entries.
__global__ void __launch_bounds__(kRowsPerCta) rel_resid_kernel(
    int N, const int *__restrict__ indexL, const int *__restrict__ itemL, const int *__restrict__ indexU,
    const int *__restrict__ itemU, const double *__restrict__ D, const double *__restrict__ AL,
    const double *__restrict__ AU, const double *__restrict__ X, const double *__restrict__ B,
    double *scratch) {
  __shared__ double sh[32];
  __shared__ int is_last;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double rr = 0.0, bb = 0.0;
  if (i < N) {
    const double *d = D + 9 * size_t(i);
    const double x0 = X[3 * i], x1 = X[3 * i + 1], x2 = X[3 * i + 2];
    double y0 = d[0] * x0 + d[1] * x1 + d[2] * x2;
    double y1 = d[3] * x0 + d[4] * x1 + d[5] * x2;
    double y2 = d[6] * x0 + d[7] * x1 + d[8] * x2;
    for (int pass = 0; pass < 2; pass++) {
      const int *index = pass ? indexU : indexL;
      const int *item = pass ? itemU : itemL;
      const double *A = pass ? AU : AL;
      for (int j = index[i]; j < index[i + 1]; j++) {
        const int c = item[j] - 1;
        if (c < 0 || c >= N) {
          atomicAdd(reinterpret_cast<unsigned int *>(scratch + kBadItems), 1u);
          continue;
        }
        const double *a = A + 9 * size_t(j);
        const double c0 = X[3 * c], c1 = X[3 * c + 1], c2 = X[3 * c + 2];
        y0 += a[0] * c0 + a[1] * c1 + a[2] * c2;
        y1 += a[3] * c0 + a[4] * c1 + a[5] * c2;
        y2 += a[6] * c0 + a[7] * c1 + a[8] * c2;
      }
    }
    const double b0 = B[3 * i], b1 = B[3 * i + 1], b2 = B[3 * i + 2];
    const double r0 = b0 - y0, r1 = b1 - y1, r2 = b2 - y2;
    rr = r0 * r0 + r1 * r1 + r2 * r2;
    bb = b0 * b0 + b1 * b1 + b2 * b2;
  }
  rr = block_sum(rr, sh);
  bb = block_sum(bb, sh);
  unsigned int *counter = reinterpret_cast<unsigned int *>(scratch + kCounter);
  if (threadIdx.x == 0) {
    scratch[blockIdx.x] = rr;
    scratch[kMaxParts + blockIdx.x] = bb;
    __threadfence();
    is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double srr = 0.0, sbb = 0.0;
  for (int k = threadIdx.x; k < int(gridDim.x); k += blockDim.x) {
    srr += __ldcg(&scratch[k]);
    sbb += __ldcg(&scratch[kMaxParts + k]);
  }
  srr = block_sum(srr, sh);
  sbb = block_sum(sbb, sh);
  if (threadIdx.x == 0) {
    if (sbb == 0.0) sbb = 1.0;  // hecmw_rel_resid_L2_33: b.b = 0 counts as 1
    scratch[kResult] = sqrt(srr / sbb);
    *counter = 0u;
  }
}

// Device address of the scratch array on the current device (looked up once).
cudaError_t scratch_on_current_device(double **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    double *p = nullptr;
    e = cudaGetSymbolAddress(reinterpret_cast<void **>(&p), g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" {

HECMW33_API void hecmw33_gpu_rel_resid_noalloc(const int *N, const int *d_indexL, const int *d_itemL,
                                               const int *d_indexU, const int *d_itemU, const double *d_D,
                                               const double *d_AL, const double *d_AU, const double *d_X,
                                               const double *d_B, double *resid, int *ierr) {
  if (!ierr) return;
  *ierr = 0;
  if (!resid || !d_indexL || !d_itemL || !d_indexU || !d_itemU || !d_D || !d_AL || !d_AU || !d_X || !d_B) {
    h33::set_last_error("hecmw33_gpu_rel_resid_noalloc: a null pointer among resid and the device arrays");
    *ierr = HECMW33_ERR_BAD_INPUT;
    return;
  }
  const int n = N ? *N : -1;
  if (n <= 0 || n > kMaxRows) {
    h33::set_last_error("hecmw33_gpu_rel_resid_noalloc: N = " + std::to_string(n) + " outside 1.." +
                        std::to_string(kMaxRows) + " (the size of its static scratch array)");
    *ierr = HECMW33_ERR_BAD_INPUT;
    return;
  }
  double *scratch = nullptr;
  cudaError_t e = scratch_on_current_device(&scratch);
  const int grid = (n + kRowsPerCta - 1) / kRowsPerCta;
  if (e == cudaSuccess)  // arrival counter and bad-item count
    e = cudaMemsetAsync(scratch + kCounter, 0, 2 * sizeof(double), 0);
  if (e == cudaSuccess) {
    rel_resid_kernel<<<grid, kRowsPerCta, 0, 0>>>(n, d_indexL, d_itemL, d_indexU, d_itemU, d_D, d_AL, d_AU,
                                                  d_X, d_B, scratch);
    e = cudaGetLastError();
  }
  double tail[3] = {0.0, 0.0, 0.0};  // result, arrival counter, bad-item count
  if (e == cudaSuccess) e = cudaMemcpy(tail, scratch + kResult, sizeof(tail), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    h33::set_last_error(std::string("hecmw33_gpu_rel_resid_noalloc: ") + cudaGetErrorString(e));
    *ierr = HECMW33_ERR_CUDA;
    return;
  }
  unsigned int bad = 0;
  static_assert(sizeof(unsigned int) <= sizeof(double), "bad-item count fits its slot");
  std::memcpy(&bad, &tail[2], sizeof(bad));
  if (bad != 0) {
    h33::set_last_error("hecmw33_gpu_rel_resid_noalloc: " + std::to_string(bad) +
                        " itemL/itemU entries outside 1..N (a matrix with external nodes, NP > N, is not "
                        "accepted)");
    *ierr = HECMW33_ERR_BAD_INPUT;
    return;
  }
  *resid = tail[0];
}

}  // extern "C"
