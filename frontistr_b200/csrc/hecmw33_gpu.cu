// hecmw33_gpu.cu -- host side of the B200 3x3-block CG solver and its C ABI
// (include/hecmw33_gpu.h).
//
// Flow of one hecmw33_gpu_solve call (the drop-in for hecmw_solve,
// hecmw1/src/solver/main/hecmw_solver.f90:9-88, METHOD=1):
//   1. set_matrix: validate the hecmwST arrays, build the sliced block-ELL layout of
//      the unified matrix on first use (symbolic), upload D|AL|AU, pack (numeric).
//   2. zero-RHS test (hecmw_solver_Iterative.f90:284-323), zero-diagonal test (:255-282),
//      preconditioner recycle policy (hecmw_matrix_misc.F90:858-877).
//   3. preconditioner setup per flags 97/98: SSOR (RCM + multicolour ordering,
//      reordered L/U in colour order, diagonal LU), DIAG, or block ILU(0).
//   4. the whole CG loop (hecmw_solver_CG.f90:164-279) runs as ONE CUDA graph launch:
//      a prologue (r = b - A x0, ||b||^2) and a conditional WHILE node whose body is one
//      iteration; the device decides when the loop ends (cudaGraphSetConditional).
//   5. true relative residual and the converged/diverged flags (Iterative.f90:131-157).
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "h33_common.cuh"
#include "h33_kernels.cuh"
#include "h33_setup.h"

namespace h33 {

namespace {

thread_local std::string g_last_error;

// NVTX range for profilers (no-op without a tool attached).
struct Range {
  explicit Range(const char *name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
};

// HECMW33_GRAPH=0 selects stream mode: the same kernels launched from the host in
// chunks of kStreamChunk iterations, the host reading the done flag in between
// (used by profilers that replay single launches).
bool graph_mode() {
  const char *e = std::getenv("HECMW33_GRAPH");
  return !(e && e[0] == '0');
}
constexpr int kStreamChunk = 16;

double wall() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Device copy of a sliced layout plus its values.
template <class T>
struct DevSell {
  int nslices = 0, nslots = 0;
  DevArray<int> row0, nrows, slot0, len, rowlen, col, src;
  DevArray<T> val;
  std::vector<int> group_slice;

  void upload(const SellLayout &L, cudaStream_t s) {
    nslices = L.nslices;
    nslots = int(L.nslots);
    row0.upload(L.row0, s);
    nrows.upload(L.nrows, s);
    slot0.upload(L.slot0, s);
    len.upload(L.len, s);
    rowlen.upload(L.rowlen, s);
    col.upload(L.col, s);
    src.upload(L.src, s);
    val.alloc(size_t(nslots) * 288);
    group_slice = L.group_slice;
  }
  SellView<T> view() const {
    return SellView<T>{nslices, row0.p, nrows.p, slot0.p, len.p, rowlen.p, col.p, val.p};
  }
  void pack(const double *raw, cudaStream_t s, int nsm) {
    if (nslots == 0) return;
    const int total = nslots * 32;
    const int grid = std::min((total + kThreads - 1) / kThreads, nsm * 8);
    pack_sell_kernel<T><<<grid, kThreads, 0, s>>>(val.p, src.p, nslots, raw);
    H33_CUDA(cudaGetLastError());
  }
  size_t bytes() const {
    return row0.bytes() + nrows.bytes() + slot0.bytes() + len.bytes() + rowlen.bytes() + col.bytes() +
           src.bytes() + val.bytes();
  }
};

struct Precond {
  int kind = 0;  // 1 SSOR, 3 DIAG, 10 ILU(0)
  bool valid = false;
  int ncolor_in = 0;
  int generation = 0;
  // colour / level schedules
  DevSell<double> lo, up;
  DevArray<int> perm_fwd, perm_bwd;
  DevArray<double> alu_fwd, alu_bwd;  // SoA, 9 x N
  bool alu_shared = true;
  int ncolor = 0;
  std::vector<int> colorindex, perm;  // SSOR: host copies (0-based)
  DevArray<double> ilu_raw;           // ILU(0) factor blocks, raw numbering
};

struct Solver {
  int device = 0;
  cudaStream_t stream = nullptr;
  int nsm = 148;
  int occ_spmv = 4, occ_sweep = 4, occ_vec = 8;
  // matrix
  bool has_matrix = false;
  int N = 0, NPL = 0, NPU = 0;
  int generation = 0;
  bool zero_diag = false;
  std::vector<int> indexL, itemL, indexU, itemU;
  DevArray<double> raw;
  DevSell<double> A;
  // vectors and scalars
  DevArray<double> b, x, r, z, p, q, w, zp;
  DevArray<double> partials;
  DevArray<CgState> state;
  DevArray<CgParams> params;
  CgParams *h_params = nullptr;
  CgState *h_state = nullptr;
  DevArray<int> d_err;
  Precond pc;
  // graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_key[4] = {-1, -1, -1, -1};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int build_counter = 0;  // monotonic id of preconditioner builds (graph cache key)
  // last-solve record
  int last_iter = 0, last_kernels = 0, kernels_per_iter = 0, prologue_kernels = 0;
  double last_solve_s = 0.0, last_setup_s = 0.0;

  Solver() {
    H33_CUDA(cudaGetDevice(&device));
    H33_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    H33_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    H33_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_spmv, spmv_kernel<double, 2>, kThreads, 0));
    H33_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sweep, sweep_bwd_kernel<double, true>, kThreads, 0));
    H33_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_vec, update_xr_kernel, kThreads, 0));
    occ_spmv = std::max(occ_spmv, 1);
    occ_sweep = std::max(occ_sweep, 1);
    occ_vec = std::max(occ_vec, 1);
    H33_CUDA(cudaMallocHost(&h_params, sizeof(CgParams)));
    H33_CUDA(cudaMallocHost(&h_state, sizeof(CgState)));
    state.alloc(1);
    params.alloc(1);
    d_err.alloc(1);
    H33_CUDA(cudaEventCreate(&ev0));
    H33_CUDA(cudaEventCreate(&ev1));
  }
  ~Solver() {
    drop_graph();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (h_params) cudaFreeHost(h_params);
    if (h_state) cudaFreeHost(h_state);
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
  }
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    graph_key[0] = -1;
  }
  int n3() const { return 3 * N; }
  int grid_vec() const { return std::max(1, std::min((n3() + kThreads - 1) / kThreads, nsm * occ_vec)); }
  int grid_spmv() const {
    const int need = (A.nslices + kWarpsPerCta - 1) / kWarpsPerCta;
    return std::max(1, std::min(need, nsm * occ_spmv));
  }
  int grid_sweep(int nslices) const {
    const int need = (nslices + kWarpsPerCta - 1) / kWarpsPerCta;
    return std::max(1, std::min(need, nsm * occ_sweep));
  }
  void sync() { H33_CUDA(cudaStreamSynchronize(stream)); }
};

std::mutex g_mu;
std::map<int, std::unique_ptr<Solver>> g_handles;
int g_next_handle = 1;

Solver &get(const int *handle) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!handle) throw Failure(HECMW33_ERR_BAD_HANDLE, "null handle");
  auto it = g_handles.find(*handle);
  if (it == g_handles.end()) throw Failure(HECMW33_ERR_BAD_HANDLE, "unknown solver handle");
  return *it->second;
}

// Restores the caller's current device on scope exit.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) H33_CUDA(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// ---------------------------------------------------------------------------
// Matrix upload
void validate(int N, int NP, int NPL, int NPU, const int *indexL, const int *itemL,
              const int *indexU, const int *itemU) {
  if (N <= 0) throw Failure(HECMW33_ERR_BAD_INPUT, "N must be positive");
  if (NP != N) throw Failure(HECMW33_ERR_BAD_INPUT, "NP != N: one GPU domain has no halo nodes");
  if (!indexL || !indexU || (NPL > 0 && !itemL) || (NPU > 0 && !itemU))
    throw Failure(HECMW33_ERR_BAD_INPUT, "null profile array");
  if (indexL[0] != 0 || indexU[0] != 0 || indexL[N] != NPL || indexU[N] != NPU)
    throw Failure(HECMW33_ERR_BAD_INPUT, "indexL/indexU inconsistent with NPL/NPU");
  for (int i = 0; i < N; i++) {
    if (indexL[i + 1] < indexL[i] || indexU[i + 1] < indexU[i])
      throw Failure(HECMW33_ERR_BAD_INPUT, "index arrays must be non-decreasing");
    int prev = 0;
    for (int j = indexL[i]; j < indexL[i + 1]; j++) {
      const int c = itemL[j];
      if (c <= prev || c >= i + 1) throw Failure(HECMW33_ERR_BAD_INPUT, "itemL must be ascending ids < row");
      prev = c;
    }
    prev = i + 1;
    for (int j = indexU[i]; j < indexU[i + 1]; j++) {
      const int c = itemU[j];
      if (c <= prev || c > N) throw Failure(HECMW33_ERR_BAD_INPUT, "itemU must be ascending ids in (row, N]");
      prev = c;
    }
  }
}

void set_matrix(Solver &S, int N, int NP, int NPL, int NPU, const int *indexL, const int *itemL,
                const int *indexU, const int *itemU, const double *D, const double *AL,
                const double *AU, const int *Iarray) {
  const bool symbolic = !S.has_matrix || N != S.N || NPL != S.NPL || NPU != S.NPU || Iarray == nullptr ||
                        Iarray[97] != 0;
  if (symbolic) {
    validate(N, NP, NPL, NPU, indexL, itemL, indexU, itemU);
    S.has_matrix = false;
    S.N = N;
    S.NPL = NPL;
    S.NPU = NPU;
    S.indexL.assign(indexL, indexL + N + 1);
    S.itemL.assign(itemL, itemL + NPL);
    S.indexU.assign(indexU, indexU + N + 1);
    S.itemU.assign(itemU, itemU + NPU);
    Profile prof{N, S.indexL.data(), S.itemL.data(), S.indexU.data(), S.itemU.data()};
    BlockRows rows;
    unified_rows(prof, rows);
    SellLayout lay;
    build_sell(rows, std::vector<int>{0, N}, lay);
    S.A.upload(lay, S.stream);
    const size_t n3 = size_t(3) * N;
    for (auto *v : {&S.b, &S.x, &S.r, &S.z, &S.p, &S.q, &S.w, &S.zp}) v->alloc(n3);
    S.partials.alloc(size_t(std::max(N / 32 + 64, S.nsm * 16)) + 1024);
    S.generation++;
    S.pc.valid = false;
    S.drop_graph();
  }
  const size_t nb = size_t(N) + NPL + NPU;
  S.raw.alloc(9 * nb);
  H33_CUDA(cudaMemcpyAsync(S.raw.p, D, sizeof(double) * 9 * N, cudaMemcpyHostToDevice, S.stream));
  if (NPL)
    H33_CUDA(cudaMemcpyAsync(S.raw.p + 9 * size_t(N), AL, sizeof(double) * 9 * NPL, cudaMemcpyHostToDevice, S.stream));
  if (NPU)
    H33_CUDA(cudaMemcpyAsync(S.raw.p + 9 * (size_t(N) + NPL), AU, sizeof(double) * 9 * NPU,
                             cudaMemcpyHostToDevice, S.stream));
  S.A.pack(S.raw.p, S.stream, S.nsm);
  S.zero_diag = false;
  for (int i = 0; i < N && !S.zero_diag; i++)
    for (int j = 0; j < 3; j++)
      if (std::fabs(D[9 * size_t(i) + 4 * j]) == 0.0) S.zero_diag = true;
  S.has_matrix = true;
  S.sync();
}

// ---------------------------------------------------------------------------
// Preconditioners
void diag_alu(Solver &S, DevArray<double> &alu, const double *blocks, const int *perm, double sigma,
              int lu_done) {
  alu.alloc(size_t(9) * S.N);
  H33_CUDA(cudaMemsetAsync(S.d_err.p, 0, sizeof(int), S.stream));
  const int grid = std::max(1, std::min((S.N + kThreads - 1) / kThreads, S.nsm * 8));
  alu_kernel<double><<<grid, kThreads, 0, S.stream>>>(blocks, perm, S.N, sigma, lu_done, alu.p, S.d_err.p);
  H33_CUDA(cudaGetLastError());
}

void setup_ssor(Solver &S, int ncolor_in, double sigma, bool symbolic) {
  Precond &P = S.pc;
  if (symbolic) {
    Profile prof{S.N, S.indexL.data(), S.itemL.data(), S.indexU.data(), S.itemU.data()};
    std::vector<int> perm_rcm, iperm_rcm, perm, iperm, colorindex;
    ordering_rcm(prof, perm_rcm, iperm_rcm);
    P.ncolor = ordering_mc(prof, perm_rcm, ncolor_in, colorindex, perm, iperm);
    BlockRows lower, upper;
    reordered_rows(prof, perm, iperm, lower, upper);
    SellLayout lo, up;
    build_sell(lower, colorindex, lo);
    build_sell(upper, colorindex, up);
    P.lo.upload(lo, S.stream);
    P.up.upload(up, S.stream);
    P.perm_fwd.upload(perm, S.stream);
    P.colorindex = colorindex;
    P.perm = perm;
    P.alu_shared = true;
  }
  P.lo.pack(S.raw.p, S.stream, S.nsm);
  P.up.pack(S.raw.p, S.stream, S.nsm);
  diag_alu(S, P.alu_fwd, S.raw.p, P.perm_fwd.p, sigma, 0);
}

void setup_bilu0(Solver &S, double sigma, bool symbolic) {
  Precond &P = S.pc;
  Profile prof{S.N, S.indexL.data(), S.itemL.data(), S.indexU.data(), S.itemU.data()};
  if (symbolic) {
    std::vector<int> ord_f, lev_f, ord_b, lev_b;
    level_schedule(prof, true, ord_f, lev_f);
    level_schedule(prof, false, ord_b, lev_b);
    BlockRows lower, upper;
    const int N = S.N, NPL = S.NPL;
    lower.ptr.assign(size_t(N) + 1, 0);
    upper.ptr.assign(size_t(N) + 1, 0);
    for (int pos = 0; pos < N; pos++) {
      const int i = ord_f[pos];
      lower.ptr[pos + 1] = lower.ptr[pos] + (S.indexL[i + 1] - S.indexL[i]);
      const int k = ord_b[pos];
      upper.ptr[pos + 1] = upper.ptr[pos] + (S.indexU[k + 1] - S.indexU[k]);
    }
    lower.col.resize(size_t(lower.ptr[N]));
    lower.src.resize(size_t(lower.ptr[N]));
    upper.col.resize(size_t(upper.ptr[N]));
    upper.src.resize(size_t(upper.ptr[N]));
    for (int pos = 0; pos < N; pos++) {
      const int i = ord_f[pos];
      int64_t w = lower.ptr[pos];
      for (int j = S.indexL[i]; j < S.indexL[i + 1]; j++) {
        lower.col[w] = S.itemL[j] - 1;
        lower.src[w++] = N + j;
      }
      const int k = ord_b[pos];
      w = upper.ptr[pos];
      for (int j = S.indexU[k]; j < S.indexU[k + 1]; j++) {
        upper.col[w] = S.itemU[j] - 1;
        upper.src[w++] = N + NPL + j;
      }
    }
    SellLayout lo, up;
    build_sell(lower, lev_f, lo);
    build_sell(upper, lev_b, up);
    P.lo.upload(lo, S.stream);
    P.up.upload(up, S.stream);
    P.perm_fwd.upload(ord_f, S.stream);
    P.perm_bwd.upload(ord_b, S.stream);
    P.alu_shared = false;
    P.ncolor = 0;
  }
  // numeric factorisation on the host, from the resident values
  const size_t nb = size_t(S.N) + S.NPL + S.NPU;
  std::vector<double> host(9 * nb);
  H33_CUDA(cudaMemcpyAsync(host.data(), S.raw.p, sizeof(double) * host.size(), cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  std::vector<double> Dlu, ALlu, AUlu;
  const int rc = factor_bilu0(prof, host.data(), host.data() + 9 * size_t(S.N),
                              host.data() + 9 * (size_t(S.N) + S.NPL), sigma, Dlu, ALlu, AUlu);
  if (rc) throw Failure(HECMW33_ERR_ILU_ZERO_PIVOT, "block ILU(0): zero pivot (the reference stops here)");
  std::copy(Dlu.begin(), Dlu.end(), host.begin());
  std::copy(ALlu.begin(), ALlu.end(), host.begin() + 9 * size_t(S.N));
  std::copy(AUlu.begin(), AUlu.end(), host.begin() + 9 * (size_t(S.N) + S.NPL));
  P.ilu_raw.upload(host.data(), host.size(), S.stream);
  P.lo.pack(P.ilu_raw.p, S.stream, S.nsm);
  P.up.pack(P.ilu_raw.p, S.stream, S.nsm);
  diag_alu(S, P.alu_fwd, P.ilu_raw.p, P.perm_fwd.p, 1.0, 1);
  diag_alu(S, P.alu_bwd, P.ilu_raw.p, P.perm_bwd.p, 1.0, 1);
  S.sync();
}

// hecmw_mat_recycle_precond_setting (hecmw_matrix_misc.F90:858-877)
void recycle_precond_setting(int *Iarray) {
  int &nrecycle = Iarray[95], &numfact = Iarray[96];
  const int symbfact = Iarray[97], maxrecycle = Iarray[34];
  if (symbfact >= 1) {
    numfact = 1;
    nrecycle = 0;
  } else if (numfact > 1) {
    nrecycle = 0;
    numfact = 1;
  } else if (numfact == 1) {
    if (nrecycle < maxrecycle) {
      numfact = 0;
      nrecycle++;
    } else {
      nrecycle = 0;
    }
  }
}

// hecmw_precond_setup (hecmw_precond.f90:30-58) with the reuse test of each
// preconditioner's setup (e.g. hecmw_precond_SSOR_33.F90:74-82).
void precond_setup(Solver &S, int precond, int ncolor_in, double sigma, int *Iarray) {
  const int kind = precond == 2 ? 1 : precond;
  if (kind != 1 && kind != 3 && kind != 10)
    throw Failure(HECMW33_ERR_INCONS_PC, "PRECOND " + std::to_string(precond) +
                                             " is not available in the GPU drop-in (1, 2, 3, 10 are)");
  Precond &P = S.pc;
  const bool reuse = P.valid && P.kind == kind && Iarray[97] == 0 && Iarray[96] == 0 &&
                     (kind != 1 || P.ncolor_in == ncolor_in);
  if (reuse) return;
  const bool symbolic = !P.valid || P.kind != kind || (kind == 1 && P.ncolor_in != ncolor_in);
  if (symbolic) {
    P = Precond();
  }
  P.kind = kind;
  P.ncolor_in = ncolor_in;
  if (kind == 1) setup_ssor(S, ncolor_in, sigma, symbolic);
  else if (kind == 3) diag_alu(S, P.alu_fwd, S.raw.p, nullptr, sigma, 0);
  else setup_bilu0(S, sigma, symbolic);
  int err = 0;
  H33_CUDA(cudaMemcpyAsync(&err, S.d_err.p, sizeof(int), cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  (void)err;  // a zero pivot in SSOR/DIAG gives Inf entries, as in the reference (no check there)
  P.valid = true;
  if (symbolic) {
    // new device buffers: graphs that captured the old ones must go
    P.generation = ++S.build_counter;
    S.drop_graph();
  }
  Iarray[97] = 0;
  Iarray[96] = 0;
}

// ---------------------------------------------------------------------------
// Launch sequences (captured into graphs or run directly)

// z = M^-1 r, one pass; FUSE_RHO adds the RHO reduction + finisher.
template <bool FUSE_RHO>
void launch_sweep(Solver &S, const double *rin, double *zout, CgState *st) {
  Precond &P = S.pc;
  cudaStream_t s = S.stream;
  if (P.kind == 3) {
    diag_kernel<double, FUSE_RHO><<<S.grid_vec(), kThreads, 0, s>>>(P.alu_fwd.p, S.N, rin, zout, st, S.partials.p);
    return;
  }
  const SellView<double> L = P.lo.view(), U = P.up.view();
  const double *alu_b = P.alu_shared ? P.alu_fwd.p : P.alu_bwd.p;
  const int *perm_b = P.alu_shared ? P.perm_fwd.p : P.perm_bwd.p;
  const int gf = int(P.lo.group_slice.size()) - 1;
  for (int g = 0; g < gf; g++) {
    const int sb = P.lo.group_slice[g], se = P.lo.group_slice[g + 1];
    if (se <= sb) continue;
    sweep_fwd_kernel<double><<<S.grid_sweep(se - sb), kThreads, 0, s>>>(L, P.perm_fwd.p, P.alu_fwd.p, S.N, rin,
                                                                        zout, sb, se, st);
  }
  const int gb = int(P.up.group_slice.size()) - 1;
  int total = 0;
  for (int g = gb - 1; g >= 0; g--) {
    const int sb = P.up.group_slice[g], se = P.up.group_slice[g + 1];
    total += S.grid_sweep(std::max(se - sb, 1));
  }
  int base = 0;
  for (int g = gb - 1; g >= 0; g--) {
    const int sb = P.up.group_slice[g], se = P.up.group_slice[g + 1];
    const int grid = S.grid_sweep(std::max(se - sb, 1));
    // a group without slices still launches (one idle CTA) so that the reduction
    // ticket count stays exact
    sweep_bwd_kernel<double, FUSE_RHO><<<grid, kThreads, 0, s>>>(U, perm_b, alu_b, S.N, rin, zout, sb, se, st,
                                                                 S.partials.p, base, total);
    base += grid;
  }
}

// hecmw_precond_apply (hecmw_precond.f90:86-172): z = M^-1 r with iterPREmax passes.
// When st is given and iterPREmax == 1 the RHO reduction is fused into the sweep;
// otherwise (st given) RHO is computed by a separate dot.
void launch_precond(Solver &S, int iterpremax, const double *r, double *z, CgState *st) {
  cudaStream_t s = S.stream;
  const int n3 = S.n3();
  if (iterpremax <= 0) {
    copy_kernel<<<S.grid_vec(), kThreads, 0, s>>>(r, z, n3, st);
    if (st) dot_kernel<1><<<S.grid_vec(), kThreads, 0, s>>>(r, z, n3, st, S.partials.p, 0, 0);
    return;
  }
  if (iterpremax == 1) {
    if (st) launch_sweep<true>(S, r, z, st);
    else launch_sweep<false>(S, r, z, nullptr);
    return;
  }
  const double *in = r;
  for (int it = 1; it <= iterpremax; it++) {
    launch_sweep<false>(S, in, S.zp.p, st);
    if (it == 1) copy_kernel<<<S.grid_vec(), kThreads, 0, s>>>(S.zp.p, z, n3, st);
    else add_kernel<<<S.grid_vec(), kThreads, 0, s>>>(S.zp.p, z, n3, st);
    if (it == iterpremax) break;
    spmv_kernel<double, 1><<<S.grid_spmv(), kThreads, 0, s>>>(S.A.view(), z, S.w.p, r, nullptr, nullptr);
    in = S.w.p;
  }
  if (st) dot_kernel<1><<<S.grid_vec(), kThreads, 0, s>>>(r, z, n3, st, S.partials.p, 0, 0);
}

void launch_prologue(Solver &S, cudaGraphConditionalHandle h, int use_cond) {
  cudaStream_t s = S.stream;
  CgState *st = S.state.p;
  cg_init_kernel<<<1, 32, 0, s>>>(st, S.params.p);
  spmv_kernel<double, 1><<<S.grid_spmv(), kThreads, 0, s>>>(S.A.view(), S.x.p, S.r.p, S.b.p, nullptr, nullptr);
  dot_kernel<0><<<S.grid_vec(), kThreads, 0, s>>>(S.b.p, S.b.p, S.n3(), st, S.partials.p, h, use_cond);
}

void launch_iteration(Solver &S, int iterpremax, cudaGraphConditionalHandle h, int use_cond) {
  cudaStream_t s = S.stream;
  CgState *st = S.state.p;
  const int n3 = S.n3();
  iter_begin_kernel<<<1, 32, 0, s>>>(st, h, use_cond);
  launch_precond(S, iterpremax, S.r.p, S.z.p, st);
  update_p_kernel<<<S.grid_vec(), kThreads, 0, s>>>(S.z.p, S.p.p, n3, st);
  spmv_kernel<double, 2><<<S.grid_spmv(), kThreads, 0, s>>>(S.A.view(), S.p.p, S.q.p, nullptr, st, S.partials.p);
  update_xr_kernel<<<S.grid_vec(), kThreads, 0, s>>>(S.x.p, S.p.p, S.r.p, S.q.p, n3, st, S.partials.p);
  resid_ctl_kernel<double><<<S.grid_spmv(), kThreads, 0, s>>>(S.A.view(), S.x.p, S.r.p, S.b.p, st, S.partials.p,
                                                              h, use_cond);
}

void build_graph(Solver &S, int iterpremax) {
  const int key[4] = {S.generation, S.pc.generation, S.pc.kind, iterpremax};
  if (S.exec && std::equal(key, key + 4, S.graph_key)) return;
  S.drop_graph();
  cudaGraph_t g = nullptr;
  H33_CUDA(cudaGraphCreate(&g, 0));
  S.graph = g;
  cudaGraphConditionalHandle h;
  H33_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
  // prologue
  H33_CUDA(cudaStreamBeginCaptureToGraph(S.stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  launch_prologue(S, h, 1);
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  H33_CUDA(cudaStreamGetCaptureInfo(S.stream, &cs, nullptr, nullptr, &deps, &ndeps));
  std::vector<cudaGraphNode_t> dep(deps, deps + ndeps);
  cudaGraph_t g2 = nullptr;
  H33_CUDA(cudaStreamEndCapture(S.stream, &g2));
  // WHILE node whose body is one CG iteration
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  H33_CUDA(cudaGraphAddNode(&cnode, g, dep.data(), dep.size(), &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  H33_CUDA(cudaStreamBeginCaptureToGraph(S.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  launch_iteration(S, iterpremax, h, 1);
  cudaGraph_t b2 = nullptr;
  H33_CUDA(cudaStreamEndCapture(S.stream, &b2));
  H33_CUDA(cudaGraphInstantiate(&S.exec, g, 0));
  std::copy(key, key + 4, S.graph_key);
  size_t nbody = 0, nall = 0;
  H33_CUDA(cudaGraphGetNodes(body, nullptr, &nbody));
  H33_CUDA(cudaGraphGetNodes(g, nullptr, &nall));
  S.kernels_per_iter = int(nbody);
  S.prologue_kernels = int(nall) - 1;  // minus the conditional node
}

// Relative residual ||b - A x|| / ||b|| on the device (hecmw_rel_resid_L2_33).
double rel_resid_device(Solver &S) {
  cudaStream_t s = S.stream;
  CgState *st = S.state.p;
  spmv_kernel<double, 1><<<S.grid_spmv(), kThreads, 0, s>>>(S.A.view(), S.x.p, S.w.p, S.b.p, nullptr, nullptr);
  dot_kernel<2><<<S.grid_vec(), kThreads, 0, s>>>(S.w.p, S.w.p, S.n3(), st, S.partials.p, 0, 0);
  double rr = 0.0;
  H33_CUDA(cudaMemcpyAsync(&rr, &st->rr_true, sizeof(double), cudaMemcpyDeviceToHost, s));
  S.sync();
  double bb = S.h_state->bnrm2;
  if (bb == 0.0) bb = 1.0;
  return std::sqrt(rr / bb);
}

double dot_device(Solver &S, const double *a, const double *b) {
  CgState *st = S.state.p;
  dot_kernel<2><<<S.grid_vec(), kThreads, 0, S.stream>>>(a, b, S.n3(), st, S.partials.p, 0, 0);
  double v = 0.0;
  H33_CUDA(cudaMemcpyAsync(&v, &st->rr_true, sizeof(double), cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  return v;
}

// The hecmw_solve / hecmw_solve_iterative sequence on resident B (S.b) and X (S.x).
int solve_resident(Solver &S, int *Iarray, double *Rarray, int *iter, double *resid, double *times) {
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix: call hecmw33_gpu_set_matrix first");
  const double t0 = wall();
  *iter = 0;
  *resid = 0.0;
  if (times) times[0] = times[1] = times[2] = 0.0;
  // zero right-hand side (hecmw_solver.f90:32-37)
  const double bb = dot_device(S, S.b.p, S.b.p);
  if (bb == 0.0) {
    H33_CUDA(cudaMemsetAsync(S.x.p, 0, sizeof(double) * S.n3(), S.stream));
    S.sync();
    Iarray[80] = 1;
    Iarray[81] = 0;
    return HECMW33_ERR_ZERO_RHS;
  }
  const int MAXIT = Iarray[0], METHOD = Iarray[1], PRECOND = Iarray[2], iterPREmax = Iarray[4];
  const int NCOLOR_IN = Iarray[33];
  const double TOL = Rarray[0];
  double sigma = Rarray[1];
  const bool auto_sigma = sigma < 0.0;
  if (auto_sigma) sigma = 1.0;
  if (S.zero_diag && PRECOND < 10 && iterPREmax > 0) return HECMW33_ERR_ZERO_DIAG;
  if (METHOD != 1)
    throw Failure(HECMW33_ERR_INCONS_PC, "METHOD " + std::to_string(METHOD) + ": the GPU drop-in implements CG (1)");
  recycle_precond_setting(Iarray);
  {
    Range rg("hecmw33_precond_setup");
    if (iterPREmax > 0) precond_setup(S, PRECOND, NCOLOR_IN, sigma, Iarray);
    if (graph_mode()) build_graph(S, iterPREmax);
  }
  Range rs("hecmw33_solve");
  const double t1 = wall();
  int error = 0;
  float ms_total = 0.0f;
  const bool use_graph = graph_mode();
  for (;;) {
    Iarray[80] = 0;
    Iarray[81] = 0;
    S.h_params->tol = TOL;
    S.h_params->maxit = MAXIT;
    S.h_params->iterpremax = iterPREmax;
    H33_CUDA(cudaMemcpyAsync(S.params.p, S.h_params, sizeof(CgParams), cudaMemcpyHostToDevice, S.stream));
    H33_CUDA(cudaEventRecord(S.ev0, S.stream));
    if (use_graph) {
      H33_CUDA(cudaGraphLaunch(S.exec, S.stream));
      H33_CUDA(cudaEventRecord(S.ev1, S.stream));
      H33_CUDA(cudaMemcpyAsync(S.h_state, S.state.p, sizeof(CgState), cudaMemcpyDeviceToHost, S.stream));
      S.sync();
    } else {
      launch_prologue(S, 0, 0);
      for (int done = 0, it = 0; !done && it <= MAXIT + kStreamChunk; it += kStreamChunk) {
        for (int k = 0; k < kStreamChunk; k++) launch_iteration(S, iterPREmax, 0, 0);
        H33_CUDA(cudaGetLastError());
        H33_CUDA(cudaMemcpyAsync(S.h_state, S.state.p, sizeof(CgState), cudaMemcpyDeviceToHost, S.stream));
        S.sync();
        done = S.h_state->done;
      }
      H33_CUDA(cudaEventRecord(S.ev1, S.stream));
      S.sync();
    }
    float ms = 0.0f;
    H33_CUDA(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
    ms_total += ms;
    const CgState &st = *S.h_state;
    error = st.error;
    if (!st.done && !st.zero_rhs)
      throw Failure(HECMW33_ERR_TIMEOUT, "device CG loop ended without a decision (internal error)");
    *iter = st.iter;
    *resid = st.resid;
    if (st.zero_rhs) {  // not reached after the host-side test, kept for completeness
      *iter = 0;
      *resid = 0.0;
    }
    if (error == HECMW33_ERR_DIVERGE_PC || error == HECMW33_ERR_DIVERGE_MAT || error == HECMW33_ERR_DIVERGE_NAN) {
      Iarray[81] = 1;
      // Iterative.f90:133-137; the reference's retry reuses the factorisation
      // already built (flags 97/98 are cleared), continuing from the current X
      if (PRECOND >= 10 && PRECOND < 20 && auto_sigma && sigma < 2.0) {
        sigma = sigma + 0.1;
        continue;
      }
    }
    break;
  }
  const double resid2 = rel_resid_device(S);
  if (resid2 < TOL) Iarray[80] = 1;
  {
    // launches: zero-RHS dot, per graph launch the prologue plus one body per
    // executed iteration (iterations that stopped early still launched the body),
    // and the true-residual SpMV + dot
    const int executed = std::min(S.h_state->iter, MAXIT);
    S.last_iter = *iter;
    S.last_kernels = 1 + S.prologue_kernels + std::max(executed, 0) * S.kernels_per_iter + 2;
    S.last_solve_s = ms_total * 1e-3;
    S.last_setup_s = t1 - t0;
  }
  if (times) {
    times[0] = t1 - t0;
    times[1] = ms_total * 1e-3;
    times[2] = 0.0;
  }
  return error;
}

void fail(int *ierr, int code, const char *msg) {
  g_last_error = msg;
  if (ierr) *ierr = code;
}

}  // namespace

}  // namespace h33

using namespace h33;

#define H33_ENTRY_BEGIN \
  try {
#define H33_ENTRY_END                                           \
  }                                                             \
  catch (const Failure &f) {                                    \
    fail(ierr, f.code, f.what());                               \
  }                                                             \
  catch (const std::bad_alloc &) {                              \
    fail(ierr, HECMW33_ERR_CUDA, "host allocation failed");     \
  }                                                             \
  catch (const std::exception &e) {                             \
    fail(ierr, HECMW33_ERR_CUDA, e.what());                     \
  }

extern "C" {

HECMW33_API void hecmw33_gpu_create(int *handle, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  auto s = std::make_unique<Solver>();
  std::lock_guard<std::mutex> lk(g_mu);
  const int id = g_next_handle++;
  g_handles[id] = std::move(s);
  *handle = id;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_destroy(const int *handle, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  std::unique_ptr<Solver> victim;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = handle ? g_handles.find(*handle) : g_handles.end();
    if (it == g_handles.end()) throw Failure(HECMW33_ERR_BAD_HANDLE, "unknown solver handle");
    victim = std::move(it->second);
    g_handles.erase(it);
  }
  DeviceGuard dg(victim->device);
  victim.reset();
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_set_matrix(const int *handle, const int *N, const int *NP, const int *NPL,
                                        const int *NPU, const int *indexL, const int *itemL,
                                        const int *indexU, const int *itemU, const double *D,
                                        const double *AL, const double *AU, const int *Iarray,
                                        int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  set_matrix(S, *N, *NP, *NPL, *NPU, indexL, itemL, indexU, itemU, D, AL, AU, Iarray);
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_solve_resident(const int *handle, const double *B, double *X, int *Iarray,
                                            double *Rarray, int *iter, double *resid, double *times,
                                            int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix: call hecmw33_gpu_set_matrix first");
  const size_t bytes = sizeof(double) * S.n3();
  H33_CUDA(cudaMemcpyAsync(S.b.p, B, bytes, cudaMemcpyHostToDevice, S.stream));
  H33_CUDA(cudaMemcpyAsync(S.x.p, X, bytes, cudaMemcpyHostToDevice, S.stream));
  const int rc = solve_resident(S, Iarray, Rarray, iter, resid, times);
  H33_CUDA(cudaMemcpyAsync(X, S.x.p, bytes, cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  if (ierr) *ierr = rc;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_solve_resident_device(const int *handle, const double *dB, double *dX,
                                                   int *Iarray, double *Rarray, int *iter,
                                                   double *resid, double *times, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix: call hecmw33_gpu_set_matrix first");
  const size_t bytes = sizeof(double) * S.n3();
  H33_CUDA(cudaMemcpyAsync(S.b.p, dB, bytes, cudaMemcpyDeviceToDevice, S.stream));
  H33_CUDA(cudaMemcpyAsync(S.x.p, dX, bytes, cudaMemcpyDeviceToDevice, S.stream));
  const int rc = solve_resident(S, Iarray, Rarray, iter, resid, times);
  H33_CUDA(cudaMemcpyAsync(dX, S.x.p, bytes, cudaMemcpyDeviceToDevice, S.stream));
  S.sync();
  if (ierr) *ierr = rc;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_solve(const int *handle, const int *N, const int *NP, const int *NPL,
                                   const int *NPU, const int *indexL, const int *itemL, const int *indexU,
                                   const int *itemU, const double *D, const double *AL, const double *AU,
                                   const double *B, double *X, int *Iarray, double *Rarray, int *iter,
                                   double *resid, double *times, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  const double t0 = wall();
  set_matrix(S, *N, *NP, *NPL, *NPU, indexL, itemL, indexU, itemU, D, AL, AU, Iarray);
  const double tm = wall() - t0;
  const size_t bytes = sizeof(double) * S.n3();
  H33_CUDA(cudaMemcpyAsync(S.b.p, B, bytes, cudaMemcpyHostToDevice, S.stream));
  H33_CUDA(cudaMemcpyAsync(S.x.p, X, bytes, cudaMemcpyHostToDevice, S.stream));
  const int rc = solve_resident(S, Iarray, Rarray, iter, resid, times);
  H33_CUDA(cudaMemcpyAsync(X, S.x.p, bytes, cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  if (times) times[0] += tm;
  if (ierr) *ierr = rc;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_matvec(const int *handle, const double *X, double *Y, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix: call hecmw33_gpu_set_matrix first");
  const size_t bytes = sizeof(double) * S.n3();
  H33_CUDA(cudaMemcpyAsync(S.w.p, X, bytes, cudaMemcpyHostToDevice, S.stream));
  spmv_kernel<double, 0><<<S.grid_spmv(), kThreads, 0, S.stream>>>(S.A.view(), S.w.p, S.zp.p, nullptr, nullptr,
                                                                    nullptr);
  H33_CUDA(cudaGetLastError());
  H33_CUDA(cudaMemcpyAsync(Y, S.zp.p, bytes, cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_precond_apply(const int *handle, const double *R, double *Z, int *Iarray,
                                           double *Rarray, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix: call hecmw33_gpu_set_matrix first");
  const int iterPREmax = Iarray[4];
  double sigma = Rarray[1];
  if (sigma < 0.0) sigma = 1.0;
  if (iterPREmax > 0) precond_setup(S, Iarray[2], Iarray[33], sigma, Iarray);
  const size_t bytes = sizeof(double) * S.n3();
  H33_CUDA(cudaMemcpyAsync(S.r.p, R, bytes, cudaMemcpyHostToDevice, S.stream));
  launch_precond(S, iterPREmax, S.r.p, S.z.p, nullptr);
  H33_CUDA(cudaGetLastError());
  H33_CUDA(cudaMemcpyAsync(Z, S.z.p, bytes, cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_get_colouring(const int *handle, int *ncolor, int *colorindex, int *perm,
                                           int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  if (!S.pc.valid || S.pc.kind != 1) throw Failure(HECMW33_ERR_NO_MATRIX, "no SSOR preconditioner built");
  *ncolor = S.pc.ncolor;
  for (int c = 0; c <= S.pc.ncolor; c++) colorindex[c] = S.pc.colorindex[c];
  for (int i = 0; i < S.N; i++) perm[i] = S.pc.perm[i] + 1;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_colour_schedule(const int *N, const int *indexL, const int *itemL,
                                             const int *indexU, const int *itemU, const int *ncolor_in,
                                             int *ncolor, int *colorindex, int *perm, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  const int n = *N;
  validate(n, n, indexL[n], indexU[n], indexL, itemL, indexU, itemU);
  Profile prof{n, indexL, itemL, indexU, itemU};
  std::vector<int> perm_rcm, iperm_rcm, pm, ipm, ci;
  ordering_rcm(prof, perm_rcm, iperm_rcm);
  *ncolor = ordering_mc(prof, perm_rcm, *ncolor_in, ci, pm, ipm);
  for (int c = 0; c <= *ncolor; c++) colorindex[c] = ci[c];
  for (int i = 0; i < n; i++) perm[i] = pm[i] + 1;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_last_solve_info(const int *handle, int *info, double *dinfo, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  for (int i = 0; i < 8; i++) {
    info[i] = 0;
    dinfo[i] = 0.0;
  }
  info[0] = S.last_iter;
  info[1] = S.last_kernels;
  info[2] = S.pc.valid ? int(S.pc.lo.group_slice.size() + S.pc.up.group_slice.size()) - 2 : 0;
  info[3] = S.kernels_per_iter;
  const double N = S.N, NPL = S.NPL, NPU = S.NPU, NZ = N + NPL + NPU;
  info[4] = int(NZ);
  info[5] = S.A.nslices;
  info[6] = S.A.nslots;
  dinfo[0] = S.last_solve_s;
  dinfo[1] = S.last_setup_s;
  const double spmv = 72.0 * NZ + 4.0 * (NPL + NPU) + 8.0 * (N + 1) + 24.0 * N + 24.0 * N;
  // SSOR sweeps: off-diagonal blocks + their columns once, diagonal LU twice, two
  // vector passes each way; vector updates: r, z, p, q, x (minimum fused traffic)
  const double sweeps = 72.0 * (NPL + NPU) + 4.0 * (NPL + NPU) + 2.0 * 72.0 * N + 2.0 * 4.0 * 2.0 * (N + 1) +
                        2.0 * 2.0 * 24.0 * N;
  const double vec = 10.0 * 24.0 * N;
  dinfo[2] = spmv;
  dinfo[3] = spmv + sweeps + vec;
  size_t held = S.raw.bytes() + S.A.bytes() + S.pc.lo.bytes() + S.pc.up.bytes() + S.pc.alu_fwd.bytes() +
                S.pc.alu_bwd.bytes() + S.pc.ilu_raw.bytes();
  for (auto *v : {&S.b, &S.x, &S.r, &S.z, &S.p, &S.q, &S.w, &S.zp}) held += v->bytes();
  dinfo[4] = double(held);
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_time_spmv(const int *handle, const int *reps, double *ms_per_launch, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix");
  const int n = std::max(1, *reps);
  spmv_kernel<double, 0><<<S.grid_spmv(), kThreads, 0, S.stream>>>(S.A.view(), S.x.p, S.zp.p, nullptr, nullptr, nullptr);
  H33_CUDA(cudaEventRecord(S.ev0, S.stream));
  for (int i = 0; i < n; i++)
    spmv_kernel<double, 0><<<S.grid_spmv(), kThreads, 0, S.stream>>>(S.A.view(), S.x.p, S.zp.p, nullptr, nullptr,
                                                                      nullptr);
  H33_CUDA(cudaGetLastError());
  H33_CUDA(cudaEventRecord(S.ev1, S.stream));
  S.sync();
  float ms = 0.0f;
  H33_CUDA(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
  *ms_per_launch = double(ms) / n;
  H33_ENTRY_END
}

HECMW33_API int hecmw33_gpu_last_error(char *buf, int len) {
  const int n = int(g_last_error.size());
  if (buf && len > 0) {
    const int m = std::min(n, len - 1);
    std::memcpy(buf, g_last_error.data(), size_t(m));
    buf[m] = 0;
  }
  return n;
}

}  // extern "C"
