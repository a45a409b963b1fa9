// hecmw33_batch.cu -- batched solves: many independent systems (the diagonal blocks
// of one hecmwST matrix) in one persistent, graph-captured launch (h33_batch.cuh),
// with a launch-schedule autotuner whose choices are kept in a JSON-lines cache.
//
// No counterpart in the reference beyond the per-system algorithm: each system is
// solved as hecmw_solve would solve it alone (hecmw_solver.f90:9-88 with
// hecmw_solve_CG, hecmw_solver_CG.f90:19-289, and the SSOR_33 / DIAG_33
// preconditioners in the reference's ordering).
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "h33_batch.cuh"
#include "h33_common.cuh"
#include "h33_setup.h"

namespace h33 {
void set_last_error(const std::string &msg);  // message for hecmw33_gpu_last_error

namespace {

double bwall() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct DevSellB {
  int nslices = 0, nslots = 0, lanes = 1;
  DevArray<int> row0, nrows, slot0, len, rowlen, col, src;
  DevArray<double> val;
  void upload(const SellLayout &L, cudaStream_t s) {
    nslices = L.nslices;
    lanes = L.lanes;
    nslots = int(L.nslots);
    row0.upload(L.row0, s);
    nrows.upload(L.nrows, s);
    slot0.upload(L.slot0, s);
    len.upload(L.len, s);
    rowlen.upload(L.rowlen, s);
    col.upload(L.col, s);
    src.upload(L.src, s);
    val.alloc(size_t(std::max(nslots, 1)) * 288);
  }
  void pack(const double *raw, cudaStream_t s, int nsm) {
    if (nslots == 0) return;
    const int total = nslots * 32;
    const int grid = std::min((total + kThreads - 1) / kThreads, nsm * 8);
    pack_sell_kernel<double><<<grid, kThreads, 0, s>>>(val.p, src.p, nslots, raw);
    H33_CUDA(cudaGetLastError());
  }
  SellView<double> view() const {
    return SellView<double>{nslices, row0.p, nrows.p, slot0.p, len.p, rowlen.p, col.p, val.p};
  }
  size_t bytes() const {
    return row0.bytes() + nrows.bytes() + slot0.bytes() + len.bytes() + rowlen.bytes() + col.bytes() + src.bytes() +
           val.bytes();
  }
};

// Launch schedule: lanes per row of the sweep layouts (rows per warp = 32 / lanes),
// cluster size of the big-system teams and the share of systems (by estimated work,
// largest first) that teams take.
struct Schedule {
  int lanes = 8;
  int cluster = 4;
  double big_frac = 0.15;
};

struct Batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  int nsm = 148;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // problem
  bool ready = false;
  int nsys = 0, N = 0, NPL = 0, NPU = 0;
  std::vector<int> node0;  // nsys + 1
  std::vector<int> indexL, itemL, indexU, itemU;
  std::vector<int> zero_diag;  // per system
  // preconditioner build parameters
  int kind = 0, ncolor_in = -1, lanes_built = 0;
  double sigma = 1.0;
  std::vector<std::vector<int>> colour_rows;  // per system: colour boundaries (local positions)
  std::vector<int> perm_h;                    // global position -> node
  // device data
  DevArray<double> raw, alu;
  DevSellB A, lo, up;
  DevArray<int> lo_gs, up_gs, perm, d_err;
  std::vector<BatchSys> sys_h;
  DevArray<BatchSys> sys_d;
  DevArray<int> big, small, queue;
  DevArray<BatchOut> out;
  BatchOut *h_out = nullptr;
  DevArray<BatchArgs> d_args;
  BatchArgs *h_args = nullptr;
  DevArray<double> b, x, r, z, p, q;
  // schedule and statistics
  Schedule sched;
  bool tuned = false;
  std::vector<int> last_iter;  // per system, from the previous solve (work estimate)
  int grid = 0, nbig = 0, nsmall = 0;
  float last_ms = 0.0f;
  double last_setup_s = 0.0;
  // the graph of one solve (queue reset + persistent kernel)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int gkey[4] = {-1, -1, -1, -1};

  Batch() {
    H33_CUDA(cudaGetDevice(&device));
    H33_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    H33_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    H33_CUDA(cudaEventCreate(&ev0));
    H33_CUDA(cudaEventCreate(&ev1));
    queue.alloc(2);
    d_err.alloc(1);
    d_args.alloc(1);
    H33_CUDA(cudaMallocHost(&h_args, sizeof(BatchArgs)));
  }
  ~Batch() {
    drop_graph();
    if (h_out) cudaFreeHost(h_out);
    if (h_args) cudaFreeHost(h_args);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
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
    gkey[0] = -1;
  }
  void sync() { H33_CUDA(cudaStreamSynchronize(stream)); }
};

std::mutex g_bmu;
std::map<int, std::unique_ptr<Batch>> g_batches;
int g_next_batch = 1;

Batch &get_batch(const int *h) {
  std::lock_guard<std::mutex> lk(g_bmu);
  if (!h) throw Failure(HECMW33_ERR_BAD_HANDLE, "null batch handle");
  auto it = g_batches.find(*h);
  if (it == g_batches.end()) throw Failure(HECMW33_ERR_BAD_HANDLE, "unknown batch handle");
  return *it->second;
}

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) H33_CUDA(cudaSetDevice(dev));
  }
  ~DevGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// The profile of system s renumbered to its own nodes (1-based ids).
struct SubProfile {
  std::vector<int> indexL, itemL, indexU, itemU;
  Profile view(int n) const { return Profile{n, indexL.data(), itemL.data(), indexU.data(), itemU.data()}; }
};

SubProfile sub_profile(const Batch &B, int s) {
  const int a = B.node0[s], e = B.node0[s + 1], n = e - a;
  SubProfile sp;
  sp.indexL.resize(size_t(n) + 1);
  sp.indexU.resize(size_t(n) + 1);
  const int l0 = B.indexL[a], u0 = B.indexU[a];
  for (int i = 0; i <= n; i++) {
    sp.indexL[i] = B.indexL[a + i] - l0;
    sp.indexU[i] = B.indexU[a + i] - u0;
  }
  sp.itemL.resize(size_t(B.indexL[e] - l0));
  sp.itemU.resize(size_t(B.indexU[e] - u0));
  for (size_t j = 0; j < sp.itemL.size(); j++) sp.itemL[j] = B.itemL[l0 + j] - a;
  for (size_t j = 0; j < sp.itemU.size(); j++) sp.itemU[j] = B.itemU[u0 + j] - a;
  return sp;
}

// Symbolic setup of the preconditioner layouts for `lanes` lanes per row: per-system
// orderings (in parallel, once), one global position order (system by system), the
// sliced lower / upper layouts whose groups are the systems' colours.
void build_precond_layout(Batch &B, int lanes) {
  const int nsys = B.nsys;
  Profile prof{B.N, B.indexL.data(), B.itemL.data(), B.indexU.data(), B.itemU.data()};
  if (B.colour_rows.size() != size_t(nsys) || B.lanes_built == 0) {
    B.perm_h.assign(size_t(B.N), 0);
    B.colour_rows.assign(size_t(nsys), {});
    std::vector<std::vector<int>> perms(static_cast<size_t>(nsys));
#pragma omp parallel for schedule(dynamic)
    for (int s = 0; s < nsys; s++) {
      const int n = B.node0[s + 1] - B.node0[s];
      if (B.kind == 3) {
        perms[s].resize(size_t(n));
        std::iota(perms[s].begin(), perms[s].end(), 0);
        B.colour_rows[s] = {0, n};
        continue;
      }
      const SubProfile sp = sub_profile(B, s);
      const Profile p = sp.view(n);
      std::vector<int> pr, ipr, pm, ipm, ci;
      ordering_rcm(p, pr, ipr);
      ordering_mc(p, pr, B.ncolor_in, ci, pm, ipm);
      perms[s] = pm;
      B.colour_rows[s] = ci;
    }
    for (int s = 0; s < nsys; s++)
      for (size_t i = 0; i < perms[s].size(); i++) B.perm_h[B.node0[s] + i] = B.node0[s] + perms[s][i];
  }
  std::vector<int> iperm(static_cast<size_t>(B.N), 0);
  for (int i = 0; i < B.N; i++) iperm[B.perm_h[i]] = i;
  std::vector<int> group_rows{0};
  for (int s = 0; s < nsys; s++) {
    B.sys_h[s].g0 = int(group_rows.size()) - 1;
    for (size_t c = 1; c < B.colour_rows[s].size(); c++) group_rows.push_back(B.node0[s] + B.colour_rows[s][c]);
    B.sys_h[s].g1 = int(group_rows.size()) - 1;
  }
  BlockRows lower, upper;
  if (B.kind == 3) {
    lower.ptr.assign(size_t(B.N) + 1, 0);
    upper.ptr.assign(size_t(B.N) + 1, 0);
  } else {
    reordered_rows(prof, B.perm_h, iperm, lower, upper);
  }
  SellLayout lo, up;
  build_sell(lower, group_rows, lo, lanes);
  build_sell(upper, group_rows, up, lanes);
  B.lo.upload(lo, B.stream);
  B.up.upload(up, B.stream);
  B.lo_gs.upload(lo.group_slice, B.stream);
  B.up_gs.upload(up.group_slice, B.stream);
  B.perm.upload(B.perm_h, B.stream);
  B.lanes_built = lanes;
  B.lo.pack(B.raw.p, B.stream, B.nsm);
  B.up.pack(B.raw.p, B.stream, B.nsm);
  B.alu.alloc(size_t(9) * B.N);
  H33_CUDA(cudaMemsetAsync(B.d_err.p, 0, sizeof(int), B.stream));
  const int g = std::max(1, std::min((B.N + kThreads - 1) / kThreads, B.nsm * 8));
  alu_kernel<double><<<g, kThreads, 0, B.stream>>>(B.raw.p, B.perm.p, B.N, B.sigma, 0, B.alu.p, B.d_err.p);
  H33_CUDA(cudaGetLastError());
  B.sys_d.upload(B.sys_h, B.stream);
  B.drop_graph();
  B.sync();
}

void batch_set_matrix(Batch &B, int nsys, const int *sys_ptr, int N, int NP, int NPL, int NPU, const int *indexL,
                      const int *itemL, const int *indexU, const int *itemU, const double *D, const double *AL,
                      const double *AU, const int *Iarray, const double *Rarray) {
  const double t0 = bwall();
  if (nsys < 1 || !sys_ptr) throw Failure(HECMW33_ERR_BAD_INPUT, "nsys must be positive");
  const std::string msg = check_profile(N, NP, NPL, NPU, indexL, itemL, indexU, itemU);
  if (!msg.empty()) throw Failure(HECMW33_ERR_BAD_INPUT, msg);
  if (sys_ptr[0] != 0 || sys_ptr[nsys] != N) throw Failure(HECMW33_ERR_BAD_INPUT, "sys_ptr must run from 0 to N");
  for (int s = 0; s < nsys; s++)
    if (sys_ptr[s + 1] <= sys_ptr[s]) throw Failure(HECMW33_ERR_BAD_INPUT, "every system needs at least one node");
  // block-diagonal: the blocks of a row stay inside its system (items are sorted)
  for (int s = 0; s < nsys; s++)
    for (int i = sys_ptr[s]; i < sys_ptr[s + 1]; i++) {
      if (indexL[i + 1] > indexL[i] && itemL[indexL[i]] - 1 < sys_ptr[s])
        throw Failure(HECMW33_ERR_BAD_INPUT, "matrix couples two systems (itemL)");
      if (indexU[i + 1] > indexU[i] && itemU[indexU[i + 1] - 1] - 1 >= sys_ptr[s + 1])
        throw Failure(HECMW33_ERR_BAD_INPUT, "matrix couples two systems (itemU)");
    }
  const int PRECOND = Iarray ? Iarray[2] : 1;
  const int kind = (PRECOND == 1 || PRECOND == 2) ? 1 : PRECOND;
  if (kind != 1 && kind != 3)
    throw Failure(HECMW33_ERR_INCONS_PC, "PRECOND " + std::to_string(PRECOND) +
                                             ": batched solves use SSOR (1, 2) or DIAG (3)");
  const int ncolor_in = Iarray ? Iarray[33] : 10;
  double sigma = Rarray ? Rarray[1] : 1.0;
  if (sigma < 0.0) sigma = 1.0;
  const bool symbolic = !B.ready || N != B.N || NPL != B.NPL || NPU != B.NPU || nsys != B.nsys ||
                        !std::equal(sys_ptr, sys_ptr + nsys + 1, B.node0.begin()) || kind != B.kind ||
                        (kind == 1 && ncolor_in != B.ncolor_in) || (Iarray && Iarray[97] != 0);
  B.sigma = sigma;
  if (symbolic) {
    B.ready = false;
    B.nsys = nsys;
    B.N = N;
    B.NPL = NPL;
    B.NPU = NPU;
    B.kind = kind;
    B.ncolor_in = ncolor_in;
    B.node0.assign(sys_ptr, sys_ptr + nsys + 1);
    B.indexL.assign(indexL, indexL + N + 1);
    B.itemL.assign(itemL, itemL + NPL);
    B.indexU.assign(indexU, indexU + N + 1);
    B.itemU.assign(itemU, itemU + NPU);
    B.colour_rows.clear();
    B.lanes_built = 0;
    B.last_iter.assign(size_t(nsys), 0);
    Profile prof{N, B.indexL.data(), B.itemL.data(), B.indexU.data(), B.itemU.data()};
    BlockRows rows;
    unified_rows(prof, rows);
    SellLayout lay;
    build_sell(rows, B.node0, lay, 1);  // groups = systems: no slice straddles two
    B.A.upload(lay, B.stream);
    B.sys_h.assign(size_t(nsys), BatchSys{});
    for (int s = 0; s < nsys; s++) {
      BatchSys &y = B.sys_h[s];
      y.n = sys_ptr[s + 1] - sys_ptr[s];
      y.node0 = sys_ptr[s];
      y.a0 = lay.group_slice[s];
      y.a1 = lay.group_slice[s + 1];
    }
    const size_t n3 = size_t(3) * N;
    for (auto *v : {&B.b, &B.x, &B.r, &B.z, &B.p, &B.q}) v->alloc(n3);
    B.out.alloc(size_t(nsys));
    if (B.h_out) cudaFreeHost(B.h_out);
    B.h_out = nullptr;
    H33_CUDA(cudaMallocHost(&B.h_out, sizeof(BatchOut) * nsys));
    B.big.alloc(size_t(nsys));
    B.small.alloc(size_t(nsys));
  }
  const size_t nb = size_t(N) + NPL + NPU;
  B.raw.alloc(9 * nb);
  H33_CUDA(cudaMemcpyAsync(B.raw.p, D, sizeof(double) * 9 * N, cudaMemcpyHostToDevice, B.stream));
  if (NPL)
    H33_CUDA(cudaMemcpyAsync(B.raw.p + 9 * size_t(N), AL, sizeof(double) * 9 * NPL, cudaMemcpyHostToDevice, B.stream));
  if (NPU)
    H33_CUDA(cudaMemcpyAsync(B.raw.p + 9 * (size_t(N) + NPL), AU, sizeof(double) * 9 * NPU, cudaMemcpyHostToDevice,
                             B.stream));
  B.A.pack(B.raw.p, B.stream, B.nsm);
  B.zero_diag.assign(size_t(nsys), 0);
  for (int s = 0; s < nsys; s++)
    for (int i = sys_ptr[s]; i < sys_ptr[s + 1] && !B.zero_diag[s]; i++)
      for (int j = 0; j < 3; j++)
        if (std::fabs(D[9 * size_t(i) + 4 * j]) == 0.0) B.zero_diag[s] = 1;
  if (symbolic) {
    build_precond_layout(B, B.sched.lanes);
  } else {
    // values only: repack the sweep layouts and refactor the diagonal blocks
    B.lo.pack(B.raw.p, B.stream, B.nsm);
    B.up.pack(B.raw.p, B.stream, B.nsm);
    const int g = std::max(1, std::min((N + kThreads - 1) / kThreads, B.nsm * 8));
    alu_kernel<double><<<g, kThreads, 0, B.stream>>>(B.raw.p, B.perm.p, N, B.sigma, 0, B.alu.p, B.d_err.p);
    H33_CUDA(cudaGetLastError());
  }
  B.ready = true;
  B.sync();
  B.last_setup_s = bwall() - t0;
}

// ---- autotuner cache (JSON lines: {"key": ..., "lanes": L, "cluster": C, "big_frac": f, "ms": t})
std::string cache_path() {
  const char *e = std::getenv("HECMW33_AUTOTUNE_CACHE");
  if (e && *e) return e;
  const char *home = std::getenv("HOME");
  return std::string(home ? home : ".") + "/.cache/frontistr_b200_autotune.jsonl";
}

std::string batch_key(const Batch &B, int iterpremax) {
  // the schedule depends on the device, the system sizes and the preconditioner
  uint64_t h = 1469598103934665603ull;
  for (int v : B.node0) h = (h ^ uint64_t(v)) * 1099511628211ull;
  char buf[256];
  std::snprintf(buf, sizeof(buf), "batch:sm%d:n%d:nz%d:sys%d:pc%d:pre%d:%016llx", B.nsm, B.N, B.N + B.NPL + B.NPU,
                B.nsys, B.kind, iterpremax, (unsigned long long)h);
  return buf;
}

bool valid_schedule(int lanes, int cluster, double bf) {
  return (lanes == 2 || lanes == 4 || lanes == 8 || lanes == 16) &&
         (cluster == 1 || cluster == 2 || cluster == 4 || cluster == 8) && bf >= 0.0 && bf <= 1.0;
}

bool cache_load(const std::string &key, Schedule &s) {
  FILE *f = std::fopen(cache_path().c_str(), "r");
  if (!f) return false;
  char line[2048];
  bool found = false;
  const std::string tag = "\"key\": \"" + key + "\"";
  while (std::fgets(line, sizeof(line), f)) {
    const std::string t(line);
    if (t.find(tag) == std::string::npos) continue;
    const size_t a = t.find("\"lanes\": "), c = t.find("\"cluster\": "), b = t.find("\"big_frac\": ");
    if (a == std::string::npos || c == std::string::npos || b == std::string::npos) continue;
    const int lanes = std::atoi(t.c_str() + a + 9);
    const int cl = std::atoi(t.c_str() + c + 11);
    const double bf = std::atof(t.c_str() + b + 12);
    if (valid_schedule(lanes, cl, bf)) {
      s = Schedule{lanes, cl, bf};
      found = true;  // the last matching line wins
    }
  }
  std::fclose(f);
  return found;
}

void cache_store(const std::string &key, const Schedule &s, double ms) {
  FILE *f = std::fopen(cache_path().c_str(), "a");
  if (!f) return;  // no writable cache: the schedule is kept for this handle only
  std::fprintf(f, "{\"key\": \"%s\", \"lanes\": %d, \"cluster\": %d, \"big_frac\": %.3f, \"ms\": %.4f}\n",
               key.c_str(), s.lanes, s.cluster, s.big_frac, ms);
  std::fclose(f);
}

// ---- one solve
cudaLaunchConfig_t launch_config(Batch &B, int cluster, int grid, cudaLaunchAttribute *attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(grid), 1, 1);
  cfg.blockDim = dim3(kThreads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = B.stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = unsigned(cluster);
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

template <int K>
void launch_batch_k(Batch &B, const BatchArgs *a, int cluster, int grid) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = launch_config(B, cluster, grid, attr);
  H33_CUDA(cudaLaunchKernelEx(&cfg, batch_cg_kernel<K>, a));
}

// CTAs of the persistent grid: as many clusters as can be resident at once.
template <int K>
int resident_grid(Batch &B, int cluster) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = launch_config(B, cluster, cluster * B.nsm, attr);
  int ncl = 0;
  H33_CUDA(cudaOccupancyMaxActiveClusters(&ncl, batch_cg_kernel<K>, &cfg));
  return std::max(1, ncl) * cluster;
}

void launch_batch(Batch &B, const BatchArgs *a, int cluster, int grid) {
  switch (B.lanes_built) {
    case 2: return launch_batch_k<2>(B, a, cluster, grid);
    case 4: return launch_batch_k<4>(B, a, cluster, grid);
    case 16: return launch_batch_k<16>(B, a, cluster, grid);
    default: return launch_batch_k<8>(B, a, cluster, grid);
  }
}

int batch_grid(Batch &B, int cluster) {
  switch (B.lanes_built) {
    case 2: return resident_grid<2>(B, cluster);
    case 4: return resident_grid<4>(B, cluster);
    case 16: return resident_grid<16>(B, cluster);
    default: return resident_grid<8>(B, cluster);
  }
}

// Queues for this solve: systems by decreasing estimated work (blocks x expected
// iterations: the previous solve's count, else a size-based guess); the first
// big_frac of them go to cluster teams when cluster > 1.
void make_queues(Batch &B, const Schedule &sc) {
  std::vector<std::pair<double, int>> w;
  for (int s = 0; s < B.nsys; s++) {
    if (B.sys_h[s].skip) continue;
    const int a = B.node0[s], e = B.node0[s + 1];
    const double blocks = double(e - a) + double(B.indexL[e] - B.indexL[a]) + double(B.indexU[e] - B.indexU[a]);
    const double it = B.last_iter[s] > 0 ? double(B.last_iter[s]) : 10.0 * std::cbrt(double(e - a));
    w.push_back({blocks * it, s});
  }
  std::stable_sort(w.begin(), w.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
  const int n = int(w.size());
  int nbig = sc.cluster > 1 ? int(std::lround(sc.big_frac * n)) : 0;
  nbig = std::min(std::max(nbig, 0), n);
  std::vector<int> big(static_cast<size_t>(std::max(nbig, 1))), small(static_cast<size_t>(std::max(n - nbig, 1)));
  for (int i = 0; i < nbig; i++) big[i] = w[i].second;
  for (int i = nbig; i < n; i++) small[i - nbig] = w[i].second;
  H33_CUDA(cudaMemcpyAsync(B.big.p, big.data(), sizeof(int) * big.size(), cudaMemcpyHostToDevice, B.stream));
  H33_CUDA(cudaMemcpyAsync(B.small.p, small.data(), sizeof(int) * small.size(), cudaMemcpyHostToDevice, B.stream));
  B.sync();  // the host vectors go out of scope
  B.nbig = nbig;
  B.nsmall = n - nbig;
}

// One batched solve on resident b/x with schedule sc; returns the device ms.
float run_batch(Batch &B, const Schedule &sc, int iterpremax, double tol, int maxit) {
  if (B.lanes_built != sc.lanes) build_precond_layout(B, sc.lanes);
  for (int s = 0; s < B.nsys; s++) B.sys_h[s].skip = (B.zero_diag[s] && iterpremax > 0) ? 1 : 0;
  B.sys_d.upload(B.sys_h, B.stream);
  make_queues(B, sc);
  const int grid = batch_grid(B, sc.cluster);
  BatchArgs a;
  a.A = B.A.view();
  a.lo = B.lo.view();
  a.up = B.up.view();
  a.lo_gs = B.lo_gs.p;
  a.up_gs = B.up_gs.p;
  a.perm = B.perm.p;
  a.alu = B.alu.p;
  a.npos = B.N;
  a.kind = B.kind;
  a.iterpremax = iterpremax;
  a.sys = B.sys_d.p;
  a.big = B.big.p;
  a.small = B.small.p;
  a.nbig = B.nbig;
  a.nsmall = B.nsmall;
  a.queue = B.queue.p;
  a.b = B.b.p;
  a.x = B.x.p;
  a.r = B.r.p;
  a.z = B.z.p;
  a.p = B.p.p;
  a.q = B.q.p;
  a.out = B.out.p;
  a.tol = tol;
  a.maxit = maxit;
  *B.h_args = a;
  H33_CUDA(cudaMemcpyAsync(B.d_args.p, B.h_args, sizeof(BatchArgs), cudaMemcpyHostToDevice, B.stream));
  // the solve as one graph: queue reset + the persistent kernel (its arguments are
  // read from d_args, so the graph depends only on the launch shape)
  const int key[4] = {sc.lanes, sc.cluster, grid, 0};
  if (!(B.exec && std::equal(key, key + 4, B.gkey))) {
    B.drop_graph();
    H33_CUDA(cudaStreamBeginCapture(B.stream, cudaStreamCaptureModeThreadLocal));
    H33_CUDA(cudaMemsetAsync(B.queue.p, 0, 2 * sizeof(int), B.stream));
    launch_batch(B, B.d_args.p, sc.cluster, grid);
    H33_CUDA(cudaStreamEndCapture(B.stream, &B.graph));
    H33_CUDA(cudaGraphInstantiate(&B.exec, B.graph, 0));
    std::copy(key, key + 4, B.gkey);
  }
  B.grid = grid;
  H33_CUDA(cudaEventRecord(B.ev0, B.stream));
  H33_CUDA(cudaGraphLaunch(B.exec, B.stream));
  H33_CUDA(cudaEventRecord(B.ev1, B.stream));
  H33_CUDA(cudaMemcpyAsync(B.h_out, B.out.p, sizeof(BatchOut) * B.nsys, cudaMemcpyDeviceToHost, B.stream));
  B.sync();
  float ms = 0.0f;
  H33_CUDA(cudaEventElapsedTime(&ms, B.ev0, B.ev1));
  return ms;
}

struct Flags {
  int iterpremax, maxit;
  double tol;
};

Flags check_flags(Batch &B, const int *Iarray, const double *Rarray) {
  if (!B.ready) throw Failure(HECMW33_ERR_NO_MATRIX, "no batch matrix: call hecmw33_gpu_batch_set_matrix first");
  if (Iarray[1] != 1)
    throw Failure(HECMW33_ERR_INCONS_PC, "METHOD " + std::to_string(Iarray[1]) + ": the GPU drop-in implements CG (1)");
  const int PRECOND = Iarray[2];
  const int kind = (PRECOND == 1 || PRECOND == 2) ? 1 : PRECOND;
  if (kind != B.kind || (kind == 1 && Iarray[33] != B.ncolor_in))
    throw Failure(HECMW33_ERR_INCONS_PC, "PRECOND / ncolor_in differ from hecmw33_gpu_batch_set_matrix's");
  if (Iarray[4] > 1) throw Failure(HECMW33_ERR_INCONS_PC, "batched solves take iterPREmax 0 or 1");
  return Flags{Iarray[4], Iarray[0], Rarray[0]};
}

int collect(Batch &B, int *iter, double *resid, int *error, double *true_resid, int *Iarray) {
  int rc = 0, conv = 1, div = 0;
  for (int s = 0; s < B.nsys; s++) {
    if (B.sys_h[s].skip) {
      iter[s] = 0;
      resid[s] = 0.0;
      error[s] = HECMW33_ERR_ZERO_DIAG;
      if (true_resid) true_resid[s] = 1.0;
      conv = 0;
    } else {
      const BatchOut &o = B.h_out[s];
      iter[s] = o.iter;
      resid[s] = o.resid;
      error[s] = o.error;
      if (true_resid) true_resid[s] = o.true_resid;
      B.last_iter[s] = o.iter;
      if (!o.converged) conv = 0;
    }
    if (error[s] == HECMW33_ERR_DIVERGE_PC || error[s] == HECMW33_ERR_DIVERGE_MAT ||
        error[s] == HECMW33_ERR_DIVERGE_NAN)
      div = 1;
    if (!rc && error[s] != 0 && error[s] != HECMW33_ERR_ZERO_RHS) rc = error[s];
  }
  Iarray[80] = conv;
  Iarray[81] = div;
  return rc;
}

void load_bx(Batch &B, const double *Bv, const double *X, bool device) {
  const size_t bytes = sizeof(double) * 3 * size_t(B.N);
  const cudaMemcpyKind k = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  H33_CUDA(cudaMemcpyAsync(B.b.p, Bv, bytes, k, B.stream));
  H33_CUDA(cudaMemcpyAsync(B.x.p, X, bytes, k, B.stream));
}

void store_x(Batch &B, double *X, bool device) {
  const size_t bytes = sizeof(double) * 3 * size_t(B.N);
  H33_CUDA(cudaMemcpyAsync(X, B.x.p, bytes, device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, B.stream));
  B.sync();
}

// Autotune on the caller's B/X: one warm solve (it sets the per-system iteration
// counts that order the queues), then one timed solve per schedule, each from the
// same X (X itself is not modified); the fastest is kept.  Coordinate search: the
// cluster size with every system given to teams, the team share at the best size,
// then the lanes at the best of those (9 timed solves; the full grid of sizes and
// shares took 13).  Layout rebuilds and graph captures happen outside the timed
// region.
double autotune(Batch &B, const Flags &f, const double *Bv, const double *X, bool device) {
  const int L0 = B.sched.lanes;
  auto note_iters = [&]() {
    for (int s = 0; s < B.nsys; s++)
      if (!B.sys_h[s].skip) B.last_iter[s] = B.h_out[s].iter;
  };
  load_bx(B, Bv, X, device);
  run_batch(B, B.sched, f.iterpremax, f.tol, f.maxit);
  note_iters();
  double best_ms = 1e300;
  Schedule best = B.sched;
  auto trial = [&](const Schedule &sc) {
    load_bx(B, Bv, X, device);
    const float ms = run_batch(B, sc, f.iterpremax, f.tol, f.maxit);
    if (ms < best_ms) {
      best_ms = ms;
      best = sc;
    }
  };
  trial(Schedule{L0, 1, 0.0});
  for (int c : {2, 4, 8}) trial(Schedule{L0, c, 1.0});
  if (best.cluster > 1) {
    const int c = best.cluster;
    for (double bf : {0.1, 0.25, 0.5}) trial(Schedule{L0, c, bf});
  }
  for (int L : {4, 8, 16}) {
    if (L == L0) continue;
    Schedule sc = best;
    sc.lanes = L;
    trial(sc);
  }
  B.sched = best;
  B.tuned = true;
  return best_ms;
}

int batch_solve(Batch &B, const double *Bv, double *X, bool device, int *Iarray, double *Rarray, int *iter,
                double *resid, int *error, double *true_resid, double *times) {
  const Flags f = check_flags(B, Iarray, Rarray);
  const double t0 = bwall();
  // HECMW33_BATCH_SCHEDULE="lanes,cluster,big_frac" fixes the schedule (experiments)
  if (const char *e = std::getenv("HECMW33_BATCH_SCHEDULE")) {
    int L = 0, C = 0;
    double bf = -1.0;
    if (std::sscanf(e, "%d,%d,%lf", &L, &C, &bf) == 3 && valid_schedule(L, C, bf)) {
      B.sched = Schedule{L, C, bf};
      B.tuned = true;
    }
  }
  if (!B.tuned) {
    Schedule sc = B.sched;
    if (cache_load(batch_key(B, f.iterpremax), sc)) {
      B.sched = sc;
      B.tuned = true;
    }
  }
  load_bx(B, Bv, X, device);
  nvtxRangePushA("hecmw33_batch_solve");
  const float ms = run_batch(B, B.sched, f.iterpremax, f.tol, f.maxit);
  nvtxRangePop();
  B.last_ms = ms;
  store_x(B, X, device);
  if (times) {
    times[0] = bwall() - t0 - ms * 1e-3;
    times[1] = ms * 1e-3;
    times[2] = 0.0;
  }
  return collect(B, iter, resid, error, true_resid, Iarray);
}

void fail(int *ierr, int code, const char *msg) {
  set_last_error(msg);
  if (ierr) *ierr = code;
}

}  // namespace
}  // namespace h33

using namespace h33;

#define HB_BEGIN try {
#define HB_END                                              \
  }                                                         \
  catch (const Failure &f) {                                \
    fail(ierr, f.code, f.what());                           \
  }                                                         \
  catch (const std::bad_alloc &) {                          \
    fail(ierr, HECMW33_ERR_CUDA, "host allocation failed"); \
  }                                                         \
  catch (const std::exception &e) {                         \
    fail(ierr, HECMW33_ERR_CUDA, e.what());                 \
  }

extern "C" {

HECMW33_API void hecmw33_gpu_batch_create(int *handle, int *ierr) {
  if (ierr) *ierr = 0;
  HB_BEGIN
  auto b = std::make_unique<Batch>();
  std::lock_guard<std::mutex> lk(g_bmu);
  const int id = g_next_batch++;
  g_batches[id] = std::move(b);
  *handle = id;
  HB_END
}

HECMW33_API void hecmw33_gpu_batch_destroy(const int *handle, int *ierr) {
  if (ierr) *ierr = 0;
  HB_BEGIN
  std::unique_ptr<Batch> victim;
  {
    std::lock_guard<std::mutex> lk(g_bmu);
    auto it = handle ? g_batches.find(*handle) : g_batches.end();
    if (it == g_batches.end()) throw Failure(HECMW33_ERR_BAD_HANDLE, "unknown batch handle");
    victim = std::move(it->second);
    g_batches.erase(it);
  }
  DevGuard dg(victim->device);
  victim.reset();
  HB_END
}

HECMW33_API void hecmw33_gpu_batch_set_matrix(const int *handle, const int *nsys, const int *sys_ptr, const int *N,
                                              const int *NP, const int *NPL, const int *NPU, const int *indexL,
                                              const int *itemL, const int *indexU, const int *itemU, const double *D,
                                              const double *AL, const double *AU, const int *Iarray,
                                              const double *Rarray, int *ierr) {
  if (ierr) *ierr = 0;
  HB_BEGIN
  Batch &B = get_batch(handle);
  DevGuard dg(B.device);
  batch_set_matrix(B, *nsys, sys_ptr, *N, *NP, *NPL, *NPU, indexL, itemL, indexU, itemU, D, AL, AU, Iarray, Rarray);
  HB_END
}

HECMW33_API void hecmw33_gpu_batch_solve(const int *handle, const double *B, double *X, int *Iarray, double *Rarray,
                                         int *iter, double *resid, int *error, double *true_resid, double *times,
                                         int *ierr) {
  if (ierr) *ierr = 0;
  HB_BEGIN
  Batch &Bt = get_batch(handle);
  DevGuard dg(Bt.device);
  const int rc = batch_solve(Bt, B, X, false, Iarray, Rarray, iter, resid, error, true_resid, times);
  if (ierr) *ierr = rc;
  HB_END
}

HECMW33_API void hecmw33_gpu_batch_solve_device(const int *handle, const double *dB, double *dX, int *Iarray,
                                                double *Rarray, int *iter, double *resid, int *error,
                                                double *true_resid, double *times, int *ierr) {
  if (ierr) *ierr = 0;
  HB_BEGIN
  Batch &Bt = get_batch(handle);
  DevGuard dg(Bt.device);
  const int rc = batch_solve(Bt, dB, dX, true, Iarray, Rarray, iter, resid, error, true_resid, times);
  if (ierr) *ierr = rc;
  HB_END
}

HECMW33_API void hecmw33_gpu_batch_autotune(const int *handle, const double *B, const double *X, const int *Iarray,
                                            const double *Rarray, int *ierr) {
  if (ierr) *ierr = 0;
  HB_BEGIN
  Batch &Bt = get_batch(handle);
  DevGuard dg(Bt.device);
  const Flags f = check_flags(Bt, Iarray, Rarray);
  const double ms = autotune(Bt, f, B, X, false);
  cache_store(batch_key(Bt, f.iterpremax), Bt.sched, ms);
  HB_END
}

HECMW33_API void hecmw33_gpu_batch_info(const int *handle, int *info, double *dinfo, int *ierr) {
  if (ierr) *ierr = 0;
  HB_BEGIN
  Batch &B = get_batch(handle);
  for (int i = 0; i < 16; i++) {
    info[i] = 0;
    dinfo[i] = 0.0;
  }
  info[0] = B.sched.lanes;
  info[1] = B.sched.cluster;
  info[2] = B.nbig;
  info[3] = B.nsmall;
  info[4] = B.grid;
  info[5] = B.tuned ? 1 : 0;
  info[6] = B.nsys;
  info[7] = 1;  // kernels per solve (the persistent kernel)
  long long total_iter = 0;
  int max_iter = 0;
  for (int s = 0; s < B.nsys; s++) {
    total_iter += B.last_iter[s];
    max_iter = std::max(max_iter, B.last_iter[s]);
  }
  info[8] = int(std::min<long long>(total_iter, 2147483647ll));
  info[9] = max_iter;
  dinfo[0] = B.last_ms * 1e-3;
  dinfo[1] = B.last_setup_s;
  dinfo[2] = B.sched.big_frac;
  const size_t held = B.raw.bytes() + B.alu.bytes() + B.A.bytes() + B.lo.bytes() + B.up.bytes() + 6 * B.b.bytes();
  dinfo[3] = double(held);
  HB_END
}

}  // extern "C"
