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
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <cmath>
#include <cstring>
#include <map>
#include <type_traits>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "h33_assemble.cuh"
#include "h33_bicg.cuh"
#include "h33_coarse.cuh"
#include "h33_common.cuh"
#include "h33_cr.cuh"
#include "h33_domain.cuh"
#include "h33_gmres.cuh"
#include "h33_gnn.cuh"
#include "h33_kernels.cuh"
#include "h33_layout.cuh"
#include "h33_multi.cuh"
#include "h33_setup.h"
#include "h33_vecops.cuh"

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

// Programmatic dependent launch for every kernel of the solver, opt-in with
// HECMW33_PDL=1: a kernel may be scheduled while its predecessor drains and waits on
// the device (pdl_entry) for the predecessor's results.  Measured on the 100^3 cube it
// changes nothing (0.808 s with, 0.809 s without; stream launches 0.815 s): the
// iteration is bound by the kernels themselves, not by the gaps between them.
bool pdl_mode() {
  const char *e = std::getenv("HECMW33_PDL");
  return e && e[0] == '1';
}

// colour_prologue's mode for the SSOR colour launches of values stored as TV: every
// launch is programmatic (the next colour starts its static work while this one
// drains), and that work brings into L2 the columns -- the head of each slot's
// chain of dependent loads -- with the values where they are BF16, with the
// diagonal LU entries where the values are wider.
// Measured on the 100^3 cube (FP64 / mode-1 solve, s): none 0.741 / 0.622;
// programmatic only 0.736 / 0.622; + values, columns and LU 0.781 / 0.604; FP64 with
// columns 0.719, LU 0.731, columns and LU 0.715; BF16 with values 0.612, columns
// 0.607, columns and LU 0.607, values and columns 0.600.  Prefetching the FP64
// values crowds the vectors out of L2 (their slot ranges are 4x the BF16 ones).
template <class TV>
constexpr int sweep_pre() {
  return sizeof(TV) <= 2 ? (1 | 2 | 4) : (1 | 4 | 8);
}

// level_prologue's mode for the node-order level launches of the block ILU sweeps:
// programmatic launches whose static work, before the wait for the previous level,
// brings into L2 the level's values, columns and diagonal LU entries (a level of the
// natural-order schedule is a few MB, far from crowding the vectors out of L2).
// HECMW33_LEVEL_PRE overrides it (0 = plain launches).
template <class TV>
int level_pre() {
  static const int v = [] {
    const char *e = std::getenv("HECMW33_LEVEL_PRE");
    return e ? std::atoi(e) : (1 | 2 | 4 | 8);
  }();
  return v;
}

// HECMW33_MR_TILED=1: the multi-RHS loop's SpMM stages p through shared memory
// (mr_spmm_tiled_kernel).  Opt-in: on the 100^3 cube with 16 load cases it measured
// 4.06 s against 3.77 s untiled -- a CTA waits for its tile's copies before it
// computes, and the ~60 KB tile leaves room for three CTAs per SM, too few to hide
// that wait.
bool mr_tiled_mode() {
  const char *e = std::getenv("HECMW33_MR_TILED");
  return e && e[0] == '1';
}

template <typename... KArgs, typename... Args>
void launch_ks(cudaStream_t s, void (*kern)(KArgs...), int grid, int block, size_t smem, Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(grid), 1, 1);
  cfg.blockDim = dim3(unsigned(block), 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_mode() ? 1 : 0;
  H33_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
}

// As launch_k, with programmatic stream serialisation on or off explicitly.
template <typename... KArgs, typename... Args>
void launch_kp(cudaStream_t s, bool pdl, void (*kern)(KArgs...), int grid, int block, Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(grid), 1, 1);
  cfg.blockDim = dim3(unsigned(block), 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  H33_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
}

template <typename... KArgs, typename... Args>
void launch_k(cudaStream_t s, void (*kern)(KArgs...), int grid, int block, Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(grid), 1, 1);
  cfg.blockDim = dim3(unsigned(block), 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_mode() ? 1 : 0;
  H33_CUDA(cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...));
}

// Lanes per row of the preconditioner sweep layouts (HECMW33_SWEEP_LANES overrides;
// 4, 8 or 16).  Several lanes per row shorten each row's dependent load
// chain and multiply the warps of a colour, which the sweeps need: a colour holds
// a tenth of the rows, too few one-lane rows to cover HBM latency.
int sweep_lanes() {
  const char *e = std::getenv("HECMW33_SWEEP_LANES");
  const int k = e ? std::atoi(e) : 4;
  return (k == 4 || k == 8 || k == 16) ? k : 4;
}

double wall() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// HECMW33_SETUP_TRACE=1 prints the wall time of each setup phase (host orderings,
// layouts, uploads, device packing, graph capture) on stderr, the device synchronised
// at every mark so that a phase owns its own device work.  Off: one branch per mark.
void setup_mark(const char *what) {
  static const bool on = [] {
    const char *e = std::getenv("HECMW33_SETUP_TRACE");
    return e && e[0] == '1';
  }();
  static double last = 0.0;
  if (!on) return;
  cudaDeviceSynchronize();
  const double t = wall();
  std::fprintf(stderr, "[setup] %-36s %9.1f ms\n", what, last > 0.0 ? 1e3 * (t - last) : 0.0);
  last = t;
}

// Device copy of a sliced layout plus its values.
template <class T>
struct DevSell {
  int nslices = 0, nslots = 0;
  DevArray<int> row0, nrows, slot0, len, rowlen, col, src;
  DevArray<T> val;
  DevArray<float> val32;  // FP32 copy of val (mixed precision), same layout
  DevArray<__nv_bfloat16> val16;  // BF16 copy of val (low-precision preconditioner), same layout
  std::vector<int> group_slice, group_rows;
  std::vector<int> run_ptr, run_slice, run_slot, run_len;  // run tables (multicolour SSOR layouts)

  int lanes = 1;
  void upload(const SellLayout &L, cudaStream_t s) {
    upload_shape(L, s);
    H33_CUDA(cudaMemcpyAsync(col.p, L.col.data(), col.bytes(), cudaMemcpyHostToDevice, s));
    H33_CUDA(cudaMemcpyAsync(src.p, L.src.data(), src.bytes(), cudaMemcpyHostToDevice, s));
  }
  // Everything but the blocks' columns and raw ids, which a fill kernel writes into
  // col and src (cleared here to the padding: column 0, raw id -1).
  void upload_shape(const SellLayout &L, cudaStream_t s) {
    nslices = L.nslices;
    lanes = L.lanes;
    nslots = int(L.nslots);
    row0.upload(L.row0, s);
    nrows.upload(L.nrows, s);
    slot0.upload(L.slot0, s);
    len.upload(L.len, s);
    rowlen.upload(L.rowlen, s);
    col.alloc(size_t(nslots) * 32);
    src.alloc(size_t(nslots) * 32);
    col.zero(s);
    if (src.n) H33_CUDA(cudaMemsetAsync(src.p, 0xff, src.bytes(), s));
    val.alloc(size_t(nslots) * 288);
    group_slice = L.group_slice;
    run_ptr = L.run_ptr;
    run_slice = L.run_slice;
    run_slot = L.run_slot;
    run_len = L.run_len;
  }
  SellView<T> view() const {
    return SellView<T>{nslices, row0.p, nrows.p, slot0.p, len.p, rowlen.p, col.p, val.p};
  }
  SellView<float> view32() const {
    return SellView<float>{nslices, row0.p, nrows.p, slot0.p, len.p, rowlen.p, col.p, val32.p};
  }
  SellView<__nv_bfloat16> view16() const {
    return SellView<__nv_bfloat16>{nslices, row0.p, nrows.p, slot0.p, len.p, rowlen.p, col.p, val16.p};
  }
  void pack(const double *raw, cudaStream_t s, int nsm) {
    if (nslots == 0) return;
    const int total = nslots * 32;
    const int grid = std::min((total + kThreads - 1) / kThreads, nsm * 8);
    launch_k(s, pack_sell_kernel<T>, grid, kThreads, val.p, src.p, nslots, raw);
    H33_CUDA(cudaGetLastError());
  }
  size_t bytes() const {
    return row0.bytes() + nrows.bytes() + slot0.bytes() + len.bytes() + rowlen.bytes() + col.bytes() +
           src.bytes() + val.bytes() + val32.bytes() + val16.bytes();
  }
};

struct Precond {
  int kind = 0;  // 1 SSOR, 3 DIAG, 10 block ILU(p)
  int ilu_level = 0;   // p of the block ILU (PRECOND 10, 11, 12)
  FilledProfile fill;  // its factor pattern when p > 0
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
  DevArray<double> ilu_raw;           // block ILU factor blocks: D | L | U in factor-pattern order
  DevArray<float> alu32_fwd, alu32_bwd;
  int numeric_version = 0, fp32_version = -1, lowp_version = -1;
  bool pos_cols = false;  // lo/up columns are colour positions (multicolour SSOR)
  double sigma = 0.0;     // SIGMA_DIAG of the last numeric setup
};

// The learned preconditioner: node graph of the matrix, weights, activations and
// the (r, e) pairs recorded from earlier solves (training data).
struct Learned {
  int graph_generation = -1, feat_version = -1;
  int n = 0, nedges = 0;
  DevArray<int> ptr, col, rev, src;
  DevArray<float> feat, s;
  bool have_weights = false;
  int weights_version = 0;
  int adam_step = 0;
  DevArray<float> theta, m1, m2, grad, gacc;
  DevArray<__nv_bfloat16> theta_bf16;
  DevArray<int> row_of;
  int built_for = -1, w_version = -1;
  DevArray<float> w, x, h[4], m[3], gm, dh, dhp, part;
  int nparts = 0, stride = 0;
  DevArray<float> t_z, t_zs, t_d, t_q, t_dz;  // training scratch (3N)
  // recorded pairs (FP32): r_k, e_k, SSOR(r_k) and e_k.r_k
  bool recording = false;
  int max_pairs = 16;
  std::vector<DevArray<float>> pr, pe, pzs;
  std::vector<double> per;
  DevArray<double> losses;
  GnnGraph graph() const { return GnnGraph{n, nedges, ptr.p, col.p, rev.p, feat.p, s.p}; }
  // the smoother of the two-grid cycle: SSOR on its own layouts in first-fit colour
  // order, rebuilt with the matrix structure (symbolic) and with every numeric setup
  // of the solve's SSOR (same SIGMA_DIAG)
  Precond sm;
  int sm_built_for = -1, sm_numeric_for = -1;
  // the coarse space the network shapes (h33_coarse.cuh): aggregation and patterns
  // (per matrix structure), prolongator, A P, dense coarse inverse (per matrix values
  // and weights), application and training vectors
  // coarse smoothing weights: 0 the network's omega, 1 omega = 0 (unsmoothed
  // aggregation), 2 omega = 1/2 everywhere (the untrained network's output)
  int coarse_mode = 0;
  struct Coarse {
    int built_for = -1, mask_version = -1, t0_version = -1;
    int op_precond = -1, op_weights = -1, op_mode = -1;  // what the coarse inverse was built from
    bool ok = false;                                    // coarse inverse usable
    int n = 0, nagg = 0, nc = 0;
    DevArray<int> agg, pptr, pagg, rptr, rnode, rpos, qptr, qagg, cptr, cagg, uptr, ucol, usrc;
    DevArray<float> mask, x, out, omega, dout;
    DevArray<double> t0, p, q, ac, gjc, gjb, gjd, bc, y, v, t0y, apy, dots;
    DevArray<float> p32, q32, ainv32;  // FP32 copies for the application in a solve
    DevArray<int> err;
    float *one = nullptr;  // device 1.0f (the decode scale of the backward pass)
    DevArray<float> one_buf;
    CoarseApply apply_view() {
      return CoarseApply{n, nagg, nc, pptr.p, pagg.p, qptr.p, qagg.p, rptr.p, rnode.p, rpos.p,
                         p32.p, q32.p, ainv32.p};
    }
    CoarseView view() {
      return CoarseView{n,      nagg,   nc,     agg.p,  pptr.p, pagg.p, rptr.p, rnode.p, rpos.p,
                        qptr.p, qagg.p, cptr.p, cagg.p, uptr.p, ucol.p, usrc.p, mask.p,  t0.p,
                        p.p,    q.p,    ac.p};
    }
  } C;
};

// One instantiated CG graph and the key of the device buffers it captured.
struct GraphSlot {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int key[5] = {-1, -1, -1, -1, -1};
  int kernels_per_iter = 0, prologue_kernels = 0;
  void drop() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    key[0] = -1;
  }
};

// One domain of a decomposed mesh (N internal of NP local nodes): the blocks of
// internal rows at external columns, the communication table and the caller's
// exchange / allreduce, the external values of X and of the CG direction, and the
// host staging of the exchanged values.
struct DomainState {
  bool on = false;
  int NP = 0, n_ext = 0, NPL = 0, NPU = 0;
  // A_IE: interface rows (internal row, its blocks at external positions)
  int n_irows = 0;
  std::vector<int> au_src;  // per A_II upper block: its index in the caller's AU
  std::vector<int> ie_src;  // per A_IE block: its index in the caller's AU
  DevArray<int> irow, iptr, icol;
  DevArray<double> ival;
  // communication
  bool has_table = false;
  int n_exp = 0, n_imp = 0;
  DevArray<int> exp_idx, imp_idx;
  DevArray<double> send_d, recv_d, xe_x, xe_p, xe_z;
  double *send_h = nullptr, *recv_h = nullptr;
  hecmw33_exchange_fn exchange = nullptr;
  hecmw33_allreduce_fn allreduce = nullptr;
  void *ctx = nullptr;
  void free_host() {
    if (send_h) cudaFreeHost(send_h);
    if (recv_h) cudaFreeHost(recv_h);
    send_h = recv_h = nullptr;
  }
  void clear_table() {
    has_table = false;
    n_exp = n_imp = 0;
    exchange = nullptr;
    allreduce = nullptr;
    ctx = nullptr;
    free_host();
  }
  void reset() {
    clear_table();
    on = false;
    NP = n_ext = NPL = NPU = n_irows = 0;
    au_src.clear();
    ie_src.clear();
  }
  ~DomainState() { free_host(); }
};

struct Solver {
  int device = 0;
  cudaStream_t stream = nullptr;
  int nsm = 148;
  int occ_spmv = 4, occ_sweep = 4, occ_vec = 8, occ_sweep_uni = 4;
  // matrix
  bool has_matrix = false;
  int N = 0, NPL = 0, NPU = 0;
  int generation = 0;
  bool zero_diag = false;
  std::vector<int> indexL, itemL, indexU, itemU;
  DevArray<int> d_indexL, d_itemL, d_indexU, d_itemU;  // the same profile on the device (layout fills)
  DevArray<double> raw;
  DevSell<double> A;
  // vectors and scalars
  DevArray<double> b, x, r, z, p, q, w, zp;
  DevArray<double> dpos;  // the learned smoother's y - z per colour position (lower_resid_kernel)
  DevArray<double> partials;
  DevArray<CgState> state;
  DevArray<CgParams> params;
  CgParams *h_params = nullptr;
  CgState *h_state = nullptr;
  DevArray<int> d_err;
  Precond pc;
  // FP32 copies for the mixed-precision refinement
  DevArray<float> bf, xf, rf, zf, pf, qf, wf, zpf;
  // flexible CG buffers (SSOR output and previous residual) and the learned preconditioner
  DevArray<double> zs, rold;
  DevArray<float> zsf, roldf;
  DevArray<double> zpos;  // SSOR sweep intermediate in colour-position order (FP64 / FP32)
  DevArray<float> zposf;
  // SCALING=YES: row and column of every raw block, the scaled copy of the raw
  // values and the unscaled right-hand side while a scaled solve runs
  // BiCGSTAB vectors: r_tld, s, s_tld, t ({p_tld} and {v} use z and q)
  DevArray<double> b_rt, b_s, b_st, b_t;
  // GMRES(m): Krylov basis (m+1 vectors), w, zq, av; the small system (H, s, y, ss,
  // scalars) and the breakdown flag
  DevArray<double> g_V, g_w, g_zq, g_av, g_small;
  DevArray<double> gp_W;  // GPBiCG: its twelve work vectors
  DevArray<double> gr_W;  // GMRESR / GMRESREN: u, c, uin, cin (xi, eta), BFGS pairs, vecR, tmp
  DomainState dom;
  // MPCs of the mesh (hecmwST_local_mesh%mpc): slave DOF, master DOFs and
  // coefficients of every MPC whose DOFs are all 1-3, the sum of mpc_const^2; active
  // during a solve with MPC_METHOD = 2
  struct {
    int n = 0;      // MPCs the T operator applies
    int n_raw = 0;  // hecMESH%mpc%n_mpc as given (the zero-RHS check's condition)
    bool active = false;
    double const2 = 0.0;
    DevArray<int> slave, ptr, idx;
    DevArray<double> val, t, w;
  } mpc;
  // ESTCOND: ALPHA / BETA history of the CG (2 per iteration) and the last estimate
  bool lanczos_on = false;
  DevArray<double> lanczos_buf;
  bool rhist_on = false;  // ITERLOG: RESID history of the CG / BiCGSTAB graph loops
  DevArray<double> rhist_buf;
  bool iterlog = false;   // ITERLOG (Iarray(21) = 1) for the host-driven methods
  int last_lanczos_n = 0;
  double last_emin = 0.0, last_emax = 0.0;
  DevArray<int> g_flag;
  DevArray<int> blk_row, blk_col;
  DevArray<double> raw_scaled, scale, b_unscaled;
  int blk_generation = -1;
  // HEX8 assembly on the device: mesh, per-block element contribution lists, the
  // element blocks, the profile on the device and the constraint tables
  struct {
    int n_node = 0, n_elem = 0, generation = -1;
    DevArray<double> coords, E, nu, Ke, bc_value, U, fe;
    DevArray<int> conn, code, bc_first, bc_last, indexL, itemL, indexU, itemU, flag;
    DevArray<int64_t> ptr;
  } asmb;
  Learned L;
  int values_version = 0, a32_version = -1;
  double bnrm2 = 0.0;
  // graphs (FP64 drop-in, FP32 inner solve)
  GraphSlot g64, g32;
  // multi-RHS CG: node-major RHS-minor vectors (48 doubles per node), per-RHS states
  DevArray<double> mb, mx, mr, mz, mp, mq, mw, mzp, mzpos, mpart;
  DevArray<double> mzs, mrold, mbc, my, mdpos;  // the learned multi-RHS cycle (zs, r_old, P^T w, Ac^-1 P^T w, y - zs)
  DevArray<CgState> mst;
  DevArray<MultiCtl> mctl;
  CgState *h_mst = nullptr;
  MultiCtl *h_mctl = nullptr;
  GraphSlot gm;
  int occ_mr = 4;
  // pinned staging of pageable host -> device copies (upload_pageable)
  void *stage[2] = {nullptr, nullptr};
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};
  // the multi-RHS vector kernels (fewer registers than the sweeps): the streamed updates
  // (mr_update_xr_kernel), the learned iteration's RHO pass with its P y gathers and its
  // (A P) y residual
  int occ_mru = 4, occ_mrv = 4, occ_mrq = 4;
  // tiled SpMM of the multi-RHS loop: per 16-row tile its distinct columns, and each
  // block's place in that list
  DevArray<int> mt_ptr, mt_cols;
  DevArray<uint16_t> mt_lidx;
  int mt_generation = -1, mt_maxcols = 0, mt_occ = 0, mt_ntiles = 0;
  // A again with 16 lanes per row for the multi-RHS SpMM (mr_spmv_kernel<., 16>)
  DevSell<double> Amr;
  int amr_generation = -1, amr_values = -1;
  SellView<double> amr_view() const { return Amr.view(); }
  int grid_amr() const { return grid_mr(Amr.nslices * (32 / kMrLanes)); }
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int build_counter = 0;  // monotonic id of preconditioner builds (graph cache key)
  // last-solve record
  int last_iter = 0, last_outer = 0, last_kernels = 0, last_learned = 0, last_fallback = 0;
  double last_solve_s = 0.0, last_setup_s = 0.0, last_true_resid = 0.0;

  Solver() {
    H33_CUDA(cudaGetDevice(&device));
    H33_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    H33_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    H33_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_spmv, spmv_kernel<double, 2>, kThreads, 0));
    H33_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sweep, sweep_bwd_kernel<double, double, double, 8, true>, kThreads, 0));
    H33_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sweep_uni, sweep_bwd_uni_kernel<double, double, double, 4, true>, kThreads, 0));
    occ_sweep_uni = std::max(occ_sweep_uni, 1);
    H33_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_vec, update_xr_kernel<double>, kThreads, 0));
    H33_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_mr, mr_sweep_bwd_kernel<8, true, true>, kThreads, 0));
    H33_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_mru, mr_update_xr_kernel, kThreads, 0));
    H33_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_mrv, mr_fcg_rho_kernel, kThreads, 0));
    H33_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_mrq, mr_coarse_resid_kernel, kThreads, 0));
    occ_spmv = std::max(occ_spmv, 1);
    occ_sweep = std::max(occ_sweep, 1);
    occ_vec = std::max(occ_vec, 1);
    occ_mr = std::max(occ_mr, 1);
    occ_mru = std::max(occ_mru, 1);
    occ_mrv = std::max(occ_mrv, 1);
    occ_mrq = std::max(occ_mrq, 1);
    H33_CUDA(cudaMallocHost(&h_params, sizeof(CgParams)));
    std::memset(h_params, 0, sizeof(CgParams));
    H33_CUDA(cudaMallocHost(&h_state, sizeof(CgState)));
    H33_CUDA(cudaMallocHost(&h_mst, sizeof(CgState) * kMaxRhs));
    H33_CUDA(cudaMallocHost(&h_mctl, sizeof(MultiCtl)));
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
    if (h_mst) cudaFreeHost(h_mst);
    if (h_mctl) cudaFreeHost(h_mctl);
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
    for (int b = 0; b < 2; b++) {
      if (stage_ev[b]) cudaEventDestroy(stage_ev[b]);
      if (stage[b]) cudaFreeHost(stage[b]);
    }
  }
  void drop_graph() {
    g64.drop();
    g32.drop();
    gm.drop();
  }
  int n3() const { return 3 * N; }
  int grid_vec() const { return std::max(1, std::min((n3() + kThreads - 1) / kThreads, nsm * occ_vec)); }
  int grid_spmv() const {
    const int need = (A.nslices + kWarpsPerCta - 1) / kWarpsPerCta;
    return std::max(1, std::min(need, nsm * occ_spmv));
  }
  int grid_sweep_uni(int nslices) const {
    const int need = (nslices + kWarpsPerCta - 1) / kWarpsPerCta;
    return std::max(1, std::min(need, nsm * occ_sweep_uni));
  }
  int grid_sweep(int nslices) const {
    const int need = (nslices + kWarpsPerCta - 1) / kWarpsPerCta;
    return std::max(1, std::min(need, nsm * occ_sweep));
  }
  // multi-RHS kernels: one half-warp per block row
  int grid_mr(int rows) const { return std::max(1, std::min((rows + 15) / 16, nsm * occ_mr)); }
  // a half-warp per row, at most occ resident CTAs per SM
  int grid_rows(int rows, int occ) const { return std::max(1, std::min((rows + 15) / 16, nsm * occ)); }
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
  const std::string msg = check_profile(N, NP, NPL, NPU, indexL, itemL, indexU, itemU);
  if (!msg.empty()) throw Failure(HECMW33_ERR_BAD_INPUT, msg);
}

// Symbolic part of set_matrix: host copy of the profile, SpMV layout, vectors.
// HECMW33_HOST_LAYOUT=1 builds the sliced layouts wholly on the host (unified_rows,
// reordered_rows, build_sell: the reference for the device fill, which gives the same
// layouts entry for entry); read at every symbolic setup.
bool host_layouts() {
  const char *e = std::getenv("HECMW33_HOST_LAYOUT");
  return e && e[0] == '1';
}

// Host -> device copy of a caller's buffer on S.stream.  Pinned (or registered) memory
// goes straight to the DMA engine (device or managed memory as a plain copy); pageable
// memory goes through two pinned staging buffers, host threads filling one while the
// other's DMA runs (a pageable cudaMemcpyAsync stages through one driver thread: about
// 11 GB/s for the cube's 2 GB of values).  Returns once the last chunk is queued; the
// data are then stream-ordered.
constexpr size_t kStageBytes = size_t(32) << 20;
void upload_host(Solver &S, void *dst, const void *src, size_t bytes) {
  if (bytes == 0) return;
  cudaPointerAttributes attr{};
  const bool known = cudaPointerGetAttributes(&attr, src) == cudaSuccess;
  (void)cudaGetLastError();  // an unregistered pointer may leave an error behind on older drivers
  if (known && attr.type != cudaMemoryTypeUnregistered) {  // pinned, registered, managed or device memory
    H33_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, S.stream));
    return;
  }
  if (bytes < kStageBytes) {
    H33_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, S.stream));
    return;
  }
  for (int b = 0; b < 2; b++) {
    if (!S.stage[b]) {
      H33_CUDA(cudaHostAlloc(&S.stage[b], kStageBytes, cudaHostAllocDefault));
      H33_CUDA(cudaEventCreateWithFlags(&S.stage_ev[b], cudaEventDisableTiming));
    }
  }
  const char *from = static_cast<const char *>(src);
  char *to = static_cast<char *>(dst);
  constexpr size_t kPiece = size_t(1) << 20;
  for (size_t off = 0, k = 0; off < bytes; off += kStageBytes, k++) {
    const int b = int(k & 1);
    const size_t n = std::min(kStageBytes, bytes - off);
    H33_CUDA(cudaEventSynchronize(S.stage_ev[b]));  // the buffer's previous DMA is done
    char *st = static_cast<char *>(S.stage[b]);
    const int64_t np = int64_t((n + kPiece - 1) / kPiece);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < np; i++) {
      const size_t o = size_t(i) * kPiece;
      std::memcpy(st + o, from + off + o, std::min(kPiece, n - o));
    }
    H33_CUDA(cudaMemcpyAsync(to + off, st, n, cudaMemcpyHostToDevice, S.stream));
    H33_CUDA(cudaEventRecord(S.stage_ev[b], S.stream));
  }
}

// Device -> host copy into a caller's or the library's pageable buffer, complete on
// return: through the same two pinned staging buffers, the DMA of one chunk running
// while host threads copy the previous one out (pinned or device destinations take a
// plain copy).
void download_host(Solver &S, void *dst, const void *src, size_t bytes) {
  if (bytes == 0) return;
  cudaPointerAttributes attr{};
  const bool known = cudaPointerGetAttributes(&attr, dst) == cudaSuccess;
  (void)cudaGetLastError();
  if ((known && attr.type != cudaMemoryTypeUnregistered) || bytes < kStageBytes) {
    H33_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, S.stream));
    S.sync();
    return;
  }
  for (int b = 0; b < 2; b++) {
    if (!S.stage[b]) {
      H33_CUDA(cudaHostAlloc(&S.stage[b], kStageBytes, cudaHostAllocDefault));
      H33_CUDA(cudaEventCreateWithFlags(&S.stage_ev[b], cudaEventDisableTiming));
    }
  }
  const char *from = static_cast<const char *>(src);
  char *to = static_cast<char *>(dst);
  const size_t nchunks = (bytes + kStageBytes - 1) / kStageBytes;
  auto issue = [&](size_t k) {  // DMA of chunk k into its staging buffer (stream-ordered after its last use)
    const int b = int(k & 1);
    const size_t off = k * kStageBytes, n = std::min(kStageBytes, bytes - off);
    H33_CUDA(cudaMemcpyAsync(S.stage[b], from + off, n, cudaMemcpyDeviceToHost, S.stream));
    H33_CUDA(cudaEventRecord(S.stage_ev[b], S.stream));
  };
  constexpr size_t kPiece = size_t(1) << 20;
  issue(0);
  for (size_t k = 0; k < nchunks; k++) {
    if (k + 1 < nchunks) issue(k + 1);
    const int b = int(k & 1);
    H33_CUDA(cudaEventSynchronize(S.stage_ev[b]));  // chunk k has landed
    const size_t off = k * kStageBytes, n = std::min(kStageBytes, bytes - off);
    const char *st = static_cast<const char *>(S.stage[b]);
    const int64_t np = int64_t((n + kPiece - 1) / kPiece);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < np; i++) {
      const size_t o = size_t(i) * kPiece;
      std::memcpy(to + off + o, st + o, std::min(kPiece, n - o));
    }
  }
}

DevProfile dev_profile(const Solver &S) {
  return DevProfile{S.N, S.NPL, S.d_indexL.p, S.d_itemL.p, S.d_indexU.p, S.d_itemU.p};
}

// The matrix's unified rows (L, D, U of each row) in a sliced layout of `lanes` lanes
// per row, rows in input order as one group: the shape from the rows' block counts on
// the host, the blocks placed by fill_unified_kernel.
void build_unified(Solver &S, DevSell<double> &D, int lanes) {
  const int N = S.N;
  if (host_layouts()) {
    Profile prof{N, S.indexL.data(), S.itemL.data(), S.indexU.data(), S.itemU.data()};
    BlockRows rows;
    unified_rows(prof, rows);
    SellLayout lay;
    build_sell(rows, std::vector<int>{0, N}, lay, lanes);
    D.upload(lay, S.stream);
    return;
  }
  std::vector<int> count(static_cast<size_t>(N));
  for (int i = 0; i < N; i++)
    count[size_t(i)] = (S.indexL[size_t(i) + 1] - S.indexL[size_t(i)]) + 1 + (S.indexU[size_t(i) + 1] - S.indexU[size_t(i)]);
  SellLayout lay;
  sell_shape(count.data(), std::vector<int>{0, N}, lay, lanes);
  D.upload_shape(lay, S.stream);
  const int grid = std::max(1, std::min((N + kThreads - 1) / kThreads, S.nsm * 8));
  launch_k(S.stream, fill_unified_kernel, grid, kThreads, dev_profile(S), lanes, static_cast<const int *>(D.slot0.p),
           D.col.p, D.src.p);
  H33_CUDA(cudaGetLastError());
}

void set_profile(Solver &S, int N, int NPL, int NPU, const int *indexL, const int *itemL, const int *indexU,
                 const int *itemU) {
  S.has_matrix = false;
  if (N != S.N) S.mpc.n = S.mpc.n_raw = 0;  // the MPC DOF indices belong to the old mesh
  S.N = N;
  S.NPL = NPL;
  S.NPU = NPU;
  S.indexL.assign(indexL, indexL + N + 1);
  S.itemL.assign(itemL, itemL + NPL);
  S.indexU.assign(indexU, indexU + N + 1);
  S.itemU.assign(itemU, itemU + NPU);
  S.d_indexL.upload(S.indexL, S.stream);
  S.d_itemL.upload(S.itemL, S.stream);
  S.d_indexU.upload(S.indexU, S.stream);
  S.d_itemU.upload(S.itemU, S.stream);
  setup_mark("set_matrix: profile up");
  build_unified(S, S.A, 1);
  const size_t n3 = size_t(3) * N;
  for (auto *v : {&S.b, &S.x, &S.r, &S.z, &S.p, &S.q, &S.w, &S.zp}) v->alloc(n3);
  S.partials.alloc(size_t(std::max(N / 32 + 64, S.nsm * 16)) + 1024);
  S.generation++;
  S.pc.valid = false;
  S.drop_graph();
}

void set_matrix_square(Solver &S, int N, int NPL, int NPU, const int *indexL, const int *itemL,
                       const int *indexU, const int *itemU, const double *D, const double *AL, const double *AU,
                       const int *Iarray);

// A domain of a decomposed mesh (N < NP): the internal block A_II (rows and columns
// 1..N) goes to the usual layouts, the internal rows' blocks at external columns to
// the interface list; rows N+1..NP are not read by the solve.
void set_matrix_domain(Solver &S, int N, int NP, int NPL, int NPU, const int *indexL, const int *itemL,
                       const int *indexU, const int *itemU, const double *D, const double *AL, const double *AU,
                       const int *Iarray) {
  validate(N, NP, NPL, NPU, indexL, itemL, indexU, itemU);
  DomainState &d = S.dom;
  const bool same_nodes = d.on && d.NP == NP && S.has_matrix && S.N == N;  // the table stays valid
  const bool symbolic = !d.on || d.NP != NP || d.NPL != NPL || d.NPU != NPU || !S.has_matrix || N != S.N ||
                        Iarray == nullptr || Iarray[97] != 0;
  std::vector<int> indexU2(size_t(N) + 1, 0), itemU2;
  if (symbolic) {
    d.au_src.clear();
    d.ie_src.clear();
    std::vector<int> irow, iptr{0}, icol;
    for (int i = 0; i < N; i++) {
      bool iface = false;
      for (int j = indexU[i]; j < indexU[i + 1]; j++) {
        const int c = itemU[j];
        if (c <= N) {
          itemU2.push_back(c);
          d.au_src.push_back(j);
        } else {
          icol.push_back(c - N - 1);
          d.ie_src.push_back(j);
          iface = true;
        }
      }
      indexU2[size_t(i) + 1] = int(itemU2.size());
      if (iface) {
        irow.push_back(i);
        iptr.push_back(int(icol.size()));
      }
    }
    d.n_irows = int(irow.size());
    d.irow.upload(irow, S.stream);
    d.iptr.upload(iptr, S.stream);
    d.icol.upload(icol, S.stream);
  } else {
    for (int i = 0, k = 0; i < N; i++) {
      for (int j = indexU[i]; j < indexU[i + 1]; j++)
        if (itemU[j] <= N) itemU2.push_back(itemU[j]), k++;
      indexU2[size_t(i) + 1] = k;
    }
  }
  const int NPU2 = int(d.au_src.size());
  std::vector<double> AU2(9 * size_t(std::max(NPU2, 1))), IE(9 * std::max<size_t>(d.ie_src.size(), 1));
  for (int k = 0; k < NPU2; k++) std::memcpy(&AU2[9 * size_t(k)], AU + 9 * size_t(d.au_src[size_t(k)]), 9 * sizeof(double));
  for (size_t k = 0; k < d.ie_src.size(); k++) std::memcpy(&IE[9 * k], AU + 9 * size_t(d.ie_src[k]), 9 * sizeof(double));
  d.ival.upload(IE.data(), 9 * d.ie_src.size(), S.stream);
  int *flags = nullptr;
  std::vector<int> ia;
  if (Iarray) {
    ia.assign(Iarray, Iarray + 100);
    if (symbolic) ia[97] = 1;  // the compact profile is new
    flags = ia.data();
  }
  set_matrix_square(S, N, indexL[N], NPU2, indexL, itemL, indexU2.data(), itemU2.data(), D, AL, AU2.data(), flags);
  d.on = true;
  d.NP = NP;
  d.NPL = NPL;
  d.NPU = NPU;
  d.n_ext = NP - N;
  d.xe_x.alloc(3 * size_t(std::max(d.n_ext, 1)));
  d.xe_p.alloc(3 * size_t(std::max(d.n_ext, 1)));
  d.xe_z.alloc(3 * size_t(std::max(d.n_ext, 1)));
  if (!same_nodes) d.clear_table();
  S.sync();
}

void set_matrix(Solver &S, int N, int NP, int NPL, int NPU, const int *indexL, const int *itemL,
                const int *indexU, const int *itemU, const double *D, const double *AL,
                const double *AU, const int *Iarray) {
  if (NP != N) {
    set_matrix_domain(S, N, NP, NPL, NPU, indexL, itemL, indexU, itemU, D, AL, AU, Iarray);
    return;
  }
  if (S.dom.on) {
    S.dom.reset();
    S.has_matrix = false;  // a new profile
  }
  validate(N, NP, NPL, NPU, indexL, itemL, indexU, itemU);
  set_matrix_square(S, N, NPL, NPU, indexL, itemL, indexU, itemU, D, AL, AU, Iarray);
}

void set_matrix_square(Solver &S, int N, int NPL, int NPU, const int *indexL, const int *itemL,
                       const int *indexU, const int *itemU, const double *D, const double *AL, const double *AU,
                       const int *Iarray) {
  const bool symbolic = !S.has_matrix || N != S.N || NPL != S.NPL || NPU != S.NPU || Iarray == nullptr ||
                        Iarray[97] != 0;
  setup_mark("set_matrix: start");
  if (symbolic) set_profile(S, N, NPL, NPU, indexL, itemL, indexU, itemU);
  setup_mark("set_matrix: profile + SpMV layout");
  const size_t nb = size_t(N) + NPL + NPU;
  S.raw.alloc(9 * nb);
  upload_host(S, S.raw.p, D, sizeof(double) * 9 * size_t(N));
  if (NPL) upload_host(S, S.raw.p + 9 * size_t(N), AL, sizeof(double) * 9 * size_t(NPL));
  if (NPU) upload_host(S, S.raw.p + 9 * (size_t(N) + NPL), AU, sizeof(double) * 9 * size_t(NPU));
  S.A.pack(S.raw.p, S.stream, S.nsm);
  S.values_version++;
  S.zero_diag = false;
  for (int i = 0; i < N && !S.zero_diag; i++)
    for (int j = 0; j < 3; j++)
      if (std::fabs(D[9 * size_t(i) + 4 * j]) == 0.0) S.zero_diag = true;
  S.has_matrix = true;
  S.sync();
  setup_mark("set_matrix: values up + packed");
}

// ---------------------------------------------------------------------------
// Preconditioners
void diag_alu(Solver &S, DevArray<double> &alu, const double *blocks, const int *perm, double sigma,
              int lu_done) {
  alu.alloc(size_t(9) * S.N);
  H33_CUDA(cudaMemsetAsync(S.d_err.p, 0, sizeof(int), S.stream));
  const int grid = std::max(1, std::min((S.N + kThreads - 1) / kThreads, S.nsm * 8));
  launch_k(S.stream, alu_kernel<double>, grid, kThreads, blocks, perm, S.N, sigma, lu_done, alu.p, S.d_err.p);
  H33_CUDA(cudaGetLastError());
}

// SSOR in P: the reference's RCM + multicolour ordering (greedy = false, the drop-in),
// or first-fit colours in the input order (greedy = true: the learned preconditioner's
// smoother, which is not bound to the reference's schedule).
void setup_ssor(Solver &S, Precond &P, int ncolor_in, double sigma, bool symbolic, bool greedy) {
  P.sigma = sigma;
  if (symbolic) {
    Profile prof{S.N, S.indexL.data(), S.itemL.data(), S.indexU.data(), S.itemU.data()};
    std::vector<int> perm_rcm, iperm_rcm, perm, iperm, colorindex;
    setup_mark("ssor: start");
    if (greedy) {
      P.ncolor = ordering_greedy(prof, colorindex, perm, iperm);
      setup_mark("ssor: first-fit colouring");
    } else {
      ordering_rcm(prof, perm_rcm, iperm_rcm);
      setup_mark("ssor: RCM");
      P.ncolor = ordering_mc(prof, perm_rcm, ncolor_in, colorindex, perm, iperm);
      setup_mark("ssor: multicolouring");
    }
    const int lanes = sweep_lanes();
    if (host_layouts()) {
      BlockRows lower_ref, upper_ref, lower, upper;
      reordered_rows(prof, perm, iperm, lower_ref, upper_ref);
      // the device sweeps gather from their colour-ordered intermediate: columns as
      // positions (the same blocks in the same order; only the index names change)
      for (auto *br : {&lower_ref, &upper_ref})
        for (int &c : br->col) c = iperm[c];
      // inside each colour the device places its rows by slot count (rows of one
      // colour never read each other, so the sweep's arithmetic per row is unchanged):
      // the slices of a colour then need few distinct slot counts and little padding
      std::vector<int> order, iorder(size_t(S.N));
      order_rows_by_length(lower_ref, upper_ref, colorindex, lanes, order);
      for (int i = 0; i < S.N; i++) iorder[size_t(order[size_t(i)])] = i;
      permute_rows(lower_ref, order, iorder, lower);
      permute_rows(upper_ref, order, iorder, upper);
      std::vector<int> perm_dev(size_t(S.N));
      for (int i = 0; i < S.N; i++) perm_dev[size_t(i)] = perm[size_t(order[size_t(i)])];
      SellLayout lo, up;
      build_sell(lower, colorindex, lo, lanes, kMaxRuns);
      build_sell(upper, colorindex, up, lanes, kMaxRuns);
      P.lo.upload(lo, S.stream);
      P.up.upload(up, S.stream);
      P.perm_fwd.upload(perm_dev, S.stream);
    } else {
      // the same layouts with the O(blocks) work on the device: the rows' lower and
      // upper block counts in the new order (count_parts_kernel), the row order inside
      // each colour and the layouts' shape from those counts on the host, the blocks
      // placed by fill_reordered_kernel
      const int N = S.N;
      const DevProfile dp = dev_profile(S);
      DevArray<int> d_perm, d_iperm, d_nl, d_nu, d_order, d_iorder, d_row_slice;
      d_perm.upload(perm, S.stream);
      d_iperm.upload(iperm, S.stream);
      d_nl.alloc(size_t(N));
      d_nu.alloc(size_t(N));
      const int grid = std::max(1, std::min((N + kThreads - 1) / kThreads, S.nsm * 8));
      launch_k(S.stream, count_parts_kernel, grid, kThreads, dp, static_cast<const int *>(d_iperm.p), d_nl.p, d_nu.p);
      H33_CUDA(cudaGetLastError());
      std::vector<int> nl(static_cast<size_t>(N)), nu(static_cast<size_t>(N));
      H33_CUDA(cudaMemcpyAsync(nl.data(), d_nl.p, sizeof(int) * size_t(N), cudaMemcpyDeviceToHost, S.stream));
      H33_CUDA(cudaMemcpyAsync(nu.data(), d_nu.p, sizeof(int) * size_t(N), cudaMemcpyDeviceToHost, S.stream));
      S.sync();
      setup_mark("  ssor layouts: row counts (device)");
      const size_t nn = static_cast<size_t>(N);
      std::vector<int> order, iorder(nn), cl(nn), cu(nn), perm_dev(nn);
      order_rows_by_counts(nl.data(), nu.data(), N, colorindex, lanes, order);
      for (int q = 0; q < N; q++) {
        const int i = order[size_t(q)];
        iorder[size_t(i)] = q;
        cl[size_t(q)] = nl[size_t(i)];
        cu[size_t(q)] = nu[size_t(i)];
        perm_dev[size_t(q)] = perm[size_t(i)];
      }
      SellLayout lo, up;
      sell_shape(cl.data(), colorindex, lo, lanes, kMaxRuns);
      sell_shape(cu.data(), colorindex, up, lanes, kMaxRuns);
      // both parts cut the colours into the same slices (same groups, same rows per slice)
      std::vector<int> row_slice(nn);
      for (int sl = 0; sl < lo.nslices; sl++)
        for (int r = 0; r < lo.nrows[size_t(sl)]; r++) row_slice[size_t(lo.row0[size_t(sl)] + r)] = sl;
      setup_mark("  ssor layouts: row order, shape (host)");
      P.lo.upload_shape(lo, S.stream);
      P.up.upload_shape(up, S.stream);
      setup_mark("  ssor layouts: shape up, arrays allocated");
      d_order.upload(order, S.stream);
      d_iorder.upload(iorder, S.stream);
      d_row_slice.upload(row_slice, S.stream);
      const int gw = std::max(1, std::min((N + kWarpsPerCta - 1) / kWarpsPerCta, S.nsm * 8));
      launch_k(S.stream, fill_reordered_kernel<true>, gw, kThreads, dp, static_cast<const int *>(d_perm.p),
               static_cast<const int *>(d_iperm.p), static_cast<const int *>(d_order.p),
               static_cast<const int *>(d_iorder.p), static_cast<const int *>(d_row_slice.p),
               static_cast<const int *>(P.lo.row0.p), static_cast<const int *>(P.lo.slot0.p), lanes, P.lo.col.p,
               P.lo.src.p);
      launch_k(S.stream, fill_reordered_kernel<false>, gw, kThreads, dp, static_cast<const int *>(d_perm.p),
               static_cast<const int *>(d_iperm.p), static_cast<const int *>(d_order.p),
               static_cast<const int *>(d_iorder.p), static_cast<const int *>(d_row_slice.p),
               static_cast<const int *>(P.up.row0.p), static_cast<const int *>(P.up.slot0.p), lanes, P.up.col.p,
               P.up.src.p);
      H33_CUDA(cudaGetLastError());
      P.perm_fwd.upload(perm_dev, S.stream);
      S.sync();  // the fills read the temporaries above
      setup_mark("  ssor layouts: blocks placed (device)");
    }
    setup_mark("ssor: layouts");
    P.pos_cols = true;
    // padding blocks gather zpos[0]: it must hold finite values from the start
    S.zpos.alloc(size_t(3) * S.N);
    S.zpos.zero(S.stream);
    P.lo.group_rows = colorindex;
    P.up.group_rows = colorindex;
    P.colorindex = colorindex;
    P.perm = perm;  // the reference's ordering (reported); the device uses perm_dev
    P.alu_shared = true;
  }
  P.lo.pack(S.raw.p, S.stream, S.nsm);
  P.up.pack(S.raw.p, S.stream, S.nsm);
  diag_alu(S, P.alu_fwd, S.raw.p, P.perm_fwd.p, sigma, 0);
  setup_mark("ssor: value packing + diagonal LU");
}

// Block ILU(p) (hecmw_precond_BILU_33.f90): p = 0 on the matrix's own pattern
// (FORM_ILU0_33), p = 1, 2 on the fill pattern of FORM_ILU1_33 / FORM_ILU2_33.  The
// factorisation runs on the host from the resident values; the forward and backward
// solves run on the device in level schedules of the factor pattern.
void setup_bilu(Solver &S, int level, double sigma, bool symbolic) {
  Precond &P = S.pc;
  const Profile prof0{S.N, S.indexL.data(), S.itemL.data(), S.indexU.data(), S.itemU.data()};
  if (symbolic) {
    if (level > 0) bilu_fill(prof0, level, P.fill);
    const Profile prof = level > 0 ? P.fill.view() : prof0;
    std::vector<int> ord_f, lev_f, ord_b, lev_b;
    level_schedule(prof, true, ord_f, lev_f);
    level_schedule(prof, false, ord_b, lev_b);
    if (level == 0 && !host_layouts()) {
      // the matrix's own pattern: the shapes from the rows' counts, the blocks placed
      // on the device from the resident profile (fill_ordered_kernel)
      const int N = S.N, lanes = sweep_lanes();
      const size_t nn = static_cast<size_t>(N);
      std::vector<int> cl(nn), cu(nn);
      for (int q = 0; q < N; q++) {
        cl[size_t(q)] = S.indexL[size_t(ord_f[size_t(q)]) + 1] - S.indexL[size_t(ord_f[size_t(q)])];
        cu[size_t(q)] = S.indexU[size_t(ord_b[size_t(q)]) + 1] - S.indexU[size_t(ord_b[size_t(q)])];
      }
      SellLayout lo, up;
      sell_shape(cl.data(), lev_f, lo, lanes);
      sell_shape(cu.data(), lev_b, up, lanes);
      std::vector<int> rs_f(nn), rs_b(nn);
      for (int sl = 0; sl < lo.nslices; sl++)
        for (int r = 0; r < lo.nrows[size_t(sl)]; r++) rs_f[size_t(lo.row0[size_t(sl)] + r)] = sl;
      for (int sl = 0; sl < up.nslices; sl++)
        for (int r = 0; r < up.nrows[size_t(sl)]; r++) rs_b[size_t(up.row0[size_t(sl)] + r)] = sl;
      P.lo.upload_shape(lo, S.stream);
      P.up.upload_shape(up, S.stream);
      P.perm_fwd.upload(ord_f, S.stream);
      P.perm_bwd.upload(ord_b, S.stream);
      DevArray<int> d_rsf, d_rsb;
      d_rsf.upload(rs_f, S.stream);
      d_rsb.upload(rs_b, S.stream);
      const DevProfile dp = dev_profile(S);
      const int grid = std::max(1, std::min((N + kThreads - 1) / kThreads, S.nsm * 8));
      launch_k(S.stream, fill_ordered_kernel<false>, grid, kThreads, dp, static_cast<const int *>(P.perm_fwd.p),
               static_cast<const int *>(d_rsf.p), static_cast<const int *>(P.lo.row0.p),
               static_cast<const int *>(P.lo.slot0.p), lanes, P.lo.col.p, P.lo.src.p);
      launch_k(S.stream, fill_ordered_kernel<true>, grid, kThreads, dp, static_cast<const int *>(P.perm_bwd.p),
               static_cast<const int *>(d_rsb.p), static_cast<const int *>(P.up.row0.p),
               static_cast<const int *>(P.up.slot0.p), lanes, P.up.col.p, P.up.src.p);
      H33_CUDA(cudaGetLastError());
      S.sync();  // the fills read the row-slice tables above
    } else {  // the filled pattern of ILU(1)/(2), or HECMW33_HOST_LAYOUT=1: on the host
      BlockRows lower, upper;
      const int N = S.N, NPL = prof.NPL();
      lower.ptr.assign(size_t(N) + 1, 0);
      upper.ptr.assign(size_t(N) + 1, 0);
      for (int pos = 0; pos < N; pos++) {
        const int i = ord_f[pos];
        lower.ptr[pos + 1] = lower.ptr[pos] + (prof.indexL[i + 1] - prof.indexL[i]);
        const int k = ord_b[pos];
        upper.ptr[pos + 1] = upper.ptr[pos] + (prof.indexU[k + 1] - prof.indexU[k]);
      }
      lower.col.resize(size_t(lower.ptr[N]));
      lower.src.resize(size_t(lower.ptr[N]));
      upper.col.resize(size_t(upper.ptr[N]));
      upper.src.resize(size_t(upper.ptr[N]));
      for (int pos = 0; pos < N; pos++) {
        const int i = ord_f[pos];
        int64_t w = lower.ptr[pos];
        for (int j = prof.indexL[i]; j < prof.indexL[i + 1]; j++) {
          lower.col[w] = prof.itemL[j] - 1;
          lower.src[w++] = N + j;
        }
        const int k = ord_b[pos];
        w = upper.ptr[pos];
        for (int j = prof.indexU[k]; j < prof.indexU[k + 1]; j++) {
          upper.col[w] = prof.itemU[j] - 1;
          upper.src[w++] = N + NPL + j;
        }
      }
      SellLayout lo, up;
      build_sell(lower, lev_f, lo, sweep_lanes());
      build_sell(upper, lev_b, up, sweep_lanes());
      P.lo.upload(lo, S.stream);
      P.up.upload(up, S.stream);
      P.perm_fwd.upload(ord_f, S.stream);
      P.perm_bwd.upload(ord_b, S.stream);
    }
    P.alu_shared = false;
    P.ncolor = 0;
    P.ilu_level = level;
  }
  // numeric factorisation on the host, from the resident values
  const size_t nb = size_t(S.N) + S.NPL + S.NPU;
  std::vector<double> host(9 * nb);
  download_host(S, host.data(), S.raw.p, sizeof(double) * host.size());
  double *D = host.data(), *AL = host.data() + 9 * size_t(S.N), *AU = host.data() + 9 * (size_t(S.N) + S.NPL);
  if (level == 0) {
    // ILU(0) keeps the matrix's pattern: factored in place, uploaded in the raw layout
    if (factor_bilu0_inplace(prof0, D, AL, AU, sigma))
      throw Failure(HECMW33_ERR_ILU_ZERO_PIVOT, "block ILU: zero pivot (the reference stops here)");
    P.ilu_raw.alloc(host.size());
    upload_host(S, P.ilu_raw.p, host.data(), sizeof(double) * host.size());
  } else {
    std::vector<double> Dlu, ALlu, AUlu;
    if (factor_bilu_fill(P.fill, level, D, AL, AU, sigma, Dlu, ALlu, AUlu))
      throw Failure(HECMW33_ERR_ILU_ZERO_PIVOT, "block ILU: zero pivot (the reference stops here)");
    P.ilu_raw.alloc(Dlu.size() + ALlu.size() + AUlu.size());
    upload_host(S, P.ilu_raw.p, Dlu.data(), sizeof(double) * Dlu.size());
    upload_host(S, P.ilu_raw.p + Dlu.size(), ALlu.data(), sizeof(double) * ALlu.size());
    upload_host(S, P.ilu_raw.p + Dlu.size() + ALlu.size(), AUlu.data(), sizeof(double) * AUlu.size());
    S.sync();  // the factors' vectors go at the end of this scope
  }
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
  const int kind = precond == 2 ? 1 : (precond >= 10 && precond <= 12 ? 10 : precond);
  const int level = kind == 10 ? precond - 10 : 0;
  if (kind != 1 && kind != 3 && kind != 10)
    throw Failure(HECMW33_ERR_INCONS_PC, "PRECOND " + std::to_string(precond) +
                                             " is not available in the GPU drop-in (1, 2, 3, 10, 11, 12 are)");
  Precond &P = S.pc;
  const bool same = P.valid && P.kind == kind && (kind != 1 || P.ncolor_in == ncolor_in) &&
                    (kind != 10 || P.ilu_level == level);
  const bool reuse = same && Iarray[97] == 0 && Iarray[96] == 0;
  if (reuse) return;
  const bool symbolic = !same;
  if (symbolic) {
    P = Precond();
  }
  P.kind = kind;
  P.ncolor_in = ncolor_in;
  if (kind == 1) setup_ssor(S, P, ncolor_in, sigma, symbolic, false);
  else if (kind == 3) diag_alu(S, P.alu_fwd, S.raw.p, nullptr, sigma, 0);
  else setup_bilu(S, level, sigma, symbolic);
  int err = 0;
  H33_CUDA(cudaMemcpyAsync(&err, S.d_err.p, sizeof(int), cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  (void)err;  // a zero pivot in SSOR/DIAG gives Inf entries, as in the reference (no check there)
  P.valid = true;
  P.numeric_version = ++S.build_counter;
  if (symbolic) {
    // new device buffers: graphs that captured the old ones must go
    P.generation = ++S.build_counter;
    S.drop_graph();
  }
  Iarray[97] = 0;
  Iarray[96] = 0;
}

// The learned preconditioner's smoother (Learned::sm) for the current matrix and the
// solve's SSOR setup.  First-fit colours give far fewer colour launches than the
// reference's multicolouring (8 against 17 on a structured hexahedral mesh).
void ensure_smoother(Solver &S) {
  Learned &L = S.L;
  Precond &P = L.sm;
  const bool symbolic = !P.valid || L.sm_built_for != S.generation;
  if (!symbolic && L.sm_numeric_for == S.pc.numeric_version) return;
  if (symbolic) P = Precond();
  P.kind = 1;
  setup_ssor(S, P, 0, S.pc.sigma, symbolic, true);
  int err = 0;
  H33_CUDA(cudaMemcpyAsync(&err, S.d_err.p, sizeof(int), cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  (void)err;  // as the solve's SSOR: a zero pivot gives Inf entries, not an error
  P.valid = true;
  P.numeric_version = ++S.build_counter;
  if (symbolic) {
    P.generation = ++S.build_counter;
    S.drop_graph();
  }
  L.sm_built_for = S.generation;
  L.sm_numeric_for = S.pc.numeric_version;
}

// ---------------------------------------------------------------------------
// Launch sequences (captured into graphs or run directly), for the working
// precision R: double (the drop-in) or float (the inner solves of the
// mixed-precision refinement, on FP32 copies of the same sliced layouts).

template <class R>
struct Views {
  SellView<R> A, lo, up;
  const R *alu_f, *alu_b;
  R *b, *x, *r, *z, *p, *q, *w, *zp, *zs, *rold;
  // low-precision preconditioner (lowp = 1): BF16 sweep values, FP32 diagonal LU,
  // arithmetic still in R
  int lowp;
  SellView<__nv_bfloat16> lo16, up16;
  const float *alu32_f, *alu32_b;
  R *zpos;  // the sweeps' intermediate in colour-position order (multicolour SSOR)
  const Precond *pc;  // whose schedule the sweeps follow
};

// Views of the solve's vectors and of the preconditioner pc (default: the drop-in's).
Views<double> views(Solver &S, double, int lowp = 0, const Precond *pc = nullptr) {
  const Precond &P = pc ? *pc : S.pc;
  return Views<double>{S.A.view(),   P.lo.view(),   P.up.view(), P.alu_fwd.p,
                       P.alu_shared ? P.alu_fwd.p : P.alu_bwd.p,
                       S.b.p, S.x.p, S.r.p, S.z.p, S.p.p, S.q.p, S.w.p, S.zp.p, S.zs.p, S.rold.p,
                       lowp, P.lo.view16(), P.up.view16(), P.alu32_fwd.p,
                       P.alu_shared ? P.alu32_fwd.p : P.alu32_bwd.p, S.zpos.p, &P};
}
Views<float> views(Solver &S, float, int lowp = 0, const Precond *pc = nullptr) {
  const Precond &P = pc ? *pc : S.pc;
  return Views<float>{S.A.view32(),   P.lo.view32(),   P.up.view32(), P.alu32_fwd.p,
                      P.alu_shared ? P.alu32_fwd.p : P.alu32_bwd.p,
                      S.bf.p, S.xf.p, S.rf.p, S.zf.p, S.pf.p, S.qf.p, S.wf.p, S.zpf.p, S.zsf.p, S.roldf.p,
                      lowp, P.lo.view16(), P.up.view16(), P.alu32_fwd.p,
                      P.alu_shared ? P.alu32_fwd.p : P.alu32_bwd.p, S.zposf.p, &P};
}

// z = M^-1 r, one pass; FUSE_RHO adds the RHO reduction + finisher.  K = lanes per
// row of the sweep layouts.
// Node-order sweeps: the ILU(0) level schedules.
template <class R, class TV, class TA, bool FUSE_RHO, int K>
void launch_sweep_node(Solver &S, const Precond &P, const SellView<TV> &lo, const SellView<TV> &up,
                       const TA *alu_f, const TA *alu_b, const R *rin, R *zout, CgState *st) {
  cudaStream_t s = S.stream;
  const int *perm_b = P.alu_shared ? P.perm_fwd.p : P.perm_bwd.p;
  const int pre = level_pre<TV>();
  const int gf = int(P.lo.group_slice.size()) - 1;
  for (int g = 0; g < gf; g++) {
    const int sb = P.lo.group_slice[g], se = P.lo.group_slice[g + 1];
    if (se <= sb) continue;
    launch_kp(s, (pre & 1) != 0, sweep_fwd_kernel<R, TV, TA, K>, S.grid_sweep(se - sb), kThreads, lo, P.perm_fwd.p,
              alu_f, S.N, rin, zout, sb, se, static_cast<const CgState *>(st), pre);
  }
  const int gb = int(P.up.group_slice.size()) - 1;
  int total = 0;
  for (int g = gb - 1; g >= 0; g--)
    total += S.grid_sweep(std::max(P.up.group_slice[g + 1] - P.up.group_slice[g], 1));
  int base = 0;
  for (int g = gb - 1; g >= 0; g--) {
    const int sb = P.up.group_slice[g], se = P.up.group_slice[g + 1];
    const int grid = S.grid_sweep(std::max(se - sb, 1));
    // a group without slices still launches (one idle CTA) so that the reduction
    // ticket count stays exact
    launch_kp(s, (pre & 1) != 0, sweep_bwd_kernel<R, TV, TA, K, FUSE_RHO>, grid, kThreads, up, perm_b, alu_b, S.N,
              rin, zout, sb, se, st, S.partials.p, base, total, pre);
    base += grid;
  }
}

// Run-table colour layout (multicolour SSOR): intermediate in colour-position order.
RunShape run_shape(const DevSell<double> &D, int g) {
  RunShape sh{};
  sh.row0 = D.group_rows[size_t(g)];
  sh.row1 = D.group_rows[size_t(g) + 1];
  const int r0 = D.run_ptr[size_t(g)], r1 = D.run_ptr[size_t(g) + 1];
  sh.nruns = r1 - r0;
  if (sh.nruns == 0) {  // a colour without rows
    sh.nruns = 1;
    return sh;
  }
  if (sh.nruns > kMaxRuns) throw Failure(HECMW33_ERR_CUDA, "run table out of range");
  for (int r = 0; r < sh.nruns; r++) {
    sh.slice[r] = D.run_slice[size_t(r0 + r)];
    sh.slot[r] = D.run_slot[size_t(r0 + r)];
    sh.len[r] = D.run_len[size_t(r0 + r)];
  }
  sh.slice[sh.nruns] = D.group_slice[size_t(g) + 1] - D.group_slice[size_t(g)];
  return sh;
}

template <class R, class TV, class TA, bool FUSE_RHO, int K>
void launch_sweep_uni(Solver &S, const Precond &P, const SellView<TV> &lo, const SellView<TV> &up,
                      const TA *alu_f, const R *rin, R *zout, R *zpos, CgState *st, R *dpos = nullptr) {
  cudaStream_t s = S.stream;
  const int gf = int(P.lo.group_slice.size()) - 1;
  for (int g = 0; g < gf; g++) {
    const int ns = P.lo.group_slice[g + 1] - P.lo.group_slice[g];
    if (ns <= 0) continue;
    constexpr int pre = sweep_pre<TV>();
    launch_kp(s, true, sweep_fwd_uni_kernel<R, TV, TA, K>, S.grid_sweep_uni(ns), kThreads, lo,
              P.perm_fwd.p, alu_f, S.N, rin, zpos, ns, run_shape(P.lo, g), static_cast<const CgState *>(st), pre);
  }
  const int gb = int(P.up.group_slice.size()) - 1;
  int total = 0;
  for (int g = gb - 1; g >= 0; g--) total += S.grid_sweep_uni(std::max(P.up.group_slice[g + 1] - P.up.group_slice[g], 1));
  int base = 0;
  for (int g = gb - 1; g >= 0; g--) {
    const int ns = P.up.group_slice[g + 1] - P.up.group_slice[g];
    const int grid = S.grid_sweep_uni(std::max(ns, 1));
    // a colour without slices still launches (one idle CTA) so that the reduction
    // ticket count stays exact
    constexpr int pre = sweep_pre<TV>();
    bool done = false;
    if constexpr (!FUSE_RHO && std::is_same<R, double>::value && std::is_same<TV, double>::value) {
      if (dpos) {  // the learned FP64 smoother's pre-smoothing (lower_resid_kernel)
        launch_kp(s, true, sweep_bwd_uni_kernel<R, TV, TA, K, FUSE_RHO, true>, grid, kThreads, up, P.perm_fwd.p,
                  alu_f, S.N, rin, zout, zpos, ns, run_shape(P.up, g), st, S.partials.p, base, total, pre, dpos);
        done = true;
      }
    }
    if (!done)
      launch_kp(s, true, sweep_bwd_uni_kernel<R, TV, TA, K, FUSE_RHO, false>, grid, kThreads, up, P.perm_fwd.p,
                alu_f, S.N, rin, zout, zpos, ns, run_shape(P.up, g), st, S.partials.p, base, total, pre,
                static_cast<R *>(nullptr));
    base += grid;
  }
}

// Lanes per row are 4, 8 or 16 (sweep_lanes()).
template <class R, class TV, class TA, bool FUSE_RHO>
void launch_sweep_t(Solver &S, const Precond &P, const SellView<TV> &lo, const SellView<TV> &up,
                    const TA *alu_f, const TA *alu_b, const R *rin, R *zout, R *zpos, CgState *st,
                    R *dpos = nullptr) {
  if (P.kind == 3) {
    launch_k(S.stream, diag_kernel<R, TA, FUSE_RHO>, S.grid_vec(), kThreads, alu_f, S.N, rin, zout, st,
             S.partials.p);
    return;
  }
  if (P.pos_cols) {
    switch (P.lo.lanes) {
      case 8: return launch_sweep_uni<R, TV, TA, FUSE_RHO, 8>(S, P, lo, up, alu_f, rin, zout, zpos, st, dpos);
      case 16: return launch_sweep_uni<R, TV, TA, FUSE_RHO, 16>(S, P, lo, up, alu_f, rin, zout, zpos, st, dpos);
      default: return launch_sweep_uni<R, TV, TA, FUSE_RHO, 4>(S, P, lo, up, alu_f, rin, zout, zpos, st, dpos);
    }
  }
  switch (P.lo.lanes) {
    case 8: return launch_sweep_node<R, TV, TA, FUSE_RHO, 8>(S, P, lo, up, alu_f, alu_b, rin, zout, st);
    case 16: return launch_sweep_node<R, TV, TA, FUSE_RHO, 16>(S, P, lo, up, alu_f, alu_b, rin, zout, st);
    default: return launch_sweep_node<R, TV, TA, FUSE_RHO, 4>(S, P, lo, up, alu_f, alu_b, rin, zout, st);
  }
}

// dpos (may be null; multicolour layouts only): the backward sweep's correction y - z
// per colour position, for lower_resid_kernel.
template <class R, bool FUSE_RHO>
void launch_sweep(Solver &S, const Views<R> &V, const R *rin, R *zout, CgState *st, R *dpos = nullptr) {
  if (V.lowp)
    launch_sweep_t<R, __nv_bfloat16, float, FUSE_RHO>(S, *V.pc, V.lo16, V.up16, V.alu32_f, V.alu32_b, rin, zout,
                                                      V.zpos, st, dpos);
  else
    launch_sweep_t<R, R, R, FUSE_RHO>(S, *V.pc, V.lo, V.up, V.alu_f, V.alu_b, rin, zout, V.zpos, st, dpos);
}

// w = r - A z after z = launch_sweep(r) with dpos: lower_resid_kernel over the
// preconditioner's lower layout, in its storage (BF16 values in precision mode 1).
template <class TV>
void launch_lower_resid(Solver &S, const Precond &P, const SellView<TV> &lo, const double *dpos, double *w,
                        CgState *st) {
  const int grid = std::max(1, std::min((P.lo.nslices + kWarpsPerCta - 1) / kWarpsPerCta, S.nsm * S.occ_sweep_uni));
  const CgState *cst = st;
  switch (P.lo.lanes) {
    case 8: launch_k(S.stream, lower_resid_kernel<double, TV, 8>, grid, kThreads, lo, P.perm_fwd.p, dpos, w, cst); break;
    case 16: launch_k(S.stream, lower_resid_kernel<double, TV, 16>, grid, kThreads, lo, P.perm_fwd.p, dpos, w, cst); break;
    default: launch_k(S.stream, lower_resid_kernel<double, TV, 4>, grid, kThreads, lo, P.perm_fwd.p, dpos, w, cst); break;
  }
}

// hecmw_precond_apply (hecmw_precond.f90:86-172): z = M^-1 r with iterPREmax passes.
// When st is given and iterPREmax == 1 the RHO reduction is fused into the sweep;
// otherwise (st given) RHO is computed by a separate dot.
template <class R>
void launch_precond(Solver &S, const Views<R> &V, int iterpremax, const R *r, R *z, CgState *st) {
  cudaStream_t s = S.stream;
  const int n3 = S.n3();
  if (iterpremax <= 0) {
    launch_k(s, copy_kernel<R>, S.grid_vec(), kThreads, r, z, n3, st);
    if (st) launch_k(s, dot_kernel<R, 1>, S.grid_vec(), kThreads, r, z, n3, st, S.partials.p, 0, 0);
    return;
  }
  if (iterpremax == 1) {
    if (st) launch_sweep<R, true>(S, V, r, z, st);
    else launch_sweep<R, false>(S, V, r, z, nullptr);
    return;
  }
  const R *in = r;
  for (int it = 1; it <= iterpremax; it++) {
    launch_sweep<R, false>(S, V, in, V.zp, st);
    if (it == 1) launch_k(s, copy_kernel<R>, S.grid_vec(), kThreads, V.zp, z, n3, st);
    else launch_k(s, add_kernel<R>, S.grid_vec(), kThreads, V.zp, z, n3, st);
    if (it == iterpremax) break;
    launch_k(s, spmv_kernel<R, 1>, S.grid_spmv(), kThreads, V.A, z, V.w, r, nullptr, nullptr);
    in = V.w;
  }
  if (st) launch_k(s, dot_kernel<R, 1>, S.grid_vec(), kThreads, r, z, n3, st, S.partials.p, 0, 0);
}

template <class R>
void launch_prologue(Solver &S, const Views<R> &V, cudaGraphConditionalHandle h, int use_cond) {
  cudaStream_t s = S.stream;
  CgState *st = S.state.p;
  launch_k(s, cg_init_kernel, 1, 32, st, S.params.p);
  launch_k(s, spmv_kernel<R, 1>, S.grid_spmv(), kThreads, V.A, V.x, V.r, V.b, nullptr, nullptr);
  launch_k(s, dot_kernel<R, 0>, S.grid_vec(), kThreads, V.b, V.b, S.n3(), st, S.partials.p, h, use_cond);
}

template <class R>
void launch_iteration(Solver &S, const Views<R> &V, int iterpremax, cudaGraphConditionalHandle h, int use_cond) {
  cudaStream_t s = S.stream;
  CgState *st = S.state.p;
  const int n3 = S.n3();
  launch_k(s, iter_begin_kernel, 1, 32, st, h, use_cond);
  launch_precond<R>(S, V, iterpremax, V.r, V.z, st);
  launch_k(s, update_p_kernel<R>, S.grid_vec(), kThreads, V.z, V.p, n3, st);
  launch_k(s, spmv_kernel<R, 2>, S.grid_spmv(), kThreads, V.A, V.p, V.q, nullptr, st, S.partials.p);
  launch_k(s, update_xr_kernel<R>, S.grid_vec(), kThreads, V.x, V.p, V.r, V.q, n3, st, S.partials.p);
  launch_k(s, resid_ctl_kernel<R>, S.grid_spmv(), kThreads, V.A, V.x, V.r, V.b, st, S.partials.p, h, use_cond);
}

// Network application z = zs + gamma W_out h3 (or z = zs when it is off), R-precision
// vectors, BF16 weights, FP32 activations.
// hecmw_precond_apply without the RHO reduction (BiCGSTAB computes its own dots);
// st (optional) only lets the kernels skip work once the loop has ended.
template <class R>
void launch_precond_plain(Solver &S, const Views<R> &V, int iterpremax, const R *r, R *z, CgState *st) {
  cudaStream_t s = S.stream;
  const int n3 = S.n3();
  if (iterpremax <= 0) {
    launch_k(s, copy_kernel<R>, S.grid_vec(), kThreads, r, z, n3, st);
    return;
  }
  const R *in = r;
  for (int it = 1; it <= iterpremax; it++) {
    launch_sweep<R, false>(S, V, in, it == 1 && iterpremax == 1 ? z : V.zp, st);
    if (iterpremax == 1) break;
    if (it == 1) launch_k(s, copy_kernel<R>, S.grid_vec(), kThreads, V.zp, z, n3, st);
    else launch_k(s, add_kernel<R>, S.grid_vec(), kThreads, V.zp, z, n3, st);
    if (it == iterpremax) break;
    launch_k(s, spmv_kernel<R, 1>, S.grid_spmv(), kThreads, V.A, z, V.w, r, nullptr, nullptr);
    in = V.w;
  }
}

// BiCGSTAB prologue (hecmw_solver_BiCGSTAB.f90:125-137): r = b - A x, r_tld = r,
// BNRM2 = b.b (which also decides whether the loop runs).
void launch_prologue_bicg(Solver &S, const Views<double> &V, cudaGraphConditionalHandle h, int use_cond) {
  cudaStream_t s = S.stream;
  CgState *st = S.state.p;
  launch_k(s, cg_init_kernel, 1, 32, st, static_cast<const CgParams *>(S.params.p));
  launch_k(s, spmv_kernel<double, 1>, S.grid_spmv(), kThreads, V.A, V.x, V.r, V.b, nullptr, nullptr);
  launch_k(s, copy_kernel<double>, S.grid_vec(), kThreads, V.r, S.b_rt.p, S.n3(), static_cast<const CgState *>(nullptr));
  launch_k(s, dot_kernel<double, 0>, S.grid_vec(), kThreads, V.b, V.b, S.n3(), st, S.partials.p, h, use_cond);
}

// One BiCGSTAB iteration (:161-271): {p_tld} in z, {v} in q.
void launch_iteration_bicg(Solver &S, const Views<double> &V, int iterpremax, cudaGraphConditionalHandle h,
                           int use_cond) {
  cudaStream_t s = S.stream;
  CgState *st = S.state.p;
  const int n3 = S.n3();
  launch_k(s, iter_begin_kernel, 1, 32, st, h, use_cond);
  launch_k(s, bicg_rho_kernel<double>, S.grid_vec(), kThreads, V.r, S.b_rt.p, n3, st, S.partials.p);
  launch_k(s, bicg_p_kernel<double>, S.grid_vec(), kThreads, V.r, V.p, V.q, n3, static_cast<const CgState *>(st));
  launch_precond_plain<double>(S, V, iterpremax, V.p, V.z, st);
  launch_k(s, bicg_spmv_kernel<double, 0>, S.grid_spmv(), kThreads, V.A, V.z, V.q, S.b_rt.p, st, S.partials.p);
  launch_k(s, bicg_s_kernel<double>, S.grid_vec(), kThreads, S.b_s.p, V.r, V.q, n3, static_cast<const CgState *>(st));
  launch_precond_plain<double>(S, V, iterpremax, S.b_s.p, S.b_st.p, st);
  launch_k(s, bicg_spmv_kernel<double, 1>, S.grid_spmv(), kThreads, V.A, S.b_st.p, S.b_t.p, S.b_s.p, st,
           S.partials.p);
  launch_k(s, bicg_update_kernel<double>, S.grid_vec(), kThreads, V.x, V.z, S.b_st.p, V.r, S.b_s.p, S.b_t.p, n3, st,
           S.partials.p);
  launch_k(s, resid_ctl_kernel<double>, S.grid_spmv(), kThreads, V.A, V.x, V.r, V.b, st, S.partials.p, h, use_cond);
}

// BiCGSTAB runs in FP64 only (the FP32 inner solves of modes 2 and 3 are CG).
template <class R>
void launch_prologue_bicg_t(Solver &S, const Views<R> &V, cudaGraphConditionalHandle h, int use_cond) {
  if constexpr (std::is_same<R, double>::value) launch_prologue_bicg(S, V, h, use_cond);
  else throw Failure(HECMW33_ERR_BAD_INPUT, "BiCGSTAB runs in FP64 only");
}
template <class R>
void launch_iteration_bicg_t(Solver &S, const Views<R> &V, int iterpremax, cudaGraphConditionalHandle h,
                             int use_cond) {
  if constexpr (std::is_same<R, double>::value) launch_iteration_bicg(S, V, iterpremax, h, use_cond);
  else throw Failure(HECMW33_ERR_BAD_INPUT, "BiCGSTAB runs in FP64 only");
}

void ensure_bicg(Solver &S) {
  const size_t n3 = size_t(S.n3());
  for (auto *v : {&S.b_rt, &S.b_s, &S.b_st, &S.b_t})
    if (v->n != n3) {
      v->alloc(n3);
      v->zero(S.stream);
    }
}

// z = zs + P Ac^-1 P^T r: the learned two-level preconditioner's coarse correction
// (defined with the coarse space below).
template <class R>
void launch_coarse(Solver &S, const R *zs, const R *r, R *z, CgState *st);

// The coarse correction inside the two-grid cycle: zc = zs + P Ac^-1 P^T w and
// w -= A P Ac^-1 P^T w (defined with the coarse space below).
template <class R>
void launch_coarse_cycle(Solver &S, const R *zs, R *w, R *zc, CgState *st);

// HECMW33_LOWER_RESID=0: the two-grid cycle's residual r - A zs by an SpMV (with the
// FP32 copy of A in precision mode 1) instead of lower_resid_kernel.
bool lower_resid_mode() {
  static const bool v = [] {
    const char *e = std::getenv("HECMW33_LOWER_RESID");
    return !(e && e[0] == '0');
  }();
  return v;
}

// HECMW33_COARSE_FORM: 0 (default) the symmetric two-grid form, 1 the additive form.
// Measured on the 100^3 cube (BF16-stored SSOR, omega = 1/2): two-grid 62 iterations,
// additive 115; the two-grid form is the one whose convergence the training loss
// (the error energy left outside the coarse space after one SSOR step) measures.
int coarse_form() {
  static const int v = [] {
    const char *e = std::getenv("HECMW33_COARSE_FORM");
    return e ? std::atoi(e) : 0;
  }();
  return v;
}

// y = r - A x inside the preconditioner: with the FP32 copy of A when the SSOR is
// BF16-stored (precision mode 1), else in the working precision.
template <class R>
void precond_resid(Solver &S, const Views<R> &V, const R *x, R *y) {
  if constexpr (std::is_same<R, double>::value) {
    if (V.lowp) {
      launch_k(S.stream, spmv_kernel<double, 1, float>, S.grid_spmv(), kThreads, S.A.view32(), x, y,
               static_cast<const double *>(V.r), static_cast<CgState *>(nullptr), static_cast<double *>(nullptr));
      return;
    }
  }
  launch_k(S.stream, spmv_kernel<R, 1>, S.grid_spmv(), kThreads, V.A, x, y, static_cast<const R *>(V.r),
           static_cast<CgState *>(nullptr), static_cast<double *>(nullptr));
}

// The learned two-level preconditioner z = M^-1 r.  Symmetric two-grid form:
//   zs = SSOR(r);  zc = zs + P Ac^-1 P^T (r - A zs);  z = zc + SSOR(r - A zc)
// (pre-smoothing, coarse correction, post-smoothing: symmetric because SSOR is); the
// residual r - A zc comes from r - A zs less (A P) y with the stored A P;
// additive form: z = SSOR(r) + P Ac^-1 P^T r.  With the correction off (fallback)
// z = SSOR(r).
template <class R>
void launch_learned_precond(Solver &S, const Views<R> &V, CgState *st) {
  cudaStream_t s = S.stream;
  if (coarse_form() == 1) {
    launch_sweep<R, false>(S, V, V.r, V.zs, st);
    launch_coarse<R>(S, V.zs, V.r, V.z, st);
    return;
  }
  // w = r - A zs: from the pre-smoothing sweep's correction and the smoother's lower
  // triangle when the identity holds with A's own values (multicolour layout, unit
  // SIGMA_DIAG, FP64 smoother), else by an SpMV.  With the BF16-stored smoother the
  // identity would give the residual of the BF16 operator instead (measured: 3 more
  // iterations on a 16x16x32 box), so precision mode 1 keeps the SpMV.
  bool lower = false;
  if constexpr (std::is_same<R, double>::value)
    lower = !V.lowp && V.pc->pos_cols && V.pc->sigma == 1.0 && S.dpos.n == size_t(S.n3()) && lower_resid_mode();
  if (lower) {
    if constexpr (std::is_same<R, double>::value) {
      launch_sweep<R, false>(S, V, V.r, V.zs, st, S.dpos.p);
      launch_lower_resid(S, *V.pc, V.lo, S.dpos.p, V.w, st);
    }
  } else {
    launch_sweep<R, false>(S, V, V.r, V.zs, st);
    precond_resid<R>(S, V, V.zs, V.w);
  }
  launch_coarse_cycle<R>(S, V.zs, V.w, V.zp, st);  // zp = zc, w = r - A zc
  launch_sweep<R, false>(S, V, V.w, V.z, st);
  launch_k(s, coarse_post_kernel<R>, S.grid_vec(), kThreads, static_cast<const R *>(V.zp),
           static_cast<const R *>(V.zs), V.z, S.n3(), static_cast<const CgState *>(st));
}

// One flexible-CG iteration with the learned two-level preconditioner: SSOR, then the
// coarse correction of the space the network shapes (iterPREmax = 1).  The correction
// may be switched off on the device (fallback); its kernels then only copy the SSOR
// output.
template <class R>
void launch_iteration_flex(Solver &S, const Views<R> &V, cudaGraphConditionalHandle h, int use_cond) {
  cudaStream_t s = S.stream;
  CgState *st = S.state.p;
  const int n3 = S.n3();
  launch_k(s, iter_begin_kernel, 1, 32, st, h, use_cond);
  launch_learned_precond<R>(S, V, st);
  launch_k(s, fcg_rho_kernel<R>, S.grid_vec(), kThreads, V.z, V.r, V.rold, n3, st, S.partials.p);
  launch_k(s, update_p_kernel<R>, S.grid_vec(), kThreads, V.z, V.p, n3, st);
  launch_k(s, spmv_kernel<R, 2>, S.grid_spmv(), kThreads, V.A, V.p, V.q, nullptr, st, S.partials.p);
  launch_k(s, update_xr_flex_kernel<R>, S.grid_vec(), kThreads, V.x, V.p, V.r, V.rold, V.q, n3, st, S.partials.p);
  launch_k(s, resid_ctl_kernel<R>, S.grid_spmv(), kThreads, V.A, V.x, V.r, V.b, st, S.partials.p, h, use_cond);
}

// Mixed precision with reliable updates (graph body in FP32, FP64 pieces inside).
// Prologue: r64 = b - A x64, ||b||^2 (FP64), r32 = float(r64), x32 = 0.
void launch_prologue_reliable(Solver &S, cudaGraphConditionalHandle h, int use_cond) {
  cudaStream_t s = S.stream;
  CgState *st = S.state.p;
  launch_k(s, cg_init_kernel, 1, 32, st, S.params.p);
  launch_k(s, spmv_kernel<double, 1>, S.grid_spmv(), kThreads, S.A.view(), S.x.p, S.r.p, S.b.p, nullptr, nullptr);
  launch_k(s, dot_kernel<double, 0>, S.grid_vec(), kThreads, S.b.p, S.b.p, S.n3(), st, S.partials.p, h, use_cond);
  launch_k(s, ru_init_kernel, S.grid_vec(), kThreads, S.r.p, S.rf.p, S.xf.p, S.n3(), st, S.partials.p, h, use_cond);
}

// One FP32 CG (or flexible CG with the network) iteration followed by the FP64
// reliable update when due.
void launch_iteration_reliable(Solver &S, int iterpremax, bool learned, cudaGraphConditionalHandle h,
                               int use_cond) {
  cudaStream_t s = S.stream;
  CgState *st = S.state.p;
  const int n3 = S.n3();
  const Views<float> V = views(S, 0.0f, 0, learned ? &S.L.sm : nullptr);
  launch_k(s, iter_begin_kernel, 1, 32, st, h, use_cond);
  if (learned) {
    launch_learned_precond<float>(S, V, st);
    launch_k(s, fcg_rho_kernel<float>, S.grid_vec(), kThreads, V.z, V.r, V.rold, n3, st, S.partials.p);
  } else {
    launch_precond<float>(S, V, iterpremax, V.r, V.z, st);
  }
  launch_k(s, update_p_kernel<float>, S.grid_vec(), kThreads, V.z, V.p, n3, st);
  launch_k(s, spmv_kernel<float, 2>, S.grid_spmv(), kThreads, V.A, V.p, V.q, nullptr, st, S.partials.p);
  if (learned)
    launch_k(s, update_xr_flex_kernel<float>, S.grid_vec(), kThreads, V.x, V.p, V.r, V.rold, V.q, n3, st, S.partials.p);
  else
    launch_k(s, update_xr_kernel<float>, S.grid_vec(), kThreads, V.x, V.p, V.r, V.q, n3, st, S.partials.p);
  launch_k(s, ru_update_x_kernel, S.grid_vec(), kThreads, S.x.p, S.xf.p, n3, st);
  launch_k(s, ru_resid_kernel, S.grid_spmv(), kThreads, S.A.view(), S.x.p, S.r.p, S.b.p, S.rf.p, st, S.partials.p, h,
                                                     use_cond);
}

template <class R>
GraphSlot &slot_of(Solver &S) {
  return sizeof(R) == sizeof(double) ? S.g64 : S.g32;
}

// mode bit 1: flexible CG with the learned preconditioner; bit 2: FP32 CG with FP64
// reliable updates (R = float)
template <class R>
void build_graph(Solver &S, int iterpremax, int mode = 0) {
  GraphSlot &G = slot_of<R>(S);
  const int flexible = mode & 1;
  const int lowp = (mode & 4) ? 1 : 0;
  const int key[5] = {S.generation, S.pc.generation, S.pc.kind, iterpremax,
                      mode + (flexible ? S.L.graph_generation * 4 : 0)};
  if (G.exec && std::equal(key, key + 5, G.key)) return;
  G.drop();
  const Views<R> V = views(S, R(), lowp, flexible ? &S.L.sm : nullptr);
  cudaGraph_t g = nullptr;
  H33_CUDA(cudaGraphCreate(&g, 0));
  G.graph = g;
  cudaGraphConditionalHandle h;
  H33_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
  // prologue
  H33_CUDA(cudaStreamBeginCaptureToGraph(S.stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  if (mode & 2) launch_prologue_reliable(S, h, 1);
  else if (mode & 8) launch_prologue_bicg_t(S, V, h, 1);
  else launch_prologue<R>(S, V, h, 1);
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
  if (mode & 2) launch_iteration_reliable(S, iterpremax, flexible != 0, h, 1);
  else if (mode & 8) launch_iteration_bicg_t(S, V, iterpremax, h, 1);
  else if (flexible) launch_iteration_flex<R>(S, V, h, 1);
  else launch_iteration<R>(S, V, iterpremax, h, 1);
  cudaGraph_t b2 = nullptr;
  H33_CUDA(cudaStreamEndCapture(S.stream, &b2));
  H33_CUDA(cudaGraphInstantiate(&G.exec, g, 0));
  std::copy(key, key + 5, G.key);
  size_t nbody = 0, nall = 0;
  H33_CUDA(cudaGraphGetNodes(body, nullptr, &nbody));
  H33_CUDA(cudaGraphGetNodes(g, nullptr, &nall));
  G.kernels_per_iter = int(nbody);
  G.prologue_kernels = int(nall) - 1;  // minus the conditional node
}

// One CG run on the device in precision R (graph or stream mode); returns the final
// state in S.h_state and the device time in ms; counts launched kernels.
template <class R>
float run_cg(Solver &S, int iterpremax, double tol, int maxit, int *kernels, int inner = 0, int learned = 0,
             int reliable = 0, double ru_delta = 1e-4, int lowp = 0, int method = 1) {
  const Views<R> V = views(S, R(), lowp, learned ? &S.L.sm : nullptr);
  const int mode = (learned ? 1 : 0) | (reliable ? 2 : 0) | (lowp ? 4 : 0) | (method == 2 ? 8 : 0);
  S.h_params->tol = tol;
  S.h_params->maxit = maxit;
  S.h_params->iterpremax = iterpremax;
  S.h_params->inner = inner || reliable;
  S.h_params->flexible = learned;
  // a coarse matrix that was not positive definite leaves the correction off (SSOR-CG)
  S.h_params->use_gnn = learned && S.L.C.ok;
  S.h_params->reliable = reliable;
  S.h_params->ru_delta = ru_delta;
  S.h_params->method = method;
  // ESTCOND: the plain FP64-recurrence CG records ALPHA and BETA
  const bool lanczos = S.lanczos_on && !learned && !reliable && !inner && method == 1;
  S.h_params->lanczos = lanczos ? S.lanczos_buf.p : nullptr;
  S.h_params->lanczos_cap = lanczos ? int(S.lanczos_buf.n / 2) : 0;
  // ITERLOG: the same plain CG records RESID per iteration
  const bool rhist = S.rhist_on && !learned && !reliable && !inner && (method == 1 || method == 2);
  S.h_params->rhist = rhist ? S.rhist_buf.p : nullptr;
  S.h_params->rhist_cap = rhist ? int(S.rhist_buf.n) : 0;
  H33_CUDA(cudaMemcpyAsync(S.params.p, S.h_params, sizeof(CgParams), cudaMemcpyHostToDevice, S.stream));
  H33_CUDA(cudaEventRecord(S.ev0, S.stream));
  if (graph_mode()) {
    build_graph<R>(S, iterpremax, mode);
    H33_CUDA(cudaGraphLaunch(slot_of<R>(S).exec, S.stream));
    H33_CUDA(cudaEventRecord(S.ev1, S.stream));
    H33_CUDA(cudaMemcpyAsync(S.h_state, S.state.p, sizeof(CgState), cudaMemcpyDeviceToHost, S.stream));
    S.sync();
    const GraphSlot &G = slot_of<R>(S);
    const int executed = std::max(std::min(S.h_state->guard, maxit + 1), 0);
    if (kernels) *kernels += G.prologue_kernels + executed * G.kernels_per_iter;
  } else {
    if (reliable) launch_prologue_reliable(S, 0, 0);
    else if (mode & 8) launch_prologue_bicg_t(S, V, 0, 0);
    else launch_prologue<R>(S, V, 0, 0);
    int launched = 0;
    for (int done = 0, it = 0; !done && it <= maxit + kStreamChunk; it += kStreamChunk) {
      for (int k = 0; k < kStreamChunk; k++) {
        if (reliable) launch_iteration_reliable(S, iterpremax, learned != 0, 0, 0);
        else if (mode & 8) launch_iteration_bicg_t(S, V, iterpremax, 0, 0);
        else if (learned) launch_iteration_flex<R>(S, V, 0, 0);
        else launch_iteration<R>(S, V, iterpremax, 0, 0);
      }
      launched += kStreamChunk;
      H33_CUDA(cudaGetLastError());
      H33_CUDA(cudaMemcpyAsync(S.h_state, S.state.p, sizeof(CgState), cudaMemcpyDeviceToHost, S.stream));
      S.sync();
      done = S.h_state->done;
    }
    H33_CUDA(cudaEventRecord(S.ev1, S.stream));
    S.sync();
    (void)launched;
  }
  float ms = 0.0f;
  H33_CUDA(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
  const CgState &st = *S.h_state;
  if (!st.done && !st.zero_rhs)
    throw Failure(HECMW33_ERR_TIMEOUT, "device CG loop ended without a decision (internal error)");
  return ms;
}

// Relative residual ||b - A x|| / ||b|| on the device (hecmw_rel_resid_L2_33).
double rel_resid_device(Solver &S) {
  cudaStream_t s = S.stream;
  CgState *st = S.state.p;
  launch_k(s, spmv_kernel<double, 1>, S.grid_spmv(), kThreads, S.A.view(), S.x.p, S.w.p, S.b.p, nullptr, nullptr);
  launch_k(s, dot_kernel<double, 2>, S.grid_vec(), kThreads, S.w.p, S.w.p, S.n3(), st, S.partials.p, 0, 0);
  double rr = 0.0;
  H33_CUDA(cudaMemcpyAsync(&rr, &st->rr_true, sizeof(double), cudaMemcpyDeviceToHost, s));
  S.sync();
  double bb = S.bnrm2;
  if (bb == 0.0) bb = 1.0;
  return std::sqrt(rr / bb);
}

double dot_device_f(Solver &S, const float *a, const float *b) {
  CgState *st = S.state.p;
  launch_k(S.stream, dot_kernel<float, 2>, S.grid_vec(), kThreads, a, b, S.n3(), st, S.partials.p, 0, 0);
  double v = 0.0;
  H33_CUDA(cudaMemcpyAsync(&v, &st->rr_true, sizeof(double), cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  return v;
}

double dot_device(Solver &S, const double *a, const double *b) {
  CgState *st = S.state.p;
  launch_k(S.stream, dot_kernel<double, 2>, S.grid_vec(), kThreads, a, b, S.n3(), st, S.partials.p, 0, 0);
  double v = 0.0;
  H33_CUDA(cudaMemcpyAsync(&v, &st->rr_true, sizeof(double), cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  return v;
}

// FP32 copies of one preconditioner's values (same layouts).
void ensure_fp32_pc(Solver &S, Precond &P) {
  auto conv = [&](const double *a, float *b, size_t n) {
    if (n == 0) return;
    const int grid = int(std::min<size_t>((n + kThreads - 1) / kThreads, size_t(S.nsm) * 16));
    launch_k(S.stream, convert_kernel<float>, grid, kThreads, a, b, n);
    H33_CUDA(cudaGetLastError());
  };
  if (P.fp32_version != P.numeric_version) {
    for (auto *d : {&P.lo, &P.up}) {
      d->val32.alloc(d->val.n);
      conv(d->val.p, d->val32.p, d->val.n);
    }
    P.alu32_fwd.alloc(P.alu_fwd.n);
    conv(P.alu_fwd.p, P.alu32_fwd.p, P.alu_fwd.n);
    if (!P.alu_shared) {
      P.alu32_bwd.alloc(P.alu_bwd.n);
      conv(P.alu_bwd.p, P.alu32_bwd.p, P.alu_bwd.n);
    }
    P.fp32_version = P.numeric_version;
  }
}

// FP32 copies of the matrix and preconditioner values (same sliced layouts),
// refreshed when the FP64 values changed.
void ensure_fp32(Solver &S) {
  auto conv = [&](const double *a, float *b, size_t n) {
    if (n == 0) return;
    const int grid = int(std::min<size_t>((n + kThreads - 1) / kThreads, size_t(S.nsm) * 16));
    launch_k(S.stream, convert_kernel<float>, grid, kThreads, a, b, n);
    H33_CUDA(cudaGetLastError());
  };
  if (S.a32_version != S.values_version) {
    S.A.val32.alloc(S.A.val.n);
    conv(S.A.val.p, S.A.val32.p, S.A.val.n);
    S.a32_version = S.values_version;
  }
  ensure_fp32_pc(S, S.pc);
  const size_t n3 = size_t(S.n3());
  for (auto *v : {&S.bf, &S.xf, &S.rf, &S.zf, &S.pf, &S.qf, &S.wf, &S.zpf}) v->alloc(n3);
  if (S.zposf.n != n3) {
    S.zposf.alloc(n3);
    S.zposf.zero(S.stream);  // padding blocks gather zposf[0]
  }
}

// ---------------------------------------------------------------------------
// Learned preconditioner (host side)

// Node graph of the matrix (CSR of off-diagonal neighbours, reverse edges, raw
// block ids) and the scaled features; rebuilt when the profile / values change.
void learned_graph(Solver &S) {
  Learned &L = S.L;
  const int N = S.N;
  if (L.graph_generation < 0 || L.built_for != S.generation) {
    const int NPL = S.NPL;
    std::vector<int> ptr(size_t(N) + 1, 0);
    for (int i = 0; i < N; i++)
      ptr[size_t(i) + 1] = ptr[size_t(i)] + (S.indexL[size_t(i) + 1] - S.indexL[size_t(i)]) +
                           (S.indexU[size_t(i) + 1] - S.indexU[size_t(i)]);
    const int ne = ptr[size_t(N)];
    L.n = N;
    L.nedges = ne;
    L.ptr.upload(ptr, S.stream);
    if (host_layouts()) {
      std::vector<int> col, src, row_of, rev;
      col.reserve(size_t(ne));
      for (int i = 0; i < N; i++) {
        for (int j = S.indexL[i]; j < S.indexL[i + 1]; j++) {
          col.push_back(S.itemL[j] - 1);
          src.push_back(N + j);
          row_of.push_back(i);
        }
        for (int j = S.indexU[i]; j < S.indexU[i + 1]; j++) {
          col.push_back(S.itemU[j] - 1);
          src.push_back(N + NPL + j);
          row_of.push_back(i);
        }
      }
      rev.assign(size_t(ne), 0);
#pragma omp parallel for schedule(static)
      for (int e = 0; e < ne; e++) {
        const int i = row_of[e], j = col[e];
        const int *b = col.data() + ptr[j], *en = col.data() + ptr[j + 1];
        const int *f = std::lower_bound(b, en, i);
        rev[e] = (f != en && *f == i) ? int(f - col.data()) : e;
      }
      L.col.upload(col, S.stream);
      L.src.upload(src, S.stream);
      L.row_of.upload(row_of, S.stream);
      L.rev.upload(rev, S.stream);
    } else {
      // the edges, their raw ids, rows and reverses placed on the device from the
      // resident profile
      for (auto *a : {&L.col, &L.src, &L.row_of, &L.rev}) a->alloc(size_t(ne));
      const int gr = std::max(1, std::min((N + kThreads - 1) / kThreads, S.nsm * 8));
      launch_k(S.stream, fill_edges_kernel, gr, kThreads, dev_profile(S), static_cast<const int *>(L.ptr.p), L.col.p,
               L.src.p, L.row_of.p);
      const int ge = std::max(1, std::min((ne + kThreads - 1) / kThreads, S.nsm * 16));
      launch_k(S.stream, edge_reverse_kernel, ge, kThreads, N, static_cast<const int *>(L.ptr.p),
               static_cast<const int *>(L.col.p), static_cast<const int *>(L.row_of.p), ne, L.rev.p);
      H33_CUDA(cudaGetLastError());
    }
    L.feat.alloc(size_t(9) * std::max(ne, 1));
    L.s.alloc(size_t(N));
    L.w.alloc(size_t(kGnnLayers) * std::max(ne, 1));
    for (auto &h : L.h) h.alloc(size_t(N) * kGnnWidth);
    L.built_for = S.generation;
    L.graph_generation = ++S.build_counter;
    L.feat_version = -1;
  }
  if (L.feat_version != S.values_version) {
    const int grid = std::max(1, std::min((N + kThreads - 1) / kThreads, S.nsm * 8));
    launch_k(S.stream, gnn_node_scale_kernel, grid, kThreads, S.raw.p, N, L.s.p);
    const int ge = int(std::max<int64_t>(1, std::min<int64_t>((int64_t(9) * L.nedges + kThreads - 1) / kThreads,
                                                               int64_t(S.nsm) * 16)));
    launch_k(S.stream, gnn_edge_feat_kernel, ge, kThreads, L.graph(), L.row_of.p, L.src.p, S.raw.p, L.feat.p);
    H33_CUDA(cudaGetLastError());
    L.feat_version = S.values_version;
    L.w_version = -1;
  }
}

// Edge weights of the current weights (BF16 copy for inference, FP32 for training).
void learned_edge_weights(Solver &S, bool bf16) {
  Learned &L = S.L;
  const int ge = std::max(1, std::min((L.nedges + kThreads - 1) / kThreads, S.nsm * 16));
  if (bf16) launch_k(S.stream, gnn_edge_weights_kernel<__nv_bfloat16>, ge, kThreads, L.graph(), L.theta_bf16.p, L.w.p);
  else launch_k(S.stream, gnn_edge_weights_kernel<float>, ge, kThreads, L.graph(), L.theta.p, L.w.p);
  H33_CUDA(cudaGetLastError());
  L.w_version = bf16 ? L.weights_version : -1;
}

// ---- the coarse space of the learned two-level preconditioner -----------------
// HECMW33_COARSE_AGG: the largest number of aggregates (default 2000: 9x9x9-node
// aggregates on a 101^3-node mesh, a 4,239-DOF coarse matrix).
int coarse_max_aggregates() {
  static const int v = [] {
    const char *e = std::getenv("HECMW33_COARSE_AGG");
    return e ? std::max(1, std::atoi(e)) : 2000;
  }();
  return v;
}

// Aggregates, patterns and buffers (once per matrix structure).
void coarse_structure(Solver &S) {
  auto &C = S.L.C;
  if (C.built_for == S.generation) return;
  Profile prof{S.N, S.indexL.data(), S.itemL.data(), S.indexU.data(), S.itemU.data()};
  Aggregation ag;
  aggregate_nodes(prof, coarse_max_aggregates(), ag);
  // the unified rows (L, D, U per row) as CSR: the row pointers from the block counts,
  // the blocks placed on the device (on the host with HECMW33_HOST_LAYOUT=1)
  std::vector<int> uptr(size_t(S.N) + 1, 0);
  int64_t nu = 0;
  for (int i = 0; i < S.N; i++) {
    nu += (S.indexL[size_t(i) + 1] - S.indexL[size_t(i)]) + 1 + (S.indexU[size_t(i) + 1] - S.indexU[size_t(i)]);
    if (nu > int64_t(std::numeric_limits<int>::max()))
      throw Failure(HECMW33_ERR_BAD_INPUT, "coarse space: too many blocks for 32-bit row pointers");
    uptr[size_t(i) + 1] = int(nu);
  }
  C.uptr.upload(uptr, S.stream);
  if (host_layouts()) {
    BlockRows u;
    unified_rows(prof, u);
    C.ucol.upload(u.col, S.stream);
    C.usrc.upload(u.src, S.stream);
  } else {
    C.ucol.alloc(size_t(nu));
    C.usrc.alloc(size_t(nu));
    const int gr = std::max(1, std::min((S.N + kThreads - 1) / kThreads, S.nsm * 8));
    launch_k(S.stream, fill_unified_csr_kernel, gr, kThreads, dev_profile(S), static_cast<const int *>(C.uptr.p),
             C.ucol.p, C.usrc.p);
    H33_CUDA(cudaGetLastError());
  }
  C.n = S.N;
  C.nagg = ag.n_agg;
  C.nc = 3 * ag.n_agg;
  C.agg.upload(ag.agg, S.stream);
  C.pptr.upload(ag.pptr, S.stream);
  C.pagg.upload(ag.pagg, S.stream);
  C.rptr.upload(ag.rptr, S.stream);
  C.rnode.upload(ag.rnode, S.stream);
  C.rpos.upload(ag.rpos, S.stream);
  C.qptr.upload(ag.qptr, S.stream);
  C.qagg.upload(ag.qagg, S.stream);
  C.cptr.upload(ag.cptr, S.stream);
  C.cagg.upload(ag.cagg, S.stream);
  const size_t n3 = size_t(S.n3()), nnzp = ag.pagg.size(), nnzq = ag.qagg.size(), nc = size_t(C.nc);
  C.mask.alloc(n3);
  C.x.alloc(size_t(S.N) * 6);
  C.out.alloc(n3);
  C.omega.alloc(n3);
  C.dout.alloc(n3);
  C.t0.alloc(9 * nnzp);
  C.p.alloc(9 * nnzp);
  C.q.alloc(9 * nnzq);
  C.ac.alloc(nc * nc);
  C.gjc.alloc(nc * kGjBlock);
  C.gjb.alloc(nc * kGjBlock);
  C.gjd.alloc(size_t(kGjBlock) * kGjBlock);
  C.bc.alloc(nc);
  C.y.alloc(nc);
  C.v.alloc(n3);
  C.t0y.alloc(n3);
  C.apy.alloc(n3);
  C.dots.alloc(64);
  C.err.alloc(1);
  if (!C.one) {
    const float one = 1.0f;
    C.one_buf.upload(&one, 1, S.stream);
    C.one = C.one_buf.p;
  }
  C.built_for = S.generation;
  C.mask_version = C.t0_version = -1;
  C.op_precond = C.op_weights = C.op_mode = -1;
  C.ok = false;
  S.sync();
}

// DOF mask, the network's static input and T0 (per matrix values).
void coarse_values(Solver &S) {
  auto &C = S.L.C;
  if (C.t0_version == S.values_version) return;
  const int gt = std::max(1, std::min((S.N + kThreads - 1) / kThreads, S.nsm * 8));
  const int gw = std::max(1, std::min((S.N + kWarpsPerCta - 1) / kWarpsPerCta, S.nsm * 16));
  launch_k(S.stream, coarse_mask_kernel, gw, kThreads, C.view(), static_cast<const double *>(S.raw.p));
  launch_k(S.stream, coarse_features_kernel, gt, kThreads, C.view(), C.x.p);
  launch_k(S.stream, coarse_t0_kernel, gw, kThreads, C.view(), static_cast<const double *>(S.raw.p));
  H33_CUDA(cudaGetLastError());
  C.t0_version = S.values_version;
}

// omega = sigmoid(W_out h3) of the network on the static features: BF16 weights
// (inference) or FP32 master weights with the activations kept (training).
void coarse_omega(Solver &S, bool bf16, bool keep) {
  Learned &L = S.L;
  auto &C = L.C;
  cudaStream_t s = S.stream;
  const GnnGraph g = L.graph();
  const int gw = std::max(1, std::min((S.N + kWarpsPerCta - 1) / kWarpsPerCta, S.nsm * 8));
  const int gt = std::max(1, std::min((S.N + kThreads - 1) / kThreads, S.nsm * 8));
  learned_edge_weights(S, bf16);
  if (bf16) {
    const __nv_bfloat16 *th = L.theta_bf16.p;
    launch_k(s, gnn_encode_static_kernel<__nv_bfloat16>, gt, kThreads, S.N, th, static_cast<const float *>(C.x.p),
             L.h[0].p);
    for (int l = 0; l < kGnnLayers; l++)
      launch_k(s, gnn_layer_kernel<__nv_bfloat16>, gw, kThreads, g, th, l, static_cast<const float *>(L.w.p),
               static_cast<const float *>(L.h[l].p), static_cast<float *>(nullptr), L.h[l + 1].p,
               static_cast<const CgState *>(nullptr));
    launch_k(s, gnn_omega_kernel<__nv_bfloat16>, gt, kThreads, S.N, th, static_cast<const float *>(L.h[3].p), C.out.p,
             C.omega.p);
  } else {
    const float *th = L.theta.p;
    launch_k(s, gnn_encode_static_kernel<float>, gt, kThreads, S.N, th, static_cast<const float *>(C.x.p), L.h[0].p);
    for (int l = 0; l < kGnnLayers; l++)
      launch_k(s, gnn_layer_kernel<float>, gw, kThreads, g, th, l, static_cast<const float *>(L.w.p),
               static_cast<const float *>(L.h[l].p), keep ? L.m[l].p : static_cast<float *>(nullptr), L.h[l + 1].p,
               static_cast<const CgState *>(nullptr));
    launch_k(s, gnn_omega_kernel<float>, gt, kThreads, S.N, th, static_cast<const float *>(L.h[3].p), C.out.p,
             C.omega.p);
  }
  H33_CUDA(cudaGetLastError());
}

// P from omega (nullptr: omega = 0, the unsmoothed aggregation), A P, Ac = P^T A P
// and its inverse in place (blocked Gauss-Jordan).  Returns false when a pivot of Ac
// was not positive (the coarse correction is then not applied).
bool coarse_operator(Solver &S, const float *omega) {
  auto &C = S.L.C;
  cudaStream_t s = S.stream;
  const CoarseView cv = C.view();
  const int gt = std::max(1, std::min((S.N + kThreads - 1) / kThreads, S.nsm * 8));
  const int gw = std::max(1, std::min((S.N + kWarpsPerCta - 1) / kWarpsPerCta, S.nsm * 16));
  launch_k(s, coarse_p_kernel, gt, kThreads, cv, omega);
  launch_k(s, coarse_ap_kernel, gw, kThreads, cv, static_cast<const double *>(S.raw.p));
  C.ac.zero(s);
  C.err.zero(s);
  launch_k(s, coarse_ac_kernel, std::max(1, S.nsm * 8), kThreads, cv);
  coarse_zero_diag_kernel<<<std::max(1, (C.nc + 255) / 256), 256, 0, s>>>(C.ac.p, C.nc);
  const int n = C.nc;
  H33_CUDA(cudaFuncSetAttribute(gj_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kGjUpdateSmem)));
  const dim3 tiles(unsigned((n + kGjTileJ - 1) / kGjTileJ), unsigned((n + kGjTileI - 1) / kGjTileI));
  for (int k0 = 0; k0 < n; k0 += kGjBlock) {
    const int nb = std::min(kGjBlock, n - k0);
    gj_diag_kernel<<<1, 1024, 0, s>>>(C.ac.p, n, k0, nb, C.gjd.p, C.err.p);
    gj_col_kernel<<<std::max(1, (n + 7) / 8), 256, 0, s>>>(C.ac.p, n, k0, nb, C.gjd.p, C.gjc.p, C.gjb.p);
    gj_update_kernel<<<tiles, 256, kGjUpdateSmem, s>>>(C.ac.p, n, k0, nb, C.gjc.p, C.gjb.p);
  }
  const unsigned nt = unsigned((n + 31) / 32);
  gj_mirror_kernel<<<dim3(nt, nt), 256, 0, s>>>(C.ac.p, n);
  // FP32 copies for the application
  auto conv = [&](const DevArray<double> &a, DevArray<float> &b) {
    b.alloc(a.n);
    const int grid = int(std::min<size_t>((a.n + kThreads - 1) / kThreads, size_t(S.nsm) * 16));
    launch_k(s, convert_kernel<float>, std::max(grid, 1), kThreads, static_cast<const double *>(a.p), b.p, a.n);
  };
  conv(C.p, C.p32);
  conv(C.q, C.q32);
  conv(C.ac, C.ainv32);
  H33_CUDA(cudaGetLastError());
  int err = 0;
  H33_CUDA(cudaMemcpyAsync(&err, C.err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  S.sync();
  C.ok = err == 0;
  return C.ok;
}

// z = zs + P Ac^-1 P^T r (or z = zs when the correction is off), in the solve's stream.
// z = zs + P Ac^-1 P^T r (additive form), with the FP32 copies.
template <class R>
void launch_coarse(Solver &S, const R *zs, const R *r, R *z, CgState *st) {
  auto &C = S.L.C;
  cudaStream_t s = S.stream;
  const CoarseApply ca = C.apply_view();
  const int gt = std::max(1, std::min((S.N + kThreads - 1) / kThreads, S.nsm * 8));
  launch_k(s, coarse_restrict32_kernel<R>, std::max(1, C.nagg), 256, ca, r, C.bc.p,
           static_cast<const CgState *>(st));
  launch_k(s, coarse_gemv32_kernel, std::max(1, std::min((C.nc + kWarpsPerCta - 1) / kWarpsPerCta, S.nsm * 8)),
           kThreads, C.nc, static_cast<const float *>(C.ainv32.p), static_cast<const double *>(C.bc.p), C.y.p,
           static_cast<const CgState *>(st));
  launch_k(s, coarse_prolong32_kernel<R>, gt, kThreads, ca, static_cast<const double *>(C.y.p), zs, z,
           static_cast<const CgState *>(st));
}

template <class R>
void launch_coarse_cycle(Solver &S, const R *zs, R *w, R *zc, CgState *st) {
  auto &C = S.L.C;
  cudaStream_t s = S.stream;
  const CoarseApply ca = C.apply_view();
  const int gt = std::max(1, std::min((S.N + kThreads - 1) / kThreads, S.nsm * 8));
  launch_k(s, coarse_restrict32_kernel<R>, std::max(1, C.nagg), 256, ca, static_cast<const R *>(w), C.bc.p,
           static_cast<const CgState *>(st));
  launch_k(s, coarse_gemv32_kernel, std::max(1, std::min((C.nc + kWarpsPerCta - 1) / kWarpsPerCta, S.nsm * 8)),
           kThreads, C.nc, static_cast<const float *>(C.ainv32.p), static_cast<const double *>(C.bc.p), C.y.p,
           static_cast<const CgState *>(st));
  launch_k(s, coarse_prolong_resid32_kernel<R>, gt, kThreads, ca, static_cast<const double *>(C.y.p), zs, zc, w,
           static_cast<const CgState *>(st));
}

void learned_set_weights(Solver &S, const float *theta_host, bool reset_adam) {
  Learned &L = S.L;
  const int n = GnnOffsets::make().total;
  L.theta.upload(theta_host, size_t(n), S.stream);
  std::vector<__nv_bfloat16> b(static_cast<size_t>(n));
  for (int k = 0; k < n; k++) b[size_t(k)] = __float2bfloat16(theta_host[k]);
  L.theta_bf16.upload(b.data(), b.size(), S.stream);
  if (reset_adam || L.m1.n != size_t(n)) {
    L.m1.alloc(size_t(n));
    L.m2.alloc(size_t(n));
    L.m1.zero(S.stream);
    L.m2.zero(S.stream);
    L.adam_step = 0;
  }
  L.grad.alloc(size_t(n));
  L.gacc.alloc(size_t(n));
  L.have_weights = true;
  L.weights_version++;
  S.sync();
}

// Deterministic initial weights (scaled Gaussian; the output layer starts at zero).
void learned_init_weights(Solver &S, uint64_t seed) {
  const GnnOffsets o = GnnOffsets::make();
  std::vector<float> th(size_t(o.total), 0.0f);
  uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
  auto normal = [&]() {
    auto next = [&]() {
      uint64_t z = (st += 0x9E3779B97F4A7C15ull);
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      return double((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
    };
    double u1 = next(), u2 = next();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  };
  for (int k = 0; k < kGnnWidth * 6; k++) th[size_t(o.W_in + k)] = float(normal() / std::sqrt(6.0));
  for (int l = 0; l < kGnnLayers; l++) {
    for (int k = 0; k < 9; k++) th[size_t(o.u[l] + k)] = float(0.3 * normal());
    th[size_t(o.c[l])] = 0.5f;
    for (int k = 0; k < kGnnWidth * kGnnWidth; k++) {
      th[size_t(o.Ws[l] + k)] = float(normal() / std::sqrt(double(kGnnWidth)));
      th[size_t(o.Wm[l] + k)] = float(normal() / std::sqrt(double(kGnnWidth)) / 8.0);
    }
  }
  // W_out = 0: the untrained network gives omega = 1/2 everywhere
  for (int k = 0; k < 3 * kGnnWidth; k++) th[size_t(o.W_out + k)] = 0.0f;
  learned_set_weights(S, th.data(), true);
}

// Ready for inference inside a solve: the coarse space of the current matrix values,
// preconditioner and weights (the network's omega with BF16 weights, or the fixed
// omega of coarse_mode 1 / 2), its inverse, and the flexible-CG buffers.
void learned_prepare_inference(Solver &S) {
  Learned &L = S.L;
  auto &C = L.C;
  if (L.coarse_mode == 0 && !L.have_weights)
    throw Failure(HECMW33_ERR_INCONS_PC, "learned preconditioner requested but not trained");
  if (!(S.pc.valid && S.pc.kind == 1))
    throw Failure(HECMW33_ERR_INCONS_PC, "the learned preconditioner works after SSOR (PRECOND 1 or 2)");
  if (S.dom.on)
    throw Failure(HECMW33_ERR_INCONS_PC, "the learned preconditioner takes a whole mesh (one domain) only");
  ensure_smoother(S);
  if (L.coarse_mode == 0) {  // the network's graph and features (the fixed weights need neither)
    learned_graph(S);
    setup_mark("learned: network graph");
  }
  coarse_structure(S);
  setup_mark("learned: aggregates, P and A P structure");
  coarse_values(S);
  setup_mark("learned: coarse values");
  if (S.a32_version != S.values_version) {  // FP32 A for the residuals of the mode-1 preconditioner
    S.A.val32.alloc(S.A.val.n);
    const size_t n = S.A.val.n;
    launch_k(S.stream, convert_kernel<float>, int(std::min<size_t>((n + kThreads - 1) / kThreads, size_t(S.nsm) * 16)),
             kThreads, static_cast<const double *>(S.A.val.p), S.A.val32.p, n);
    H33_CUDA(cudaGetLastError());
    S.a32_version = S.values_version;
  }
  const int wv = L.coarse_mode == 0 ? L.weights_version : -1;
  if (C.op_precond != S.pc.numeric_version || C.op_weights != wv || C.op_mode != L.coarse_mode) {
    const float *omega = nullptr;
    if (L.coarse_mode == 0) {
      coarse_omega(S, true, false);
      omega = C.omega.p;
    } else if (L.coarse_mode == 2) {
      std::vector<float> half(size_t(S.n3()), 0.5f);
      C.omega.upload(half, S.stream);
      omega = C.omega.p;
    }
    setup_mark("learned: FP32 A, omega");
    coarse_operator(S, omega);
    setup_mark("learned: Ac and its inverse");
    C.op_precond = S.pc.numeric_version;
    C.op_weights = wv;
    C.op_mode = L.coarse_mode;
  }
  const size_t n3 = size_t(S.n3());
  S.zs.alloc(n3);
  S.dpos.alloc(n3);
  S.rold.alloc(n3);
  S.zsf.alloc(n3);
  S.roldf.alloc(n3);
}

// Training buffers (activations saved for the backward pass).
void learned_train_buffers(Solver &S) {
  Learned &L = S.L;
  const size_t nw = size_t(S.N) * kGnnWidth;
  for (auto &m : L.m) m.alloc(nw);
  L.x.alloc(size_t(S.N) * 6);
  L.gm.alloc(nw);
  L.dh.alloc(nw);
  L.dhp.alloc(nw);
  const size_t n3 = size_t(S.n3());
  for (auto *v : {&L.t_z, &L.t_zs, &L.t_d, &L.t_q, &L.t_dz}) v->alloc(n3);
  L.nparts = std::max(1, std::min((S.N + kWarpsPerCta - 1) / kWarpsPerCta, S.nsm * 4));
  L.stride = GnnOffsets::make().total;
  L.part.alloc(size_t(L.nparts) * L.stride);
}

// One pass of the training loss over pairs (r_k, e_k, e_k.r_k) with the FP32 master
// weights: the network's omega (activations kept for the backward pass), the coarse
// operator, then per pair  y = Ac^-1 P^T r,  loss_k = (e.r - (P^T r).y) / e.r  (the
// energy of e outside the coarse space, relative to its energy) and its gradient in
// out (coarse_grad_kernel).  With backward, the network's backward pass turns the mean
// gradient into L.gacc.  Returns the mean loss.
double learned_coarse_pass(Solver &S, const std::vector<const float *> &pr, const std::vector<double> &per,
                           bool backward) {
  Learned &L = S.L;
  auto &C = L.C;
  cudaStream_t s = S.stream;
  const int np = int(pr.size());
  const int n3 = S.n3();
  coarse_omega(S, false, backward);
  if (!coarse_operator(S, C.omega.p))
    throw Failure(HECMW33_ERR_INCONS_PC, "learned preconditioner: the coarse matrix is not positive definite");
  const CoarseView cv = C.view();
  const int gt = std::max(1, std::min((S.N + kThreads - 1) / kThreads, S.nsm * 8));
  const int gr = std::max(1, std::min((C.nagg + kWarpsPerCta - 1) / kWarpsPerCta, S.nsm * 8));
  const int gg = std::max(1, std::min((C.nc + kWarpsPerCta - 1) / kWarpsPerCta, S.nsm * 8));
  C.dout.zero(s);
  L.losses.alloc(size_t(std::max(np, 1)));
  for (int k = 0; k < np; k++) {
    launch_k(s, coarse_restrict_kernel<float>, gr, kThreads, cv, pr[size_t(k)], C.bc.p,
             static_cast<const CgState *>(nullptr));
    launch_k(s, coarse_gemv_kernel, gg, kThreads, C.nc, static_cast<const double *>(C.ac.p),
             static_cast<const double *>(C.bc.p), C.y.p, static_cast<const CgState *>(nullptr));
    launch_k(s, coarse_prolong_kernel<float>, gt, kThreads, cv, static_cast<const double *>(C.y.p),
             static_cast<const float *>(nullptr), static_cast<float *>(nullptr), C.v.p, C.t0y.p,
             static_cast<const CgState *>(nullptr));
    launch_k(s, spmv_kernel<double, 0>, S.grid_spmv(), kThreads, S.A.view(), static_cast<const double *>(C.v.p),
             C.apy.p, static_cast<const double *>(nullptr), static_cast<CgState *>(nullptr),
             static_cast<double *>(nullptr));
    launch_k(s, coarse_grad_kernel<float>, S.grid_vec(), kThreads, n3, pr[size_t(k)],
             static_cast<const double *>(C.apy.p), static_cast<const double *>(C.t0y.p),
             static_cast<const float *>(C.omega.p), 1.0 / (per[size_t(k)] * np), C.dout.p);
    coarse_dot_kernel<<<1, 256, 0, s>>>(C.nc, C.bc.p, C.y.p, L.losses.p + k);
  }
  H33_CUDA(cudaGetLastError());
  if (backward) {
    const GnnGraph g = L.graph();
    const int gw = std::max(1, std::min((S.N + kWarpsPerCta - 1) / kWarpsPerCta, S.nsm * 8));
    const int npart = L.nparts, stride = L.stride;
    launch_k(s, gnn_decode_bwd_kernel, npart, kThreads, S.N, static_cast<const float *>(L.theta.p),
             static_cast<const float *>(L.h[3].p), static_cast<const float *>(C.dout.p),
             static_cast<const float *>(C.one), L.dh.p, L.part.p, stride);
    for (int l = kGnnLayers - 1; l >= 0; l--) {
      launch_k(s, gnn_layer_bwd_kernel, npart, kThreads, g, static_cast<const float *>(L.theta.p), l,
               static_cast<const float *>(L.w.p), static_cast<const float *>(L.h[l].p),
               static_cast<const float *>(L.h[l + 1].p), static_cast<const float *>(L.m[l].p),
               static_cast<const float *>(L.dh.p), L.gm.p, L.dhp.p, L.part.p, stride);
      launch_k(s, gnn_layer_bwd_gather_kernel, gw, kThreads, g, l, static_cast<const float *>(L.w.p),
               static_cast<const float *>(L.gm.p), L.dhp.p);
      std::swap(L.dh, L.dhp);
    }
    launch_k(s, gnn_encode_bwd_kernel, npart, kThreads, S.N, static_cast<const float *>(C.x.p),
             static_cast<const float *>(L.dh.p), L.part.p, stride);
    launch_k(s, gnn_reduce_grads_kernel, (stride + 255) / 256, 256, static_cast<const float *>(L.part.p), npart,
             stride, L.gacc.p, stride);
    H33_CUDA(cudaGetLastError());
  }
  std::vector<double> by(size_t(std::max(np, 1)));
  H33_CUDA(cudaMemcpyAsync(by.data(), L.losses.p, sizeof(double) * size_t(np), cudaMemcpyDeviceToHost, s));
  S.sync();
  double m = 0.0;
  for (int k = 0; k < np; k++) m += (per[size_t(k)] - by[size_t(k)]) / per[size_t(k)];
  return np ? m / np : 0.0;
}

// FP64 CG in stream mode, one iteration per host step, keeping x at iterations
// 1, 2, 4, 8, ... (x_0 = the start); after convergence every kept x_k gives a
// training pair (r_k = b - A x_k, e_k = x* - x_k) for the learned preconditioner.
float record_cg(Solver &S, int iterpremax, double tol, int maxit, int *kernels) {
  Learned &L = S.L;
  const Views<double> V = views(S, 0.0);
  const size_t n3 = size_t(S.n3());
  S.h_params->tol = tol;
  S.h_params->maxit = maxit;
  S.h_params->iterpremax = iterpremax;
  S.h_params->inner = 0;
  S.h_params->flexible = 0;
  S.h_params->use_gnn = 0;
  S.h_params->reliable = 0;
  S.h_params->ru_delta = 1.0;
  S.h_params->method = 1;
  S.h_params->lanczos = nullptr;
  S.h_params->lanczos_cap = 0;
  S.h_params->rhist = nullptr;
  S.h_params->rhist_cap = 0;
  H33_CUDA(cudaMemcpyAsync(S.params.p, S.h_params, sizeof(CgParams), cudaMemcpyHostToDevice, S.stream));
  H33_CUDA(cudaEventRecord(S.ev0, S.stream));
  launch_prologue<double>(S, V, 0, 0);
  std::vector<DevArray<double>> snaps;
  int next = 1;
  for (int it = 1; it <= maxit + 1; it++) {
    if (it == next && snaps.size() < 24) {
      snaps.emplace_back();
      snaps.back().alloc(n3);
      H33_CUDA(cudaMemcpyAsync(snaps.back().p, S.x.p, n3 * sizeof(double), cudaMemcpyDeviceToDevice, S.stream));
      next *= 2;
    }
    launch_iteration<double>(S, V, iterpremax, 0, 0);
    H33_CUDA(cudaGetLastError());
    H33_CUDA(cudaMemcpyAsync(S.h_state, S.state.p, sizeof(CgState), cudaMemcpyDeviceToHost, S.stream));
    S.sync();
    if (S.h_state->done) break;
  }
  H33_CUDA(cudaEventRecord(S.ev1, S.stream));
  S.sync();
  float ms = 0.0f;
  H33_CUDA(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
  if (kernels) *kernels += 3 + S.h_state->iter * 40;
  if (S.h_state->error == 0 && S.h_state->converged) {
    const int gt = S.grid_vec();
    for (auto &x : snaps) {
      DevArray<float> pr, pe;
      pr.alloc(n3);
      pe.alloc(n3);
      launch_k(S.stream, spmv_kernel<double, 1>, S.grid_spmv(), kThreads, S.A.view(), x.p, S.w.p, S.b.p, nullptr,
                                                                        nullptr);
      launch_k(S.stream, narrow_kernel, gt, kThreads, S.w.p, pr.p, int(n3));
      launch_k(S.stream, diff_narrow_kernel, gt, kThreads, S.x.p, x.p, pe.p, int(n3));
      H33_CUDA(cudaGetLastError());
      // e.r of the stored FP32 pair (FP64 accumulation) -- the normaliser of its loss
      const double er = dot_device_f(S, pe.p, pr.p);
      if (!(er > 0.0)) continue;
      L.pr.push_back(std::move(pr));
      L.pe.push_back(std::move(pe));
      L.pzs.emplace_back();
      L.per.push_back(er);
      while (int(L.pr.size()) > L.max_pairs) {
        L.pr.erase(L.pr.begin());
        L.pe.erase(L.pe.begin());
        L.pzs.erase(L.pzs.begin());
        L.per.erase(L.per.begin());
      }
    }
    S.sync();
  }
  return ms;
}

// Trains the network on the recorded pairs, smoothed once by the two-grid cycle's
// SSOR smoother (Learned::sm): Adam on the mean
// loss of learned_coarse_pass.  loss[0] = mean loss before the first step, loss[1] =
// after the last.
void learned_train(Solver &S, int steps, double lr, double *loss) {
  Learned &L = S.L;
  const int np = int(L.pr.size());
  if (np == 0) throw Failure(HECMW33_ERR_BAD_INPUT, "no recorded pairs: enable recording and solve first");
  if (!(S.pc.valid && S.pc.kind == 1))
    throw Failure(HECMW33_ERR_INCONS_PC, "training needs the SSOR preconditioner of the matrix");
  learned_graph(S);
  learned_train_buffers(S);
  coarse_structure(S);
  coarse_values(S);
  if (!L.have_weights) learned_init_weights(S, 12345);
  // The coarse correction has to capture what SSOR leaves: each pair's error after
  // one SSOR step, e' = e - SSOR(r), with r' = A e' (FP64, stored as FP32).
  std::vector<DevArray<float>> sr(static_cast<size_t>(np));
  std::vector<double> ser(static_cast<size_t>(np));
  std::vector<const float *> pr;
  {
    auto &C = L.C;
    ensure_smoother(S);
    const Views<double> V = views(S, 0.0, 0, &S.L.sm);
    const int gt = S.grid_vec(), n3 = S.n3();
    for (int k = 0; k < np; k++) {
      launch_k(S.stream, coarse_widen_kernel, gt, kThreads, static_cast<const float *>(L.pr[size_t(k)].p),
               static_cast<const double *>(nullptr), S.w.p, n3);
      launch_sweep<double, false>(S, V, S.w.p, C.v.p, nullptr);
      launch_k(S.stream, coarse_widen_kernel, gt, kThreads, static_cast<const float *>(L.pe[size_t(k)].p),
               static_cast<const double *>(C.v.p), C.t0y.p, n3);
      launch_k(S.stream, spmv_kernel<double, 0>, S.grid_spmv(), kThreads, S.A.view(),
               static_cast<const double *>(C.t0y.p), C.apy.p, static_cast<const double *>(nullptr),
               static_cast<CgState *>(nullptr), static_cast<double *>(nullptr));
      sr[size_t(k)].alloc(size_t(n3));
      launch_k(S.stream, narrow_kernel, gt, kThreads, static_cast<const double *>(C.apy.p), sr[size_t(k)].p, n3);
      H33_CUDA(cudaGetLastError());
      ser[size_t(k)] = dot_device(S, C.t0y.p, C.apy.p);
      if (!(ser[size_t(k)] > 0.0)) throw Failure(HECMW33_ERR_CUDA, "learned training: a smoothed pair lost its energy");
      pr.push_back(sr[size_t(k)].p);
    }
  }
  const int nparam = GnnOffsets::make().total;
  loss[0] = learned_coarse_pass(S, pr, ser, false);
  for (int it = 0; it < steps; it++) {
    learned_coarse_pass(S, pr, ser, true);
    L.adam_step++;
    launch_k(S.stream, gnn_adam_kernel, (nparam + 255) / 256, 256, L.theta.p, static_cast<const float *>(L.gacc.p),
             L.m1.p, L.m2.p, nparam, float(lr), 0.9f, 0.999f, 1e-8f, L.adam_step, 1.0f, L.theta_bf16.p);
    H33_CUDA(cudaGetLastError());
  }
  loss[1] = learned_coarse_pass(S, pr, ser, false);
  L.weights_version++;
}

// BF16 copies of the preconditioner's sweep values and FP32 copies of its diagonal
// LU (same layouts), refreshed when the preconditioner's values changed.
void ensure_lowp(Solver &S, Precond &P) {
  if (P.lowp_version == P.numeric_version) return;
  auto grid = [&](size_t n) { return int(std::max<size_t>(1, std::min<size_t>((n + kThreads - 1) / kThreads, size_t(S.nsm) * 16))); };
  for (auto *d : {&P.lo, &P.up}) {
    d->val16.alloc(d->val.n);
    if (d->val.n) launch_k(S.stream, convert_bf16_kernel, grid(d->val.n), kThreads, d->val.p, d->val16.p, d->val.n);
  }
  P.alu32_fwd.alloc(P.alu_fwd.n);
  if (P.alu_fwd.n) launch_k(S.stream, convert_kernel<float>, grid(P.alu_fwd.n), kThreads, P.alu_fwd.p, P.alu32_fwd.p, P.alu_fwd.n);
  if (!P.alu_shared) {
    P.alu32_bwd.alloc(P.alu_bwd.n);
    launch_k(S.stream, convert_kernel<float>, grid(P.alu_bwd.n), kThreads, P.alu_bwd.p, P.alu32_bwd.p, P.alu_bwd.n);
  }
  H33_CUDA(cudaGetLastError());
  P.lowp_version = P.numeric_version;
  P.fp32_version = -1;  // the FP32 ALU copy now follows the low-precision path
}
void ensure_lowp(Solver &S) { ensure_lowp(S, S.pc); }

// Checks and preconditioner setup shared by the FP64 and mixed solves
// (hecmw_solve + hecmw_solve_iterative up to the CG call).  Returns 0 to go on,
// or the code to return (2002 with X = 0, 2001).
// Row and column (0-based nodes) of every raw block, for the kernels that need a
// block's position (scaling, constraints); rebuilt when the profile changes.
void ensure_block_rc(Solver &S) {
  if (S.blk_generation == S.generation) return;
  const int N = S.N;
  const int64_t nb = int64_t(N) + S.NPL + S.NPU;
  std::vector<int> br(static_cast<size_t>(nb)), bc(static_cast<size_t>(nb));
  for (int i = 0; i < N; i++) {
    br[size_t(i)] = bc[size_t(i)] = i;
    for (int j = S.indexL[i]; j < S.indexL[i + 1]; j++) {
      br[size_t(N) + j] = i;
      bc[size_t(N) + j] = S.itemL[j] - 1;
    }
    for (int j = S.indexU[i]; j < S.indexU[i + 1]; j++) {
      br[size_t(N) + S.NPL + j] = i;
      bc[size_t(N) + S.NPL + j] = S.itemU[j] - 1;
    }
  }
  S.blk_row.upload(br, S.stream);
  S.blk_col.upload(bc, S.stream);
  S.blk_generation = S.generation;
}

// SCALING=YES (Iarray(7), hecmw_solver_scaling_33.f90:20-208): the solve runs on
// S A S, S b with S = diag(1/sqrt|D_kk|), and X is multiplied by S after each CG
// (hecmw_solver_CG.f90:102,283).  The device works on a scaled copy of the resident
// values (the borrowed host arrays are never written); restore() brings back the
// unscaled values and right-hand side, so the driver's final true residual is that
// of the unscaled system, as in hecmw_solver_Iterative.f90:153.
struct ScaleScope {
  Solver &S;
  bool on, active = false;
  ScaleScope(Solver &S_, bool on_) : S(S_), on(on_) {
    if (!on) return;
    const int N = S.N;
    const int64_t nb = int64_t(N) + S.NPL + S.NPU;
    ensure_block_rc(S);
    const int n3 = S.n3();
    S.scale.alloc(size_t(n3));
    S.raw_scaled.alloc(S.raw.n);
    S.b_unscaled.alloc(size_t(n3));
    const int gv = S.grid_vec();
    launch_k(S.stream, scale_vector_kernel, gv, kThreads, static_cast<const double *>(S.raw.p), N, S.scale.p);
    const int gb = std::max(1, std::min(int((9 * nb + kThreads - 1) / kThreads), S.nsm * 8));
    launch_k(S.stream, scale_blocks_kernel, gb, kThreads, static_cast<const double *>(S.raw.p), S.raw_scaled.p,
             static_cast<const int *>(S.blk_row.p), static_cast<const int *>(S.blk_col.p),
             static_cast<const double *>(S.scale.p), nb);
    H33_CUDA(cudaMemcpyAsync(S.b_unscaled.p, S.b.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, S.stream));
    launch_k(S.stream, mul_vec_kernel, gv, kThreads, S.b.p, static_cast<const double *>(S.scale.p), n3);
    std::swap(S.raw, S.raw_scaled);
    S.A.pack(S.raw.p, S.stream, S.nsm);
    S.values_version++;
    active = true;
  }
  // X = S X (hecmw_solver_scaling_bk_33, :144-147)
  void x_back() {
    if (on) launch_k(S.stream, mul_vec_kernel, S.grid_vec(), kThreads, S.x.p, static_cast<const double *>(S.scale.p),
                     S.n3());
  }
  void restore() {
    if (!active) return;
    active = false;
    std::swap(S.raw, S.raw_scaled);
    S.A.pack(S.raw.p, S.stream, S.nsm);
    S.values_version++;
    H33_CUDA(cudaMemcpyAsync(S.b.p, S.b_unscaled.p, sizeof(double) * S.n3(), cudaMemcpyDeviceToDevice, S.stream));
  }
  ~ScaleScope() {
    if (!active) return;  // an error path: put the unscaled values back, errors ignored
    std::swap(S.raw, S.raw_scaled);
    const int total = S.A.nslots * 32;
    if (total > 0)
      pack_sell_kernel<double><<<std::min((total + kThreads - 1) / kThreads, S.nsm * 8), kThreads, 0, S.stream>>>(
          S.A.val.p, S.A.src.p, S.A.nslots, S.raw.p);
    S.values_version++;
    cudaMemcpyAsync(S.b.p, S.b_unscaled.p, sizeof(double) * S.n3(), cudaMemcpyDeviceToDevice, S.stream);
  }
};

// HEX8 assembly on the device (the caller side of hecmw_solve): profile
// (hecmw_mat_con) and per-block contribution lists on the host when `symbolic`,
// element blocks and their element-order sums on the device, nodal loads F, then
// the constraints (hecmw_mat_ass_bc) in list order.  Leaves the matrix and the
// right-hand side resident, as set_matrix and a B upload would.
// Material: linear elastic (E, nu per element) or, when U is given, compressible
// Neo-Hookean (C10, D1) at nodal displacements U: tangent K(U) and right-hand side
// F - f_int(U); *inverted receives the number of elements with J <= 0.
struct HexMaterial {
  const double *E = nullptr, *nu = nullptr;  // linear elastic
  const double *U = nullptr;                 // Neo-Hookean
  double C10 = 0.0, D1 = 0.0;
};

void assemble_hex8(Solver &S, int n_node, const double *coords, int n_elem, const int *conn,
                   const HexMaterial &mat, const double *F, int n_bc, const int *bc_node, const int *bc_dof,
                   const double *bc_value, bool symbolic, int *inverted = nullptr) {
  auto &M = S.asmb;
  if (n_node < 1 || n_elem < 1) throw Failure(HECMW33_ERR_BAD_INPUT, "empty mesh");
  if (S.dom.on) {  // the assembled mesh is one whole domain
    S.dom.reset();
    symbolic = true;
  }
  if (!symbolic && (M.generation != S.generation || M.n_node != n_node || M.n_elem != n_elem))
    symbolic = true;
  if (symbolic) {
    std::vector<int> iL, tL, iU, tU;
    try {
      element_profile(n_node, n_elem, 8, conn, iL, tL, iU, tU);
    } catch (const std::exception &e) {
      throw Failure(HECMW33_ERR_BAD_INPUT, e.what());
    }
    set_profile(S, n_node, iL[size_t(n_node)], iU[size_t(n_node)], iL.data(), tL.data(), iU.data(), tU.data());
    std::vector<int64_t> ptr;
    std::vector<int> code;
    element_contributions(n_node, n_elem, 8, conn, iL, tL, iU, tU, ptr, code);
    M.ptr.upload(ptr, S.stream);
    M.code.upload(code, S.stream);
    M.conn.upload(conn, size_t(n_elem) * 8, S.stream);
    M.indexL.upload(iL, S.stream);
    M.indexU.upload(iU, S.stream);
    M.itemL.upload(tL.empty() ? std::vector<int>{0} : tL, S.stream);
    M.itemU.upload(tU.empty() ? std::vector<int>{0} : tU, S.stream);
    M.Ke.alloc(size_t(n_elem) * 576);
    M.n_node = n_node;
    M.n_elem = n_elem;
    M.generation = S.generation;
  }
  ensure_block_rc(S);
  cudaStream_t s = S.stream;
  M.coords.upload(coords, size_t(3) * n_node, s);
  const int64_t nb = int64_t(n_node) + S.NPL + S.NPU;
  S.raw.alloc(size_t(9 * nb));
  const int64_t ne64 = int64_t(n_elem) * 64;
  const bool nh = mat.U != nullptr;
  M.flag.alloc(2);
  H33_CUDA(cudaMemsetAsync(M.flag.p, 0, 2 * sizeof(int), s));
  if (nh) {
    M.U.upload(mat.U, size_t(3) * n_node, s);
    M.fe.alloc(size_t(n_elem) * 24);
    launch_k(s, neohooke_element_kernel, int((ne64 + 127) / 128), 128, static_cast<const double *>(M.coords.p),
             static_cast<const double *>(M.U.p), static_cast<const int *>(M.conn.p), n_elem, mat.C10, mat.D1,
             M.Ke.p, M.fe.p, M.flag.p + 1);
  } else {
    M.E.upload(mat.E, size_t(n_elem), s);
    M.nu.upload(mat.nu, size_t(n_elem), s);
    launch_k(s, hex8_element_kernel, int((ne64 + 255) / 256), 256, static_cast<const double *>(M.coords.p),
             static_cast<const int *>(M.conn.p), n_elem, static_cast<const double *>(M.E.p),
             static_cast<const double *>(M.nu.p), M.Ke.p);
  }
  launch_k(s, hex8_gather_kernel, int((9 * nb + 255) / 256), 256, static_cast<const double *>(M.Ke.p),
           static_cast<const int64_t *>(M.ptr.p), static_cast<const int *>(M.code.p), nb, S.raw.p);
  // right-hand side: nodal loads (minus the internal forces), then the constraints
  if (F) H33_CUDA(cudaMemcpyAsync(S.b.p, F, sizeof(double) * 3 * n_node, cudaMemcpyHostToDevice, s));
  else H33_CUDA(cudaMemsetAsync(S.b.p, 0, sizeof(double) * 3 * n_node, s));
  if (nh)
    launch_k(s, node_force_gather_kernel, (3 * n_node + 255) / 256, 256, static_cast<const double *>(M.fe.p),
             static_cast<const int64_t *>(M.ptr.p), static_cast<const int *>(M.code.p), n_node, S.b.p);
  if (n_bc > 0) {
    std::vector<int> first(size_t(3) * n_node, -1), last(size_t(3) * n_node, -1);
    for (int k = 0; k < n_bc; k++) {
      if (bc_node[k] < 1 || bc_node[k] > n_node || bc_dof[k] < 1 || bc_dof[k] > 3)
        throw Failure(HECMW33_ERR_BAD_INPUT, "constraint node or dof out of range");
      const size_t at = size_t(3) * (bc_node[k] - 1) + (bc_dof[k] - 1);
      if (first[at] < 0) first[at] = k;
      last[at] = k;
    }
    M.bc_first.upload(first, s);
    M.bc_last.upload(last, s);
    M.bc_value.upload(bc_value, size_t(n_bc), s);
    const BcArgs args{n_node, M.indexL.p, M.itemL.p, M.indexU.p, M.itemU.p, M.bc_first.p, M.bc_last.p,
                      M.bc_value.p};
    launch_k(s, bc_rhs_kernel, (3 * n_node + 255) / 256, 256, args, static_cast<const double *>(S.raw.p), S.b.p);
    launch_k(s, bc_matrix_kernel, int((9 * nb + 255) / 256), 256, args, static_cast<const int *>(S.blk_row.p),
             static_cast<const int *>(S.blk_col.p), nb, S.raw.p);
  }
  S.A.pack(S.raw.p, s, S.nsm);
  S.values_version++;
  launch_k(s, zero_diag_kernel, std::max(1, std::min((n_node + kThreads - 1) / kThreads, S.nsm * 8)), kThreads,
           static_cast<const double *>(S.raw.p), n_node, M.flag.p);
  int fl[2] = {0, 0};
  H33_CUDA(cudaMemcpyAsync(fl, M.flag.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  S.sync();
  S.zero_diag = fl[0] != 0;
  if (inverted) *inverted = fl[1];
  S.has_matrix = true;
}

int prepare_solve(Solver &S, int *Iarray, double *Rarray, double *sigma, bool *auto_sigma) {
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix: call hecmw33_gpu_set_matrix first");
  // zero right-hand side (hecmw_solver.f90:32-37; hecmw_solver_Iterative.f90:284-323,
  // with the MPC constants)
  S.bnrm2 = dot_device(S, S.b.p, S.b.p);
  if (S.bnrm2 + (S.mpc.n_raw > 0 ? S.mpc.const2 : 0.0) == 0.0) {
    H33_CUDA(cudaMemsetAsync(S.x.p, 0, sizeof(double) * S.n3(), S.stream));
    S.sync();
    Iarray[80] = 1;
    Iarray[81] = 0;
    return HECMW33_ERR_ZERO_RHS;
  }
  const int METHOD = Iarray[1], PRECOND = Iarray[2], iterPREmax = Iarray[4];
  *sigma = Rarray[1];
  *auto_sigma = *sigma < 0.0;
  if (*auto_sigma) *sigma = 1.0;
  if (S.zero_diag && PRECOND < 10 && iterPREmax > 0) return HECMW33_ERR_ZERO_DIAG;
  if (METHOD < 1 || METHOD > 7)
    throw Failure(HECMW33_ERR_INCONS_PC, "METHOD " + std::to_string(METHOD) + ": undefined (1-7)");
  if (METHOD == 2 || Iarray[7] == 2 || METHOD == 7 || Iarray[7] == 7) ensure_bicg(S);
  recycle_precond_setting(Iarray);
  Range rg("hecmw33_precond_setup");
  if (iterPREmax > 0) precond_setup(S, PRECOND, Iarray[33], *sigma, Iarray);
  return 0;
}

// Sturm count of the symmetric tridiagonal matrix (d, e): how many of its eigenvalues
// lie below x.
int sturm_count(const std::vector<double> &d, const std::vector<double> &e, int n, double x) {
  int c = 0;
  double q = 1.0;
  for (int i = 0; i < n; i++) {
    q = d[size_t(i)] - x - (i ? e[size_t(i) - 1] * e[size_t(i) - 1] / q : 0.0);
    if (q == 0.0) q = -std::numeric_limits<double>::min();
    if (q < 0.0) c++;
  }
  return c;
}

// The k-th smallest eigenvalue (0-based) of the leading n x n tridiagonal by bisection
// inside the Gershgorin interval, to the resolution of double precision.
double tridiag_eigen(const std::vector<double> &d, const std::vector<double> &e, int n, int k) {
  double lo = d[0], hi = d[0];
  for (int i = 0; i < n; i++) {
    const double r = (i ? std::fabs(e[size_t(i) - 1]) : 0.0) + (i + 1 < n ? std::fabs(e[size_t(i)]) : 0.0);
    lo = std::min(lo, d[size_t(i)] - r);
    hi = std::max(hi, d[size_t(i)] + r);
  }
  for (int it = 0; it < 200; it++) {
    const double mid = 0.5 * (lo + hi);
    if (mid <= lo || mid >= hi) break;
    if (sturm_count(d, e, n, mid) > k) hi = mid;
    else lo = mid;
  }
  return 0.5 * (lo + hi);
}

// hecmw_estimate_condition_CG (hecmw_estimate_condition.F90:14-99) for the ALPHA /
// BETA history of a CG solve: the Lanczos tridiagonal of hecmw_solver_CG.f90:256-263
// (D(1) = 1/ALPHA(1), D(k) = 1/ALPHA(k) + BETA(k)/ALPHA(k-1), E(k-1) =
// sqrt(BETA(k))/ALPHA(k-1)), its extreme eigenvalues every ESTCOND iterations and at
// the end of a solve without error, printed as the reference prints them.  The
// eigenvalues come from bisection on the Sturm count (the reference calls LAPACK's
// dstegr).
void condition_report(Solver &S, const std::vector<double> &ab, int n, int estcond, int error) {
  std::vector<double> d(size_t(std::max(n, 1))), e(size_t(std::max(n, 1)));
  auto estimate = [&](int m) {
    if (m <= 1) return;
    const double emin = tridiag_eigen(d, e, m, 0), emax = tridiag_eigen(d, e, m, m - 1);
    std::printf("emin=%13.6E, emax=%13.6E, emax/emin=%13.6E\n", emin, emax, emax / emin);
    S.last_emin = emin;
    S.last_emax = emax;
  };
  for (int k = 1; k <= n; k++) {
    const double alpha = ab[2 * size_t(k - 1)], beta = ab[2 * size_t(k - 1) + 1];
    if (k == 1) {
      d[0] = 1.0 / alpha;
    } else {
      const double alpha1 = ab[2 * size_t(k - 2)];
      d[size_t(k) - 1] = 1.0 / alpha + beta / alpha1;
      e[size_t(k) - 2] = std::sqrt(beta) / alpha1;
    }
    if (k % estcond == 0) estimate(k);
  }
  if (error == 0) estimate(n);
  std::fflush(stdout);
  S.last_lanczos_n = n;
}

// Singular values of the n x n column-major matrix a (overwritten) by one-sided Jacobi
// rotations (Hestenes): columns are orthogonalised pairwise until every pair is
// orthogonal to rounding; the singular values are then the column norms.
std::vector<double> jacobi_singular_values(std::vector<double> a, int n) {
  for (int sweep = 0; sweep < 60; sweep++) {
    bool rotated = false;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        double alpha = 0.0, beta = 0.0, gamma = 0.0;
        for (int i = 0; i < n; i++) {
          const double x = a[size_t(p) * n + i], y = a[size_t(q) * n + i];
          alpha += x * x;
          beta += y * y;
          gamma += x * y;
        }
        if (gamma == 0.0 || std::fabs(gamma) <= 1e-15 * std::sqrt(alpha * beta)) continue;
        rotated = true;
        const double zeta = (beta - alpha) / (2.0 * gamma);
        const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / std::sqrt(1.0 + t * t), sn = c * t;
        for (int i = 0; i < n; i++) {
          const double x = a[size_t(p) * n + i], y = a[size_t(q) * n + i];
          a[size_t(p) * n + i] = c * x - sn * y;
          a[size_t(q) * n + i] = sn * x + c * y;
        }
      }
    if (!rotated) break;
  }
  std::vector<double> sv(size_t(std::max(n, 0)));
  for (int j = 0; j < n; j++) {
    double s2 = 0.0;
    for (int i = 0; i < n; i++) s2 += a[size_t(j) * n + i] * a[size_t(j) * n + i];
    sv[size_t(j)] = std::sqrt(s2);
  }
  return sv;
}

// hecmw_estimate_condition_GMRES (hecmw_estimate_condition.F90:102-170) on the
// device's Hessenberg (column-major, leading dimension ld, 1-based (k, j) at
// H[(j-1) ld + k-1]) after step I: the I x I block whose entries below the first
// subdiagonal are zero, its extreme singular values printed as the reference
// prints them (the reference calls LAPACK's dgesdd).
void gmres_condition(Solver &S, const double *dH, int ld, int I) {
  if (I <= 0) return;
  std::vector<double> H(size_t(ld) * ld);
  H33_CUDA(cudaMemcpy(H.data(), dH, sizeof(double) * H.size(), cudaMemcpyDeviceToHost));
  const int n = std::min(I, ld);
  std::vector<double> a(size_t(n) * n, 0.0);
  for (int j = 1; j <= n; j++)
    for (int k = 1; k <= std::min(j + 1, n); k++) a[size_t(j - 1) * n + (k - 1)] = H[size_t(j - 1) * ld + (k - 1)];
  const std::vector<double> sv = jacobi_singular_values(a, n);
  const double emin = *std::min_element(sv.begin(), sv.end()), emax = *std::max_element(sv.begin(), sv.end());
  std::printf("emin=%13.6E, emax=%13.6E, emax/emin=%13.6E\n", emin, emax, emax / emin);
  std::fflush(stdout);
  S.last_emin = emin;
  S.last_emax = emax;
  S.last_lanczos_n = n;
}

// hecmw_solve_GMRES (hecmw_solver_GMRES.f90:123-411) on the resident B and X in FP64:
// right-preconditioned GMRES(NREST) with modified Gram-Schmidt and Givens rotations.
// Returns the device-side seconds; sets *error (0 or 3001), *iter and *resid.
float run_gmres(Solver &S, int iterpremax, double tol, int maxit, int nrest, int lowp, int *kernels, int *error,
                int *iter, double *resid, int estcond = 0) {
  cudaStream_t s = S.stream;
  const int n3 = S.n3();
  int m = nrest;
  if (m >= n3 - 1) m = n3 - 2;  // :93
  if (m < 1) throw Failure(HECMW33_ERR_BAD_INPUT, "GMRES needs NREST >= 1");
  const int ld = m + 7, CS = m + 1, SN = m + 2;
  S.g_V.alloc(size_t(m + 1) * n3);
  for (auto *v : {&S.g_w, &S.g_zq, &S.g_av}) v->alloc(size_t(n3));
  const size_t nsmall = size_t(ld) * ld + 3 * size_t(ld + 2) + 3;
  S.g_small.alloc(nsmall);
  S.g_flag.alloc(1);
  H33_CUDA(cudaMemsetAsync(S.g_small.p, 0, sizeof(double) * nsmall, s));
  double *base = S.g_small.p;
  GmresDev g{base, base + size_t(ld) * ld, base + size_t(ld) * ld + (ld + 2), base + nsmall - 3,
             base + nsmall - 2, base + nsmall - 1, S.g_flag.p, ld};
  double *ss = base + size_t(ld) * ld + 2 * size_t(ld + 2);
  const Views<double> V = views(S, 0.0, lowp);
  CgState *st = S.state.p;
  S.h_params->tol = tol;
  S.h_params->maxit = maxit;
  S.h_params->iterpremax = iterpremax;
  S.h_params->inner = S.h_params->flexible = S.h_params->use_gnn = S.h_params->reliable = 0;
  S.h_params->ru_delta = 0.0;
  S.h_params->method = 3;
  S.h_params->lanczos = nullptr;
  S.h_params->lanczos_cap = 0;
  S.h_params->rhist = nullptr;
  S.h_params->rhist_cap = 0;
  H33_CUDA(cudaMemcpyAsync(S.params.p, S.h_params, sizeof(CgParams), cudaMemcpyHostToDevice, s));
  H33_CUDA(cudaEventRecord(S.ev0, s));
  launch_k(s, cg_init_kernel, 1, 32, st, static_cast<const CgParams *>(S.params.p));
  int launched = 1;
  auto vec = [&](int k) { return S.g_V.p + size_t(k) * n3; };
  auto precond = [&](const double *in, double *out) { launch_precond_plain<double>(S, V, iterpremax, in, out, nullptr); };
  auto finish = [&](int irow) {  // [H]{y} = {s}; {av} = V y; {zq} = M^-1 {av}; {x} += {zq}
    launch_k(s, gmres_trisolve_kernel, 1, 32, g, irow, ss);
    launch_k(s, gmres_combine_kernel, S.grid_vec(), kThreads, static_cast<const double *>(S.g_V.p), size_t(n3),
             irow, g, n3, S.g_av.p);
    precond(S.g_av.p, S.g_zq.p);
    launch_k(s, gmres_update_x_kernel, S.grid_vec(), kThreads, static_cast<const double *>(S.g_zq.p), S.x.p, n3);
    launched += 4;
  };
  // {r} = {b} - [A]{x0}, BNRM2
  launch_k(s, spmv_kernel<double, 1>, S.grid_spmv(), kThreads, V.A, V.x, V.r, V.b, nullptr, nullptr);
  const double bnrm2 = dot_device(S, S.b.p, S.b.p);
  *error = 0;
  *iter = 0;
  *resid = 0.0;
  int I = 0;
  bool exit_outer = false;
  while (!exit_outer) {
    I = 0;
    const double dnrm2 = dot_device(S, S.r.p, S.r.p);
    if (dnrm2 == 0.0) break;  // converged
    const double rnorm = std::sqrt(dnrm2);
    launch_k(s, gmres_start_kernel, S.grid_vec(), kThreads, static_cast<const double *>(S.r.p), vec(0), n3,
             1.0 / rnorm);
    H33_CUDA(cudaMemsetAsync(g.s, 0, sizeof(double) * (ld + 2), s));
    H33_CUDA(cudaMemcpyAsync(g.s + 1, &rnorm, sizeof(double), cudaMemcpyHostToDevice, s));
    H33_CUDA(cudaMemsetAsync(S.g_flag.p, 0, sizeof(int), s));
    launched++;
    for (I = 1; I <= m; I++) {
      (*iter)++;
      precond(vec(I - 1), S.g_zq.p);
      launch_k(s, spmv_kernel<double, 0>, S.grid_spmv(), kThreads, V.A, static_cast<const double *>(S.g_zq.p),
               S.g_w.p, static_cast<const double *>(nullptr), static_cast<CgState *>(nullptr),
               static_cast<double *>(nullptr));
      for (int K = 1; K <= I; K++) {
        launch_k(s, gmres_dot_kernel, S.grid_vec(), kThreads, static_cast<const double *>(S.g_w.p),
                 static_cast<const double *>(vec(K - 1)), n3, g, K, I, st, S.partials.p);
        launch_k(s, gmres_orth_kernel, S.grid_vec(), kThreads, S.g_w.p, static_cast<const double *>(vec(K - 1)),
                 n3, g, K, I);
      }
      launch_k(s, gmres_norm_kernel, S.grid_vec(), kThreads, static_cast<const double *>(S.g_w.p), n3, g, I, st,
               S.partials.p);
      launch_k(s, gmres_scale_kernel, S.grid_vec(), kThreads, static_cast<const double *>(S.g_w.p), vec(I), n3, g);
      launch_k(s, gmres_givens_kernel, 1, 32, g, I, CS, SN, bnrm2);
      launched += 5 + 2 * I;
      int brk = 0;
      double rs = 0.0;
      H33_CUDA(cudaMemcpyAsync(&brk, S.g_flag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      H33_CUDA(cudaMemcpyAsync(&rs, g.resid, sizeof(double), cudaMemcpyDeviceToHost, s));
      S.sync();
      if (brk) break;  // {w} = 0: the reference leaves the inner loop (:231)
      *resid = rs;
      if (S.iterlog) std::printf("%8d%8d%16.6E\n", *iter, I + 1, rs);  // :286-287
      if (estcond > 0 && *iter % estcond == 0) gmres_condition(S, g.H, ld, I);  // :290-291
      if (rs <= tol) {
        finish(I);
        exit_outer = true;
        break;
      }
      if (*iter > maxit) {
        *error = HECMW33_ERR_NOCONV_MAXIT;
        exit_outer = true;
        break;
      }
    }
    if (exit_outer) break;
    // current solution and the true residual of the restart (:331-377)
    finish(m);
    launch_k(s, spmv_kernel<double, 1>, S.grid_spmv(), kThreads, V.A, V.x, V.r, V.b, nullptr, nullptr);
    const double d2 = dot_device(S, S.r.p, S.r.p);
    *resid = std::sqrt(d2 / bnrm2);
    launched += 2;
    if (*resid <= tol) break;
    if (*iter > maxit) {
      *error = HECMW33_ERR_NOCONV_MAXIT;
      break;
    }
  }
  if (*error == HECMW33_ERR_NOCONV_MAXIT) finish(I);  // :382-411
  if (estcond > 0) gmres_condition(S, g.H, ld, I);     // :416-417
  H33_CUDA(cudaEventRecord(S.ev1, s));
  S.sync();
  float ms = 0.0f;
  H33_CUDA(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
  if (kernels) *kernels += launched;
  return ms;
}

// hecmw_solve_CR (hecmw_solver_CR.f90:108-296) on the resident B and X in FP64:
// preconditioned conjugate residual with the recursive residual {rt} and explicit
// true-residual checks (every 100th iteration, at RESID_REC <= TOL and at MAXIT).
// Vectors: x, rt = S.r, z = S.z, p = S.p, ap = S.q, map / az / wk in the BiCGSTAB
// buffers.  Returns the device-side seconds; sets *error, *iter, *resid.
float run_cr(Solver &S, int iterpremax, double tol, int maxit, int lowp, int *kernels, int *error, int *iter,
             double *resid) {
  cudaStream_t s = S.stream;
  const int n3 = S.n3();
  constexpr int kCheckTrue = 100;  // N_ITER_CHECK_TRUE_R
  ensure_bicg(S);
  double *x = S.x.p, *rt = S.r.p, *z = S.z.p, *p = S.p.p, *ap = S.q.p;
  double *map = S.b_s.p, *az = S.b_t.p, *wk = S.b_st.p;
  const Views<double> V = views(S, 0.0, lowp);
  int launched = 0;
  auto spmv = [&](const double *in, double *out) {
    launch_k(s, spmv_kernel<double, 0>, S.grid_spmv(), kThreads, V.A, in, out, static_cast<const double *>(nullptr),
             static_cast<CgState *>(nullptr), static_cast<double *>(nullptr));
    launched++;
  };
  auto resid_into = [&](double *out) {  // out = b - A x
    launch_k(s, spmv_kernel<double, 1>, S.grid_spmv(), kThreads, V.A, static_cast<const double *>(x), out,
             static_cast<const double *>(S.b.p), static_cast<CgState *>(nullptr), static_cast<double *>(nullptr));
    launched++;
  };
  auto precond = [&](const double *in, double *out) { launch_precond_plain<double>(S, V, iterpremax, in, out, nullptr); };
  H33_CUDA(cudaEventRecord(S.ev0, s));
  *error = 0;
  *iter = 0;
  *resid = 0.0;
  resid_into(rt);
  const double bnrm2 = dot_device(S, S.b.p, S.b.p);
  double rTAr_old = 0.0;
  int MAXIT = maxit;
  {
    const double dnrm2 = dot_device(S, rt, rt);
    *resid = std::sqrt(dnrm2 / bnrm2);
    if (*resid <= tol) {
      MAXIT = 0;
    } else {
      precond(rt, z);
      H33_CUDA(cudaMemcpyAsync(p, z, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
      spmv(z, az);
      H33_CUDA(cudaMemcpyAsync(ap, az, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
      rTAr_old = dot_device(S, z, az);
      if (rTAr_old != rTAr_old) {
        *error = HECMW33_ERR_DIVERGE_NAN;
        MAXIT = 0;
      } else if (rTAr_old <= 0.0) {
        *error = HECMW33_ERR_DIVERGE_MAT;
        MAXIT = 0;
      }
    }
  }
  int it = 1;
  for (it = 1; it <= MAXIT; it++) {
    precond(ap, map);
    const double apTap = dot_device(S, ap, map);
    if (apTap != apTap) {
      *error = HECMW33_ERR_DIVERGE_NAN;
      break;
    } else if (apTap <= 0.0) {
      *error = HECMW33_ERR_DIVERGE_PC;
      break;
    }
    const double alpha = rTAr_old / apTap;
    launch_k(s, cr_update_kernel, S.grid_vec(), kThreads, x, static_cast<const double *>(p), rt,
             static_cast<const double *>(ap), z, static_cast<const double *>(map), n3, alpha);
    launched++;
    const double dnrm2 = dot_device(S, rt, rt);
    const double resid_rec = std::sqrt(dnrm2 / bnrm2);
    bool true_checked = false;
    double resid_true = 0.0;
    if (resid_rec <= tol || it % kCheckTrue == 0 || it == MAXIT) {
      resid_into(wk);
      resid_true = std::sqrt(dot_device(S, wk, wk) / bnrm2);
      true_checked = true;
    }
    *resid = true_checked ? resid_true : resid_rec;
    if (S.iterlog) std::printf("%7d%16.6E\n", it, *resid);  // hecmw_solver_CR.f90:249
    if (true_checked) {
      if (resid_true <= tol) break;
      if (it == MAXIT) {
        *error = HECMW33_ERR_NOCONV_MAXIT;
        break;
      }
    }
    spmv(z, az);
    const double rTAr = dot_device(S, z, az);
    if (rTAr != rTAr) {
      *error = HECMW33_ERR_DIVERGE_NAN;
      break;
    } else if (rTAr <= 0.0) {
      *error = HECMW33_ERR_DIVERGE_MAT;
      break;
    }
    const double beta = rTAr / rTAr_old;
    rTAr_old = rTAr;
    launch_k(s, cr_direction_kernel, S.grid_vec(), kThreads, p, static_cast<const double *>(z), ap,
             static_cast<const double *>(az), n3, beta);
    launched++;
  }
  *iter = MAXIT == 0 ? 0 : it;  // (:296; a completed DO loop would leave MAXIT+1)
  H33_CUDA(cudaEventRecord(S.ev1, s));
  S.sync();
  float ms = 0.0f;
  H33_CUDA(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
  if (kernels) *kernels += launched;
  return ms;
}

// hecmw_solve_GPBiCG (hecmw_solver_GPBiCG.f90:117-322, pol_coef_vanilla2 :458-506) on
// the resident B and X in FP64, the vector operations in the reference's order.
float run_gpbicg(Solver &S, int iterpremax, double tol, int maxit, int lowp, int *kernels, int *error, int *iter,
                 double *resid) {
  cudaStream_t s = S.stream;
  const int n3 = S.n3();
  constexpr int kRecompute = 20;  // N_ITER_RECOMPUTE_R
  constexpr double kOmega = 0.707106781;
  S.gp_W.alloc(size_t(12) * n3);
  H33_CUDA(cudaMemsetAsync(S.gp_W.p, 0, sizeof(double) * 12 * size_t(n3), s));  // WW = 0
  auto col = [&](int k) { return S.gp_W.p + size_t(k) * n3; };
  double *R = S.r.p, *RT = col(0), *T = col(1), *TT = col(2), *T0 = col(3), *P = col(4), *PT = col(5);
  double *U = col(6), *W1 = col(7), *Y = col(8), *Z = col(9), *WK = col(10), *W2 = col(11), *X = S.x.p;
  const Views<double> V = views(S, 0.0, lowp);
  int launched = 0;
  const int gv = S.grid_vec();
  auto axpy = [&](double a, const double *x, double *y) {
    launch_k(s, vec_axpy_kernel, gv, kThreads, y, a, x, n3);
    launched++;
  };
  auto xpay = [&](double a, const double *x, double *y) {
    launch_k(s, vec_xpay_kernel, gv, kThreads, y, a, x, n3);
    launched++;
  };
  auto axpyz = [&](double a, const double *x, const double *y, double *z) {
    launch_k(s, vec_axpyz_kernel, gv, kThreads, z, a, x, y, n3);
    launched++;
  };
  auto axpby = [&](double a, double b, const double *x, double *y) {
    launch_k(s, vec_axpby_kernel, gv, kThreads, y, a, b, x, n3);
    launched++;
  };
  auto copy = [&](const double *x, double *y) {
    H33_CUDA(cudaMemcpyAsync(y, x, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
  };
  auto matvec = [&](const double *in, double *out) {
    launch_k(s, spmv_kernel<double, 0>, S.grid_spmv(), kThreads, V.A, in, out, static_cast<const double *>(nullptr),
             static_cast<CgState *>(nullptr), static_cast<double *>(nullptr));
    launched++;
  };
  auto matresid = [&](double *out) {
    launch_k(s, spmv_kernel<double, 1>, S.grid_spmv(), kThreads, V.A, static_cast<const double *>(X), out,
             static_cast<const double *>(S.b.p), static_cast<CgState *>(nullptr), static_cast<double *>(nullptr));
    launched++;
  };
  auto precond = [&](const double *in, double *out) { launch_precond_plain<double>(S, V, iterpremax, in, out, nullptr); };
  auto dot = [&](const double *a, const double *b) { return dot_device(S, a, b); };
  H33_CUDA(cudaEventRecord(S.ev0, s));
  matresid(R);
  copy(R, RT);
  const double bnrm2 = dot(S.b.p, S.b.p);
  double RHO = dot(RT, R), BETA = 0.0, ALPHA = 0.0, QSI = 0.0, ETA = 0.0;
  *error = 0;
  *resid = 0.0;
  int it;
  for (it = 1; it <= maxit; it++) {
    copy(R, WK);  // {r} = M^-1 {r} (:169-170)
    precond(WK, R);
    if (it > 1) {  // {p} = {r} + BETA ({p} - {u}) (:179-184)
      axpy(-1.0, U, P);
      xpay(BETA, R, P);
    } else {
      copy(R, P);
    }
    matvec(P, PT);  // (:195)
    const double RHO1 = dot(RT, PT);
    ALPHA = RHO / RHO1;
    axpyz(-1.0, W1, PT, Y);  // (:210-213)
    xpay(ALPHA, T, Y);
    axpy(-1.0, WK, Y);
    axpyz(-ALPHA, PT, WK, T);
    precond(T, TT);  // (:226-229)
    precond(T0, W2);
    copy(W2, T0);
    precond(PT, W2);
    matvec(TT, WK);  // (:235-236)
    copy(WK, TT);
    {  // pol_coef_vanilla2 (:458-506)
      const double c1 = dot(T, T), c2 = dot(TT, TT), c3 = dot(T, TT);
      double gamma1 = 0.0, gamma2 = 0.0;
      if (it > 1) {
        const double c4 = dot(Y, Y), c5 = dot(Y, TT), c6 = dot(Y, T);
        gamma1 = c6 / c4;
        gamma2 = c5 / c4;
      }
      const double c = c3 / std::sqrt(c1 * c2);
      if (std::fabs(c) > kOmega) QSI = c * std::sqrt(c1 / c2);
      else if (c >= 0.0) QSI = kOmega * std::sqrt(c1 / c2);
      else QSI = -kOmega * std::sqrt(c1 / c2);
      ETA = gamma1 - QSI * gamma2;
    }
    if (it > 1) {  // {u}, {z} (:260-273)
      xpay(BETA, T0, U);
      axpy(-1.0, R, U);
      axpby(QSI, ETA, W2, U);
      axpby(-ALPHA, ETA, U, Z);
      axpy(QSI, R, Z);
    } else {
      axpyz(-1.0, R, T0, U);
      axpby(QSI, ETA, W2, U);
      axpby(-ALPHA, ETA, U, Z);
      axpy(QSI, R, Z);
    }
    axpy(ALPHA, P, X);  // (:279-281)
    axpy(1.0, Z, X);
    copy(T, T0);
    if (it % kRecompute == 0) {  // (:284-290)
      matresid(R);
    } else {
      axpyz(-ETA, Y, T, R);
      axpy(-QSI, TT, R);
    }
    const double DNRM2 = dot(R, R), COEF1 = dot(R, RT);
    BETA = ALPHA * COEF1 / (QSI * RHO);
    axpyz(BETA, PT, TT, W1);
    *resid = std::sqrt(DNRM2 / bnrm2);
    if (S.iterlog) std::printf("%5d%16.6E\n", it, *resid);  // hecmw_solver_GPBiCG.f90:306-308
    RHO = COEF1;
    if (*resid <= tol) {  // (:311-319)
      if (it % kRecompute == 0) break;
      matresid(R);
      *resid = std::sqrt(dot(R, R) / bnrm2);
      if (*resid <= tol) break;
    }
    if (it == maxit) *error = HECMW33_ERR_NOCONV_MAXIT;
  }
  *iter = it;  // a completed DO loop leaves MAXIT+1
  H33_CUDA(cudaEventRecord(S.ev1, s));
  S.sync();
  float ms = 0.0f;
  H33_CUDA(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
  if (kernels) *kernels += launched;
  return ms;
}

// hecmw_solve_GMRESR (hecmw_solver_GMRESR.f90:158-232, with the NBFGS = Iarray(60)
// quasi-Newton correction of the preconditioned direction) and hecmw_solve_GMRESREN
// (hecmw_solver_GMRESREN.f90:136-207) on the resident B and X in FP64: truncated
// GCR-type methods restarted after NREST steps, whose direction is the
// preconditioned residual (GMRESR) or is built from the renormalised xi/eta pair
// (GMRESREN).  GMRESREN's second orthogonalisation takes the coefficient left by the
// previous step (the reference computes, then ignores, {c}{cin}); that is kept.
float run_gmresr(Solver &S, int iterpremax, double tol, int maxit, int nrest, int nbfgs, bool ren, int lowp,
                 int *kernels, int *error, int *iter, double *resid) {
  cudaStream_t s = S.stream;
  const int n3 = S.n3();
  if (nrest < 1) throw Failure(HECMW33_ERR_BAD_INPUT, "GMRESR needs NREST >= 1");
  if (ren) nbfgs = 0;
  if (nbfgs < 0) nbfgs = 0;
  const int ncol = 4 * nrest + (ren ? 2 * nrest : 0) + 2 * nbfgs + 2;
  S.gr_W.alloc(size_t(ncol) * n3);
  H33_CUDA(cudaMemsetAsync(S.gr_W.p, 0, sizeof(double) * ncol * size_t(n3), s));
  auto col = [&](int k) { return S.gr_W.p + size_t(k) * n3; };
  // 1-based columns as in the reference
  auto u = [&](int i) { return col(i - 1); };
  auto c = [&](int i) { return col(nrest + i - 1); };
  auto uin = [&](int i) { return col(2 * nrest + i - 1); };
  auto cin = [&](int i) { return col(3 * nrest + i - 1); };
  auto xi = [&](int i) { return col(4 * nrest + i - 1); };
  auto eta = [&](int i) { return col(5 * nrest + i - 1); };
  const int bf0 = 4 * nrest + (ren ? 2 * nrest : 0);
  auto sB = [&](int i) { return col(bf0 + i - 1); };
  auto yB = [&](int i) { return col(bf0 + nbfgs + i - 1); };
  double *vecR = col(ncol - 2), *tmp = col(ncol - 1), *X = S.x.p;
  const Views<double> V = views(S, 0.0, lowp);
  int launched = 0;
  const int gv = S.grid_vec();
  auto axpy = [&](double a, const double *x, double *y) {
    launch_k(s, vec_axpy_kernel, gv, kThreads, y, a, x, n3);
    launched++;
  };
  auto xpay = [&](double a, const double *x, double *y) {
    launch_k(s, vec_xpay_kernel, gv, kThreads, y, a, x, n3);
    launched++;
  };
  auto axpyz = [&](double a, const double *x, const double *y, double *z) {
    launch_k(s, vec_axpyz_kernel, gv, kThreads, z, a, x, y, n3);
    launched++;
  };
  auto scal = [&](double a, const double *x, double *y) {  // hecmw_axpby_R(a, 0)
    launch_k(s, vec_axpby_kernel, gv, kThreads, y, a, 0.0, x, n3);
    launched++;
  };
  auto matvec = [&](const double *in, double *out) {
    launch_k(s, spmv_kernel<double, 0>, S.grid_spmv(), kThreads, V.A, in, out, static_cast<const double *>(nullptr),
             static_cast<CgState *>(nullptr), static_cast<double *>(nullptr));
    launched++;
  };
  auto precond = [&](const double *in, double *out) { launch_precond_plain<double>(S, V, iterpremax, in, out, nullptr); };
  auto dot = [&](const double *a, const double *b) { return dot_device(S, a, b); };
  H33_CUDA(cudaEventRecord(S.ev0, s));
  const double bnrm2 = dot(S.b.p, S.b.p);
  std::vector<int> idx(size_t(std::max(nbfgs, 1)));
  for (int k = 0; k < nbfgs; k++) idx[size_t(k)] = k + 1;
  std::vector<double> rho(size_t(std::max(nbfgs, 1))), alpha(size_t(std::max(nbfgs, 1)));
  int ib = 0, it = 0;
  double coef = 0.0;
  *error = 0;
  *resid = 0.0;
  bool done = false;
  while (!done) {  // OUTER
    launch_k(s, spmv_kernel<double, 1>, S.grid_spmv(), kThreads, V.A, static_cast<const double *>(X), vecR,
             static_cast<const double *>(S.b.p), static_cast<CgState *>(nullptr), static_cast<double *>(nullptr));
    launched++;
    for (int I = 1; I <= nrest; I++) {
      it++;
      if (ren) {
        precond(vecR, eta(1));
        matvec(eta(1), xi(1));
        xpay(-1.0, vecR, xi(1));
        for (int o = 1; o <= I - 1; o++) {
          const double a = dot(c(o), xi(o));
          axpyz(-a, c(o), xi(o), xi(o + 1));
          axpyz(a, u(o), eta(o), eta(o + 1));
        }
        precond(xi(I), uin(1));
      } else if (ib == 0) {
        precond(vecR, uin(1));
      } else {
        H33_CUDA(cudaMemcpyAsync(tmp, vecR, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
        for (int k = 1; k <= ib; k++) {
          const int q = idx[size_t(k - 1)];
          rho[size_t(k - 1)] = 1.0 / dot(sB(q), yB(q));
          alpha[size_t(k - 1)] = rho[size_t(k - 1)] * dot(sB(q), tmp);
          axpy(-alpha[size_t(k - 1)], yB(q), tmp);
        }
        precond(tmp, uin(1));
        for (int k = ib; k >= 1; k--) {
          const int q = idx[size_t(k - 1)];
          const double coef2 = rho[size_t(k - 1)] * dot(yB(q), uin(1));
          axpy(alpha[size_t(k - 1)] - coef2, sB(q), uin(1));
        }
      }
      matvec(uin(1), cin(1));
      for (int o = 1; o <= I - 1; o++) {
        if (!ren) coef = dot(c(o), cin(o));
        axpyz(-coef, c(o), cin(o), cin(o + 1));
        axpyz(-coef, u(o), uin(o), uin(o + 1));
      }
      coef = 1.0 / std::sqrt(dot(cin(I), cin(I)));
      scal(coef, cin(I), c(I));
      scal(coef, uin(I), u(I));
      if (ren) {
        coef = dot(c(I), xi(I));
        axpy(coef, u(I), X);
        axpy(1.0, eta(I), X);
        axpyz(-coef, c(I), xi(I), vecR);
      } else {
        coef = dot(c(I), vecR);
        axpy(coef, u(I), X);
        axpy(-coef, c(I), vecR);
        if (nbfgs > 0) {
          ib++;
          if (ib == nbfgs + 1) {
            const int t = idx[0];
            for (int k = 0; k < nbfgs - 1; k++) idx[size_t(k)] = idx[size_t(k) + 1];
            idx[size_t(nbfgs - 1)] = t;
            ib--;
          }
          scal(coef, c(I), yB(idx[size_t(ib - 1)]));
          scal(coef, u(I), sB(idx[size_t(ib - 1)]));
        }
      }
      *resid = std::sqrt(dot(vecR, vecR) / bnrm2);
      if (S.iterlog) std::printf("%7d%16.6E\n", it, *resid);  // GMRESR.f90:227, GMRESREN.f90:199
      if (*resid <= tol) {
        done = true;
        break;
      }
      if (it > maxit) {
        *error = HECMW33_ERR_NOCONV_MAXIT;
        done = true;
        break;
      }
    }
  }
  *iter = it;
  // hecmw_precond_clear at the end of the solve: the next solve builds the
  // preconditioner again
  S.pc.valid = false;
  H33_CUDA(cudaEventRecord(S.ev1, s));
  S.sync();
  float ms = 0.0f;
  H33_CUDA(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
  if (kernels) *kernels += launched;
  return ms;
}

// The hecmw_solve / hecmw_solve_iterative sequence on resident B (S.b) and X (S.x),
// FP64 throughout (the drop-in).
int solve_fp64(Solver &S, int *Iarray, double *Rarray, int *iter, double *resid, double *times, int lowp = 0) {
  const double t0 = wall();
  *iter = 0;
  *resid = 0.0;
  if (times) times[0] = times[1] = times[2] = 0.0;
  double sigma;
  bool auto_sigma;
  setup_mark("solve: start");
  ScaleScope scaling(S, Iarray[6] != 0);
  const int pre = prepare_solve(S, Iarray, Rarray, &sigma, &auto_sigma);
  if (pre) {
    scaling.restore();
    return pre;
  }
  setup_mark("solve: precond_setup");
  const int MAXIT = Iarray[0], PRECOND = Iarray[2], iterPREmax = Iarray[4], METHOD2 = Iarray[7];
  const double TOL = Rarray[0];
  int method = Iarray[1];
  int learned = (Iarray[42] == 1 && method == 1) ? 1 : 0;  // the learned two-level preconditioner
  S.L.coarse_mode = (Iarray[43] >= 0 && Iarray[43] <= 2) ? Iarray[43] : 0;
  if (learned) {
    learned_prepare_inference(S);
    setup_mark("solve: learned smoother + coarse space");
  }
  const int ESTCOND = Iarray[13];  // hecmw_mat_get_estcond
  S.lanczos_on = ESTCOND > 0 && method == 1 && !learned;
  S.last_lanczos_n = 0;
  S.last_emin = S.last_emax = 0.0;
  if (S.lanczos_on) S.lanczos_buf.alloc(2 * size_t(std::max(MAXIT, 1)));
  S.rhist_on = Iarray[20] == 1 && (method == 1 || method == 2) && !learned;  // hecmw_mat_get_iterlog
  S.iterlog = Iarray[20] == 1;
  if (S.rhist_on) S.rhist_buf.alloc(size_t(std::max(MAXIT, 1)));
  if (lowp && iterPREmax > 0) {
    // a learned solve sweeps with its smoother only: the solve's SSOR needs its BF16
    // copy when a plain solve (or the METHOD2 hand-over below) uses it
    if (learned) ensure_lowp(S, S.L.sm);
    else ensure_lowp(S);
  } else {
    lowp = 0;
  }
  setup_mark("solve: BF16 copies, buffers");
  const bool record = S.L.recording && !learned && method == 1;
  if (graph_mode() && !record && (method == 1 || method == 2))
    build_graph<double>(S, iterPREmax, learned | (lowp ? 4 : 0) | (method == 2 ? 8 : 0));
  setup_mark("solve: graph capture + instantiate");
  Range rs("hecmw33_solve");
  const double t1 = wall();
  int error = 0, kernels = 1;
  float ms_total = 0.0f;
  for (;;) {
    Iarray[80] = 0;
    Iarray[81] = 0;
    if (method == 3) {
      ms_total += run_gmres(S, iterPREmax, TOL, MAXIT, Iarray[5], lowp, &kernels, &error, iter, resid, ESTCOND);
    } else if (method == 7) {
      ms_total += run_cr(S, iterPREmax, TOL, MAXIT, lowp, &kernels, &error, iter, resid);
    } else if (method == 4) {
      ms_total += run_gpbicg(S, iterPREmax, TOL, MAXIT, lowp, &kernels, &error, iter, resid);
    } else if (method == 5 || method == 6) {
      ms_total += run_gmresr(S, iterPREmax, TOL, MAXIT, Iarray[5], Iarray[59], method == 6, lowp, &kernels, &error,
                             iter, resid);
    } else {
      if (record) ms_total += record_cg(S, iterPREmax, TOL, MAXIT, &kernels);
      else ms_total += run_cg<double>(S, iterPREmax, TOL, MAXIT, &kernels, 0, learned, 0, 1e-4, lowp, method);
      const CgState &st = *S.h_state;
      error = st.error;
      *iter = st.iter;
      *resid = st.resid;
      if (S.rhist_on && (method == 1 || method == 2) && !record) {  // ITERATION HISTORY (CG.f90:251-253,
                                                                      // BiCGSTAB.f90:254-256)
        const int n = std::min(st.rhist_n, int(S.rhist_buf.n));
        std::vector<double> h(size_t(std::max(n, 1)));
        if (n > 0) H33_CUDA(cudaMemcpy(h.data(), S.rhist_buf.p, sizeof(double) * size_t(n), cudaMemcpyDeviceToHost));
        for (int k = 1; k <= n; k++) std::printf("%7d%16.6E\n", k, h[size_t(k) - 1]);
        std::fflush(stdout);
      }
      if (S.lanczos_on && method == 1 && !record) {
        const int n = std::min(st.lanczos_n, int(S.lanczos_buf.n / 2));
        std::vector<double> ab(2 * size_t(std::max(n, 1)));
        if (n > 0)
          H33_CUDA(cudaMemcpy(ab.data(), S.lanczos_buf.p, sizeof(double) * 2 * size_t(n), cudaMemcpyDeviceToHost));
        condition_report(S, ab, n, ESTCOND, error);
      }
    }
    scaling.x_back();  // the end of each hecmw_solve_CG call
    if (error == HECMW33_ERR_DIVERGE_PC || error == HECMW33_ERR_DIVERGE_MAT || error == HECMW33_ERR_DIVERGE_NAN) {
      Iarray[81] = 1;
      // Iterative.f90:133-137; the reference's retry reuses the factorisation
      // already built (flags 97/98 are cleared), continuing from the current X
      if (PRECOND >= 10 && PRECOND < 20 && auto_sigma && sigma < 2.0) {
        sigma = sigma + 0.1;
        continue;
      } else if (method == 1 && METHOD2 > 1) {
        // Iterative.f90:138-142: a diverged CG hands over to METHOD2 from the current X
        if (METHOD2 > 7)
          throw Failure(HECMW33_ERR_INCONS_PC, "METHOD2 " + std::to_string(METHOD2) + ": undefined (2-7)");
        if (auto_sigma) sigma = 1.0;
        method = METHOD2;
        learned = 0;
        if (lowp) ensure_lowp(S);
        continue;
      }
    }
    break;
  }
  if (scaling.on) {
    scaling.restore();
    S.bnrm2 = dot_device(S, S.b.p, S.b.p);
  }
  const double resid2 = rel_resid_device(S);
  if (resid2 < TOL) Iarray[80] = 1;
  if (S.iterlog) std::fflush(stdout);
  S.lanczos_on = false;
  S.rhist_on = false;
  S.iterlog = false;
  S.last_learned = learned;
  S.last_fallback = S.h_state->fallback;
  S.last_iter = *iter;
  S.last_outer = 1;
  S.last_kernels = kernels + 2;
  S.last_solve_s = ms_total * 1e-3;
  S.last_setup_s = t1 - t0;
  S.last_true_resid = resid2;
  if (times) {
    times[0] = t1 - t0;
    times[1] = ms_total * 1e-3;
    times[2] = 0.0;
  }
  return error;
}

// Mixed precision (selected by Iarray(42) = 1): FP64 iterative refinement around
// FP32 preconditioned CG.  Matrix and preconditioner are FP32 copies of the FP64
// ones; inner CG vectors are FP32 while every dot product (RHO, C1, DNRM2) is
// accumulated in FP64, so ALPHA/BETA are FP64 values; the outer true residual
// r = b - A x, its norm and the correction x += d are FP64.  The inner solve stops
// at a relative residual of Rarray(42) (default 1e-4); the outer loop stops at
// Rarray(1) on the FP64 true residual.  ITER reports the total inner iterations.
int solve_mixed_restart(Solver &S, int *Iarray, double *Rarray, int *iter, double *resid, double *times) {
  const double t0 = wall();
  *iter = 0;
  *resid = 0.0;
  if (times) times[0] = times[1] = times[2] = 0.0;
  double sigma;
  bool auto_sigma;
  const int pre = prepare_solve(S, Iarray, Rarray, &sigma, &auto_sigma);
  if (pre) return pre;
  const int MAXIT = Iarray[0], iterPREmax = Iarray[4];
  const double TOL = Rarray[0];
  const double TOL_IN = Rarray[41] > 0.0 ? Rarray[41] : 1e-4;
  ensure_fp32(S);
  if (graph_mode()) build_graph<float>(S, iterPREmax);
  Range rs("hecmw33_solve_mixed");
  const double t1 = wall();
  Iarray[80] = 0;
  Iarray[81] = 0;
  const int n3 = S.n3();
  cudaStream_t s = S.stream;
  cudaEvent_t e0, e1;
  H33_CUDA(cudaEventCreate(&e0));
  H33_CUDA(cudaEventCreate(&e1));
  H33_CUDA(cudaEventRecord(e0, s));
  int kernels = 1, total_inner = 0, outer = 0, error = 0;
  // r = b - A x in FP64
  launch_k(s, spmv_kernel<double, 1>, S.grid_spmv(), kThreads, S.A.view(), S.x.p, S.r.p, S.b.p, nullptr, nullptr);
  double rr = dot_device(S, S.r.p, S.r.p);
  kernels += 2;
  double res = std::sqrt(rr / S.bnrm2);
  constexpr int kMaxOuter = 60;
  while (!(res <= TOL)) {
    if (res != res) {
      error = HECMW33_ERR_DIVERGE_NAN;
      break;
    }
    if (outer >= kMaxOuter || total_inner >= MAXIT) {
      error = HECMW33_ERR_NOCONV_MAXIT;
      break;
    }
    launch_k(s, narrow_kernel, S.grid_vec(), kThreads, S.r.p, S.bf.p, n3);
    H33_CUDA(cudaMemsetAsync(S.xf.p, 0, sizeof(float) * n3, s));
    run_cg<float>(S, iterPREmax, TOL_IN, MAXIT - total_inner, &kernels, 1);
    const CgState st = *S.h_state;
    const int inner = std::min(st.iter, MAXIT - total_inner);
    total_inner += std::max(inner, 0);
    if (st.error == HECMW33_ERR_DIVERGE_PC || st.error == HECMW33_ERR_DIVERGE_MAT ||
        st.error == HECMW33_ERR_DIVERGE_NAN) {
      error = st.error;
      Iarray[81] = 1;
      break;
    }
    launch_k(s, widen_add_kernel, S.grid_vec(), kThreads, S.xf.p, S.x.p, n3);
    launch_k(s, spmv_kernel<double, 1>, S.grid_spmv(), kThreads, S.A.view(), S.x.p, S.r.p, S.b.p, nullptr, nullptr);
    rr = dot_device(S, S.r.p, S.r.p);
    kernels += 4;
    res = std::sqrt(rr / S.bnrm2);
    outer++;
  }
  H33_CUDA(cudaEventRecord(e1, s));
  S.sync();
  float ms = 0.0f;
  H33_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *iter = total_inner;
  *resid = res;
  if (res < TOL) Iarray[80] = 1;
  S.last_iter = total_inner;
  S.last_outer = outer;
  S.last_kernels = kernels;
  S.last_solve_s = ms * 1e-3;
  S.last_setup_s = t1 - t0;
  S.last_true_resid = res;
  if (times) {
    times[0] = t1 - t0;
    times[1] = ms * 1e-3;
    times[2] = 0.0;
  }
  return error;
}

// Mixed precision with reliable updates (Iarray(42) = 1): FP32 CG + SSOR (FP32
// matrix and preconditioner copies, FP64 dot products) whose solution and residual
// are folded into FP64 -- x64 += x32, r64 = b - A x64 (FP64 SpMV), r32 = float(r64)
// -- each time the FP32 residual has fallen by Rarray(42) (default 1e-4) since the
// last update, and at the tolerance.  Convergence is decided on the FP64 true
// residual; the FP32 recurrence keeps its search direction across updates, so the
// iteration count stays close to the FP64 solve's.  With Iarray(43) = 1 the
// learned preconditioner runs after the FP32 SSOR (flexible CG).
int solve_mixed_reliable(Solver &S, int *Iarray, double *Rarray, int *iter, double *resid, double *times) {
  const double t0 = wall();
  *iter = 0;
  *resid = 0.0;
  if (times) times[0] = times[1] = times[2] = 0.0;
  double sigma;
  bool auto_sigma;
  const int pre = prepare_solve(S, Iarray, Rarray, &sigma, &auto_sigma);
  if (pre) return pre;
  const int MAXIT = Iarray[0], iterPREmax = Iarray[4];
  const double TOL = Rarray[0];
  const double DELTA = Rarray[41] > 0.0 ? Rarray[41] : 0.1;
  const int learned = Iarray[42] == 1 ? 1 : 0;
  S.L.coarse_mode = (Iarray[43] >= 0 && Iarray[43] <= 2) ? Iarray[43] : 0;
  ensure_fp32(S);
  if (learned) {
    learned_prepare_inference(S);
    ensure_fp32_pc(S, S.L.sm);
  }
  if (graph_mode()) build_graph<float>(S, iterPREmax, 2 | learned);
  Range rs("hecmw33_solve_mixed");
  const double t1 = wall();
  Iarray[80] = 0;
  Iarray[81] = 0;
  int kernels = 1;
  const float ms = run_cg<float>(S, iterPREmax, TOL, MAXIT, &kernels, 0, learned, 1, DELTA);
  const CgState st = *S.h_state;
  // fold a correction not yet carried into x64 (a stop between reliable updates)
  launch_k(S.stream, widen_add_kernel, S.grid_vec(), kThreads, S.xf.p, S.x.p, S.n3());
  const int error = st.error;
  *iter = st.iter;
  *resid = st.resid;
  if (error == HECMW33_ERR_DIVERGE_PC || error == HECMW33_ERR_DIVERGE_MAT || error == HECMW33_ERR_DIVERGE_NAN)
    Iarray[81] = 1;
  const double resid2 = rel_resid_device(S);
  if (resid2 < TOL) Iarray[80] = 1;
  S.last_learned = learned;
  S.last_fallback = st.fallback;
  S.last_iter = *iter;
  S.last_outer = st.ru_count;
  S.last_kernels = kernels + 3;
  S.last_solve_s = ms * 1e-3;
  S.last_setup_s = t1 - t0;
  S.last_true_resid = resid2;
  if (times) {
    times[0] = t1 - t0;
    times[1] = ms * 1e-3;
    times[2] = 0.0;
  }
  return error;
}

// ---------------------------------------------------------------------------
// Multi-RHS CG: up to kMaxRhs load cases per pass over the matrix (h33_multi.cuh).

template <int K, bool FUSE_RHO, bool POS>
void launch_mr_sweep_k(Solver &S, const Precond &P, const DevSell<double> &Lo, const DevSell<double> &Up,
                       const double *rin, double *zout, double *dpos = nullptr) {
  cudaStream_t s = S.stream;
  const int *perm_b = P.alu_shared ? P.perm_fwd.p : P.perm_bwd.p;
  const double *alu_b = P.alu_shared ? P.alu_fwd.p : P.alu_bwd.p;
  MultiCtl *ctl = S.mctl.p;
  const SellView<double> lo = Lo.view(), up = Up.view();
  const int gf = int(Lo.group_slice.size()) - 1;
  for (int g = 0; g < gf; g++) {
    const int sb = Lo.group_slice[g], se = Lo.group_slice[g + 1];
    if (se <= sb) continue;
    launch_k(s, mr_sweep_fwd_kernel<K, POS>, S.grid_mr((se - sb) * (32 / K)), kThreads, 
        lo, P.perm_fwd.p, P.alu_fwd.p, S.N, rin, zout, S.mzpos.p, sb, se, ctl);
  }
  const int gb = int(Up.group_slice.size()) - 1;
  int total = 0;
  for (int g = gb - 1; g >= 0; g--) {
    const int sb = Up.group_slice[g], se = Up.group_slice[g + 1];
    total += S.grid_mr(std::max(se - sb, 1) * (32 / K));
  }
  int base = 0;
  for (int g = gb - 1; g >= 0; g--) {
    const int sb = Up.group_slice[g], se = Up.group_slice[g + 1];
    const int grid = S.grid_mr(std::max(se - sb, 1) * (32 / K));
    bool done = false;
    if constexpr (POS && !FUSE_RHO) {
      if (dpos) {
        launch_k(s, mr_sweep_bwd_kernel<K, FUSE_RHO, POS, true>, grid, kThreads, up, perm_b, alu_b, S.N, rin, zout,
                 S.mzpos.p, sb, se, S.mst.p, ctl, S.mpart.p, base, total, dpos);
        done = true;
      }
    }
    if (!done)
      launch_k(s, mr_sweep_bwd_kernel<K, FUSE_RHO, POS, false>, grid, kThreads, up, perm_b, alu_b, S.N, rin, zout,
               S.mzpos.p, sb, se, S.mst.p, ctl, S.mpart.p, base, total, static_cast<double *>(nullptr));
    base += grid;
  }
}

template <bool FUSE_RHO>
void launch_mr_sweep(Solver &S, const double *rin, double *zout) {
  Precond &P = S.pc;
  if (P.kind == 3) {
    launch_k(S.stream, mr_diag_kernel<FUSE_RHO>, S.grid_mr(S.N), kThreads, P.alu_fwd.p, S.N, rin, zout, S.mst.p,
                                                                         S.mctl.p, S.mpart.p);
    return;
  }
  if (P.pos_cols) {
    switch (P.lo.lanes) {
      case 4: return launch_mr_sweep_k<4, FUSE_RHO, true>(S, P, P.lo, P.up, rin, zout);
      case 16: return launch_mr_sweep_k<16, FUSE_RHO, true>(S, P, P.lo, P.up, rin, zout);
      default: return launch_mr_sweep_k<8, FUSE_RHO, true>(S, P, P.lo, P.up, rin, zout);
    }
  }
  switch (P.lo.lanes) {
    case 4: return launch_mr_sweep_k<4, FUSE_RHO, false>(S, P, P.lo, P.up, rin, zout);
    case 16: return launch_mr_sweep_k<16, FUSE_RHO, false>(S, P, P.lo, P.up, rin, zout);
    default: return launch_mr_sweep_k<8, FUSE_RHO, false>(S, P, P.lo, P.up, rin, zout);
  }
}

// Largest number of CTAs one reduction of the multi-RHS loop uses.
int mr_max_parts(Solver &S) {
  Precond &P = S.pc;
  int m = std::max({S.grid_amr(), S.grid_mr(S.N), S.grid_rows(S.N, S.occ_mru), S.grid_rows(S.N, S.occ_mrv)});
  if (S.mt_occ > 0) m = std::max(m, std::min(S.mt_ntiles, S.nsm * S.mt_occ));
  if (P.valid && P.kind != 3) {
    const DevSell<double> &U = P.up;
    const int K = U.lanes;
    int total = 0;
    const int gb = int(U.group_slice.size()) - 1;
    for (int g = 0; g < gb; g++)
      total += S.grid_mr(std::max(U.group_slice[g + 1] - U.group_slice[g], 1) * (32 / K));
    m = std::max(m, total);
  }
  return m;
}

// hecmw_precond_apply for 16 RHS (iterPREmax passes; RHO fused when iterPREmax == 1).
void launch_mr_precond(Solver &S, int iterpremax) {
  cudaStream_t s = S.stream;
  const int n48 = S.N * kRhsStride;
  const int gv = std::max(1, std::min((n48 + kThreads - 1) / kThreads, S.nsm * S.occ_vec));
  if (iterpremax <= 0) {
    launch_k(s, copy_kernel<double>, gv, kThreads, S.mr.p, S.mz.p, n48, nullptr);
    launch_k(s, mr_dot_kernel<1>, S.grid_mr(S.N), kThreads, S.mr.p, S.mz.p, S.N, S.mst.p, S.mctl.p, S.mpart.p);
    return;
  }
  if (iterpremax == 1) {
    launch_mr_sweep<true>(S, S.mr.p, S.mz.p);
    return;
  }
  const double *in = S.mr.p;
  for (int it = 1; it <= iterpremax; it++) {
    launch_mr_sweep<false>(S, in, S.mzp.p);
    if (it == 1) launch_k(s, copy_kernel<double>, gv, kThreads, S.mzp.p, S.mz.p, n48, nullptr);
    else launch_k(s, add_kernel<double>, gv, kThreads, S.mzp.p, S.mz.p, n48, nullptr);
    if (it == iterpremax) break;
    launch_k(s, mr_spmv_kernel<1, kMrLanes>, S.grid_amr(), kThreads, S.amr_view(), S.mz.p, S.mw.p, S.mr.p, S.mst.p,
                                                                       S.mctl.p, S.mpart.p);
    in = S.mw.p;
  }
  launch_k(s, mr_dot_kernel<1>, S.grid_mr(S.N), kThreads, S.mr.p, S.mz.p, S.N, S.mst.p, S.mctl.p, S.mpart.p);
}

void launch_mr_prologue(Solver &S, int nrhs, cudaGraphConditionalHandle h, int use_cond) {
  cudaStream_t s = S.stream;
  const int gs = S.grid_amr();
  launch_k(s, mr_init_kernel, 1, 32, S.mst.p, S.mctl.p, S.params.p, nrhs);
  launch_k(s, mr_spmv_kernel<1, kMrLanes>, gs, kThreads, S.amr_view(), S.mx.p, S.mr.p, S.mb.p, S.mst.p, S.mctl.p, S.mpart.p);
  launch_k(s, mr_dot_kernel<0>, S.grid_mr(S.N), kThreads, S.mb.p, S.mb.p, S.N, S.mst.p, S.mctl.p, S.mpart.p);
  launch_k(s, mr_ctl_kernel, 1, 32, S.mst.p, S.mctl.p, h, use_cond);
}

void launch_mr_iteration(Solver &S, int iterpremax, cudaGraphConditionalHandle h, int use_cond) {
  cudaStream_t s = S.stream;
  const int gs = S.grid_amr(), gn = S.grid_rows(S.N, S.occ_mru);
  launch_k(s, mr_iter_begin_kernel, 1, 32, S.mst.p, S.mctl.p, h, use_cond);
  launch_mr_precond(S, iterpremax);
  launch_k(s, mr_update_p_kernel, gn, kThreads, S.mz.p, S.mp.p, S.N, S.mst.p, S.mctl.p);
  if (mr_tiled_mode() && S.mt_occ > 0 && S.mt_generation == S.generation)
    launch_ks(s, mr_spmm_tiled_kernel, std::min(S.mt_ntiles, S.nsm * S.mt_occ), kThreads,
              size_t(S.mt_maxcols) * kRhsStride * sizeof(double), S.A.view(), S.mt_ptr.p, S.mt_cols.p,
              S.mt_lidx.p, S.mt_ntiles, S.mp.p, S.mq.p, S.mst.p, S.mctl.p, S.mpart.p);
  else
    launch_k(s, mr_spmv_kernel<2, kMrLanes>, gs, kThreads, S.amr_view(), S.mp.p, S.mq.p, nullptr, S.mst.p, S.mctl.p, S.mpart.p);
  launch_k(s, mr_update_xr_kernel, gn, kThreads, S.mx.p, S.mp.p, S.mr.p, S.mq.p, S.N, S.mst.p, S.mctl.p, S.mpart.p);
  launch_k(s, mr_spmv_kernel<3, kMrLanes>, gs, kThreads, S.amr_view(), S.mx.p, S.mr.p, S.mb.p, S.mst.p, S.mctl.p, S.mpart.p);
  launch_k(s, mr_ctl_kernel, 1, 32, S.mst.p, S.mctl.p, h, use_cond);
}

// One flexible-CG iteration of the multi-RHS loop with the learned two-level
// preconditioner (launch_learned_precond's symmetric cycle, FP64 smoother): zs =
// SSOR(r); w = r - A zs; bc = P^T w; y = Ac^-1 bc; zc = zs + P y, w -= (A P) y;
// z = zc + SSOR(w).
void launch_mr_iteration_learned(Solver &S, cudaGraphConditionalHandle h, int use_cond) {
  cudaStream_t s = S.stream;
  Precond &P = S.L.sm;
  auto &C = S.L.C;
  const CoarseApply ca = C.apply_view();
  // the vector kernels' grids from their own occupancy, not the sweeps'
  const int gs = S.grid_amr(), gn = S.grid_rows(S.N, S.occ_mru), grho = S.grid_rows(S.N, S.occ_mrv);
  auto smooth = [&](const double *rin, double *zout, double *dpos) {
    switch (P.lo.lanes) {
      case 8: return launch_mr_sweep_k<8, false, true>(S, P, P.lo, P.up, rin, zout, dpos);
      case 16: return launch_mr_sweep_k<16, false, true>(S, P, P.lo, P.up, rin, zout, dpos);
      default: return launch_mr_sweep_k<4, false, true>(S, P, P.lo, P.up, rin, zout, dpos);
    }
  };
  launch_k(s, mr_iter_begin_kernel, 1, 32, S.mst.p, S.mctl.p, h, use_cond);
  // w = r - A zs: L (y - zs) from the pre-smoothing's correction when SIGMA_DIAG is 1
  // (as launch_learned_precond), else the SpMM
  if (P.sigma == 1.0 && lower_resid_mode()) {
    smooth(S.mr.p, S.mzs.p, S.mdpos.p);
    const SellView<double> lo = P.lo.view();
    const MultiCtl *cctl = S.mctl.p;
    const int gl = S.grid_mr(P.lo.nslices * (32 / P.lo.lanes));
    switch (P.lo.lanes) {
      case 8: launch_k(s, mr_lower_resid_kernel<8>, gl, kThreads, lo, P.perm_fwd.p, static_cast<const double *>(S.mdpos.p), S.mw.p, cctl); break;
      case 16: launch_k(s, mr_lower_resid_kernel<16>, gl, kThreads, lo, P.perm_fwd.p, static_cast<const double *>(S.mdpos.p), S.mw.p, cctl); break;
      default: launch_k(s, mr_lower_resid_kernel<4>, gl, kThreads, lo, P.perm_fwd.p, static_cast<const double *>(S.mdpos.p), S.mw.p, cctl); break;
    }
  } else {
    smooth(S.mr.p, S.mzs.p, nullptr);
    launch_k(s, mr_spmv_kernel<1, kMrLanes>, gs, kThreads, S.amr_view(), static_cast<const double *>(S.mzs.p),
             S.mw.p, static_cast<const double *>(S.mr.p), S.mst.p, S.mctl.p, S.mpart.p);
  }
  launch_k(s, mr_coarse_restrict_kernel, std::max(1, C.nagg), kThreads, ca, static_cast<const double *>(S.mw.p),
           S.mbc.p, static_cast<const MultiCtl *>(S.mctl.p));
  launch_k(s, mr_coarse_gemm_kernel, std::max(1, (C.nc + kMrGemmRows - 1) / kMrGemmRows), kThreads, C.nc,
           static_cast<const float *>(C.ainv32.p), static_cast<const double *>(S.mbc.p), S.my.p,
           static_cast<const MultiCtl *>(S.mctl.p));
  launch_k(s, mr_coarse_resid_kernel, S.grid_rows(S.N, S.occ_mrq), kThreads, ca, static_cast<const double *>(S.my.p), S.mw.p,
           static_cast<const CgState *>(S.mst.p), static_cast<const MultiCtl *>(S.mctl.p));
  smooth(S.mw.p, S.mz.p, nullptr);
  // z = SSOR(w) + (zs + P y), formed inside the RHO/DELTA pass
  launch_k(s, mr_fcg_rho_kernel, grho, kThreads, S.mz.p, static_cast<const double *>(S.mzs.p), ca,
           static_cast<const double *>(S.my.p), static_cast<const double *>(S.mr.p), static_cast<const double *>(S.mrold.p), S.N, S.mst.p, S.mctl.p,
           S.mpart.p);
  launch_k(s, mr_update_p_kernel, gn, kThreads, S.mz.p, S.mp.p, S.N, S.mst.p, S.mctl.p);
  launch_k(s, mr_spmv_kernel<2, kMrLanes>, gs, kThreads, S.amr_view(), S.mp.p, S.mq.p, nullptr, S.mst.p, S.mctl.p,
           S.mpart.p);
  launch_k(s, mr_update_xr_flex_kernel, gn, kThreads, S.mx.p, static_cast<const double *>(S.mp.p), S.mr.p,
           S.mrold.p, static_cast<const double *>(S.mq.p), S.N, S.mst.p, S.mctl.p, S.mpart.p);
  launch_k(s, mr_spmv_kernel<3, kMrLanes>, gs, kThreads, S.amr_view(), S.mx.p, S.mr.p, S.mb.p, S.mst.p, S.mctl.p,
           S.mpart.p);
  launch_k(s, mr_ctl_kernel, 1, 32, S.mst.p, S.mctl.p, h, use_cond);
}

// Graph of the whole multi-RHS loop (prologue + WHILE node), as build_graph.
void build_graph_multi(Solver &S, int iterpremax, int nrhs, bool learned = false) {
  GraphSlot &G = S.gm;
  const int key[5] = {S.generation, S.pc.generation, S.pc.kind, 2 * iterpremax + (learned ? 1 : 0), nrhs};
  if (G.exec && std::equal(key, key + 5, G.key)) return;
  G.drop();
  cudaGraph_t g = nullptr;
  H33_CUDA(cudaGraphCreate(&g, 0));
  G.graph = g;
  cudaGraphConditionalHandle h;
  H33_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
  H33_CUDA(cudaStreamBeginCaptureToGraph(S.stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  launch_mr_prologue(S, nrhs, h, 1);
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  H33_CUDA(cudaStreamGetCaptureInfo(S.stream, &cs, nullptr, nullptr, &deps, &ndeps));
  std::vector<cudaGraphNode_t> dep(deps, deps + ndeps);
  cudaGraph_t g2 = nullptr;
  H33_CUDA(cudaStreamEndCapture(S.stream, &g2));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  H33_CUDA(cudaGraphAddNode(&cnode, g, dep.data(), dep.size(), &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  H33_CUDA(cudaStreamBeginCaptureToGraph(S.stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  if (learned) launch_mr_iteration_learned(S, h, 1);
  else launch_mr_iteration(S, iterpremax, h, 1);
  cudaGraph_t b2 = nullptr;
  H33_CUDA(cudaStreamEndCapture(S.stream, &b2));
  H33_CUDA(cudaGraphInstantiate(&G.exec, g, 0));
  std::copy(key, key + 5, G.key);
  size_t nbody = 0, nall = 0;
  H33_CUDA(cudaGraphGetNodes(body, nullptr, &nbody));
  H33_CUDA(cudaGraphGetNodes(g, nullptr, &nall));
  G.kernels_per_iter = int(nbody);
  G.prologue_kernels = int(nall) - 1;
}

// Tiles of the SpMV layout for mr_spmm_tiled_kernel (built from the device layout).
void build_mr_tiles(Solver &S) {
  const DevSell<double> &A = S.A;
  const int ns = A.nslices;
  std::vector<int> row0(static_cast<size_t>(ns)), nrows(static_cast<size_t>(ns)), slot0(static_cast<size_t>(ns));
  std::vector<int> rowlen(static_cast<size_t>(ns) * 32), col(static_cast<size_t>(A.nslots) * 32);
  H33_CUDA(cudaMemcpy(nrows.data(), A.nrows.p, sizeof(int) * ns, cudaMemcpyDeviceToHost));
  H33_CUDA(cudaMemcpy(slot0.data(), A.slot0.p, sizeof(int) * ns, cudaMemcpyDeviceToHost));
  H33_CUDA(cudaMemcpy(rowlen.data(), A.rowlen.p, sizeof(int) * rowlen.size(), cudaMemcpyDeviceToHost));
  H33_CUDA(cudaMemcpy(col.data(), A.col.p, sizeof(int) * col.size(), cudaMemcpyDeviceToHost));
  const int ntiles = 2 * ns;
  std::vector<int> ptr(static_cast<size_t>(ntiles) + 1, 0), cols;
  std::vector<uint16_t> lidx(col.size(), 0);
  std::vector<int> mark(static_cast<size_t>(S.N), -1), local(static_cast<size_t>(S.N), 0);
  int maxc = 0;
  cols.reserve(size_t(ntiles) * 192);
  for (int t = 0; t < ntiles; t++) {
    const int sl = t >> 1, r0 = 16 * (t & 1), r1 = std::min(r0 + 16, nrows[sl]);
    int n = 0;
    for (int r = r0; r < r1; r++)
      for (int k = 0; k < rowlen[size_t(sl) * 32 + r]; k++) {
        const size_t at = (size_t(slot0[sl]) + k) * 32 + r;
        const int c = col[at];
        if (mark[c] != t) {
          mark[c] = t;
          local[c] = n++;
          cols.push_back(c);
        }
        lidx[at] = uint16_t(local[c]);
      }
    ptr[t + 1] = ptr[t] + n;
    maxc = std::max(maxc, n);
  }
  S.mt_ptr.upload(ptr, S.stream);
  S.mt_cols.upload(cols, S.stream);
  S.mt_lidx.upload(lidx, S.stream);
  S.mt_maxcols = maxc;
  S.mt_ntiles = ntiles;
  const size_t smem = size_t(maxc) * kRhsStride * sizeof(double);
  S.mt_occ = 0;
  if (smem <= size_t(200) * 1024) {
    H33_CUDA(cudaFuncSetAttribute(mr_spmm_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    H33_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&S.mt_occ, mr_spmm_tiled_kernel, kThreads, smem));
  }
  S.sync();
  S.mt_generation = S.generation;
}

void ensure_multi_buffers(Solver &S) {
  if (mr_tiled_mode() && S.mt_generation != S.generation) build_mr_tiles(S);
  if (S.amr_generation != S.generation) {
    build_unified(S, S.Amr, kMrLanes);
    S.amr_generation = S.generation;
    S.amr_values = -1;
  }
  if (S.amr_values != S.values_version) {
    S.Amr.pack(S.raw.p, S.stream, S.nsm);
    S.amr_values = S.values_version;
  }
  const size_t n48 = size_t(S.N) * kRhsStride;
  for (auto *v : {&S.mb, &S.mx, &S.mr, &S.mz, &S.mp, &S.mq, &S.mw, &S.mzp, &S.mzpos}) v->alloc(n48);
  S.mst.alloc(kMaxRhs);
  S.mctl.alloc(1);
  S.mpart.alloc(size_t(mr_max_parts(S)) * 2 * kMaxRhs + 1024);  // two values per CTA (mr_fcg_rho_kernel)
}

// Solves nrhs <= kMaxRhs systems A X(:, k) = B(:, k); dB and dX are device arrays in
// the column-major hecmwST layout (3N x nrhs).  Per-RHS results in iter/resid/error/
// true_resid; returns the device time in ms and counts the kernels launched.
float run_multi_chunk(Solver &S, int nrhs, const double *dB, double *dX, int iterpremax, double tol, int maxit,
                      int *iter, double *resid, int *error, double *true_resid, int *kernels, bool learned = false) {
  cudaStream_t s = S.stream;
  const int n = S.N;
  const size_t n48 = size_t(n) * kRhsStride;
  const int gp = std::max(1, std::min(int((n48 + kThreads - 1) / kThreads), S.nsm * S.occ_vec));
  launch_k(s, mr_pack_kernel, gp, kThreads, dB, S.mb.p, n, nrhs);
  launch_k(s, mr_pack_kernel, gp, kThreads, dX, S.mx.p, n, nrhs);
  S.h_params->tol = tol;
  S.h_params->maxit = maxit;
  S.h_params->iterpremax = iterpremax;
  S.h_params->inner = 0;
  S.h_params->flexible = learned ? 1 : 0;
  S.h_params->use_gnn = learned ? 1 : 0;
  S.h_params->reliable = 0;
  S.h_params->ru_delta = 0.0;
  S.h_params->method = 1;
  S.h_params->lanczos = nullptr;
  S.h_params->lanczos_cap = 0;
  S.h_params->rhist = nullptr;
  S.h_params->rhist_cap = 0;
  H33_CUDA(cudaMemcpyAsync(S.params.p, S.h_params, sizeof(CgParams), cudaMemcpyHostToDevice, s));
  H33_CUDA(cudaEventRecord(S.ev0, s));
  if (graph_mode()) {
    build_graph_multi(S, iterpremax, nrhs, learned);
    H33_CUDA(cudaGraphLaunch(S.gm.exec, s));
  } else {
    launch_mr_prologue(S, nrhs, 0, 0);
    for (int it = 0; it <= maxit + kStreamChunk; it += kStreamChunk) {
      for (int k = 0; k < kStreamChunk; k++) {
        if (learned) launch_mr_iteration_learned(S, 0, 0);
        else launch_mr_iteration(S, iterpremax, 0, 0);
      }
      H33_CUDA(cudaGetLastError());
      H33_CUDA(cudaMemcpyAsync(S.h_mctl, S.mctl.p, sizeof(MultiCtl), cudaMemcpyDeviceToHost, s));
      S.sync();
      if (S.h_mctl->all_done) break;
    }
  }
  H33_CUDA(cudaEventRecord(S.ev1, s));
  // final true residuals (hecmw_rel_resid_L2_33 per RHS) and the zero-RHS lanes
  launch_k(s, mr_spmv_kernel<1, kMrLanes>, S.grid_amr(), kThreads, S.amr_view(), S.mx.p, S.mw.p, S.mb.p, S.mst.p,
                                                                     S.mctl.p, S.mpart.p);
  launch_k(s, mr_dot_kernel<2>, S.grid_mr(n), kThreads, S.mw.p, S.mw.p, n, S.mst.p, S.mctl.p, S.mpart.p);
  launch_k(s, mr_zero_x_kernel, gp, kThreads, S.mx.p, n, S.mst.p);
  launch_k(s, mr_unpack_kernel, gp, kThreads, S.mx.p, dX, n, nrhs);
  H33_CUDA(cudaGetLastError());
  H33_CUDA(cudaMemcpyAsync(S.h_mst, S.mst.p, sizeof(CgState) * kMaxRhs, cudaMemcpyDeviceToHost, s));
  H33_CUDA(cudaMemcpyAsync(S.h_mctl, S.mctl.p, sizeof(MultiCtl), cudaMemcpyDeviceToHost, s));
  S.sync();
  float ms = 0.0f;
  H33_CUDA(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
  if (!S.h_mctl->all_done) throw Failure(HECMW33_ERR_TIMEOUT, "multi-RHS loop ended without a decision");
  if (S.h_mctl->fault) throw Failure(HECMW33_ERR_TIMEOUT, "multi-RHS SpMM: a bulk copy did not complete in time");
  for (int k = 0; k < nrhs; k++) {
    const CgState &st = S.h_mst[k];
    iter[k] = st.zero_rhs ? 0 : st.iter;
    resid[k] = st.zero_rhs ? 0.0 : st.resid;
    error[k] = st.zero_rhs ? HECMW33_ERR_ZERO_RHS : st.error;
    true_resid[k] = st.bnrm2 > 0.0 ? std::sqrt(st.rr_true / st.bnrm2) : 0.0;
  }
  if (kernels) {
    const int body = S.h_mctl->guard;
    *kernels += (graph_mode() ? S.gm.prologue_kernels + body * S.gm.kernels_per_iter : 0) + 6;
  }
  return ms;
}

// hecmw_solve for nrhs load cases on the resident matrix: the checks and the
// preconditioner setup of hecmw_solve_iterative once, then the RHS in chunks of
// kMaxRhs.  Returns the first non-zero per-RHS code other than 2002 (or 0).
int solve_multi(Solver &S, int nrhs, const double *dB, double *dX, int *Iarray, double *Rarray, int *iter,
                double *resid, int *error, double *true_resid, double *times) {
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix: call hecmw33_gpu_set_matrix first");
  if (nrhs < 1) throw Failure(HECMW33_ERR_BAD_INPUT, "nrhs must be positive");
  if (Iarray[6] != 0) throw Failure(HECMW33_ERR_BAD_INPUT, "SCALING=YES is not implemented for multi-RHS solves");
  const double t0 = wall();
  if (times) times[0] = times[1] = times[2] = 0.0;
  const int METHOD = Iarray[1], PRECOND = Iarray[2], iterPREmax = Iarray[4], MAXIT = Iarray[0];
  const double TOL = Rarray[0];
  double sigma = Rarray[1];
  if (sigma < 0.0) sigma = 1.0;
  if (S.zero_diag && PRECOND < 10 && iterPREmax > 0) return HECMW33_ERR_ZERO_DIAG;
  if (METHOD != 1)
    throw Failure(HECMW33_ERR_INCONS_PC, "METHOD " + std::to_string(METHOD) + ": the GPU drop-in implements CG (1)");
  recycle_precond_setting(Iarray);
  if (iterPREmax > 0) precond_setup(S, PRECOND, Iarray[33], sigma, Iarray);
  ensure_multi_buffers(S);
  // Iarray(43) = 1: the learned two-level preconditioner for every load case (FP64
  // smoother and recurrences; precision modes do not apply to multi-RHS solves)
  bool learned = Iarray[42] == 1;
  if (learned) {
    if (iterPREmax != 1)
      throw Failure(HECMW33_ERR_INCONS_PC, "the learned preconditioner applies one cycle per iteration (iterPREmax 1)");
    S.L.coarse_mode = (Iarray[43] >= 0 && Iarray[43] <= 2) ? Iarray[43] : 0;
    learned_prepare_inference(S);
    learned = S.L.C.ok;  // a coarse matrix that is not positive definite: plain CG for all cases
    const size_t n48 = size_t(S.N) * kRhsStride, nc16 = size_t(std::max(S.L.C.nc, 1)) * kMaxRhs;
    S.mzs.alloc(n48);
    S.mdpos.alloc(n48);
    if (S.mrold.n != n48) {
      S.mrold.alloc(n48);
      S.mrold.zero(S.stream);
    }
    S.mbc.alloc(nc16);
    S.my.alloc(nc16);
  }
  const double t1 = wall();
  Range rs("hecmw33_solve_multi");
  float ms = 0.0f;
  int kernels = 0, rc = 0, conv = 1, div = 0;
  const size_t n3 = size_t(S.n3());
  for (int k0 = 0; k0 < nrhs; k0 += kMaxRhs) {
    const int m = std::min(kMaxRhs, nrhs - k0);
    ms += run_multi_chunk(S, m, dB + n3 * k0, dX + n3 * k0, iterPREmax, TOL, MAXIT, iter + k0, resid + k0,
                          error + k0, true_resid + k0, &kernels, learned);
    for (int k = k0; k < k0 + m; k++) {
      if (!rc && error[k] != 0 && error[k] != HECMW33_ERR_ZERO_RHS) rc = error[k];
      if (!(error[k] == HECMW33_ERR_ZERO_RHS || true_resid[k] < TOL)) conv = 0;
      if (error[k] == HECMW33_ERR_DIVERGE_PC || error[k] == HECMW33_ERR_DIVERGE_MAT ||
          error[k] == HECMW33_ERR_DIVERGE_NAN)
        div = 1;
    }
  }
  Iarray[80] = conv;
  Iarray[81] = div;
  S.last_iter = *std::max_element(iter, iter + nrhs);
  S.last_outer = (nrhs + kMaxRhs - 1) / kMaxRhs;
  S.last_kernels = kernels;
  S.last_solve_s = ms * 1e-3;
  S.last_setup_s = t1 - t0;
  S.last_true_resid = *std::max_element(true_resid, true_resid + nrhs);
  S.last_learned = learned ? 1 : 0;
  S.last_fallback = 0;
  if (times) {
    times[0] = t1 - t0;
    times[1] = ms * 1e-3;
  }
  return rc;
}

// ---------------------------------------------------------------------------
// A domain of a decomposed mesh: hecmw_update_R and hecmw_allreduce_R1 through the
// caller's functions, CG (hecmw_solver_CG.f90:77-288) with the halo update before
// every product and allreduced inner products.

// hecmw_allreduce_R1 (hecmw_sum); a domain without a table sums over itself.
double domain_allreduce(Solver &S, double v) {
  const DomainState &d = S.dom;
  return (d.has_table && d.allreduce) ? d.allreduce(d.ctx, v) : v;
}

// hecmw_update_R of the vector whose internal part is v (3N, device): its external
// values land in xe (3 n_ext, device).  No neighbours: nothing changes
// (hecmw_comm_f.F90:850).
void halo_update(Solver &S, const double *v, double *xe) {
  DomainState &d = S.dom;
  if (!d.has_table || (d.n_exp == 0 && d.n_imp == 0)) return;
  cudaStream_t s = S.stream;
  const int gv = S.grid_vec();
  if (d.n_exp) {
    launch_k(s, halo_pack_kernel, gv, kThreads, v, static_cast<const int *>(d.exp_idx.p), d.n_exp, d.send_d.p);
    H33_CUDA(cudaMemcpyAsync(d.send_h, d.send_d.p, sizeof(double) * 3 * d.n_exp, cudaMemcpyDeviceToHost, s));
  }
  S.sync();
  d.exchange(d.ctx, d.send_h, d.recv_h);
  if (d.n_imp) {
    H33_CUDA(cudaMemcpyAsync(d.recv_d.p, d.recv_h, sizeof(double) * 3 * d.n_imp, cudaMemcpyHostToDevice, s));
    launch_k(s, halo_unpack_kernel, gv, kThreads, static_cast<const double *>(d.recv_d.p),
             static_cast<const int *>(d.imp_idx.p), d.n_imp, xe);
  }
}

// y = A v over the internal rows: halo update of v into xe, the A_II product, then
// the interface blocks (the reference's matvec order: external columns last).
void domain_matvec(Solver &S, const double *v, double *xe, double *y, int *launched) {
  if (S.mpc.active) {  // y = T^T A T v (hecmw_TtmatTvec_33)
    cudaStream_t s = S.stream;
    const int n3 = S.n3(), gm = std::max(1, std::min((S.mpc.n + kThreads - 1) / kThreads, S.nsm * 4));
    H33_CUDA(cudaMemcpyAsync(S.mpc.t.p, v, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    launch_k(s, mpc_tvec_kernel, gm, kThreads, static_cast<const int *>(S.mpc.slave.p),
             static_cast<const int *>(S.mpc.ptr.p), static_cast<const int *>(S.mpc.idx.p),
             static_cast<const double *>(S.mpc.val.p), S.mpc.n, v, S.mpc.t.p);
    launch_k(s, spmv_kernel<double, 0>, S.grid_spmv(), kThreads, S.A.view(), static_cast<const double *>(S.mpc.t.p),
             S.mpc.w.p, static_cast<const double *>(nullptr), static_cast<CgState *>(nullptr),
             static_cast<double *>(nullptr));
    H33_CUDA(cudaMemcpyAsync(y, S.mpc.w.p, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    launch_k(s, mpc_ttvec_kernel, gm, kThreads, static_cast<const int *>(S.mpc.slave.p),
             static_cast<const int *>(S.mpc.ptr.p), static_cast<const int *>(S.mpc.idx.p),
             static_cast<const double *>(S.mpc.val.p), S.mpc.n, static_cast<const double *>(S.mpc.w.p), y);
    *launched += 3;
    return;
  }
  halo_update(S, v, xe);
  launch_k(S.stream, spmv_kernel<double, 0>, S.grid_spmv(), kThreads, S.A.view(), v, y,
           static_cast<const double *>(nullptr), static_cast<CgState *>(nullptr), static_cast<double *>(nullptr));
  (*launched)++;
  const DomainState &d = S.dom;
  if (d.n_irows) {
    launch_k(S.stream, interface_spmv_kernel, std::max(1, std::min((d.n_irows + kThreads - 1) / kThreads, S.nsm * 8)),
             kThreads, static_cast<const int *>(d.irow.p), static_cast<const int *>(d.iptr.p),
             static_cast<const int *>(d.icol.p), static_cast<const double *>(d.ival.p), d.n_irows,
             static_cast<const double *>(xe), y);
    (*launched)++;
  }
}

// r = b - A x (hecmw_matresid_33, hecmw_solver_las_33.F90:367-399)
void domain_matresid(Solver &S, const double *x, double *xe, const double *b, double *r, int *launched) {
  domain_matvec(S, x, xe, r, launched);
  launch_k(S.stream, vec_xpay_kernel, S.grid_vec(), kThreads, r, -1.0, b, S.n3());
  (*launched)++;
}

double domain_dot(Solver &S, const double *a, const double *b) { return domain_allreduce(S, dot_device(S, a, b)); }

// hecmw_precond_apply on a domain (hecmw_precond.f90:86-172): with iterPREmax > 1 the
// outer passes form ZP = R - A Z, whose product updates the halo of Z first (Z,
// external entries included, starts at zero).
void domain_precond_apply(Solver &S, const Views<double> &V, int iterpremax, const double *r, double *z,
                          int *launched) {
  if (iterpremax <= 1) {
    launch_precond_plain<double>(S, V, iterpremax, r, z, nullptr);
    *launched += 2 * std::max(1, int(S.pc.lo.group_slice.size()));
    return;
  }
  cudaStream_t s = S.stream;
  DomainState &d = S.dom;
  d.xe_z.zero(s);
  const double *in = r;
  for (int it = 1; it <= iterpremax; it++) {
    launch_sweep<double, false>(S, V, in, V.zp, nullptr);
    *launched += 2 * std::max(1, int(S.pc.lo.group_slice.size()));
    if (it == 1) launch_k(s, copy_kernel<double>, S.grid_vec(), kThreads, static_cast<const double *>(V.zp), z, S.n3(),
                          static_cast<const CgState *>(nullptr));
    else launch_k(s, add_kernel<double>, S.grid_vec(), kThreads, static_cast<const double *>(V.zp), z, S.n3(),
                  static_cast<const CgState *>(nullptr));
    (*launched)++;
    if (it == iterpremax) break;
    domain_matresid(S, z, d.xe_z.p, r, V.w, launched);
    in = V.w;
  }
}

// hecmw_solve_CG on one domain, host-driven (every inner product is a global sum).
float run_cg_domain(Solver &S, int iterpremax, double tol, int maxit, int *error, int *iter, double *resid,
                    int *kernels) {
  cudaStream_t s = S.stream;
  DomainState &d = S.dom;
  const int n3 = S.n3(), gv = S.grid_vec();
  const Views<double> V = views(S, 0.0, 0);
  double *X = S.x.p, *R = S.r.p, *Z = S.z.p, *P = S.p.p, *Q = S.q.p;
  const double *B = S.b.p;
  int launched = 0;
  H33_CUDA(cudaEventRecord(S.ev0, s));
  d.xe_p.zero(s);  // the direction's external entries start at zero (WW is allocated zeroed)
  domain_matresid(S, X, d.xe_x.p, B, R, &launched);
  const double BNRM2 = domain_dot(S, B, B);
  *error = 0;
  *resid = 0.0;
  if (BNRM2 == 0.0) {
    maxit = 0;
    H33_CUDA(cudaMemsetAsync(X, 0, sizeof(double) * n3, s));
    d.xe_x.zero(s);
  }
  int n_indef = 0, it;
  double RHO1 = 0.0;
  for (it = 1; it <= maxit; it++) {
    domain_precond_apply(S, V, iterpremax, R, Z, &launched);
    const double RHO = domain_dot(S, R, Z);
    if (RHO == 0.0) break;
    else if (it > 1 && RHO * RHO1 <= 0) {
      if (++n_indef >= 3) {
        *error = HECMW33_ERR_DIVERGE_PC;
        break;
      }
    } else if (RHO != RHO) {
      *error = HECMW33_ERR_DIVERGE_NAN;
      break;
    }
    if (it == 1) {
      H33_CUDA(cudaMemcpyAsync(P, Z, sizeof(double) * n3, cudaMemcpyDeviceToDevice, s));
    } else {
      launch_k(s, vec_xpay_kernel, gv, kThreads, P, RHO / RHO1, static_cast<const double *>(Z), n3);
      launched++;
    }
    domain_matvec(S, P, d.xe_p.p, Q, &launched);
    const double C1 = domain_dot(S, P, Q);
    if (C1 <= 0) {
      *error = HECMW33_ERR_DIVERGE_MAT;
      break;
    } else if (C1 != C1) {
      *error = HECMW33_ERR_DIVERGE_NAN;
      break;
    }
    const double ALPHA = RHO / C1;
    launch_k(s, vec_axpy_kernel, gv, kThreads, X, ALPHA, static_cast<const double *>(P), n3);
    launched++;
    if (it % kIterRecomputeR == 0) {
      domain_matresid(S, X, d.xe_x.p, B, R, &launched);
    } else {
      launch_k(s, vec_axpy_kernel, gv, kThreads, R, -ALPHA, static_cast<const double *>(Q), n3);
      launched++;
    }
    double DNRM2 = domain_dot(S, R, R);
    *resid = std::sqrt(DNRM2 / BNRM2);
    if (*resid <= tol) {
      if (it % kIterRecomputeR == 0) break;
      domain_matresid(S, X, d.xe_x.p, B, R, &launched);
      DNRM2 = domain_dot(S, R, R);
      *resid = std::sqrt(DNRM2 / BNRM2);
      if (*resid <= tol) break;
    }
    if (it == maxit) *error = HECMW33_ERR_NOCONV_MAXIT;
    RHO1 = RHO;
  }
  halo_update(S, X, d.xe_x.p);  // hecmw_solver_CG.f90:288
  *iter = it;
  H33_CUDA(cudaEventRecord(S.ev1, s));
  S.sync();
  float ms = 0.0f;
  H33_CUDA(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
  if (kernels) *kernels += launched;
  return ms;
}

// hecmw_solve -> hecmw_solve_iterative (METHOD = 1) on one domain: allreduced zero-RHS
// and zero-diagonal checks (hecmw_solver_Iterative.f90:255-323), the recycle policy
// and the local preconditioner, CG, the sigma_diag retry of a diverged ILU, and the
// allreduced true residual.
struct MpcScope {  // the MPC operator for the duration of a solve
  Solver &S;
  MpcScope(Solver &s, bool on) : S(s) { S.mpc.active = on; }
  ~MpcScope() { S.mpc.active = false; }
};

int solve_domain(Solver &S, int *Iarray, double *Rarray, int *iter, double *resid, double *times) {
  const double t0 = wall();
  *iter = 0;
  *resid = 0.0;
  if (times) times[0] = times[1] = times[2] = 0.0;
  const bool mpc = S.mpc.n > 0 && Iarray[12] == 2;
  const char *what = S.dom.on ? "a decomposed domain" : "MPC-CG (MPC_METHOD = 2)";
  if (mpc && S.dom.on) throw Failure(HECMW33_ERR_BAD_INPUT, "MPC-CG runs on a whole (one-domain) mesh");
  if (Iarray[1] != 1) throw Failure(HECMW33_ERR_BAD_INPUT, std::string(what) + " runs CG (METHOD = 1)");
  if (Iarray[41] != 0 || Iarray[42] != 0)
    throw Failure(HECMW33_ERR_BAD_INPUT, std::string(what) + " runs the FP64 CG (Iarray(42) = Iarray(43) = 0)");
  if (Iarray[6] != 0) throw Failure(HECMW33_ERR_BAD_INPUT, std::string(what) + " runs with SCALING=NO");
  if (mpc) {
    S.mpc.t.alloc(size_t(S.n3()));
    S.mpc.w.alloc(size_t(S.n3()));
  }
  MpcScope mpc_scope(S, mpc);
  DomainState &d = S.dom;
  // hecmw_solve_check_zerorhs adds the MPC constants (hecmw_solver_Iterative.f90:305-309)
  const double bb = domain_allreduce(S, dot_device(S, S.b.p, S.b.p) + (S.mpc.n_raw > 0 ? S.mpc.const2 : 0.0));
  S.bnrm2 = bb;
  if (bb == 0.0) {
    H33_CUDA(cudaMemsetAsync(S.x.p, 0, sizeof(double) * S.n3(), S.stream));
    d.xe_x.zero(S.stream);
    S.sync();
    Iarray[80] = 1;
    Iarray[81] = 0;
    return HECMW33_ERR_ZERO_RHS;
  }
  const int MAXIT = Iarray[0], PRECOND = Iarray[2], iterPREmax = Iarray[4];
  const double TOL = Rarray[0];
  double sigma = Rarray[1];
  const bool auto_sigma = sigma < 0.0;
  if (auto_sigma) sigma = 1.0;
  if (domain_allreduce(S, S.zero_diag ? 1.0 : 0.0) > 0.0 && PRECOND < 10 && iterPREmax > 0)
    return HECMW33_ERR_ZERO_DIAG;
  recycle_precond_setting(Iarray);
  const double t1 = wall();
  int error = 0, kernels = 0;
  float ms_total = 0.0f;
  if (iterPREmax > 0) precond_setup(S, PRECOND, Iarray[33], sigma, Iarray);
  Range rs("hecmw33_solve_domain");
  for (;;) {
    Iarray[80] = 0;
    Iarray[81] = 0;
    ms_total += run_cg_domain(S, iterPREmax, TOL, MAXIT, &error, iter, resid, &kernels);
    if (error == HECMW33_ERR_DIVERGE_PC || error == HECMW33_ERR_DIVERGE_MAT || error == HECMW33_ERR_DIVERGE_NAN) {
      Iarray[81] = 1;
      // Iterative.f90:133-137: the retry's setup finds flags 97/98 cleared and keeps
      // the factorisation; CG continues from the current X
      if (PRECOND >= 10 && PRECOND < 20 && auto_sigma && sigma < 2.0) {
        sigma = sigma + 0.1;
        continue;
      }
    }
    break;
  }
  // hecmw_rel_resid_L2_33 with the halo update inside matresid
  int launched = 0;
  domain_matresid(S, S.x.p, d.xe_x.p, S.b.p, S.w.p, &launched);
  double bn = domain_dot(S, S.b.p, S.b.p);
  if (bn == 0.0) bn = 1.0;
  const double resid2 = std::sqrt(domain_dot(S, S.w.p, S.w.p) / bn);
  if (resid2 < TOL) Iarray[80] = 1;
  S.last_learned = 0;
  S.last_fallback = 0;
  S.last_iter = *iter;
  S.last_outer = 1;
  S.last_kernels = kernels + launched;
  S.last_solve_s = ms_total * 1e-3;
  S.last_setup_s = t1 - t0;
  S.last_true_resid = resid2;
  if (times) {
    times[0] = t1 - t0;
    times[1] = ms_total * 1e-3;
  }
  return error;
}

int solve_resident(Solver &S, int *Iarray, double *Rarray, int *iter, double *resid, double *times) {
  if (S.dom.on || (S.mpc.n > 0 && Iarray[12] == 2)) return solve_domain(S, Iarray, Rarray, iter, resid, times);
  if (Iarray[6] != 0 && (Iarray[41] == 2 || Iarray[41] == 3))
    throw Failure(HECMW33_ERR_BAD_INPUT, "SCALING=YES is implemented for the FP64 CG (Iarray(42) = 0 or 1)");
  if (Iarray[1] >= 2 && (Iarray[41] == 2 || Iarray[41] == 3))
    throw Failure(HECMW33_ERR_BAD_INPUT, "BiCGSTAB and GMRES run in FP64 (Iarray(42) = 0 or 1)");
  switch (Iarray[41]) {
    case 1: return solve_fp64(S, Iarray, Rarray, iter, resid, times, 1);
    case 2: return solve_mixed_restart(S, Iarray, Rarray, iter, resid, times);
    case 3: return solve_mixed_reliable(S, Iarray, Rarray, iter, resid, times);
    default: return solve_fp64(S, Iarray, Rarray, iter, resid, times, 0);
  }
}

}  // namespace

void set_last_error(const std::string &msg) { g_last_error = msg; }

namespace {

void fail(int *ierr, int code, const char *msg) {
  g_last_error = msg;
  if (ierr) *ierr = code;
}

// The external part of X (entries 3N..3NP-1) of a decomposed domain: into the
// handle's copy before the solve, back to the caller after it.
void halo_x_in(Solver &S, const double *Xe, cudaMemcpyKind kind) {
  const DomainState &d = S.dom;
  if (d.on && d.n_ext)
    H33_CUDA(cudaMemcpyAsync(d.xe_x.p, Xe, sizeof(double) * 3 * size_t(d.n_ext), kind, S.stream));
}
void halo_x_out(Solver &S, double *Xe, cudaMemcpyKind kind) {
  const DomainState &d = S.dom;
  if (d.on && d.n_ext)
    H33_CUDA(cudaMemcpyAsync(Xe, d.xe_x.p, sizeof(double) * 3 * size_t(d.n_ext), kind, S.stream));
}

void no_domain(const Solver &S, const char *what) {
  if (S.dom.on) throw Failure(HECMW33_ERR_BAD_INPUT, std::string(what) + " is for a whole (one-domain) mesh");
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

HECMW33_API void hecmw33_gpu_set_domain(const int *handle, const int *n_neighbor_pe, const int *neighbor_pe,
                                        const int *import_index, const int *import_item,
                                        const int *export_index, const int *export_item,
                                        hecmw33_exchange_fn exchange, hecmw33_allreduce_fn allreduce,
                                        void *ctx, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  if (!S.has_matrix || !S.dom.on)
    throw Failure(HECMW33_ERR_NO_MATRIX, "set_domain: first a domain matrix (N < NP) by hecmw33_gpu_set_matrix");
  DomainState &d = S.dom;
  const int nn = n_neighbor_pe ? *n_neighbor_pe : 0;
  if (nn < 0) throw Failure(HECMW33_ERR_BAD_INPUT, "n_neighbor_pe < 0");
  if (nn > 0 && (!neighbor_pe || !import_index || !export_index || !exchange || !allreduce))
    throw Failure(HECMW33_ERR_BAD_INPUT, "set_domain: null table or function");
  const int n_imp = nn ? import_index[nn] : 0, n_exp = nn ? export_index[nn] : 0;
  if (nn && (import_index[0] != 0 || export_index[0] != 0 || n_imp < 0 || n_exp < 0 ||
             (n_imp && !import_item) || (n_exp && !export_item)))
    throw Failure(HECMW33_ERR_BAD_INPUT, "set_domain: inconsistent import/export index");
  for (int k = 0; k < nn; k++)
    if (import_index[k + 1] < import_index[k] || export_index[k + 1] < export_index[k])
      throw Failure(HECMW33_ERR_BAD_INPUT, "set_domain: index arrays must be non-decreasing");
  const int N = S.N;
  std::vector<int> imp(static_cast<size_t>(n_imp)), expt(static_cast<size_t>(n_exp));
  for (int k = 0; k < n_imp; k++) {
    const int it = import_item[k];
    if (it <= N || it > d.NP) throw Failure(HECMW33_ERR_BAD_INPUT, "set_domain: import_item outside N+1..NP");
    imp[size_t(k)] = it - N - 1;
  }
  for (int k = 0; k < n_exp; k++) {
    const int it = export_item[k];
    if (it < 1 || it > N) throw Failure(HECMW33_ERR_BAD_INPUT, "set_domain: export_item outside 1..N");
    expt[size_t(k)] = it - 1;
  }
  d.clear_table();
  d.n_imp = n_imp;
  d.n_exp = n_exp;
  d.imp_idx.upload(imp, S.stream);
  d.exp_idx.upload(expt, S.stream);
  d.send_d.alloc(3 * size_t(std::max(n_exp, 1)));
  d.recv_d.alloc(3 * size_t(std::max(n_imp, 1)));
  H33_CUDA(cudaMallocHost(&d.send_h, sizeof(double) * 3 * size_t(std::max(n_exp, 1))));
  H33_CUDA(cudaMallocHost(&d.recv_h, sizeof(double) * 3 * size_t(std::max(n_imp, 1))));
  d.exchange = exchange;
  d.allreduce = allreduce;
  d.ctx = ctx;
  d.has_table = nn > 0;
  S.sync();
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_set_mpc(const int *handle, const int *n_mpc, const int *mpc_index, const int *mpc_item,
                                     const int *mpc_dof, const double *mpc_val, const double *mpc_const,
                                     int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "set_mpc: set the matrix first");
  const int n = n_mpc ? *n_mpc : 0;
  if (n < 0) throw Failure(HECMW33_ERR_BAD_INPUT, "n_mpc < 0");
  std::vector<int> slave, ptr{0}, idx;
  std::vector<double> val;
  double c2 = 0.0;
  if (n > 0) {
    if (!mpc_index || !mpc_item || !mpc_dof || !mpc_val) throw Failure(HECMW33_ERR_BAD_INPUT, "set_mpc: null array");
    if (mpc_index[0] != 0) throw Failure(HECMW33_ERR_BAD_INPUT, "set_mpc: mpc_index(0) must be 0");
    const int nn = S.N;
    for (int i = 0; i < n; i++) {
      const int j0 = mpc_index[i], j1 = mpc_index[i + 1];
      if (j1 <= j0) throw Failure(HECMW33_ERR_BAD_INPUT, "set_mpc: an MPC without terms");
      bool skip = false;  // an MPC with a DOF above 3 is left out (hecmw_solver_las_33.F90:479-481)
      for (int j = j0; j < j1; j++) {
        if (mpc_item[j] < 1 || mpc_item[j] > nn || mpc_dof[j] < 1)
          throw Failure(HECMW33_ERR_BAD_INPUT, "set_mpc: MPC term outside the mesh");
        if (mpc_dof[j] > 3) skip = true;
      }
      if (skip) continue;
      slave.push_back(3 * (mpc_item[j0] - 1) + mpc_dof[j0] - 1);
      for (int j = j0 + 1; j < j1; j++) {
        idx.push_back(3 * (mpc_item[j] - 1) + mpc_dof[j] - 1);
        val.push_back(mpc_val[j]);
      }
      ptr.push_back(int(idx.size()));
    }
    if (mpc_const)
      for (int i = 0; i < n; i++) c2 = c2 + mpc_const[i] * mpc_const[i];
  }
  S.mpc.n = int(slave.size());
  S.mpc.n_raw = n;
  S.mpc.const2 = c2;
  S.mpc.slave.upload(slave, S.stream);
  S.mpc.ptr.upload(ptr, S.stream);
  S.mpc.idx.upload(idx, S.stream);
  S.mpc.val.upload(val, S.stream);
  S.sync();
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
  halo_x_in(S, X + S.n3(), cudaMemcpyHostToDevice);
  const int rc = solve_resident(S, Iarray, Rarray, iter, resid, times);
  H33_CUDA(cudaMemcpyAsync(X, S.x.p, bytes, cudaMemcpyDeviceToHost, S.stream));
  halo_x_out(S, X + S.n3(), cudaMemcpyDeviceToHost);
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
  halo_x_in(S, dX + S.n3(), cudaMemcpyDeviceToDevice);
  const int rc = solve_resident(S, Iarray, Rarray, iter, resid, times);
  H33_CUDA(cudaMemcpyAsync(dX, S.x.p, bytes, cudaMemcpyDeviceToDevice, S.stream));
  halo_x_out(S, dX + S.n3(), cudaMemcpyDeviceToDevice);
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
  halo_x_in(S, X + S.n3(), cudaMemcpyHostToDevice);
  const int rc = solve_resident(S, Iarray, Rarray, iter, resid, times);
  H33_CUDA(cudaMemcpyAsync(X, S.x.p, bytes, cudaMemcpyDeviceToHost, S.stream));
  halo_x_out(S, X + S.n3(), cudaMemcpyDeviceToHost);
  S.sync();
  if (times) times[0] += tm;
  if (ierr) *ierr = rc;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_solve_multi(const int *handle, const int *nrhs, const double *B, double *X,
                                         int *Iarray, double *Rarray, int *iter, double *resid, int *error,
                                         double *true_resid, double *times, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  no_domain(S, "hecmw33_gpu_solve_multi");
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix: call hecmw33_gpu_set_matrix first");
  if (!nrhs || *nrhs < 1) throw Failure(HECMW33_ERR_BAD_INPUT, "nrhs must be positive");
  const size_t total = size_t(S.n3()) * size_t(*nrhs);
  DevArray<double> dB, dX;
  dB.alloc(total);
  dX.alloc(total);
  upload_host(S, dB.p, B, sizeof(double) * total);
  upload_host(S, dX.p, X, sizeof(double) * total);
  std::vector<double> tr(static_cast<size_t>(*nrhs));
  const int rc = solve_multi(S, *nrhs, dB.p, dX.p, Iarray, Rarray, iter, resid, error, tr.data(), times);
  H33_CUDA(cudaMemcpyAsync(X, dX.p, sizeof(double) * total, cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  if (true_resid) std::copy(tr.begin(), tr.end(), true_resid);
  if (ierr) *ierr = rc;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_solve_multi_device(const int *handle, const int *nrhs, const double *dB, double *dX,
                                                int *Iarray, double *Rarray, int *iter, double *resid, int *error,
                                                double *true_resid, double *times, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  no_domain(S, "hecmw33_gpu_solve_multi_device");
  if (!nrhs || *nrhs < 1) throw Failure(HECMW33_ERR_BAD_INPUT, "nrhs must be positive");
  std::vector<double> tr(static_cast<size_t>(*nrhs));
  const int rc = solve_multi(S, *nrhs, dB, dX, Iarray, Rarray, iter, resid, error, tr.data(), times);
  if (true_resid) std::copy(tr.begin(), tr.end(), true_resid);
  if (ierr) *ierr = rc;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_matvec(const int *handle, const double *X, double *Y, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  no_domain(S, "hecmw33_gpu_matvec");
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix: call hecmw33_gpu_set_matrix first");
  const size_t bytes = sizeof(double) * S.n3();
  H33_CUDA(cudaMemcpyAsync(S.w.p, X, bytes, cudaMemcpyHostToDevice, S.stream));
  launch_k(S.stream, spmv_kernel<double, 0>, S.grid_spmv(), kThreads, S.A.view(), S.w.p, S.zp.p, nullptr, nullptr,
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
  no_domain(S, "hecmw33_gpu_precond_apply");
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix: call hecmw33_gpu_set_matrix first");
  const int iterPREmax = Iarray[4];
  double sigma = Rarray[1];
  if (sigma < 0.0) sigma = 1.0;
  if (iterPREmax > 0) precond_setup(S, Iarray[2], Iarray[33], sigma, Iarray);
  const size_t bytes = sizeof(double) * S.n3();
  H33_CUDA(cudaMemcpyAsync(S.r.p, R, bytes, cudaMemcpyHostToDevice, S.stream));
  launch_precond<double>(S, views(S, 0.0), iterPREmax, S.r.p, S.z.p, nullptr);
  H33_CUDA(cudaGetLastError());
  H33_CUDA(cudaMemcpyAsync(Z, S.z.p, bytes, cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_assemble_hex8(const int *handle, const int *n_node, const double *coords,
                                           const int *n_elem, const int *conn, const double *E, const double *nu,
                                           const double *F, const int *n_bc, const int *bc_node,
                                           const int *bc_dof, const double *bc_value, const int *symbolic,
                                           int *NPL, int *NPU, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  const int nbc = n_bc ? *n_bc : 0;
  HexMaterial mat;
  mat.E = E;
  mat.nu = nu;
  assemble_hex8(S, *n_node, coords, *n_elem, conn, mat, F, nbc, bc_node, bc_dof, bc_value,
                !symbolic || *symbolic != 0);
  if (NPL) *NPL = S.NPL;
  if (NPU) *NPU = S.NPU;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_assemble_hex8_neohooke(const int *handle, const int *n_node, const double *coords,
                                                    const int *n_elem, const int *conn, const double *C10,
                                                    const double *D1, const double *U, const double *F,
                                                    const int *n_bc, const int *bc_node, const int *bc_dof,
                                                    const double *bc_value, const int *symbolic, int *NPL,
                                                    int *NPU, int *n_inverted, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  if (!U) throw Failure(HECMW33_ERR_BAD_INPUT, "nodal displacements U are required");
  const int nbc = n_bc ? *n_bc : 0;
  HexMaterial mat;
  mat.U = U;
  mat.C10 = *C10;
  mat.D1 = *D1;
  int inv = 0;
  assemble_hex8(S, *n_node, coords, *n_elem, conn, mat, F, nbc, bc_node, bc_dof, bc_value,
                !symbolic || *symbolic != 0, &inv);
  if (NPL) *NPL = S.NPL;
  if (NPU) *NPU = S.NPU;
  if (n_inverted) *n_inverted = inv;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_get_matrix(const int *handle, int *indexL, int *itemL, int *indexU, int *itemU,
                                        double *D, double *AL, double *AU, double *B, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  no_domain(S, "hecmw33_gpu_get_matrix");
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix");
  const int N = S.N;
  if (indexL) std::copy(S.indexL.begin(), S.indexL.end(), indexL);
  if (itemL) std::copy(S.itemL.begin(), S.itemL.end(), itemL);
  if (indexU) std::copy(S.indexU.begin(), S.indexU.end(), indexU);
  if (itemU) std::copy(S.itemU.begin(), S.itemU.end(), itemU);
  if (D) H33_CUDA(cudaMemcpyAsync(D, S.raw.p, sizeof(double) * 9 * N, cudaMemcpyDeviceToHost, S.stream));
  if (AL && S.NPL)
    H33_CUDA(cudaMemcpyAsync(AL, S.raw.p + 9 * size_t(N), sizeof(double) * 9 * S.NPL, cudaMemcpyDeviceToHost,
                             S.stream));
  if (AU && S.NPU)
    H33_CUDA(cudaMemcpyAsync(AU, S.raw.p + 9 * (size_t(N) + S.NPL), sizeof(double) * 9 * S.NPU,
                             cudaMemcpyDeviceToHost, S.stream));
  if (B) H33_CUDA(cudaMemcpyAsync(B, S.b.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_solve_assembled(const int *handle, double *X, int *Iarray, double *Rarray,
                                             int *iter, double *resid, double *times, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix: call hecmw33_gpu_assemble_hex8 first");
  const size_t bytes = sizeof(double) * S.n3();
  H33_CUDA(cudaMemcpyAsync(S.x.p, X, bytes, cudaMemcpyHostToDevice, S.stream));
  const int rc = solve_resident(S, Iarray, Rarray, iter, resid, times);
  H33_CUDA(cudaMemcpyAsync(X, S.x.p, bytes, cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  if (ierr) *ierr = rc;
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

HECMW33_API void hecmw33_gpu_smoother_schedule(const int *N, const int *indexL, const int *itemL,
                                               const int *indexU, const int *itemU, int *ncolor,
                                               int *colorindex, int *perm, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  const int n = *N;
  validate(n, n, indexL[n], indexU[n], indexL, itemL, indexU, itemU);
  Profile prof{n, indexL, itemL, indexU, itemU};
  std::vector<int> pm, ipm, ci;
  *ncolor = ordering_greedy(prof, ci, pm, ipm);
  for (int c = 0; c <= *ncolor; c++) colorindex[c] = ci[c];
  for (int i = 0; i < n; i++) perm[i] = pm[i] + 1;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_coarse_aggregates(const int *N, const int *indexL, const int *itemL,
                                               const int *indexU, const int *itemU, const int *max_aggregates,
                                               int *n_agg, int *agg, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  const int n = *N;
  validate(n, n, indexL[n], indexU[n], indexL, itemL, indexU, itemU);
  Profile prof{n, indexL, itemL, indexU, itemU};
  Aggregation ag;
  aggregate_nodes(prof, max_aggregates && *max_aggregates > 0 ? *max_aggregates : coarse_max_aggregates(), ag);
  *n_agg = ag.n_agg;
  for (int i = 0; i < n; i++) agg[i] = ag.agg[size_t(i)];
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_condition_estimate(const int *handle, int *n, double *emin, double *emax, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  *n = S.last_lanczos_n;
  *emin = S.last_emin;
  *emax = S.last_emax;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_last_solve_info(const int *handle, int *info, double *dinfo, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  for (int i = 0; i < 16; i++) {
    info[i] = 0;
    dinfo[i] = 0.0;
  }
  info[8] = S.last_learned;
  info[9] = S.last_fallback;
  info[10] = int(S.L.pr.size());
  info[0] = S.last_iter;
  info[1] = S.last_kernels;
  info[2] = S.pc.valid ? int(S.pc.lo.group_slice.size() + S.pc.up.group_slice.size()) - 2 : 0;
  info[3] = S.g64.kernels_per_iter ? S.g64.kernels_per_iter : S.g32.kernels_per_iter;
  info[7] = S.last_outer;
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
  held += S.pc.alu32_fwd.bytes() + S.pc.alu32_bwd.bytes();
  for (auto *v : {&S.bf, &S.xf, &S.rf, &S.zf, &S.pf, &S.qf, &S.wf, &S.zpf}) held += v->bytes();
  dinfo[4] = double(held);
  dinfo[5] = S.last_true_resid;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_time_spmv(const int *handle, const int *reps, double *ms_per_launch, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix");
  const int n = std::max(1, *reps);
  launch_k(S.stream, spmv_kernel<double, 0>, S.grid_spmv(), kThreads, S.A.view(), S.x.p, S.zp.p, nullptr, nullptr, nullptr);
  H33_CUDA(cudaEventRecord(S.ev0, S.stream));
  for (int i = 0; i < n; i++)
    launch_k(S.stream, spmv_kernel<double, 0>, S.grid_spmv(), kThreads, S.A.view(), S.x.p, S.zp.p, nullptr, nullptr,
                                                                      nullptr);
  H33_CUDA(cudaGetLastError());
  H33_CUDA(cudaEventRecord(S.ev1, S.stream));
  S.sync();
  float ms = 0.0f;
  H33_CUDA(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
  *ms_per_launch = double(ms) / n;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_time_precond(const int *handle, const int *reps, const int *lowp,
                                          double *ms_per_apply, double *bytes_per_apply, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix");
  if (!S.pc.valid) throw Failure(HECMW33_ERR_BAD_INPUT, "no preconditioner: solve once first");
  const bool smoother = lowp && (*lowp & 2);
  if (smoother) {
    if (S.pc.kind != 1) throw Failure(HECMW33_ERR_BAD_INPUT, "the learned smoother follows an SSOR setup");
    ensure_smoother(S);
  }
  Precond &P = smoother ? S.L.sm : S.pc;
  const int lp = (lowp && (*lowp & 1) && P.kind != 3) ? 1 : 0;
  if (lp) ensure_lowp(S, P);
  const Views<double> V = views(S, 0.0, lp, &P);
  const int n = std::max(1, *reps);
  // z = M^-1 r on the resident r (the last solve's residual), one pass (iterPREmax = 1)
  launch_sweep<double, false>(S, V, S.r.p, S.w.p, nullptr);
  H33_CUDA(cudaEventRecord(S.ev0, S.stream));
  for (int i = 0; i < n; i++) launch_sweep<double, false>(S, V, S.r.p, S.w.p, nullptr);
  H33_CUDA(cudaGetLastError());
  H33_CUDA(cudaEventRecord(S.ev1, S.stream));
  S.sync();
  float ms = 0.0f;
  H33_CUDA(cudaEventElapsedTime(&ms, S.ev0, S.ev1));
  *ms_per_apply = double(ms) / n;
  // algorithmic bytes of one forward + backward application: every off-diagonal block
  // once (values + column index), the diagonal LU read by both sweeps, the row
  // pointers of both triangles, and r read / z written and read back per sweep
  const double nb = double(S.NPL) + double(S.NPU), nn = double(S.N);
  const double vb = lp ? 18.0 : 72.0, ab = lp ? 36.0 : 72.0;
  if (bytes_per_apply)
    *bytes_per_apply = P.kind == 3 ? nn * (ab + 48.0)
                                   : nb * (vb + 4.0) + 2.0 * ab * nn + 2.0 * 4.0 * 2.0 * (nn + 1.0) + 2.0 * 2.0 * 24.0 * nn;
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_learn_record(const int *handle, const int *enable, const int *max_pairs,
                                          int *npairs, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  S.L.recording = enable && *enable != 0;
  if (max_pairs && *max_pairs > 0) S.L.max_pairs = *max_pairs;
  if (enable && *enable < 0) {  // forget the recorded pairs
    S.L.pr.clear();
    S.L.pe.clear();
    S.L.pzs.clear();
    S.L.per.clear();
    S.L.recording = false;
  }
  if (npairs) *npairs = int(S.L.pr.size());
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_learn_train(const int *handle, const int *steps, const double *lr, double *loss,
                                         int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  double l2[2] = {0.0, 0.0};
  learned_train(S, steps ? *steps : 100, lr ? *lr : 1e-3, l2);
  if (loss) {
    loss[0] = l2[0];
    loss[1] = l2[1];
  }
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_learn_weights(const int *handle, const int *mode, float *theta, int *n, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  const int total = GnnOffsets::make().total;
  if (*mode == 1) {
    if (*n != total) throw Failure(HECMW33_ERR_BAD_INPUT, "expected " + std::to_string(total) + " weights");
    learned_set_weights(S, theta, true);
  } else {
    if (theta && *n >= total && S.L.have_weights) {
      H33_CUDA(cudaMemcpyAsync(theta, S.L.theta.p, sizeof(float) * size_t(total), cudaMemcpyDeviceToHost, S.stream));
      S.sync();
    }
    *n = S.L.have_weights ? total : 0;
    if (!S.L.have_weights && *mode == 0) *n = total == 0 ? 0 : -total;
  }
  H33_ENTRY_END
}

HECMW33_API void hecmw33_gpu_learn_eval(const int *handle, const float *theta, const double *R, const double *E,
                                        double *Z, double *loss, float *grad, int *ierr) {
  if (ierr) *ierr = 0;
  H33_ENTRY_BEGIN
  Solver &S = get(handle);
  DeviceGuard dg(S.device);
  if (!S.has_matrix) throw Failure(HECMW33_ERR_NO_MATRIX, "no matrix");
  if (!(S.pc.valid && S.pc.kind == 1)) throw Failure(HECMW33_ERR_INCONS_PC, "build the SSOR preconditioner first");
  const int total = GnnOffsets::make().total;
  learned_graph(S);
  learned_train_buffers(S);
  coarse_structure(S);
  coarse_values(S);
  learned_set_weights(S, theta, false);
  const size_t n3 = size_t(S.n3());
  std::vector<float> rf(n3), ef(n3), wf(n3);
  for (size_t i = 0; i < n3; i++) {
    rf[i] = float(R[i]);
    ef[i] = float(E[i]);
  }
  DevArray<float> dr, de;
  dr.upload(rf, S.stream);
  de.upload(ef, S.stream);
  const double er = dot_device_f(S, de.p, dr.p);
  if (!(er > 0.0)) throw Failure(HECMW33_ERR_BAD_INPUT, "learn_eval: e.r must be positive (r = A e)");
  const double l = learned_coarse_pass(S, {dr.p}, {er}, true);
  H33_CUDA(cudaMemcpyAsync(wf.data(), S.L.C.omega.p, sizeof(float) * n3, cudaMemcpyDeviceToHost, S.stream));
  if (grad)
    H33_CUDA(cudaMemcpyAsync(grad, S.L.gacc.p, sizeof(float) * size_t(total), cudaMemcpyDeviceToHost, S.stream));
  S.sync();
  for (size_t i = 0; i < n3; i++) Z[i] = wf[i];
  if (loss) *loss = l;
  S.L.weights_version++;
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
