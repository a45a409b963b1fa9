// h33_gnn.cuh -- the learned preconditioner: a 3-layer message-passing network over
// the node graph of the matrix, applied after SSOR inside flexible CG.
//
// No counterpart in the reference solver.  The math is fixed by the CPU reference
// tests/gnn_reference.py (test infrastructure):
//   s_i   = (trace(D_i)/3)^(-1/2),  e_ij = s_i A_ij s_j (9 features per edge)
//   gamma = sqrt(mean(zs^2)) with zs = SSOR(r)
//   x_i   = [zs_i/gamma, s_i^2 r_i/gamma];  h0 = W_in x
//   w^l_ij = tanh(u_l . e_ij + c_l)
//   m^l_i = sum_j w^l_ij h^{l-1}_j;  h^l_i = tanh(Ws_l h^{l-1}_i + Wm_l m^l_i)
//   z_i   = zs_i + gamma W_out h^3_i
// Weights are trained in FP32 (master copy) and used in BF16 (rounded) for
// inference; every product is accumulated in FP32.
//
// Layout: activations are node-major, 32 channels contiguous (128 B per node in
// FP32); a warp handles one node with lane = channel, so every neighbour gather is
// one coalesced 128-byte row.  The 32x32 layer matrices sit in shared memory and
// the node's own vectors are broadcast with warp shuffles.
#pragma once

#include <cuda_bf16.h>

#include "h33_common.cuh"

namespace h33 {

constexpr int kGnnWidth = 32;
constexpr int kGnnLayers = 3;

// Offsets of the flat parameter vector (order of tests/gnn_reference.py).
struct GnnOffsets {
  int W_in, u[kGnnLayers], c[kGnnLayers], Ws[kGnnLayers], Wm[kGnnLayers], W_out, total;
  __host__ __device__ static GnnOffsets make() {
    GnnOffsets o{};
    int k = 0;
    o.W_in = k;
    k += kGnnWidth * 6;
    for (int l = 0; l < kGnnLayers; l++) {
      o.u[l] = k;
      k += 9;
      o.c[l] = k;
      k += 1;
      o.Ws[l] = k;
      k += kGnnWidth * kGnnWidth;
      o.Wm[l] = k;
      k += kGnnWidth * kGnnWidth;
    }
    o.W_out = k;
    k += 3 * kGnnWidth;
    o.total = k;
    return o;
  }
};

// The node graph: CSR over off-diagonal neighbours (ascending columns), the
// reverse-edge index, scaled block features and node scales.
struct GnnGraph {
  int n, nedges;
  const int *ptr, *col, *rev;
  const float *feat;  // nedges x 9
  const float *s;     // n
};

template <class W>
__device__ __forceinline__ float wload(const W *p) {
  return float(*p);
}
template <>
__device__ __forceinline__ float wload<__nv_bfloat16>(const __nv_bfloat16 *p) {
  return __bfloat162float(*p);
}

// w[l][e] = tanh(u_l . feat_e + c_l) for all layers
template <class W>
__global__ void gnn_edge_weights_kernel(GnnGraph g, const W *__restrict__ theta, float *__restrict__ w) {
  pdl_entry();
  const GnnOffsets o = GnnOffsets::make();
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.nedges; e += gridDim.x * blockDim.x) {
    float f[9];
#pragma unroll
    for (int k = 0; k < 9; k++) f[k] = g.feat[9 * size_t(e) + k];
#pragma unroll
    for (int l = 0; l < kGnnLayers; l++) {
      float a = wload(theta + o.c[l]);
#pragma unroll
      for (int k = 0; k < 9; k++) a += wload(theta + o.u[l] + k) * f[k];
      w[size_t(l) * g.nedges + e] = tanhf(a);
    }
  }
}

// gamma = sqrt(mean(zs^2)) from zs.zs kept in *zz (double), into *gamma (float)
__global__ void gnn_gamma_kernel(const double *zz, int n3, float *gamma) {
  pdl_entry();
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const double g2 = *zz / double(n3);
    *gamma = g2 > 0.0 ? float(sqrt(g2)) : 1.0f;
  }
}

// h0_i = W_in [zs_i/gamma, s_i^2 r_i/gamma]   (thread per node)
template <class R, class W>
__global__ void gnn_encode_kernel(GnnGraph g, const W *__restrict__ theta, const R *__restrict__ zs,
                                  const R *__restrict__ r, const float *__restrict__ gamma, float *__restrict__ x_out,
                                  float *__restrict__ h0, const CgState *st) {
  pdl_entry();
  if (st && (st->done || !st->use_gnn)) return;
  const GnnOffsets o = GnnOffsets::make();
  __shared__ float Win[kGnnWidth * 6];
  for (int k = threadIdx.x; k < kGnnWidth * 6; k += blockDim.x) Win[k] = wload(theta + o.W_in + k);
  __syncthreads();
  const float ig = 1.0f / *gamma;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
    const float s2 = g.s[i] * g.s[i];
    float x[6];
    for (int d = 0; d < 3; d++) {
      x[d] = float(zs[3 * i + d]) * ig;
      x[3 + d] = s2 * float(r[3 * i + d]) * ig;
    }
    if (x_out)
      for (int d = 0; d < 6; d++) x_out[6 * size_t(i) + d] = x[d];
    for (int c = 0; c < kGnnWidth; c++) {
      float a = 0.0f;
#pragma unroll
      for (int d = 0; d < 6; d++) a += Win[6 * c + d] * x[d];
      h0[size_t(i) * kGnnWidth + c] = a;
    }
  }
}

// One message-passing layer (warp per node, lane = channel).  The weights sit
// transposed in shared memory (WsT[k][j] = Ws[j][k]), so lane j's reads of column k
// fall in distinct banks.  The node's edges are taken 32 at a time: lane e loads
// edge e's column and weight, then every lane receives them by shuffles, so only
// the h gathers (128 contiguous bytes per edge) touch memory; the sum over the
// edges keeps their order.
template <class W>
__global__ void __launch_bounds__(kThreads) gnn_layer_kernel(GnnGraph g, const W *__restrict__ theta, int l,
                                                             const float *__restrict__ w,
                                                             const float *__restrict__ h_prev,
                                                             float *__restrict__ m_out, float *__restrict__ h_new,
                                                             const CgState *st) {
  pdl_entry();
  if (st && (st->done || !st->use_gnn)) return;
  const GnnOffsets o = GnnOffsets::make();
  __shared__ float WsT[kGnnWidth * kGnnWidth], WmT[kGnnWidth * kGnnWidth];
  for (int k = threadIdx.x; k < kGnnWidth * kGnnWidth; k += blockDim.x) {
    const int j = k / kGnnWidth, c = k % kGnnWidth;
    WsT[c * kGnnWidth + j] = wload(theta + o.Ws[l] + k);
    WmT[c * kGnnWidth + j] = wload(theta + o.Wm[l] + k);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const float *wl = w + size_t(l) * g.nedges;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < g.n; i += nwarps) {
    float m = 0.0f;
    const int e1 = g.ptr[i + 1];
    for (int e0 = g.ptr[i]; e0 < e1; e0 += 32) {
      const int ne = min(32, e1 - e0);
      int myc = 0;
      float myw = 0.0f;
      if (lane < ne) {
        myc = g.col[e0 + lane];
        myw = wl[e0 + lane];
      }
#pragma unroll 8
      for (int k = 0; k < ne; k++) {
        const int c = __shfl_sync(0xffffffffu, myc, k);
        const float wk = __shfl_sync(0xffffffffu, myw, k);
        m += wk * h_prev[size_t(c) * kGnnWidth + lane];
      }
    }
    const float hs = h_prev[size_t(i) * kGnnWidth + lane];
    float a = 0.0f;
#pragma unroll
    for (int k = 0; k < kGnnWidth; k++) {
      const float hk = __shfl_sync(0xffffffffu, hs, k);
      const float mk = __shfl_sync(0xffffffffu, m, k);
      a += WsT[k * kGnnWidth + lane] * hk + WmT[k * kGnnWidth + lane] * mk;
    }
    if (m_out) m_out[size_t(i) * kGnnWidth + lane] = m;
    h_new[size_t(i) * kGnnWidth + lane] = tanhf(a);
  }
}

// z_i = zs_i + gamma W_out h3_i  (thread per node); z = zs once the network is off
template <class R, class W>
__global__ void gnn_decode_kernel(int n, const W *__restrict__ theta, const float *__restrict__ h3,
                                  const R *__restrict__ zs, const float *__restrict__ gamma, R *__restrict__ z,
                                  const CgState *st) {
  pdl_entry();
  if (st && st->done) return;
  if (st && !st->use_gnn) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n; i += gridDim.x * blockDim.x) z[i] = zs[i];
    return;
  }
  const GnnOffsets o = GnnOffsets::make();
  __shared__ float Wo[3 * kGnnWidth];
  for (int k = threadIdx.x; k < 3 * kGnnWidth; k += blockDim.x) Wo[k] = wload(theta + o.W_out + k);
  __syncthreads();
  const float gm = *gamma;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float a[3] = {0.0f, 0.0f, 0.0f};
    for (int c = 0; c < kGnnWidth; c++) {
      const float h = h3[size_t(i) * kGnnWidth + c];
      a[0] += Wo[c] * h;
      a[1] += Wo[kGnnWidth + c] * h;
      a[2] += Wo[2 * kGnnWidth + c] * h;
    }
    for (int d = 0; d < 3; d++) z[3 * i + d] = zs[3 * i + d] + R(gm * a[d]);
  }
}

// ---- the network as the coarse-space generator (learned two-level) ----------
// Input: six static features per node (h33_coarse.cuh coarse_features_kernel);
// output: omega = sigmoid(W_out h3) per DOF, the smoothing weights of the prolongator.

// h0_i = W_in x_i   (thread per node; x precomputed, n x 6)
template <class W>
__global__ void gnn_encode_static_kernel(int n, const W *__restrict__ theta, const float *__restrict__ x,
                                         float *__restrict__ h0) {
  pdl_entry();
  const GnnOffsets o = GnnOffsets::make();
  __shared__ float Win[kGnnWidth * 6];
  for (int k = threadIdx.x; k < kGnnWidth * 6; k += blockDim.x) Win[k] = wload(theta + o.W_in + k);
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float xi[6];
    for (int d = 0; d < 6; d++) xi[d] = x[6 * size_t(i) + d];
    for (int c = 0; c < kGnnWidth; c++) {
      float a = 0.0f;
#pragma unroll
      for (int d = 0; d < 6; d++) a += Win[6 * c + d] * xi[d];
      h0[size_t(i) * kGnnWidth + c] = a;
    }
  }
}

// out_i = W_out h3_i, omega_i = 1 / (1 + exp(-out_i))   (thread per node, 3 each)
template <class W>
__global__ void gnn_omega_kernel(int n, const W *__restrict__ theta, const float *__restrict__ h3,
                                 float *__restrict__ out, float *__restrict__ omega) {
  pdl_entry();
  const GnnOffsets o = GnnOffsets::make();
  __shared__ float Wo[3 * kGnnWidth];
  for (int k = threadIdx.x; k < 3 * kGnnWidth; k += blockDim.x) Wo[k] = wload(theta + o.W_out + k);
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float a[3] = {0.0f, 0.0f, 0.0f};
    for (int c = 0; c < kGnnWidth; c++) {
      const float h = h3[size_t(i) * kGnnWidth + c];
      a[0] += Wo[c] * h;
      a[1] += Wo[kGnnWidth + c] * h;
      a[2] += Wo[2 * kGnnWidth + c] * h;
    }
    for (int d = 0; d < 3; d++) {
      if (out) out[3 * i + d] = a[d];
      omega[3 * i + d] = 1.0f / (1.0f + expf(-a[d]));
    }
  }
}

// ---- backward (training, FP32) ----------------------------------------------
// Per-CTA partial gradients are written to partials[blockIdx.x * stride + k] and
// summed by gnn_reduce_grads_kernel in a fixed order.

// dh3_i = gamma W_out^T dz_i;  dW_out partial = gamma sum_i dz_i h3_i^T (3 x 32)
__global__ void __launch_bounds__(kThreads) gnn_decode_bwd_kernel(int n, const float *__restrict__ theta,
                                                                  const float *__restrict__ h3,
                                                                  const float *__restrict__ dz,
                                                                  const float *__restrict__ gamma,
                                                                  float *__restrict__ dh3, float *__restrict__ part,
                                                                  int stride) {
  pdl_entry();
  const GnnOffsets o = GnnOffsets::make();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const float gm = *gamma;
  const float wo0 = theta[o.W_out + lane], wo1 = theta[o.W_out + kGnnWidth + lane],
              wo2 = theta[o.W_out + 2 * kGnnWidth + lane];
  float acc0 = 0.0f, acc1 = 0.0f, acc2 = 0.0f;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
    const float d0 = dz[3 * i], d1 = dz[3 * i + 1], d2 = dz[3 * i + 2];
    const float h = h3[size_t(i) * kGnnWidth + lane];
    dh3[size_t(i) * kGnnWidth + lane] = gm * (wo0 * d0 + wo1 * d1 + wo2 * d2);
    acc0 += gm * d0 * h;
    acc1 += gm * d1 * h;
    acc2 += gm * d2 * h;
  }
  __shared__ float sh[kWarpsPerCta][3 * kGnnWidth];
  sh[warp][lane] = acc0;
  sh[warp][kGnnWidth + lane] = acc1;
  sh[warp][2 * kGnnWidth + lane] = acc2;
  __syncthreads();
  for (int k = threadIdx.x; k < 3 * kGnnWidth; k += blockDim.x) {
    float s = 0.0f;
    for (int q = 0; q < kWarpsPerCta; q++) s += sh[q][k];
    part[size_t(blockIdx.x) * stride + o.W_out + k] = s;
  }
}

// Layer l backward, node part (warp per node i, lane = channel):
//   delta_i = dh_i * (1 - h_l,i^2); gm_i = Wm^T delta_i; self_i = Ws^T delta_i
//   dWs += delta_i h_{l-1,i}^T, dWm += delta_i m_i^T
//   for each edge (i,j): dw_ij = gm_i . h_{l-1,j};  du_l += dw (1-w^2) e_ij, dc_l += dw (1-w^2)
// writes gm (n x 32) and self (into dh_prev, n x 32)
__global__ void __launch_bounds__(kThreads) gnn_layer_bwd_kernel(GnnGraph g, const float *__restrict__ theta, int l,
                                                                 const float *__restrict__ w,
                                                                 const float *__restrict__ h_prev,
                                                                 const float *__restrict__ h_new,
                                                                 const float *__restrict__ m,
                                                                 const float *__restrict__ dh,
                                                                 float *__restrict__ gm_out,
                                                                 float *__restrict__ dh_prev,
                                                                 float *__restrict__ part, int stride) {
  pdl_entry();
  const GnnOffsets o = GnnOffsets::make();
  __shared__ float Ws[kGnnWidth * kGnnWidth], Wm[kGnnWidth * kGnnWidth];
  for (int k = threadIdx.x; k < kGnnWidth * kGnnWidth; k += blockDim.x) {
    Ws[k] = theta[o.Ws[l] + k];
    Wm[k] = theta[o.Wm[l] + k];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const float *wl = w + size_t(l) * g.nedges;
  float dWs[kGnnWidth], dWm[kGnnWidth];  // row `lane` of the gradients
#pragma unroll
  for (int k = 0; k < kGnnWidth; k++) dWs[k] = dWm[k] = 0.0f;
  float du = 0.0f;  // lane k < 9: d/du_l[k]; lane 9: d/dc_l
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < g.n; i += nwarps) {
    const float hn = h_new[size_t(i) * kGnnWidth + lane];
    const float delta = dh[size_t(i) * kGnnWidth + lane] * (1.0f - hn * hn);
    const float hp = h_prev[size_t(i) * kGnnWidth + lane];
    const float mi = m[size_t(i) * kGnnWidth + lane];
    float gmi = 0.0f, self = 0.0f;
#pragma unroll
    for (int k = 0; k < kGnnWidth; k++) {
      const float dk = __shfl_sync(0xffffffffu, delta, k);
      // (Wm^T delta)_lane = sum_k Wm[k][lane] delta_k
      gmi += Wm[k * kGnnWidth + lane] * dk;
      self += Ws[k * kGnnWidth + lane] * dk;
      const float hpk = __shfl_sync(0xffffffffu, hp, k);
      const float mk = __shfl_sync(0xffffffffu, mi, k);
      dWs[k] += delta * hpk;
      dWm[k] += delta * mk;
    }
    gm_out[size_t(i) * kGnnWidth + lane] = gmi;
    dh_prev[size_t(i) * kGnnWidth + lane] = self;
    for (int e = g.ptr[i]; e < g.ptr[i + 1]; e++) {
      float dw = gmi * h_prev[size_t(g.col[e]) * kGnnWidth + lane];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) dw += __shfl_xor_sync(0xffffffffu, dw, off);
      const float we = wl[e];
      const float dpre = dw * (1.0f - we * we);
      if (lane < 9) du += dpre * g.feat[9 * size_t(e) + lane];
      else if (lane == 9) du += dpre;
    }
  }
  // per-CTA sums: dWs / dWm rows via shared memory, du via shared memory
  __shared__ float sh[kWarpsPerCta][kGnnWidth];
  for (int pass = 0; pass < 2; pass++) {
    for (int k = 0; k < kGnnWidth; k++) {
      sh[warp][lane] = pass == 0 ? dWs[k] : dWm[k];
      __syncthreads();
      if (warp == 0) {
        float s = 0.0f;
        for (int q = 0; q < kWarpsPerCta; q++) s += sh[q][lane];
        // element [lane][k] of the gradient matrix
        part[size_t(blockIdx.x) * stride + (pass == 0 ? o.Ws[l] : o.Wm[l]) + lane * kGnnWidth + k] = s;
      }
      __syncthreads();
    }
  }
  {
    sh[warp][lane] = du;
    __syncthreads();
    if (warp == 0 && lane < 10) {
      float s = 0.0f;
      for (int q = 0; q < kWarpsPerCta; q++) s += sh[q][lane];
      part[size_t(blockIdx.x) * stride + (lane < 9 ? o.u[l] + lane : o.c[l])] = s;
    }
  }
}

// Layer l backward, transpose aggregation: dh_prev_j += sum_{i in N(j)} w_ij gm_i,
// with w_ij the weight of edge (i, j) = w[rev[(j, i)]]  (warp per node j).
__global__ void __launch_bounds__(kThreads) gnn_layer_bwd_gather_kernel(GnnGraph g, int l, const float *__restrict__ w,
                                                                        const float *__restrict__ gm,
                                                                        float *__restrict__ dh_prev) {
  pdl_entry();
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const float *wl = w + size_t(l) * g.nedges;
  for (int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < g.n; j += nwarps) {
    float a = dh_prev[size_t(j) * kGnnWidth + lane];
    for (int e = g.ptr[j]; e < g.ptr[j + 1]; e++) a += wl[g.rev[e]] * gm[size_t(g.col[e]) * kGnnWidth + lane];
    dh_prev[size_t(j) * kGnnWidth + lane] = a;
  }
}

// dW_in partial = sum_i dh0_i x_i^T (32 x 6)   (warp per node, lane = channel)
__global__ void __launch_bounds__(kThreads) gnn_encode_bwd_kernel(int n, const float *__restrict__ x,
                                                                  const float *__restrict__ dh0,
                                                                  float *__restrict__ part, int stride) {
  pdl_entry();
  const GnnOffsets o = GnnOffsets::make();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  float acc[6] = {0, 0, 0, 0, 0, 0};
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
    const float d = dh0[size_t(i) * kGnnWidth + lane];
#pragma unroll
    for (int k = 0; k < 6; k++) acc[k] += d * x[6 * size_t(i) + k];
  }
  __shared__ float sh[kWarpsPerCta][kGnnWidth * 6];
  for (int k = 0; k < 6; k++) sh[warp][lane * 6 + k] = acc[k];
  __syncthreads();
  for (int k = threadIdx.x; k < kGnnWidth * 6; k += blockDim.x) {
    float s = 0.0f;
    for (int q = 0; q < kWarpsPerCta; q++) s += sh[q][k];
    part[size_t(blockIdx.x) * stride + o.W_in + k] = s;
  }
}

// grad[k] = sum over CTAs of part[cta * stride + k]  (fixed order; thread per k)
__global__ void gnn_reduce_grads_kernel(const float *__restrict__ part, int nparts, int stride,
                                        float *__restrict__ grad, int nparam) {
  pdl_entry();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nparam; k += gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int q = 0; q < nparts; q++) s += part[size_t(q) * stride + k];
    grad[k] = s;
  }
}

// Adam step on the FP32 master weights; also refreshes the BF16 copy.
__global__ void gnn_adam_kernel(float *__restrict__ theta, const float *__restrict__ grad,
                                float *__restrict__ m1, float *__restrict__ m2, int nparam, float lr,
                                float b1, float b2, float eps, int step, float gscale,
                                __nv_bfloat16 *__restrict__ theta_bf16) {
  pdl_entry();
  const float c1 = 1.0f - powf(b1, float(step)), c2 = 1.0f - powf(b2, float(step));
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nparam; k += gridDim.x * blockDim.x) {
    const float gk = grad[k] * gscale;
    const float a = b1 * m1[k] + (1.0f - b1) * gk;
    const float b = b2 * m2[k] + (1.0f - b2) * gk * gk;
    m1[k] = a;
    m2[k] = b;
    theta[k] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
    if (theta_bf16) theta_bf16[k] = __float2bfloat16(theta[k]);
  }
}

// s_i = (trace(D_i)/3)^(-1/2) from the raw diagonal blocks (first n blocks of raw)
__global__ void gnn_node_scale_kernel(const double *__restrict__ raw, int n, float *__restrict__ s) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double t = (raw[9 * size_t(i)] + raw[9 * size_t(i) + 4] + raw[9 * size_t(i) + 8]) / 3.0;
    s[i] = t > 0.0 ? float(1.0 / sqrt(t)) : 1.0f;
  }
}

// feat_e = s_i A_ij s_j for edge e = (i, j), A_ij the raw block src[e] (thread per
// entry, so that the writes are contiguous)
__global__ void gnn_edge_feat_kernel(GnnGraph g, const int *__restrict__ row_of, const int *__restrict__ src,
                                     const double *__restrict__ raw, float *__restrict__ feat) {
  pdl_entry();
  const size_t total = size_t(9) * size_t(g.nedges);
  for (size_t x = size_t(blockIdx.x) * blockDim.x + threadIdx.x; x < total; x += size_t(gridDim.x) * blockDim.x) {
    const int e = int(x / 9), k = int(x % 9);
    const double f = double(g.s[row_of[e]]) * double(g.s[g.col[e]]);
    feat[x] = float(raw[9 * size_t(src[e]) + k] * f);
  }
}

// out = float(a - b)
__global__ void diff_narrow_kernel(const double *__restrict__ a, const double *__restrict__ b,
                                   float *__restrict__ out, int n) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = float(a[i] - b[i]);
}

// d = z - e
__global__ void sub_kernel(const float *__restrict__ z, const float *__restrict__ e, float *__restrict__ d, int n) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = z[i] - e[i];
}

// dz = c * q with c = 2 / (e.r)
__global__ void scale_kernel(const float *__restrict__ q, float c, float *__restrict__ dz, int n) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dz[i] = c * q[i];
}

// acc += g * c
__global__ void accum_kernel(const float *__restrict__ g, float c, float *__restrict__ acc, int n) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc[i] += c * g[i];
}

// state for a network application outside a solve (training, evaluation)
__global__ void gnn_state_kernel(CgState *st) {
  pdl_entry();
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    st->done = 0;
    st->use_gnn = 1;
    for (int i = 0; i < 8; i++) st->ticket[i] = 0u;
  }
}

}  // namespace h33
