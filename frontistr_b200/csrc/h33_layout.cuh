// h33_layout.cuh -- device fill of the sliced block-ELL layouts whose shape (slices,
// slot counts, run tables) the host computed from the rows' block counts
// (sell_shape): every block of every row is placed from the hecmwST profile resident
// on the device, so the O(blocks) work of the layouts never runs on the host.  The
// results are the host builders' (unified_rows / reordered_rows + permute_rows +
// build_sell in h33_setup.cpp) entry for entry.
#pragma once

#include <climits>
#include <cstdint>

#include "h33_common.cuh"

namespace h33 {

// hecmwST profile on the device (indexX[0..N], itemX 1-based ids).
struct DevProfile {
  int N, NPL;
  const int *indexL, *itemL, *indexU, *itemU;
};

// Block k of the row at offset r of a slice whose first slot is s0: slot s0 + k / lanes,
// lane r * lanes + k % lanes.
__device__ __forceinline__ size_t sell_at(int s0, int r, int k, int lanes) {
  return (size_t(s0) + size_t(k / lanes)) * 32 + size_t(r) * lanes + size_t(k % lanes);
}

// The unified rows (the row's L blocks, its diagonal, its U blocks, as stored) of
// rows 0..N-1 taken as one group: row i is offset i % (32 / lanes) of slice
// i / (32 / lanes).  A thread per row.
__global__ void fill_unified_kernel(DevProfile p, int lanes, const int *__restrict__ slot0, int *__restrict__ col,
                                    int *__restrict__ src) {
  pdl_entry();
  const int per_slice = 32 / lanes;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.N; i += gridDim.x * blockDim.x) {
    const int s0 = slot0[i / per_slice], r = i % per_slice;
    int k = 0;
    for (int j = p.indexL[i]; j < p.indexL[i + 1]; j++, k++) {
      const size_t at = sell_at(s0, r, k, lanes);
      col[at] = p.itemL[j] - 1;
      src[at] = p.N + j;
    }
    {
      const size_t at = sell_at(s0, r, k++, lanes);
      col[at] = i;
      src[at] = i;
    }
    for (int j = p.indexU[i]; j < p.indexU[i + 1]; j++, k++) {
      const size_t at = sell_at(s0, r, k, lanes);
      col[at] = p.itemU[j] - 1;
      src[at] = p.N + p.NPL + j;
    }
  }
}

// Blocks of old row iold below (nl) and above (nu) it in the new order iperm; external
// columns (ids above N, rows of a decomposed domain) are not counted.  Indexed by the
// new row.  A thread per row.
__global__ void count_parts_kernel(DevProfile p, const int *__restrict__ iperm, int *__restrict__ nl,
                                   int *__restrict__ nu) {
  pdl_entry();
  for (int iold = blockIdx.x * blockDim.x + threadIdx.x; iold < p.N; iold += gridDim.x * blockDim.x) {
    const int inew = iperm[iold];
    int a = 0, b = 0;
    for (int j = p.indexL[iold]; j < p.indexL[iold + 1]; j++) (iperm[p.itemL[j] - 1] < inew ? a : b)++;
    for (int j = p.indexU[iold]; j < p.indexU[iold + 1]; j++) {
      if (p.itemU[j] > p.N) continue;
      (iperm[p.itemU[j] - 1] < inew ? a : b)++;
    }
    nl[inew] = a;
    nu[inew] = b;
  }
}

// Entry e of old row iold's stored blocks (L then U): its new column (INT_MAX for an
// external column) and raw block id.
__device__ __forceinline__ void row_entry(const DevProfile &p, const int *iperm, int l0, int nL, int u0, int e,
                                          int *jnew, int *raw) {
  const int item = e < nL ? p.itemL[l0 + e] : p.itemU[u0 + e - nL];
  *raw = e < nL ? p.N + l0 + e : p.N + p.NPL + u0 + e - nL;
  *jnew = item <= p.N ? iperm[item - 1] : INT_MAX;
}

// The lower (LOWER) or upper part of the SSOR layouts: layout row q is row order[q] of
// the new order, old row perm[order[q]]; its blocks with a new column below (lower)
// or above (upper) the row's, ascending in the new column, columns renamed to layout
// rows (iorder of the new column), values by raw block id.  A warp per row: each lane
// takes blocks of the row and finds its place among the part's blocks by counting
// those with a smaller new column (new columns are distinct within a row).
template <bool LOWER>
__global__ void fill_reordered_kernel(DevProfile p, const int *__restrict__ perm, const int *__restrict__ iperm,
                                      const int *__restrict__ order, const int *__restrict__ iorder,
                                      const int *__restrict__ row_slice, const int *__restrict__ row0,
                                      const int *__restrict__ slot0, int lanes, int *__restrict__ col,
                                      int *__restrict__ src) {
  pdl_entry();
  const int lane = threadIdx.x & 31;
  const int nwarps = int((size_t(gridDim.x) * blockDim.x) >> 5);
  for (int q = int((size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5); q < p.N; q += nwarps) {
    const int inew = order[q], iold = perm[inew];
    const int s = row_slice[q], r = q - row0[s], s0 = slot0[s];
    const int l0 = p.indexL[iold], nL = p.indexL[iold + 1] - l0;
    const int u0 = p.indexU[iold], nU = p.indexU[iold + 1] - u0;
    const int n = nL + nU;
    for (int e0 = 0; e0 < n; e0 += 32) {
      const int e = e0 + lane;
      int jnew = INT_MAX, raw = -1;
      if (e < n) row_entry(p, iperm, l0, nL, u0, e, &jnew, &raw);
      const bool mine = jnew != INT_MAX && (LOWER ? jnew < inew : jnew > inew);
      int rank = 0;
      for (int f0 = 0; f0 < n; f0 += 32) {
        const int f = f0 + lane;
        int jf = INT_MAX, rf;
        if (f < n) row_entry(p, iperm, l0, nL, u0, f, &jf, &rf);
        const bool in_part = jf != INT_MAX && (LOWER ? jf < inew : jf > inew);
        const int key = in_part ? jf : INT_MAX;
        for (int t = 0; t < 32; t++) rank += __shfl_sync(0xffffffffu, key, t) < jnew ? 1 : 0;
      }
      if (mine) {
        const size_t at = sell_at(s0, r, rank, lanes);
        col[at] = iorder[jnew];
        src[at] = raw;
      }
    }
  }
}

// The block ILU layouts (level order): layout row q holds row ord[q]'s L blocks (UPPER
// false) or U blocks (UPPER true) as stored, columns as 0-based node ids, values by raw
// block id.  A thread per row.
template <bool UPPER>
__global__ void fill_ordered_kernel(DevProfile p, const int *__restrict__ ord, const int *__restrict__ row_slice,
                                    const int *__restrict__ row0, const int *__restrict__ slot0, int lanes,
                                    int *__restrict__ col, int *__restrict__ src) {
  pdl_entry();
  const int *index = UPPER ? p.indexU : p.indexL, *item = UPPER ? p.itemU : p.itemL;
  const int base = UPPER ? p.N + p.NPL : p.N;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < p.N; q += gridDim.x * blockDim.x) {
    const int i = ord[q], s = row_slice[q], r = q - row0[s], s0 = slot0[s];
    int k = 0;
    for (int j = index[i]; j < index[i + 1]; j++, k++) {
      const size_t at = sell_at(s0, r, k, lanes);
      col[at] = item[j] - 1;
      src[at] = base + j;
    }
  }
}

// The unified rows as CSR (ptr from the host's block counts): row i's L blocks, its
// diagonal, its U blocks as stored; col 0-based, src the raw block id.  A thread per row.
__global__ void fill_unified_csr_kernel(DevProfile p, const int *__restrict__ ptr, int *__restrict__ col,
                                        int *__restrict__ src) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.N; i += gridDim.x * blockDim.x) {
    int w = ptr[i];
    for (int j = p.indexL[i]; j < p.indexL[i + 1]; j++, w++) {
      col[w] = p.itemL[j] - 1;
      src[w] = p.N + j;
    }
    col[w] = i;
    src[w++] = i;
    for (int j = p.indexU[i]; j < p.indexU[i + 1]; j++, w++) {
      col[w] = p.itemU[j] - 1;
      src[w] = p.N + p.NPL + j;
    }
  }
}

// The matrix graph without its diagonal: edge ptr[i] + k of row i is its k-th stored
// off-diagonal block (L blocks, then U blocks: ascending columns), with the block's raw
// id and the edge's row.  A thread per row.
__global__ void fill_edges_kernel(DevProfile p, const int *__restrict__ ptr, int *__restrict__ col,
                                  int *__restrict__ src, int *__restrict__ row_of) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.N; i += gridDim.x * blockDim.x) {
    int w = ptr[i];
    for (int j = p.indexL[i]; j < p.indexL[i + 1]; j++, w++) {
      col[w] = p.itemL[j] - 1;
      src[w] = p.N + j;
      row_of[w] = i;
    }
    for (int j = p.indexU[i]; j < p.indexU[i + 1]; j++, w++) {
      col[w] = p.itemU[j] - 1;
      src[w] = p.N + p.NPL + j;
      row_of[w] = i;
    }
  }
}

// rev[e] for edge e = (i, j): the edge (j, i), found by bisection in row j's ascending
// columns; e itself when row j has none (an unsymmetric profile) or is not one of the
// n rows.  A thread per edge.
__global__ void edge_reverse_kernel(int n, const int *__restrict__ ptr, const int *__restrict__ col,
                                    const int *__restrict__ row_of, int ne, int *__restrict__ rev) {
  pdl_entry();
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += gridDim.x * blockDim.x) {
    const int i = row_of[e], j = col[e];
    if (j < 0 || j >= n) {
      rev[e] = e;
      continue;
    }
    int lo = ptr[j], hi = ptr[j + 1];  // first position in [lo, hi) with col >= i
    while (lo < hi) {
      const int mid = lo + ((hi - lo) >> 1);
      if (col[mid] < i) lo = mid + 1;
      else hi = mid;
    }
    rev[e] = (lo < ptr[j + 1] && col[lo] == i) ? lo : e;
  }
}

}  // namespace h33
