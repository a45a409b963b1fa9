// h33_assemble.cuh -- HEX8 linear-elastic assembly on the device.
//
//   element matrix   fistr1/src/lib/static_LIB_3d.f90:50-208 (STF_C3, INFINITESIMAL,
//                    FORM361=FI: full 2x2x2 Gauss), hex8n.f90 shape functions,
//                    isotropic D of fistr1/src/lib/physics/ElasticLinear.f90:38-60
//   scatter          hecmw1/src/solver/matrix/hecmw_mat_ass.f90:32-135 (hecmw_mat_ass_elem,
//                    elements in order, 3x3 blocks added into D/AL/AU)
//   boundary cond.   hecmw1/src/solver/matrix/hecmw_mat_ass.f90:328-463 (hecmw_mat_ass_bc)
//
// Element kernel: one thread per (element, node a, node b) computes the 3x3 block
// K_ab = sum over the 8 Gauss points of B_a^T D B_b det J, every product and sum in
// the order of the host restatement (assemble.cpp: elastic_matrix, global_deriv,
// add_btdb), with explicitly rounded operations so that no multiply-add is fused:
// the blocks are bitwise those of the host.  Gather kernel: one thread per matrix
// block sums its element contributions in element order (a per-block list built on
// the host), which is the order of a serial hecmw_mat_ass_elem loop.
#pragma once

#include "h33_common.cuh"

namespace h33 {

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }

// Ke[e][a][b][9]: the 64 blocks of element e (576 doubles, row-major 3x3 per block).
static __global__ void __launch_bounds__(256) hex8_element_kernel(const double *__restrict__ coords,
                                                                 const int *__restrict__ conn, int n_elem,
                                                                 const double *__restrict__ E,
                                                                 const double *__restrict__ nu,
                                                                 double *__restrict__ Ke) {
  pdl_entry();
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= int64_t(n_elem) * 64) return;
  const int e = int(t >> 6), a = int(t & 63) >> 3, b = int(t & 7);
  // nodal coordinates (connectivity 1-based, hex8n order)
  double x[8][3];
#pragma unroll
  for (int n = 0; n < 8; n++) {
    const int node = conn[8 * size_t(e) + n] - 1;
#pragma unroll
    for (int d = 0; d < 3; d++) x[n][d] = coords[3 * size_t(node) + d];
  }
  // isotropic D (ElasticLinear.f90:38-60): bulk and shear form
  const double Ee = E[e], ne = nu[e];
  const double Kb = (Ee / sub_rn(1.0, mul_rn(2.0, ne))) / 3.0;
  const double G = mul_rn(Ee / add_rn(1.0, ne), 0.5);
  const double d00 = add_rn(Kb, mul_rn(4.0 / 3.0, G)), d01 = sub_rn(Kb, mul_rn(2.0 / 3.0, G));
  const double D3[3][3] = {{d00, d01, d01}, {d01, d00, d01}, {d01, d01, d00}};
  const double sgn[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                            {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  const double g = 1.0 / sqrt(3.0);
  const double gp[2] = {-g, g};
  double K[3][3] = {};
  for (int lz = 0; lz < 2; lz++)
    for (int ly = 0; ly < 2; ly++)
      for (int lx = 0; lx < 2; lx++) {
        const double xi[3] = {gp[lx], gp[ly], gp[lz]};
        double deriv[8][3];
#pragma unroll
        for (int n = 0; n < 8; n++) {
          const double f0 = add_rn(1.0, mul_rn(sgn[n][0], xi[0]));
          const double f1 = add_rn(1.0, mul_rn(sgn[n][1], xi[1]));
          const double f2 = add_rn(1.0, mul_rn(sgn[n][2], xi[2]));
          deriv[n][0] = mul_rn(mul_rn(mul_rn(0.125, sgn[n][0]), f1), f2);
          deriv[n][1] = mul_rn(mul_rn(mul_rn(0.125, sgn[n][1]), f0), f2);
          deriv[n][2] = mul_rn(mul_rn(mul_rn(0.125, sgn[n][2]), f0), f1);
        }
        // Jacobian, its determinant and inverse (assemble.cpp global_deriv)
        double XJ[3][3] = {};
#pragma unroll
        for (int n = 0; n < 8; n++)
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) XJ[i][j] = add_rn(XJ[i][j], mul_rn(x[n][i], deriv[n][j]));
        double det = mul_rn(mul_rn(XJ[0][0], XJ[1][1]), XJ[2][2]);
        det = add_rn(det, mul_rn(mul_rn(XJ[1][0], XJ[2][1]), XJ[0][2]));
        det = add_rn(det, mul_rn(mul_rn(XJ[2][0], XJ[0][1]), XJ[1][2]));
        det = sub_rn(det, mul_rn(mul_rn(XJ[2][0], XJ[1][1]), XJ[0][2]));
        det = sub_rn(det, mul_rn(mul_rn(XJ[1][0], XJ[0][1]), XJ[2][2]));
        det = sub_rn(det, mul_rn(mul_rn(XJ[0][0], XJ[2][1]), XJ[1][2]));
        const double dinv = 1.0 / det;
        double XJI[3][3];
        XJI[0][0] = mul_rn(dinv, sub_rn(mul_rn(XJ[1][1], XJ[2][2]), mul_rn(XJ[2][1], XJ[1][2])));
        XJI[0][1] = mul_rn(dinv, add_rn(mul_rn(-XJ[0][1], XJ[2][2]), mul_rn(XJ[2][1], XJ[0][2])));
        XJI[0][2] = mul_rn(dinv, sub_rn(mul_rn(XJ[0][1], XJ[1][2]), mul_rn(XJ[1][1], XJ[0][2])));
        XJI[1][0] = mul_rn(dinv, add_rn(mul_rn(-XJ[1][0], XJ[2][2]), mul_rn(XJ[2][0], XJ[1][2])));
        XJI[1][1] = mul_rn(dinv, sub_rn(mul_rn(XJ[0][0], XJ[2][2]), mul_rn(XJ[2][0], XJ[0][2])));
        XJI[1][2] = mul_rn(dinv, add_rn(mul_rn(-XJ[0][0], XJ[1][2]), mul_rn(XJ[1][0], XJ[0][2])));
        XJI[2][0] = mul_rn(dinv, sub_rn(mul_rn(XJ[1][0], XJ[2][1]), mul_rn(XJ[2][0], XJ[1][1])));
        XJI[2][1] = mul_rn(dinv, add_rn(mul_rn(-XJ[0][0], XJ[2][1]), mul_rn(XJ[2][0], XJ[0][1])));
        XJI[2][2] = mul_rn(dinv, sub_rn(mul_rn(XJ[0][0], XJ[1][1]), mul_rn(XJ[1][0], XJ[0][1])));
        // global derivatives of nodes a and b
        double ga[3], gb[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
          double sa = 0.0, sb = 0.0;
#pragma unroll
          for (int j = 0; j < 3; j++) {
            sa = add_rn(sa, mul_rn(deriv[a][j], XJI[j][k]));
            sb = add_rn(sb, mul_rn(deriv[b][j], XJI[j][k]));
          }
          ga[k] = sa;
          gb[k] = sb;
        }
        // B^T D B for the (a, b) block: the nonzero entries of B's columns in Voigt
        // order (xx, yy, zz, xy, yz, zx).  Column of dof r of a node with global
        // derivatives g: rows {r, shear rows} with values below, ascending row.
        //   r=0: (0,g0) (3,g1) (5,g2);  r=1: (1,g1) (3,g0) (4,g2);  r=2: (2,g2) (4,g1) (5,g0)
        const int rows[3][3] = {{0, 3, 5}, {1, 3, 4}, {2, 4, 5}};
        const int comp[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 1, 0}};
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int c = 0; c < 3; c++) {
            // DB[k][j] for the column j = (b, c): k < 3 -> D[k][c] g_b,c; k >= 3 -> G B[k][j]
            double s = 0.0;
#pragma unroll
            for (int q = 0; q < 3; q++) {
              const int k = rows[r][q];
              const double bki = ga[comp[r][q]];
              double dbk;
              if (k < 3) {
                dbk = mul_rn(D3[k][c], gb[c]);
              } else {
                // B[k][j] of column (b, c): nonzero when c is one of the two strains of row k
                double bkj = 0.0;
#pragma unroll
                for (int q2 = 0; q2 < 3; q2++)
                  if (rows[c][q2] == k) bkj = gb[comp[c][q2]];
                dbk = mul_rn(G, bkj);
              }
              s = add_rn(s, mul_rn(bki, dbk));
            }
            K[r][c] = add_rn(K[r][c], mul_rn(s, det));
          }
      }
  double *out = Ke + 576 * size_t(e) + 9 * (8 * a + b);
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) out[3 * r + c] = K[r][c];
}

// raw[9 * blk + i] = sum of the element contributions of block blk in element order;
// contribution code = 64 e + 8 a + b (block (a, b) of element e).
static __global__ void __launch_bounds__(256) hex8_gather_kernel(const double *__restrict__ Ke,
                                                                const int64_t *__restrict__ ptr,
                                                                const int *__restrict__ code, int64_t nblocks,
                                                                double *__restrict__ raw) {
  pdl_entry();
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= 9 * nblocks) return;
  const int64_t blk = t / 9;
  const int i = int(t - 9 * blk);
  double s = 0.0;
  for (int64_t k = ptr[blk]; k < ptr[blk + 1]; k++) {
    const int c = code[k];
    s = add_rn(s, Ke[576 * size_t(c >> 6) + 9 * size_t(c & 63) + i]);
  }
  raw[t] = s;
}

// hecmw_mat_ass_bc, right-hand side part: every free row r (node n, dof q) receives
// -A(r, (m,d)) * value_k for each constrained dof (m, d) of a node m coupled to n,
// taken in the order k of the constraint list (the first occurrence of a dof counts;
// later ones see a zeroed column).  Rows of constrained dofs are set to their value
// (the last occurrence's, as the sequential assignments leave it).
// bc_first / bc_last[3 m + d] = first / last list index k constraining (m, d), -1 if free.
struct BcArgs {
  int n_node;
  const int *indexL, *itemL, *indexU, *itemU;  // device copies (1-based items)
  const int *bc_first, *bc_last;
  const double *bc_value;
};

static __global__ void __launch_bounds__(256) bc_rhs_kernel(BcArgs A, const double *__restrict__ raw, double *B) {
  pdl_entry();
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= 3 * A.n_node) return;
  const int n = row / 3, q = row - 3 * n;
  const int own = A.bc_last[row];
  if (own >= 0) {
    B[row] = A.bc_value[own];
    return;
  }
  // (k, contribution) pairs of this row, sorted by k by insertion (at most 81)
  int ks[81];
  double cs[81];
  int m = 0;
  const int NL = A.indexL[A.n_node];
  auto visit = [&](int node, const double *blk) {
    for (int d = 0; d < 3; d++) {
      const int k = A.bc_first[3 * node + d];
      if (k < 0 || m >= 81) continue;
      const double c = mul_rn(blk[3 * q + d], A.bc_value[k]);
      int p = m++;
      while (p > 0 && ks[p - 1] > k) {
        ks[p] = ks[p - 1];
        cs[p] = cs[p - 1];
        p--;
      }
      ks[p] = k;
      cs[p] = c;
    }
  };
  for (int j = A.indexL[n]; j < A.indexL[n + 1]; j++) visit(A.itemL[j] - 1, raw + 9 * (size_t(A.n_node) + j));
  visit(n, raw + 9 * size_t(n));
  for (int j = A.indexU[n]; j < A.indexU[n + 1]; j++)
    visit(A.itemU[j] - 1, raw + 9 * (size_t(A.n_node) + NL + j));
  double b = B[row];
  for (int p = 0; p < m; p++) b = sub_rn(b, cs[p]);
  B[row] = b;
}

// hecmw_mat_ass_bc, matrix part (after bc_rhs_kernel): for every constrained dof
// (n, d) its row and column are zeroed and the diagonal set to 1.  One thread per
// matrix block entry; all writes of one entry agree, so the order does not matter.
static __global__ void __launch_bounds__(256) bc_matrix_kernel(BcArgs A, const int *__restrict__ blk_row,
                                                              const int *__restrict__ blk_col, int64_t nblocks,
                                                              double *raw) {
  pdl_entry();
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= 9 * nblocks) return;
  const int64_t blk = t / 9;
  const int e = int(t - 9 * blk), r = e / 3, c = e - 3 * r;
  const int i = blk_row[blk], j = blk_col[blk];
  const bool row_fixed = A.bc_first[3 * i + r] >= 0, col_fixed = A.bc_first[3 * j + c] >= 0;
  if (!row_fixed && !col_fixed) return;
  raw[t] = (i == j && r == c) ? 1.0 : 0.0;
}

// Any zero diagonal entry of D (hecmw_solve_check_zerodiag, hecmw_solver_Iterative.f90:255-282).
static __global__ void zero_diag_kernel(const double *__restrict__ D, int n, int *flag) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int j = 0; j < 3; j++)
      if (fabs(D[9 * size_t(i) + 4 * j]) == 0.0) atomicOr(flag, 1);
}

}  // namespace h33
