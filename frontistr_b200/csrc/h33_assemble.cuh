// h33_assemble.cuh -- HEX8 assembly on the device: linear elastic and compressible
// Neo-Hookean (tangent and internal force).
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

// ---- compressible Neo-Hookean, total Lagrangian (assemble.cpp neohooke_hex8) ----
// W = C10 (J^-2/3 I1 - 3) + (J - 1)^2 / D1 (fistr1/src/lib/physics/Hyperelastic.f90:286-381).
// Operations in the host's order with rounded intrinsics; J^-2/3 is CUDA's pow, so the
// blocks agree with the host's to rounding rather than bitwise.

// S (Voigt 11 22 33 12 23 31) and D = 2 dS/dC at F; returns J.
__device__ __forceinline__ double nh_stress(const double F[3][3], double C10, double D1, double S[6],
                                            double D[6][6]) {
  const int Vi[6] = {0, 1, 2, 0, 1, 2}, Vj[6] = {0, 1, 2, 1, 2, 0};
  double C[3][3];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 3; k++) s = add_rn(s, mul_rn(F[k][i], F[k][j]));
      C[i][j] = s;
    }
  double J = mul_rn(F[0][0], sub_rn(mul_rn(F[1][1], F[2][2]), mul_rn(F[1][2], F[2][1])));
  J = sub_rn(J, mul_rn(F[0][1], sub_rn(mul_rn(F[1][0], F[2][2]), mul_rn(F[1][2], F[2][0]))));
  J = add_rn(J, mul_rn(F[0][2], sub_rn(mul_rn(F[1][0], F[2][1]), mul_rn(F[1][1], F[2][0]))));
  const double detC = mul_rn(J, J);
  double Ci[3][3];
  Ci[0][0] = sub_rn(mul_rn(C[1][1], C[2][2]), mul_rn(C[1][2], C[2][1])) / detC;
  Ci[0][1] = sub_rn(mul_rn(C[0][2], C[2][1]), mul_rn(C[0][1], C[2][2])) / detC;
  Ci[0][2] = sub_rn(mul_rn(C[0][1], C[1][2]), mul_rn(C[0][2], C[1][1])) / detC;
  Ci[1][0] = Ci[0][1];
  Ci[1][1] = sub_rn(mul_rn(C[0][0], C[2][2]), mul_rn(C[0][2], C[2][0])) / detC;
  Ci[1][2] = sub_rn(mul_rn(C[0][2], C[1][0]), mul_rn(C[0][0], C[1][2])) / detC;
  Ci[2][0] = Ci[0][2];
  Ci[2][1] = Ci[1][2];
  Ci[2][2] = sub_rn(mul_rn(C[0][0], C[1][1]), mul_rn(C[0][1], C[1][0])) / detC;
  const double I1 = add_rn(add_rn(C[0][0], C[1][1]), C[2][2]);
  const double j23 = pow(J, -2.0 / 3.0);
  const double a = mul_rn(2.0, C10);
  const double p = mul_rn(mul_rn(2.0 / D1, sub_rn(J, 1.0)), J);
  const double q = mul_rn(mul_rn(2.0 / D1, sub_rn(mul_rn(2.0, J), 1.0)), J);
  const double a23 = mul_rn(2.0, a) / 3.0, a29 = mul_rn(2.0, a) / 9.0;
#pragma unroll
  for (int v = 0; v < 6; v++) {
    const int I = Vi[v], Jv = Vj[v];
    const double dIJ = I == Jv ? 1.0 : 0.0;
    const double cij = Ci[I][Jv];
    S[v] = add_rn(mul_rn(mul_rn(a, j23), sub_rn(dIJ, mul_rn(I1 / 3.0, cij))), mul_rn(p, cij));
#pragma unroll
    for (int w = 0; w < 6; w++) {
      const int K = Vi[w], L = Vj[w];
      const double dKL = K == L ? 1.0 : 0.0;
      const double ckl = Ci[K][L];
      const double Ic = mul_rn(0.5, add_rn(mul_rn(Ci[I][K], Ci[Jv][L]), mul_rn(Ci[I][L], Ci[Jv][K])));
      const double t1 = mul_rn(mul_rn(-a23, j23), add_rn(mul_rn(dIJ, ckl), mul_rn(cij, dKL)));
      const double t2 = mul_rn(mul_rn(mul_rn(mul_rn(a29, j23), I1), cij), ckl);
      const double t3 = mul_rn(mul_rn(mul_rn(a23, j23), I1), Ic);
      const double t4 = mul_rn(mul_rn(q, cij), ckl);
      const double t5 = mul_rn(mul_rn(2.0, p), Ic);
      D[v][w] = sub_rn(add_rn(add_rn(add_rn(t1, t2), t3), t4), t5);
    }
  }
  return J;
}

// Ke[e][a][b][9] of the tangent (material + geometric) and, from the b = 0 threads,
// fe[e][a][3] of the internal force, at nodal displacements U; elements with J <= 0
// at a Gauss point are counted in *inverted.
static __global__ void __launch_bounds__(128) neohooke_element_kernel(
    const double *__restrict__ coords, const double *__restrict__ U, const int *__restrict__ conn, int n_elem,
    double C10, double D1, double *__restrict__ Ke, double *__restrict__ fe, int *inverted) {
  pdl_entry();
  const int Vi[6] = {0, 1, 2, 0, 1, 2}, Vj[6] = {0, 1, 2, 1, 2, 0};
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= int64_t(n_elem) * 64) return;
  const int e = int(t >> 6), a = int(t & 63) >> 3, b = int(t & 7);
  double X[8][3], u[8][3];
#pragma unroll
  for (int n = 0; n < 8; n++) {
    const int node = conn[8 * size_t(e) + n] - 1;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      X[n][d] = coords[3 * size_t(node) + d];
      u[n][d] = U[3 * size_t(node) + d];
    }
  }
  const double sgn[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                            {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  const double g = 1.0 / sqrt(3.0);
  const double gp[2] = {-g, g};
  double K[3][3] = {}, fa[3] = {};
  int bad = 0;
  for (int lz = 0; lz < 2; lz++)
    for (int ly = 0; ly < 2; ly++)
      for (int lx = 0; lx < 2; lx++) {
        const double xi[3] = {gp[lx], gp[ly], gp[lz]};
        double N[8][3];
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
        double XJ[3][3] = {};
#pragma unroll
        for (int n = 0; n < 8; n++)
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) XJ[i][j] = add_rn(XJ[i][j], mul_rn(X[n][i], deriv[n][j]));
        double w = mul_rn(mul_rn(XJ[0][0], XJ[1][1]), XJ[2][2]);
        w = add_rn(w, mul_rn(mul_rn(XJ[1][0], XJ[2][1]), XJ[0][2]));
        w = add_rn(w, mul_rn(mul_rn(XJ[2][0], XJ[0][1]), XJ[1][2]));
        w = sub_rn(w, mul_rn(mul_rn(XJ[2][0], XJ[1][1]), XJ[0][2]));
        w = sub_rn(w, mul_rn(mul_rn(XJ[1][0], XJ[0][1]), XJ[2][2]));
        w = sub_rn(w, mul_rn(mul_rn(XJ[0][0], XJ[2][1]), XJ[1][2]));
        const double dinv = 1.0 / w;
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
#pragma unroll
        for (int n = 0; n < 8; n++)
#pragma unroll
          for (int k = 0; k < 3; k++) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < 3; j++) s = add_rn(s, mul_rn(deriv[n][j], XJI[j][k]));
            N[n][k] = s;
          }
        double F[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll
        for (int n = 0; n < 8; n++)
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int J = 0; J < 3; J++) F[i][J] = add_rn(F[i][J], mul_rn(u[n][i], N[n][J]));
        double S[6], D[6][6];
        if (nh_stress(F, C10, D1, S, D) <= 0.0) bad = 1;
        // B columns of nodes a and b: dE_v / du_{a,k}
        double Ba[6][3], Bb[6][3];
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
          for (int v = 0; v < 6; v++) {
            const int I = Vi[v], J = Vj[v];
            Ba[v][k] = I == J ? mul_rn(F[k][I], N[a][I])
                              : add_rn(mul_rn(F[k][I], N[a][J]), mul_rn(F[k][J], N[a][I]));
            Bb[v][k] = I == J ? mul_rn(F[k][I], N[b][I])
                              : add_rn(mul_rn(F[k][I], N[b][J]), mul_rn(F[k][J], N[b][I]));
          }
        if (b == 0)
#pragma unroll
          for (int k = 0; k < 3; k++) {
            double f = 0.0;
#pragma unroll
            for (int v = 0; v < 6; v++) f = add_rn(f, mul_rn(Ba[v][k], S[v]));
            fa[k] = add_rn(fa[k], mul_rn(w, f));
          }
        double DB[6][3];
#pragma unroll
        for (int v = 0; v < 6; v++)
#pragma unroll
          for (int c = 0; c < 3; c++) {
            double s = 0.0;
#pragma unroll
            for (int x = 0; x < 6; x++) s = add_rn(s, mul_rn(D[v][x], Bb[x][c]));
            DB[v][c] = s;
          }
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int c = 0; c < 3; c++) {
            double s = 0.0;
#pragma unroll
            for (int v = 0; v < 6; v++) s = add_rn(s, mul_rn(Ba[v][r], DB[v][c]));
            K[r][c] = add_rn(K[r][c], mul_rn(w, s));
          }
        // geometric part on the block diagonal: N_a,I S_IJ N_b,J
        const double Sm[3][3] = {{S[0], S[3], S[5]}, {S[3], S[1], S[4]}, {S[5], S[4], S[2]}};
        double gab = 0.0;
#pragma unroll
        for (int I = 0; I < 3; I++)
#pragma unroll
          for (int J = 0; J < 3; J++) gab = add_rn(gab, mul_rn(mul_rn(N[a][I], Sm[I][J]), N[b][J]));
#pragma unroll
        for (int k = 0; k < 3; k++) K[k][k] = add_rn(K[k][k], mul_rn(w, gab));
      }
  double *out = Ke + 576 * size_t(e) + 9 * (8 * a + b);
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) out[3 * r + c] = K[r][c];
  if (b == 0)
#pragma unroll
    for (int k = 0; k < 3; k++) fe[24 * size_t(e) + 3 * a + k] = fa[k];
  if (a == 0 && b == 0 && bad) atomicAdd(inverted, 1);
}

// B(node) -= internal forces of the elements around the node, in element order (the
// D block's contribution list of node i holds exactly those (element, local a)).
static __global__ void __launch_bounds__(256) node_force_gather_kernel(const double *__restrict__ fe,
                                                                      const int64_t *__restrict__ ptr,
                                                                      const int *__restrict__ code, int n_node,
                                                                      double *__restrict__ B) {
  pdl_entry();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * n_node) return;
  const int i = t / 3, d = t - 3 * i;
  double s = B[t];
  for (int64_t k = ptr[i]; k < ptr[i + 1]; k++) {
    const int c = code[k];
    s = sub_rn(s, fe[24 * size_t(c >> 6) + 3 * ((c & 63) >> 3) + d]);
  }
  B[t] = s;
}

// Any zero diagonal entry of D (hecmw_solve_check_zerodiag, hecmw_solver_Iterative.f90:255-282).
static __global__ void zero_diag_kernel(const double *__restrict__ D, int n, int *flag) {
  pdl_entry();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int j = 0; j < 3; j++)
      if (fabs(D[9 * size_t(i) + 4 * j]) == 0.0) atomicOr(flag, 1);
}

}  // namespace h33
