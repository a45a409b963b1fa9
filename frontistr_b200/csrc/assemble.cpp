// assemble.cpp -- host-side generator of hecmwST_matrix systems (the caller side of
// hecmw_solve): matrix profile, linear-elastic element stiffness, scatter, nodal
// loads and displacement boundary conditions.  Built into libfistr_assemble.so.
//
// Reference behaviour restated here (paths inside the FrontISTR tree):
//   profile          hecmw1/src/solver/matrix/hecmw_mat_con.f90:21-107
//                    (per node: sorted, unique lists of lower (L) and upper (U)
//                     neighbour ids over all elements that share the node)
//   element matrix   fistr1/src/lib/static_LIB_3d.f90:50-208 (STF_C3, INFINITESIMAL)
//                    shape functions fistr1/src/lib/element/hex8n.f90:7-60,
//                    fistr1/src/lib/element/tet4n.f90:11-40, 2x2x2 / 1-point Gauss
//                    (fistr1/src/lib/element/element.f90:449-470,558-562)
//   isotropic D      fistr1/src/lib/physics/ElasticLinear.f90:38-60 (bulk/shear form)
//   scatter          hecmw1/src/solver/matrix/hecmw_mat_ass.f90:32-135 (row-major blocks)
//   boundary cond.   hecmw1/src/solver/matrix/hecmw_mat_ass.f90:328-463 (hecmw_mat_ass_bc)
//   Neo-Hookean      fistr1/src/lib/physics/Hyperelastic.f90:286-381 (compressible
//                    NEOHOOKE: W = C10 (I1bar - 3) + (J - 1)^2 / D1), total-Lagrangian
//                    element forces and tangent in the manner of fistr1/src/lib/static_LIB_3d.f90
//                    (TOTALLAG), with the material tangent derived from W (below)
//
// Node ids are 1-based in every array that leaves this file (itemL/itemU), as in
// hecmwST_matrix; element connectivity passed in is 0-based.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---- isotropic elasticity matrix (Voigt: xx, yy, zz, xy, yz, zx) -------------
void elastic_matrix(double E, double nu, double D[6][6]) {
  std::memset(D, 0, sizeof(double) * 36);
  const double K = E / (1.0 - 2.0 * nu) / 3.0;
  const double G = E / (1.0 + nu) * 0.5;
  D[0][0] = K + (4.0 / 3.0) * G;
  D[0][1] = K - (2.0 / 3.0) * G;
  D[3][3] = G;
  D[0][2] = D[0][1];
  D[1][0] = D[0][1];
  D[1][1] = D[0][0];
  D[1][2] = D[0][1];
  D[2][0] = D[0][2];
  D[2][1] = D[1][2];
  D[2][2] = D[0][0];
  D[4][4] = D[3][3];
  D[5][5] = D[3][3];
}

// Adds w * B^T D B for one integration point; gderiv[a][k] = dN_a/dx_k.
template <int NN>
void add_btdb(const double gderiv[NN][3], const double D[6][6], double w, double *K) {
  constexpr int ND = 3 * NN;
  double B[6][ND];
  std::memset(B, 0, sizeof(B));
  for (int j = 0; j < NN; j++) {
    B[0][3 * j + 0] = gderiv[j][0];
    B[1][3 * j + 1] = gderiv[j][1];
    B[2][3 * j + 2] = gderiv[j][2];
    B[3][3 * j + 0] = gderiv[j][1];
    B[3][3 * j + 1] = gderiv[j][0];
    B[4][3 * j + 1] = gderiv[j][2];
    B[4][3 * j + 2] = gderiv[j][1];
    B[5][3 * j + 0] = gderiv[j][2];
    B[5][3 * j + 2] = gderiv[j][0];
  }
  double DB[6][ND];
  for (int r = 0; r < 6; r++)
    for (int c = 0; c < ND; c++) {
      double s = 0.0;
      for (int k = 0; k < 6; k++) s += D[r][k] * B[k][c];
      DB[r][c] = s;
    }
  for (int j = 0; j < ND; j++)
    for (int i = 0; i < ND; i++) {
      double s = 0.0;
      for (int k = 0; k < 6; k++) s += B[k][i] * DB[k][j];
      K[i * ND + j] += s * w;
    }
}

// Jacobian XJ(i,j) = sum_a x_i(a) dN_a/dxi_j, its inverse and the global derivatives.
template <int NN>
double global_deriv(const double deriv[NN][3], const double x[NN][3], double gderiv[NN][3]) {
  double XJ[3][3] = {};
  for (int a = 0; a < NN; a++)
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) XJ[i][j] += x[a][i] * deriv[a][j];
  const double det = XJ[0][0] * XJ[1][1] * XJ[2][2] + XJ[1][0] * XJ[2][1] * XJ[0][2] +
                     XJ[2][0] * XJ[0][1] * XJ[1][2] - XJ[2][0] * XJ[1][1] * XJ[0][2] -
                     XJ[1][0] * XJ[0][1] * XJ[2][2] - XJ[0][0] * XJ[2][1] * XJ[1][2];
  const double d = 1.0 / det;
  double XJI[3][3];
  XJI[0][0] = d * (XJ[1][1] * XJ[2][2] - XJ[2][1] * XJ[1][2]);
  XJI[0][1] = d * (-XJ[0][1] * XJ[2][2] + XJ[2][1] * XJ[0][2]);
  XJI[0][2] = d * (XJ[0][1] * XJ[1][2] - XJ[1][1] * XJ[0][2]);
  XJI[1][0] = d * (-XJ[1][0] * XJ[2][2] + XJ[2][0] * XJ[1][2]);
  XJI[1][1] = d * (XJ[0][0] * XJ[2][2] - XJ[2][0] * XJ[0][2]);
  XJI[1][2] = d * (-XJ[0][0] * XJ[1][2] + XJ[1][0] * XJ[0][2]);
  XJI[2][0] = d * (XJ[1][0] * XJ[2][1] - XJ[2][0] * XJ[1][1]);
  XJI[2][1] = d * (-XJ[0][0] * XJ[2][1] + XJ[2][0] * XJ[0][1]);
  XJI[2][2] = d * (XJ[0][0] * XJ[1][1] - XJ[1][0] * XJ[0][1]);
  // gderiv = deriv * XJI  (dN/dx_k = sum_j dN/dxi_j * dxi_j/dx_k)
  for (int a = 0; a < NN; a++)
    for (int k = 0; k < 3; k++) {
      double s = 0.0;
      for (int j = 0; j < 3; j++) s += deriv[a][j] * XJI[j][k];
      gderiv[a][k] = s;
    }
  return det;
}

// HEX8, full 2x2x2 Gauss integration (FORM361=FI).  K is 24x24 row-major.
void stiff_hex8(const double x[8][3], double E, double nu, double *K) {
  static const double sgn[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                   {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  double D[6][6];
  elastic_matrix(E, nu, D);
  std::memset(K, 0, sizeof(double) * 576);
  const double g = 1.0 / std::sqrt(3.0);
  const double gp[2] = {-g, g};
  for (int lz = 0; lz < 2; lz++)
    for (int ly = 0; ly < 2; ly++)
      for (int lx = 0; lx < 2; lx++) {
        const double xi[3] = {gp[lx], gp[ly], gp[lz]};
        double deriv[8][3];
        for (int a = 0; a < 8; a++) {
          const double f0 = 1.0 + sgn[a][0] * xi[0], f1 = 1.0 + sgn[a][1] * xi[1],
                       f2 = 1.0 + sgn[a][2] * xi[2];
          deriv[a][0] = 0.125 * sgn[a][0] * f1 * f2;
          deriv[a][1] = 0.125 * sgn[a][1] * f0 * f2;
          deriv[a][2] = 0.125 * sgn[a][2] * f0 * f1;
        }
        double gderiv[8][3];
        const double det = global_deriv<8>(deriv, x, gderiv);
        add_btdb<8>(gderiv, D, 1.0 * det, K);
      }
}

// TET4, one-point rule with weight 1/6.  K is 12x12 row-major.
void stiff_tet4(const double x[4][3], double E, double nu, double *K) {
  static const double deriv[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  double D[6][6];
  elastic_matrix(E, nu, D);
  std::memset(K, 0, sizeof(double) * 144);
  double gderiv[4][3];
  const double det = global_deriv<4>(deriv, x, gderiv);
  add_btdb<4>(gderiv, D, det / 6.0, K);
}

// ---- compressible Neo-Hookean, total Lagrangian --------------------------------
// Voigt order of symmetric tensors: 11, 22, 33, 12, 23, 31 (as the linear element).
const int kVi[6] = {0, 1, 2, 0, 1, 2}, kVj[6] = {0, 1, 2, 1, 2, 0};

// Second Piola-Kirchhoff stress S and material tangent D = 2 dS/dC (Voigt, D_vw =
// C_IJKL) of W = C10 (J^-2/3 I1 - 3) + (J - 1)^2 / D1 at deformation gradient F:
//   S = 2 C10 J^-2/3 (I - I1/3 C^-1) + p C^-1,            p = 2/D1 (J - 1) J
//   D = -4C10/3 J^-2/3 (I (x) C^-1 + C^-1 (x) I) + 4C10/9 J^-2/3 I1 C^-1 (x) C^-1
//       + 4C10/3 J^-2/3 I1 Ic + 2/D1 (2J - 1) J C^-1 (x) C^-1 - 2p Ic,
//   Ic_IJKL = (C^-1_IK C^-1_JL + C^-1_IL C^-1_JK) / 2.
// Returns J.
double neohooke_stress(const double F[3][3], double C10, double D1, double S[6], double D[6][6]) {
  double C[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = 0.0;
      for (int k = 0; k < 3; k++) s += F[k][i] * F[k][j];
      C[i][j] = s;
    }
  const double J = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) -
                   F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                   F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
  const double detC = J * J;
  double Ci[3][3];
  Ci[0][0] = (C[1][1] * C[2][2] - C[1][2] * C[2][1]) / detC;
  Ci[0][1] = (C[0][2] * C[2][1] - C[0][1] * C[2][2]) / detC;
  Ci[0][2] = (C[0][1] * C[1][2] - C[0][2] * C[1][1]) / detC;
  Ci[1][0] = Ci[0][1];
  Ci[1][1] = (C[0][0] * C[2][2] - C[0][2] * C[2][0]) / detC;
  Ci[1][2] = (C[0][2] * C[1][0] - C[0][0] * C[1][2]) / detC;
  Ci[2][0] = Ci[0][2];
  Ci[2][1] = Ci[1][2];
  Ci[2][2] = (C[0][0] * C[1][1] - C[0][1] * C[1][0]) / detC;
  const double I1 = C[0][0] + C[1][1] + C[2][2];
  const double j23 = std::pow(J, -2.0 / 3.0);
  const double a = 2.0 * C10, p = 2.0 / D1 * (J - 1.0) * J;
  const double q = 2.0 / D1 * (2.0 * J - 1.0) * J;
  for (int v = 0; v < 6; v++) {
    const int I = kVi[v], Jv = kVj[v];
    const double dIJ = I == Jv ? 1.0 : 0.0;
    S[v] = a * j23 * (dIJ - I1 / 3.0 * Ci[I][Jv]) + p * Ci[I][Jv];
    for (int w = 0; w < 6; w++) {
      const int K = kVi[w], L = kVj[w];
      const double dKL = K == L ? 1.0 : 0.0;
      const double Ic = 0.5 * (Ci[I][K] * Ci[Jv][L] + Ci[I][L] * Ci[Jv][K]);
      D[v][w] = -(2.0 * a / 3.0) * j23 * (dIJ * Ci[K][L] + Ci[I][Jv] * dKL) +
                (2.0 * a / 9.0) * j23 * I1 * Ci[I][Jv] * Ci[K][L] + (2.0 * a / 3.0) * j23 * I1 * Ic +
                q * Ci[I][Jv] * Ci[K][L] - 2.0 * p * Ic;
    }
  }
  return J;
}

// HEX8 element at nodal displacements u (reference coordinates X), 2x2x2 Gauss:
// internal force fint (24) and tangent K (24x24 row-major, material + geometric).
// Returns 0, or 1 when J <= 0 at a Gauss point (inverted element).
int neohooke_hex8(const double X[8][3], const double u[8][3], double C10, double D1, double *K,
                  double *fint) {
  static const double sgn[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                   {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
  std::memset(K, 0, sizeof(double) * 576);
  std::memset(fint, 0, sizeof(double) * 24);
  const double g = 1.0 / std::sqrt(3.0);
  const double gp[2] = {-g, g};
  int bad = 0;
  for (int lz = 0; lz < 2; lz++)
    for (int ly = 0; ly < 2; ly++)
      for (int lx = 0; lx < 2; lx++) {
        const double xi[3] = {gp[lx], gp[ly], gp[lz]};
        double deriv[8][3];
        for (int a = 0; a < 8; a++) {
          const double f0 = 1.0 + sgn[a][0] * xi[0], f1 = 1.0 + sgn[a][1] * xi[1],
                       f2 = 1.0 + sgn[a][2] * xi[2];
          deriv[a][0] = 0.125 * sgn[a][0] * f1 * f2;
          deriv[a][1] = 0.125 * sgn[a][1] * f0 * f2;
          deriv[a][2] = 0.125 * sgn[a][2] * f0 * f1;
        }
        double N[8][3];  // dN_a / dX_J
        const double w = global_deriv<8>(deriv, X, N);
        double F[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        for (int a = 0; a < 8; a++)
          for (int i = 0; i < 3; i++)
            for (int J = 0; J < 3; J++) F[i][J] += u[a][i] * N[a][J];
        double S[6], D[6][6];
        if (neohooke_stress(F, C10, D1, S, D) <= 0.0) bad = 1;
        // B (6 x 24): dE_v / du_ak, engineering shear
        double B[6][24];
        for (int a = 0; a < 8; a++)
          for (int k = 0; k < 3; k++)
            for (int v = 0; v < 6; v++) {
              const int I = kVi[v], J = kVj[v];
              B[v][3 * a + k] = I == J ? F[k][I] * N[a][I] : F[k][I] * N[a][J] + F[k][J] * N[a][I];
            }
        for (int c = 0; c < 24; c++) {
          double f = 0.0;
          for (int v = 0; v < 6; v++) f += B[v][c] * S[v];
          fint[c] += w * f;
        }
        double DB[6][24];
        for (int v = 0; v < 6; v++)
          for (int c = 0; c < 24; c++) {
            double t = 0.0;
            for (int x = 0; x < 6; x++) t += D[v][x] * B[x][c];
            DB[v][c] = t;
          }
        for (int r = 0; r < 24; r++)
          for (int c = 0; c < 24; c++) {
            double t = 0.0;
            for (int v = 0; v < 6; v++) t += B[v][r] * DB[v][c];
            K[r * 24 + c] += w * t;
          }
        // geometric part: (N_a,I S_IJ N_b,J) on the diagonal of every 3x3 block
        const double Sm[3][3] = {{S[0], S[3], S[5]}, {S[3], S[1], S[4]}, {S[5], S[4], S[2]}};
        for (int a = 0; a < 8; a++)
          for (int b = 0; b < 8; b++) {
            double gab = 0.0;
            for (int I = 0; I < 3; I++)
              for (int J = 0; J < 3; J++) gab += N[a][I] * Sm[I][J] * N[b][J];
            for (int k = 0; k < 3; k++) K[(3 * a + k) * 24 + 3 * b + k] += w * gab;
          }
      }
  return bad;
}

int find_col(const int *item, int is, int ie, int key) {
  const int *p = std::lower_bound(item + is, item + ie, key);
  return (p != item + ie && *p == key) ? int(p - item) : -1;
}

struct Csr {
  int NP = 0;
  const int *indexL, *itemL, *indexU, *itemU;
  double *D, *AL, *AU;
};

// hecmw_mat_ass_elem: add a (nn*3)^2 element matrix into the D/AL/AU blocks.
void scatter(const Csr &m, int nn, const int *nodes, const double *K) {
  const int ND = 3 * nn;
  for (int a = 0; a < nn; a++) {
    const int ia = nodes[a] + 1;
    for (int b = 0; b < nn; b++) {
      const int ib = nodes[b] + 1;
      double *blk;
      if (ia == ib) {
        blk = m.D + 9 * size_t(ia - 1);
      } else if (ib < ia) {
        const int p = find_col(m.itemL, m.indexL[ia - 1], m.indexL[ia], ib);
        blk = m.AL + 9 * size_t(p);
      } else {
        const int p = find_col(m.itemU, m.indexU[ia - 1], m.indexU[ia], ib);
        blk = m.AU + 9 * size_t(p);
      }
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) blk[3 * r + c] += K[(3 * a + r) * ND + 3 * b + c];
    }
  }
}

// splitmix64: small seeded generator for the jittered / heterogeneous meshes.
struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return double(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
  double normal() {  // Box-Muller
    double u1 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    const double u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// Generic meshes (used for the reference's TET4 fixtures).
// Profile counts for n_elem elements of nn nodes (0-based conn).
int fistr_mesh_profile_counts(int n_node, int n_elem, int nn, const int *conn, int *NPL, int *NPU) {
  std::vector<std::vector<int>> lo(n_node), up(n_node);
  for (int e = 0; e < n_elem; e++)
    for (int j = 0; j < nn; j++)
      for (int k = 0; k < nn; k++) {
        const int a = conn[e * nn + j], b = conn[e * nn + k];
        if (a < 0 || a >= n_node || b < 0 || b >= n_node) return -1;
        if (a < b) up[a].push_back(b);
        else if (a > b) lo[a].push_back(b);
      }
  long nl = 0, nu = 0;
  for (int i = 0; i < n_node; i++) {
    std::sort(lo[i].begin(), lo[i].end());
    std::sort(up[i].begin(), up[i].end());
    nl += std::unique(lo[i].begin(), lo[i].end()) - lo[i].begin();
    nu += std::unique(up[i].begin(), up[i].end()) - up[i].begin();
  }
  *NPL = int(nl);
  *NPU = int(nu);
  return 0;
}

// Builds the profile and assembles K for TET4 (etype 341, nn=4) or HEX8 (361, nn=8)
// elements with per-element E/nu.  Output arrays are sized from
// fistr_mesh_profile_counts; D/AL/AU are overwritten.
int fistr_mesh_assemble(int n_node, const double *coords, int n_elem, int etype, const int *conn,
                        const double *E, const double *nu, int *indexL, int *itemL, int *indexU,
                        int *itemU, double *D, double *AL, double *AU) {
  const int nn = etype == 341 ? 4 : (etype == 361 ? 8 : 0);
  if (nn == 0) return -2;
  std::vector<std::vector<int>> lo(n_node), up(n_node);
  for (int e = 0; e < n_elem; e++)
    for (int j = 0; j < nn; j++)
      for (int k = 0; k < nn; k++) {
        const int a = conn[e * nn + j], b = conn[e * nn + k];
        if (a < b) up[a].push_back(b + 1);
        else if (a > b) lo[a].push_back(b + 1);
      }
  indexL[0] = indexU[0] = 0;
  for (int i = 0; i < n_node; i++) {
    std::sort(lo[i].begin(), lo[i].end());
    lo[i].erase(std::unique(lo[i].begin(), lo[i].end()), lo[i].end());
    std::sort(up[i].begin(), up[i].end());
    up[i].erase(std::unique(up[i].begin(), up[i].end()), up[i].end());
    indexL[i + 1] = indexL[i] + int(lo[i].size());
    indexU[i + 1] = indexU[i] + int(up[i].size());
    std::copy(lo[i].begin(), lo[i].end(), itemL + indexL[i]);
    std::copy(up[i].begin(), up[i].end(), itemU + indexU[i]);
  }
  std::memset(D, 0, sizeof(double) * 9 * size_t(n_node));
  std::memset(AL, 0, sizeof(double) * 9 * size_t(indexL[n_node]));
  std::memset(AU, 0, sizeof(double) * 9 * size_t(indexU[n_node]));
  Csr m{n_node, indexL, itemL, indexU, itemU, D, AL, AU};
  std::vector<double> K(size_t(3 * nn) * size_t(3 * nn));
  for (int e = 0; e < n_elem; e++) {
    if (nn == 4) {
      double x[4][3];
      for (int a = 0; a < 4; a++)
        for (int d = 0; d < 3; d++) x[a][d] = coords[3 * conn[e * 4 + a] + d];
      stiff_tet4(x, E[e], nu[e], K.data());
    } else {
      double x[8][3];
      for (int a = 0; a < 8; a++)
        for (int d = 0; d < 3; d++) x[a][d] = coords[3 * conn[e * 8 + a] + d];
      stiff_hex8(x, E[e], nu[e], K.data());
    }
    scatter(m, nn, conn + size_t(e) * nn, K.data());
  }
  return 0;
}

// hecmw_mat_ass_bc for one (node, dof) pair: node 1-based, dof 1..3.
void fistr_mat_ass_bc(int inode, int idof, double RHS, const int *indexL, const int *itemL,
                      const int *indexU, const int *itemU, double *D, double *AL, double *AU,
                      double *B) {
  const int NDOF = 3;
  // right-hand side of the fixed dof and its coupling inside the diagonal block
  B[NDOF * (inode - 1) + idof - 1] = RHS;
  double *d = D + 9 * size_t(inode - 1);
  for (int r = 1; r <= NDOF; r++)
    if (r != idof) B[NDOF * (inode - 1) + r - 1] -= d[3 * (r - 1) + idof - 1] * RHS;
  // zero row idof, then column idof with a unit diagonal
  for (int c = 0; c < NDOF; c++) d[3 * (idof - 1) + c] = 0.0;
  for (int r = 1; r <= NDOF; r++) d[3 * (r - 1) + idof - 1] = (r == idof) ? 1.0 : 0.0;
  // lower blocks of this row: zero row idof; in the mirrored upper block of
  // row `in`, move column idof to the right-hand side and zero it
  for (int k = indexL[inode - 1]; k < indexL[inode]; k++) {
    double *a = AL + 9 * size_t(k);
    for (int c = 0; c < NDOF; c++) a[3 * (idof - 1) + c] = 0.0;
    const int in = itemL[k];
    for (int ik = indexU[in - 1]; ik < indexU[in]; ik++) {
      if (itemU[ik] == inode) {
        double *u = AU + 9 * size_t(ik);
        for (int r = 1; r <= NDOF; r++) {
          B[NDOF * (in - 1) + r - 1] -= u[3 * (r - 1) + idof - 1] * RHS;
          u[3 * (r - 1) + idof - 1] = 0.0;
        }
        break;
      }
    }
  }
  for (int k = indexU[inode - 1]; k < indexU[inode]; k++) {
    double *a = AU + 9 * size_t(k);
    for (int c = 0; c < NDOF; c++) a[3 * (idof - 1) + c] = 0.0;
    const int in = itemU[k];
    for (int ik = indexL[in - 1]; ik < indexL[in]; ik++) {
      if (itemL[ik] == inode) {
        double *l = AL + 9 * size_t(ik);
        for (int r = 1; r <= NDOF; r++) {
          B[NDOF * (in - 1) + r - 1] -= l[3 * (r - 1) + idof - 1] * RHS;
          l[3 * (r - 1) + idof - 1] = 0.0;
        }
        break;
      }
    }
  }
}

// hecmw_mat_ass_bc for n (node, dof, value) triples in order (node 1-based, dof 1..3).
void fistr_mat_ass_bc_list(int n, const int *inode, const int *idof, const double *value, const int *indexL,
                           const int *itemL, const int *indexU, const int *itemU, double *D, double *AL,
                           double *AU, double *B) {
  for (int k = 0; k < n; k++)
    fistr_mat_ass_bc(inode[k], idof[k], value[k], indexL, itemL, indexU, itemU, D, AL, AU, B);
}

// ---------------------------------------------------------------------------
// Structured HEX8 boxes: nx*ny*nz unit cubes of edge h, nodes numbered
// lexicographically (x fastest), elements likewise, hex8n node order.
// Face z=0 clamped (all dofs, hecmw_mat_ass_bc semantics); a nodal force of
// `load_y` in y on every node of the face z=nz*h.  Optional seeded interior-node
// jitter (fraction of h) and log-normal E / uniform nu per element.
int fistr_box_counts(int nx, int ny, int nz, int *n_node, int *NPL, int *NPU) {
  const long nx1 = nx + 1, ny1 = ny + 1, nz1 = nz + 1;
  const long nnode = nx1 * ny1 * nz1;
  const long nz_blocks = (3 * nx1 - 2) * (3 * ny1 - 2) * (3 * nz1 - 2);
  if (nnode > 0x7fffffffL || (nz_blocks - nnode) / 2 > 0x7fffffffL) return -1;
  *n_node = int(nnode);
  *NPL = int((nz_blocks - nnode) / 2);
  *NPU = *NPL;
  return 0;
}

// Tangent stiffness and residual of a compressible Neo-Hookean HEX8 box (edge h,
// nodes as in fistr_box_assemble) at the nodal displacements U (3 per node):
// D/AL/AU = K(U), R = -f_int(U) (no external load: the Newton sequence drives the
// block by prescribed displacements).  Returns 0, or the number of elements with
// J <= 0 at a Gauss point.
int fistr_box_neohooke(int nx, int ny, int nz, double h, double C10, double D1, const double *U, int *indexL,
                       int *itemL, int *indexU, int *itemU, double *D, double *AL, double *AU, double *R) {
  const int nx1 = nx + 1, ny1 = ny + 1, nz1 = nz + 1;
  const int n_node = nx1 * ny1 * nz1;
  auto nid = [&](int ix, int iy, int iz) { return ix + nx1 * (iy + ny1 * iz); };
  indexL[0] = indexU[0] = 0;
  {
    int cl = 0, cu = 0;
    for (int iz = 0; iz < nz1; iz++)
      for (int iy = 0; iy < ny1; iy++)
        for (int ix = 0; ix < nx1; ix++) {
          const int self = nid(ix, iy, iz);
          for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
              for (int dx = -1; dx <= 1; dx++) {
                const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
                if (jx < 0 || jx > nx || jy < 0 || jy > ny || jz < 0 || jz > nz) continue;
                const int j = nid(jx, jy, jz);
                if (j < self) itemL[cl++] = j + 1;
                else if (j > self) itemU[cu++] = j + 1;
              }
          indexL[self + 1] = cl;
          indexU[self + 1] = cu;
        }
  }
  const size_t NPL = size_t(indexL[n_node]), NPU = size_t(indexU[n_node]);
  std::memset(D, 0, sizeof(double) * 9 * size_t(n_node));
  std::memset(AL, 0, sizeof(double) * 9 * NPL);
  std::memset(AU, 0, sizeof(double) * 9 * NPU);
  std::memset(R, 0, sizeof(double) * 3 * size_t(n_node));
  Csr m{n_node, indexL, itemL, indexU, itemU, D, AL, AU};
  int bad = 0;
  for (int color = 0; color < 8; color++) {
    const int px = color & 1, py = (color >> 1) & 1, pz = (color >> 2) & 1;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : bad)
    for (int ez = pz; ez < nz; ez += 2)
      for (int ey = py; ey < ny; ey += 2) {
        double Kl[576], fl[24];
        for (int ex = px; ex < nx; ex += 2) {
          const int nodes[8] = {nid(ex, ey, ez),         nid(ex + 1, ey, ez),
                                nid(ex + 1, ey + 1, ez), nid(ex, ey + 1, ez),
                                nid(ex, ey, ez + 1),     nid(ex + 1, ey, ez + 1),
                                nid(ex + 1, ey + 1, ez + 1), nid(ex, ey + 1, ez + 1)};
          const int off[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                 {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
          double X[8][3], u[8][3];
          for (int a = 0; a < 8; a++) {
            X[a][0] = (ex + off[a][0]) * h;
            X[a][1] = (ey + off[a][1]) * h;
            X[a][2] = (ez + off[a][2]) * h;
            for (int d = 0; d < 3; d++) u[a][d] = U[3 * size_t(nodes[a]) + d];
          }
          bad += neohooke_hex8(X, u, C10, D1, Kl, fl);
          scatter(m, 8, nodes, Kl);
          for (int a = 0; a < 8; a++)
            for (int d = 0; d < 3; d++) R[3 * size_t(nodes[a]) + d] -= fl[3 * a + d];
        }
      }
  }
  return bad;
}

// params: [0]=h, [1]=E0, [2]=nu0, [3]=load_y, [4]=jitter fraction (0 = none),
//         [5]=log-normal sigma of E (0 = uniform E0 as median), [6]=nu_min, [7]=nu_max
//         (nu_max <= nu_min -> uniform nu0)
// seed drives jitter and material sampling.  coords (3*n_node) is optional.
int fistr_box_assemble(int nx, int ny, int nz, const double *params, uint64_t seed, int *indexL,
                       int *itemL, int *indexU, int *itemU, double *D, double *AL, double *AU,
                       double *B, double *coords_out) {
  const double h = params[0], E0 = params[1], nu0 = params[2], load_y = params[3];
  const double jitter = params[4], sigE = params[5], numin = params[6], numax = params[7];
  const int nx1 = nx + 1, ny1 = ny + 1, nz1 = nz + 1;
  const int n_node = nx1 * ny1 * nz1;
  auto nid = [&](int ix, int iy, int iz) { return ix + nx1 * (iy + ny1 * iz); };  // 0-based

  // coordinates
  std::vector<double> X(3 * size_t(n_node));
  {
    SplitMix64 rng(seed ^ 0x5EED0001ull);
    for (int iz = 0; iz < nz1; iz++)
      for (int iy = 0; iy < ny1; iy++)
        for (int ix = 0; ix < nx1; ix++) {
          const size_t i = size_t(nid(ix, iy, iz));
          X[3 * i] = ix * h;
          X[3 * i + 1] = iy * h;
          X[3 * i + 2] = iz * h;
          const bool interior =
              ix > 0 && ix < nx && iy > 0 && iy < ny && iz > 0 && iz < nz;
          if (jitter > 0.0 && interior) {
            for (int d = 0; d < 3; d++) X[3 * i + d] += (2.0 * rng.uniform() - 1.0) * jitter * h;
          }
        }
  }
  if (coords_out) std::memcpy(coords_out, X.data(), sizeof(double) * X.size());

  // profile: the 27-point neighbourhood, ids ascending
  indexL[0] = indexU[0] = 0;
  {
    int cl = 0, cu = 0;
    for (int iz = 0; iz < nz1; iz++)
      for (int iy = 0; iy < ny1; iy++)
        for (int ix = 0; ix < nx1; ix++) {
          const int self = nid(ix, iy, iz);
          for (int dz = -1; dz <= 1; dz++)
            for (int dy = -1; dy <= 1; dy++)
              for (int dx = -1; dx <= 1; dx++) {
                const int jx = ix + dx, jy = iy + dy, jz = iz + dz;
                if (jx < 0 || jx > nx || jy < 0 || jy > ny || jz < 0 || jz > nz) continue;
                const int j = nid(jx, jy, jz);
                if (j < self) itemL[cl++] = j + 1;
                else if (j > self) itemU[cu++] = j + 1;
              }
          indexL[self + 1] = cl;
          indexU[self + 1] = cu;
        }
  }
  const size_t NPL = size_t(indexL[n_node]), NPU = size_t(indexU[n_node]);
  std::memset(D, 0, sizeof(double) * 9 * size_t(n_node));
  std::memset(AL, 0, sizeof(double) * 9 * NPL);
  std::memset(AU, 0, sizeof(double) * 9 * NPU);
  std::memset(B, 0, sizeof(double) * 3 * size_t(n_node));
  Csr m{n_node, indexL, itemL, indexU, itemU, D, AL, AU};

  // per-element materials
  const long n_elem = long(nx) * ny * nz;
  const bool hetero = sigE > 0.0 || numax > numin;
  std::vector<double> Ee, nue;
  if (hetero) {
    Ee.resize(size_t(n_elem));
    nue.resize(size_t(n_elem));
    SplitMix64 rng(seed ^ 0x5EED0002ull);
    for (long e = 0; e < n_elem; e++) {
      Ee[size_t(e)] = sigE > 0.0 ? E0 * std::exp(sigE * rng.normal()) : E0;
      nue[size_t(e)] = numax > numin ? numin + (numax - numin) * rng.uniform() : nu0;
    }
  }
  const bool uniform = !hetero && jitter <= 0.0;
  double Kref[576];
  if (uniform) {
    const double x[8][3] = {{0, 0, 0}, {h, 0, 0}, {h, h, 0}, {0, h, 0},
                            {0, 0, h}, {h, 0, h}, {h, h, h}, {0, h, h}};
    stiff_hex8(x, E0, nu0, Kref);
  }
  // 8-colour element sweep (parity in x, y, z): elements of one colour share no node
  for (int color = 0; color < 8; color++) {
    const int px = color & 1, py = (color >> 1) & 1, pz = (color >> 2) & 1;
#pragma omp parallel for collapse(2) schedule(static)
    for (int ez = pz; ez < nz; ez += 2)
      for (int ey = py; ey < ny; ey += 2) {
        double Kl[576];
        for (int ex = px; ex < nx; ex += 2) {
          const int nodes[8] = {nid(ex, ey, ez),         nid(ex + 1, ey, ez),
                                nid(ex + 1, ey + 1, ez), nid(ex, ey + 1, ez),
                                nid(ex, ey, ez + 1),     nid(ex + 1, ey, ez + 1),
                                nid(ex + 1, ey + 1, ez + 1), nid(ex, ey + 1, ez + 1)};
          const double *K = Kref;
          if (!uniform) {
            double x[8][3];
            for (int a = 0; a < 8; a++)
              for (int d = 0; d < 3; d++) x[a][d] = X[3 * size_t(nodes[a]) + d];
            const long e = long(ex) + long(nx) * (long(ey) + long(ny) * ez);
            stiff_hex8(x, hetero ? Ee[size_t(e)] : E0, hetero ? nue[size_t(e)] : nu0, Kl);
            K = Kl;
          }
          scatter(m, 8, nodes, K);
        }
      }
  }
  // nodal loads on the top face, then the clamped bottom face
  for (int iy = 0; iy < ny1; iy++)
    for (int ix = 0; ix < nx1; ix++) B[3 * size_t(nid(ix, iy, nz)) + 1] += load_y;
  for (int iy = 0; iy < ny1; iy++)
    for (int ix = 0; ix < nx1; ix++)
      for (int dof = 1; dof <= 3; dof++)
        fistr_mat_ass_bc(nid(ix, iy, 0) + 1, dof, 0.0, indexL, itemL, indexU, itemU, D, AL, AU, B);
  return 0;
}

}  // extern "C"
