/* C caller of the drop-in ABI with Fortran-layout (hecmwST_matrix) arrays, as the
 * iso_c_binding shim in frontistr_b200/fortran/hecmw_solver_gpu33.f90 passes them.
 * Builds an nx*ny*nz HEX8 cantilever with libfistr_assemble, solves it twice
 * through hecmw33_gpu_solve (second call: numeric update, recycled preconditioner)
 * and prints "iter resid converged ierr" per call. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "hecmw33_gpu.h"

int fistr_box_counts(int nx, int ny, int nz, int *n_node, int *NPL, int *NPU);
int fistr_box_assemble(int nx, int ny, int nz, const double *params, uint64_t seed, int *indexL,
                       int *itemL, int *indexU, int *itemU, double *D, double *AL, double *AU,
                       double *B, double *coords_out);

int main(int argc, char **argv) {
  const int nx = argc > 1 ? atoi(argv[1]) : 8, ny = nx, nz = 2 * nx;
  int N, NPL, NPU;
  if (fistr_box_counts(nx, ny, nz, &N, &NPL, &NPU)) return 2;
  int *indexL = calloc(N + 1, sizeof(int)), *indexU = calloc(N + 1, sizeof(int));
  int *itemL = calloc(NPL, sizeof(int)), *itemU = calloc(NPU, sizeof(int));
  double *D = calloc(9 * (size_t)N, 8), *AL = calloc(9 * (size_t)NPL, 8), *AU = calloc(9 * (size_t)NPU, 8);
  double *B = calloc(3 * (size_t)N, 8), *X = calloc(3 * (size_t)N, 8);
  const double params[8] = {1.0, 210000.0, 0.3, -1.0, 0.0, 0.0, 0.0, 0.0};
  if (fistr_box_assemble(nx, ny, nz, params, 0, indexL, itemL, indexU, itemU, D, AL, AU, B, NULL)) return 3;
  int Iarray[100] = {0};
  double Rarray[100] = {0};
  /* hecmw_mat_init defaults + METHOD=CG, PRECOND=1 */
  Iarray[0] = 20000; Iarray[1] = 1; Iarray[2] = 1; Iarray[4] = 1; Iarray[5] = 10;
  Iarray[33] = 10; Iarray[34] = 3; Iarray[96] = 1; Iarray[97] = 1; Iarray[98] = 1;
  Rarray[0] = 1e-8; Rarray[1] = 1.0;
  int handle = 0, ierr = 0, iter = 0;
  double resid = 0, times[3];
  hecmw33_gpu_create(&handle, &ierr);
  if (ierr) return 4;
  for (int call = 0; call < 2; call++) {
    for (int i = 0; i < 3 * N; i++) X[i] = 0.0;
    if (call == 1) Iarray[96] = 1; /* a later Newton iteration: recycle policy decides */
    hecmw33_gpu_solve(&handle, &N, &N, &NPL, &NPU, indexL, itemL, indexU, itemU, D, AL, AU, B, X,
                      Iarray, Rarray, &iter, &resid, times, &ierr);
    printf("%d %.6e %d %d\n", iter, resid, Iarray[80], ierr);
  }
  hecmw33_gpu_destroy(&handle, &ierr);
  return ierr;
}
