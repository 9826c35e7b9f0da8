/* A plain C caller of the library's device path, compiled and run by
 * tests/test_c_abi.py on a machine with an sm_100 GPU: include/pgfem_gpu.h and
 * libpgfem_gpu.so only, no Python, no torch.  Builds a J2 box of quadratic
 * tets (n^3 cells, stretched past yield), creates a context
 * (pgfem_gpu_create), sets the state, assembles R and K through the
 * host-buffer entry point (pgfem_gpu_assemble_RK), reads the state at t_{n+1}
 * and destroys the context.  Writes u, R, K and the state as raw doubles to
 * the given file for the test to compare with the oracle, and prints one line
 * per check. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "pgfem_gpu.h"

static int fails = 0;
#define CHECK(c, what)                                   \
  do {                                                   \
    if (c) printf("ok %s\n", what);                      \
    else { printf("FAIL %s\n", what); fails++; }         \
  } while (0)

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  const int n = 3;
  long nn = 0, ne = 0;
  int r = pgfem_mesh_box_tet(n, 10, 0, &nn, &ne, NULL, NULL, NULL);
  double *X = malloc(sizeof(double) * 3 * nn);
  int *conn = malloc(sizeof(int) * 10 * ne);
  r |= pgfem_mesh_box_tet(n, 10, 0, &nn, &ne, X, conn, NULL);
  long *id = calloc(3 * nn, sizeof(long));
  const long ndof = pgfem_generate_dof_ids(nn, ne, 10, conn, NULL, id);
  int *Ap = malloc(sizeof(int) * (ndof + 1));
  const long nnz = pgfem_psparse_apai(ne, 10, conn, id, ndof, Ap, NULL);
  int *Ai = malloc(sizeof(int) * nnz);
  pgfem_psparse_apai(ne, 10, conn, id, ndof, Ap, Ai);
  CHECK(r == PGFEM_GPU_OK && ndof == 3 * nn && nnz > 0, "mesh, DOF ids and CSR pattern");

  /* u = 0.4 % stretch along x plus a deterministic wobble */
  double *u = malloc(sizeof(double) * ndof);
  for (long a = 0; a < nn; a++)
    for (int j = 0; j < 3; j++)
      u[id[3 * a + j] - 1] = (j == 0 ? 4e-3 * X[3 * a] : 0.0) + 1e-3 / n * sin(1.0 + 3.0 * a + j);

  pgfem_mesh_desc m = {0};
  m.nn = nn;
  m.ne = ne;
  m.nne = 10;
  m.X = X;
  m.conn = conn;
  m.dof_id = id;
  m.ndof = ndof;
  pgfem_material_desc mat = {0};
  mat.model = PGFEM_MODEL_J2;
  mat.E = 200e3;
  mat.nu = 0.3;
  mat.sigma_y = 250.0;
  mat.H = 2000.0;
  mat.vol_pot = 99;
  pgfem_gpu_ctx *ctx = NULL;
  r = pgfem_gpu_create(&m, &mat, Ap, Ai, ndof, &ctx);
  CHECK(r == PGFEM_GPU_OK && ctx, "pgfem_gpu_create");
  if (!ctx) return 1;
  const long nqp = ne * 4;
  const int ns = pgfem_gpu_state_size(PGFEM_MODEL_J2);
  double *st = calloc(nqp * ns, sizeof(double));
  for (long q = 0; q < nqp; q++) st[q * ns] = st[q * ns + 4] = st[q * ns + 8] = 1.0;
  CHECK(pgfem_gpu_set_state(ctx, st) == PGFEM_GPU_OK, "pgfem_gpu_set_state");
  double *R = malloc(sizeof(double) * ndof), *K = malloc(sizeof(double) * nnz);
  pgfem_gpu_status status;
  r = pgfem_gpu_assemble_RK(ctx, u, NULL, 0.0, R, K, &status);
  CHECK(r == PGFEM_GPU_OK && status.inverted == 0 && status.other == 0, "pgfem_gpu_assemble_RK");
  double nk = 0;
  for (long k = 0; k < nnz; k++) nk += K[k] * K[k];
  CHECK(isfinite(nk) && nk > 0, "K finite and non-zero");
  double *snp1 = malloc(sizeof(double) * nqp * ns);
  CHECK(pgfem_gpu_get_state(ctx, 1, snp1) == PGFEM_GPU_OK, "pgfem_gpu_get_state");
  CHECK(pgfem_gpu_destroy(ctx) == PGFEM_GPU_OK, "pgfem_gpu_destroy");

  FILE *f = fopen(argv[1], "wb");
  CHECK(f != NULL, "output file");
  if (f) {
    fwrite(&ndof, sizeof(long), 1, f);
    fwrite(&nnz, sizeof(long), 1, f);
    fwrite(u, sizeof(double), ndof, f);
    fwrite(R, sizeof(double), ndof, f);
    fwrite(K, sizeof(double), nnz, f);
    fwrite(snp1, sizeof(double), nqp * ns, f);
    fclose(f);
  }
  return fails ? 1 : 0;
}
