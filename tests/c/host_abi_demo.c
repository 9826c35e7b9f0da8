/* A plain C caller of the library's host entry points, compiled and run by
 * tests/test_c_abi.py: what a C or C++ code (the reference is C++) links
 * against -- include/pgfem_gpu.h and libpgfem_gpu.so, no Python, no torch.
 * Builds the DOF ids and the CSR pattern of a small box mesh, reads a mesh
 * file and round-trips a restart file; prints one line per check. */
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
  if (argc < 3) return 2;
  const char *mesh_base = argv[1]; /* <base>0.in written by the test */
  const char *res_path = argv[2];

  /* box mesh, 2^3 cells x 6 linear tets, x = 0 face fixed */
  long nn = 0, ne = 0;
  int r = pgfem_mesh_box_tet(2, 4, 0, &nn, &ne, NULL, NULL, NULL);
  CHECK(r == PGFEM_GPU_OK && nn == 27 && ne == 48, "mesh sizes");
  double *X = malloc(sizeof(double) * 3 * nn);
  int *conn = malloc(sizeof(int) * 4 * ne);
  long *Pr = malloc(sizeof(long) * nn);
  r = pgfem_mesh_box_tet(2, 4, 0, &nn, &ne, X, conn, Pr);
  long *id = calloc(3 * nn, sizeof(long));
  for (long n = 0; n < nn; n++)
    if (X[3 * n] == 0.0) id[3 * n] = id[3 * n + 1] = id[3 * n + 2] = 1;
  const long ndof = pgfem_generate_dof_ids(nn, ne, 4, conn, NULL, id);
  CHECK(ndof == 3 * 27 - 3 * 9, "free DOFs");
  int *Ap = malloc(sizeof(int) * (ndof + 1));
  const long nnz = pgfem_psparse_apai(ne, 4, conn, id, ndof, Ap, NULL);
  int *Ai = malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
  pgfem_psparse_apai(ne, 4, conn, id, ndof, Ap, Ai);
  int sorted = nnz > 0 && Ap[ndof] == nnz;
  for (long i = 0; i < ndof && sorted; i++)
    for (int j = Ap[i] + 1; j < Ap[i + 1]; j++) sorted &= Ai[j - 1] < Ai[j];
  CHECK(sorted, "CSR pattern rows sorted");
  CHECK(pgfem_gpu_state_size(PGFEM_MODEL_J2) == 10 && pgfem_gpu_state_size(PGFEM_MODEL_HE) == 0, "state sizes");

  /* mesh file */
  pgfem_input *in = NULL;
  r = pgfem_input_read_mesh(mesh_base, 1, &in);
  CHECK(r == PGFEM_GPU_OK, "read mesh file");
  pgfem_input_info info;
  pgfem_input_get_info(in, &info);
  CHECK(info.nn == 14 && info.ne == 24 && info.nne == 4 && info.npres == 1, "mesh file sizes");
  double *Xi = malloc(sizeof(double) * 3 * info.nn), defl[1];
  int *ci = malloc(sizeof(int) * 4 * info.ne);
  long *codes = malloc(sizeof(long) * 3 * info.nn);
  pgfem_input_get_mesh(in, Xi, ci, codes, defl);
  CHECK(defl[0] == 1.0, "prescribed value");
  pgfem_input_destroy(in);
  r = pgfem_input_read_mesh("no/such/mesh_", 1, &in);
  CHECK(r == PGFEM_GPU_EFORMAT && pgfem_input_last_error()[0] != 0, "missing file reported");

  /* restart file round trip */
  const int bs = pgfem_restart_block_size(PGFEM_MODEL_CP);
  double u1[6] = {1, 2, 3, 4, 5, 6}, u2[6] = {-1, -2, -3, -4, -5, -6}, blocks[64], a[6], b[6], c[64];
  for (int k = 0; k < 64; k++) blocks[k] = sin(k + 1.0);
  r = pgfem_restart_format(res_path, 2, 1, 1, PGFEM_MODEL_CP, u1, u2, blocks);
  r |= pgfem_restart_parse(res_path, 2, 1, 1, PGFEM_MODEL_CP, a, b, c);
  int same = bs == 64 && r == PGFEM_GPU_OK;
  for (int k = 0; k < 6; k++) same &= a[k] == u1[k] && b[k] == u2[k];
  for (int k = 0; k < 64; k++) same &= c[k] == blocks[k];
  CHECK(same, "restart round trip");
  free(X); free(conn); free(Pr); free(id); free(Ap); free(Ai); free(Xi); free(ci); free(codes);
  return fails ? 1 : 0;
}
