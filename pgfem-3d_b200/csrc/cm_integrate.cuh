// cm_integrate.cuh -- batched constitutive update (integration_algorithm +
// update_elasticity, include/constitutive_model.h:242-757) over an array of
// deformation gradients.  Returns the material quantities the reference
// interface exchanges: S = F^-1 tau F^-T and L = 2 dS/dC obtained by pulling
// the spatial tangent back, L_IJKL = F^-1_Ii F^-1_Jj F^-1_Kk F^-1_Ll c_ijkl.
#pragma once
#include <vector>

#include "cm_models.cuh"

namespace pgb {

// Symmetric 3x3 (Voigt) -> full index helper
__device__ __forceinline__ double sv(const double *S, int i, int j) {
  const int m[3][3] = {{0, 5, 4}, {5, 1, 3}, {4, 3, 2}};
  return S[m[i][j]];
}

template <bool PLASTIC>
__global__ void k_cm_integrate(Mat mat, long nqp, const double *F_all, const double *state_n,
                               double *state_np1, double *S_out, double *L_out, int *qst) {
  const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= nqp) return;
  double F[9], Fi[9];
#pragma unroll
  for (int i = 0; i < 9; i++) F[i] = F_all[q * 9 + i];
  const double J = det3(F);
  if (!(J > 0.0) || !inv3(F, Fi)) {
    if (qst) qst[q] = 1;
    return;
  }
  double A[6] = {1, 1, 1, 0, 0, 0}, alpha = 0.0;
  if (PLASTIC) {
    const double *s = state_n + q * 10;
    A[0] = s[0]; A[1] = s[4]; A[2] = s[8]; A[3] = s[5]; A[4] = s[2]; A[5] = s[1];
    alpha = s[9];
  }
  QpTangent t;
  double Anp1[6], alpha_np1;
  const bool linear_dev = !PLASTIC && mat.dev_pot == 2;
  if (linear_dev)
    linear_dev_update(mat, F, J, t);  // t.n = b, pulled back to the identity below
  else
    spatial_update<PLASTIC>(mat, F, J, A, alpha, t, Anp1, &alpha_np1);
  if (PLASTIC) {
    double *s = state_np1 + q * 10;
    s[0] = Anp1[0]; s[1] = Anp1[5]; s[2] = Anp1[4];
    s[3] = Anp1[5]; s[4] = Anp1[1]; s[5] = Anp1[3];
    s[6] = Anp1[4]; s[7] = Anp1[3]; s[8] = Anp1[2];
    s[9] = alpha_np1;
  }
  // pull-backs: Ci = F^-1 F^-T, S = F^-1 tau F^-T, Ss, Sn, SD
  const double I6[6] = {1, 1, 1, 0, 0, 0};
  double Ci[6], S[6], Ss[6], Sn[6], SD[6];
  push_sym(Fi, I6, Ci);
  push_sym(Fi, t.tau, S);
  push_sym(Fi, t.s, Ss);
  push_sym(Fi, t.n, Sn);
  push_sym(Fi, t.D, SD);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) S_out[q * 9 + i * 3 + j] = sv(S, i, j);
  if (qst) qst[q] = 0;
  if (!L_out) return;
  double *L = L_out + q * 81;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) {
          const double cij = sv(Ci, i, j), ckl = sv(Ci, k, l);
          double v = t.a1 * 0.5 * (sv(Ci, i, k) * sv(Ci, j, l) + sv(Ci, i, l) * sv(Ci, j, k)) +
                     t.a2 * cij * ckl - (2.0 / 3.0) * (sv(Ss, i, j) * ckl + cij * sv(Ss, k, l));
          if (PLASTIC) v += sv(Sn, i, j) * (t.a4 * sv(Sn, k, l) + t.a5 * sv(SD, k, l));
          if (linear_dev) v += mat.mu * (sv(Sn, i, k) * sv(Sn, j, l) + sv(Sn, i, l) * sv(Sn, j, k));
          L[i * 27 + j * 9 + k * 3 + l] = v;
        }
}

inline int cm_integrate_host(const Mat &mat, long nqp, const double *F, double dt,
                             const double *state_n, double *state_np1, double *S, double *L,
                             int *qp_status) {
  (void)dt;
  const bool plastic = mat.model == 1;
  double *dF = nullptr, *dsn = nullptr, *dsnp1 = nullptr, *dS = nullptr, *dL = nullptr;
  int *dq = nullptr;
  auto cleanup = [&]() {
    for (void *p : {(void *)dF, (void *)dsn, (void *)dsnp1, (void *)dS, (void *)dL, (void *)dq})
      if (p) cudaFree(p);
  };
  bool ok = cudaMalloc(&dF, sizeof(double) * 9 * nqp) == cudaSuccess &&
            cudaMalloc(&dS, sizeof(double) * 9 * nqp) == cudaSuccess &&
            cudaMalloc(&dq, sizeof(int) * nqp) == cudaSuccess &&
            (!L || cudaMalloc(&dL, sizeof(double) * 81 * nqp) == cudaSuccess) &&
            (!plastic || (cudaMalloc(&dsn, sizeof(double) * 10 * nqp) == cudaSuccess &&
                          cudaMalloc(&dsnp1, sizeof(double) * 10 * nqp) == cudaSuccess));
  if (!ok) {
    cudaGetLastError();
    cleanup();
    return -3;
  }
  cudaMemcpy(dF, F, sizeof(double) * 9 * nqp, cudaMemcpyHostToDevice);
  if (plastic) cudaMemcpy(dsn, state_n, sizeof(double) * 10 * nqp, cudaMemcpyHostToDevice);
  const unsigned grid = (unsigned)((nqp + 127) / 128);
  if (plastic)
    k_cm_integrate<true><<<grid, 128>>>(mat, nqp, dF, dsn, dsnp1, dS, dL, dq);
  else
    k_cm_integrate<false><<<grid, 128>>>(mat, nqp, dF, dsn, dsnp1, dS, dL, dq);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) {
    cudaMemcpy(S, dS, sizeof(double) * 9 * nqp, cudaMemcpyDeviceToHost);
    if (L) cudaMemcpy(L, dL, sizeof(double) * 81 * nqp, cudaMemcpyDeviceToHost);
    if (plastic) cudaMemcpy(state_np1, dsnp1, sizeof(double) * 10 * nqp, cudaMemcpyDeviceToHost);
    std::vector<int> h(nqp);
    cudaMemcpy(h.data(), dq, sizeof(int) * nqp, cudaMemcpyDeviceToHost);
    if (qp_status)
      for (long i = 0; i < nqp; i++) qp_status[i] = h[i];
  }
  cleanup();
  return e == cudaSuccess ? 0 : -2;
}

}  // namespace pgb
