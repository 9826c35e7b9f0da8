// cm_models.cuh -- device-side constitutive updates of the assembly path in
// the spatial (Kirchhoff) form used by the element kernels.
//
// Both models return the Kirchhoff stress tau and the coefficients of the
// spatial tangent (push-forward of L = 2 dS/dC):
//   c = a1 I + a2 1(x)1 - 2/3 (s(x)1 + 1(x)s) + a4 n(x)n + a5 n(x)dev(n^2)
// with s = dev tau.  Symmetric tensors are stored in Voigt order
// (xx, yy, zz, yz, xz, xy).
//
//  HE  (HE_PARAM, src/plasticity_model_none.cc:69-76, 329-361): the
//      reference's compressible neo-Hookean solid -- deviatoric
//      Mooney-Rivlin with m01 = 0 (src/new_potentials.cc:333-432) plus the
//      U_Common volumetric potential (:553-604) as combined in
//      src/displacement_based_element.cc:1368-1445, pushed forward:
//      tau = mu dev(J^-2/3 F F^T) + kappa J U'(J) 1 (U the material's
//      volumetric potential: U_Common or a Doll-Schweizerhof form).
//  HE, linear deviatoric potential (devPotFlag 2, devStress_Linear /
//      matStiff_Linear, src/new_potentials.cc:364-375, 434-452): S = G (C - I)
//      + kappa J (J-1) C^-1, L = 2G I + volumetric part; pushed forward
//      tau = G (b^2 - b) + kappa J (J-1) 1 and
//      c = G (b_ik b_jl + b_il b_jk) + a1 I + a2 1(x)1, which is not of the
//      form above: the per-node element kernel adds the b-term itself
//      (template model 3), from b = F F^T carried in the tangent's n slot.
//  J2  (CM_J2P_PARAM, src/cm_j2_plasticity.cc:184-214, damage off): the
//      isochoric-split radial return of Simo (1988) / Simo & Hughes (1998)
//      Box 9.1 with linear isotropic hardening, state (Cp^-1, eqps), and the
//      exact consistent tangent of that update (non-symmetric part a5).
#pragma once
#include <cuda_runtime.h>

namespace pgb {

struct Mat {
  int model;
  int dev_pot;  // HE deviatoric potential: 2 linear, otherwise neo-Hookean
  int vol_pot;  // volumetric potential: 99 U_Common, 2 / 3 Doll-Schweizerhof (src/new_potentials.cc:553-640)
  double mu, kappa, sy, H;
  // crystal plasticity
  double gdot0, m, G0, g0, gs0, gdots, w, tol;
  int max_iter;
};

struct Sym {
  double v[6];
};

// U'(J) and U''(J) of the volumetric potential (src/new_potentials.cc:553-622):
// 99 U_Common 0.5 (J-1)^2; 2 0.5 (exp(J-1) - ln J - 1); 3 0.5 (J-1) ln J.
__device__ __forceinline__ void vol_derivs(int vol_pot, double J, double &dU, double &d2U) {
  if (vol_pot == 2) {
    const double e = exp(J - 1.0), iJ = 1.0 / J;
    dU = 0.5 * (e - iJ);
    d2U = 0.5 * (e + iJ * iJ);
  } else if (vol_pot == 3) {
    const double iJ = 1.0 / J;
    dU = 0.5 * (J - 1.0) * iJ + 0.5 * log(J);
    d2U = iJ - 0.5 * (J - 1.0) * iJ * iJ;
  } else {
    dU = J - 1.0;
    d2U = 1.0;
  }
}

__device__ __forceinline__ double sdot(const double *a, const double *b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + 2.0 * (a[3] * b[3] + a[4] * b[4] + a[5] * b[5]);
}

// y = S x for symmetric S (Voigt)
__device__ __forceinline__ void smv(const double *S, const double *x, double *y) {
  y[0] = S[0] * x[0] + S[5] * x[1] + S[4] * x[2];
  y[1] = S[5] * x[0] + S[1] * x[1] + S[3] * x[2];
  y[2] = S[4] * x[0] + S[3] * x[1] + S[2] * x[2];
}

__device__ __forceinline__ double det3(const double *m) {
  return ((m[0] * (m[4] * m[8] - m[5] * m[7])) + m[1] * (m[5] * m[6] - m[3] * m[8]) +
          m[2] * (m[3] * m[7] - m[4] * m[6]));
}

// inverse following src/utils.cc:542-562 (refused when |det| < 1e-15)
__device__ __forceinline__ bool inv3(const double *m, double *mi) {
  const double A = det3(m);
  if (!(fabs(A) >= 1.0e-15)) return false;
  const double r = 1.0 / A;
  mi[0] = r * (m[4] * m[8] - m[5] * m[7]);
  mi[1] = -r * (m[1] * m[8] - m[2] * m[7]);
  mi[2] = r * (m[1] * m[5] - m[2] * m[4]);
  mi[3] = -r * (m[3] * m[8] - m[5] * m[6]);
  mi[4] = r * (m[0] * m[8] - m[2] * m[6]);
  mi[5] = -r * (m[0] * m[5] - m[2] * m[3]);
  mi[6] = r * (m[3] * m[7] - m[4] * m[6]);
  mi[7] = -r * (m[0] * m[7] - m[1] * m[6]);
  mi[8] = r * (m[0] * m[4] - m[1] * m[3]);
  return true;
}

// B = F A F^T for a symmetric A (Voigt), result symmetric (Voigt)
__device__ __forceinline__ void push_sym(const double *F, const double *A, double *B) {
  double FA[9];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const double x[3] = {F[i * 3], F[i * 3 + 1], F[i * 3 + 2]};
    double y[3];
    smv(A, x, y);  // (A F_i.)  = row i of F A (A symmetric)
    FA[i * 3] = y[0];
    FA[i * 3 + 1] = y[1];
    FA[i * 3 + 2] = y[2];
  }
  auto row = [&](int i, int j) {
    return FA[i * 3] * F[j * 3] + FA[i * 3 + 1] * F[j * 3 + 1] + FA[i * 3 + 2] * F[j * 3 + 2];
  };
  B[0] = row(0, 0);
  B[1] = row(1, 1);
  B[2] = row(2, 2);
  B[3] = row(1, 2);
  B[4] = row(0, 2);
  B[5] = row(0, 1);
}

struct QpTangent {
  double tau[6], s[6], n[6], D[6];
  double a1, a2, a4, a5;
};

// HE / J2 update at one quadrature point.  A = Cp^-1 at t_n (identity for
// HE), alpha_n = eqps at t_n.  On a plastic step Anp1 / alpha_np1 receive the
// updated state; otherwise they are copies of the inputs.
template <bool PLASTIC_MODEL>
__device__ __forceinline__ void spatial_update(const Mat &mat, const double *F, double J,
                                               const double *A, double alpha_n, QpTangent &o,
                                               double *Anp1, double *alpha_np1) {
  const double mu = mat.mu, kap = mat.kappa;
  const double J13 = cbrt(J);
  const double J23 = 1.0 / (J13 * J13);
  double b[6];
  push_sym(F, A, b);
#pragma unroll
  for (int i = 0; i < 6; i++) b[i] *= J23;
  const double trb = b[0] + b[1] + b[2];
  const double mubar = mu * trb * (1.0 / 3.0);
  double str[6];
#pragma unroll
  for (int i = 0; i < 6; i++) str[i] = mu * b[i];
  str[0] -= mubar;
  str[1] -= mubar;
  str[2] -= mubar;
  double dU, d2U;
  vol_derivs(mat.vol_pot, J, dU, d2U);
  const double pJ = kap * J * dU;
  double r = 1.0;
  o.a4 = 0.0;
  o.a5 = 0.0;
#pragma unroll
  for (int i = 0; i < 6; i++) o.n[i] = o.D[i] = 0.0;
  bool plastic = false;
  if (PLASTIC_MODEL) {
    const double q = sqrt(sdot(str, str));
    const double kn = sqrt(2.0 / 3.0) * (mat.sy + mat.H * alpha_n);
    const double f = q - kn;
    plastic = f > 0.0;
    if (plastic) {
      const double beta0 = 1.0 + mat.H / (3.0 * mubar);
      r = 1.0 - f / (beta0 * q);
      const double iq = 1.0 / q;
#pragma unroll
      for (int i = 0; i < 6; i++) o.n[i] = str[i] * iq;
      // n^2 (symmetric) and its deviator
      const double *n = o.n;
      double n2[6];
      n2[0] = n[0] * n[0] + n[5] * n[5] + n[4] * n[4];
      n2[1] = n[5] * n[5] + n[1] * n[1] + n[3] * n[3];
      n2[2] = n[4] * n[4] + n[3] * n[3] + n[2] * n[2];
      n2[3] = n[5] * n[4] + n[1] * n[3] + n[3] * n[2];
      n2[4] = n[0] * n[4] + n[5] * n[3] + n[4] * n[2];
      n2[5] = n[0] * n[5] + n[5] * n[1] + n[4] * n[3];
      const double t3 = (n2[0] + n2[1] + n2[2]) * (1.0 / 3.0);
#pragma unroll
      for (int i = 0; i < 6; i++) o.D[i] = n2[i];
      o.D[0] -= t3;
      o.D[1] -= t3;
      o.D[2] -= t3;
      o.a4 = -2.0 * kn * mubar / (beta0 * q) -
             (1.0 - kn / q) * 2.0 * mat.H * q * q / (9.0 * beta0 * beta0 * mubar * mubar);
      o.a5 = -2.0 * kn / beta0;
      if (Anp1) {
        const double dgam = f / (2.0 * mubar * beta0);
        *alpha_np1 = alpha_n + sqrt(2.0 / 3.0) * dgam;
        // Cp^-1_{n+1} = J^{2/3} F^-1 (r s_tr/mu + trb/3 1) F^-T
        double Fi[9];
        inv3(F, Fi);
        double be[6];
#pragma unroll
        for (int i = 0; i < 6; i++) be[i] = r * str[i] / mu;
        be[0] += trb / 3.0;
        be[1] += trb / 3.0;
        be[2] += trb / 3.0;
        double Cpi[6];
        push_sym(Fi, be, Cpi);
        const double J2_3 = J13 * J13;
#pragma unroll
        for (int i = 0; i < 6; i++) Anp1[i] = J2_3 * Cpi[i];
      }
    }
    if (!plastic && Anp1) {
#pragma unroll
      for (int i = 0; i < 6; i++) Anp1[i] = A[i];
      *alpha_np1 = alpha_n;
    }
  }
#pragma unroll
  for (int i = 0; i < 6; i++) o.s[i] = r * str[i];
#pragma unroll
  for (int i = 0; i < 6; i++) o.tau[i] = o.s[i];
  o.tau[0] += pJ;
  o.tau[1] += pJ;
  o.tau[2] += pJ;
  o.a1 = 2.0 * mubar * r - 2.0 * pJ;
  o.a2 = kap * (J * dU + J * J * d2U) - (2.0 / 3.0) * mubar * r;
}

// HE with the linear deviatoric potential at one point: tau, the volumetric
// tangent coefficients (s = n = D = 0, a4 = a5 = 0) and b = F F^T in o.n.
__device__ __forceinline__ void linear_dev_update(const Mat &mat, const double *F, double J,
                                                  QpTangent &o) {
  const double G = mat.mu, kap = mat.kappa;
  const double I6[6] = {1, 1, 1, 0, 0, 0};
  double b[6];
  push_sym(F, I6, b);
  double b2[6];
  b2[0] = b[0] * b[0] + b[5] * b[5] + b[4] * b[4];
  b2[1] = b[5] * b[5] + b[1] * b[1] + b[3] * b[3];
  b2[2] = b[4] * b[4] + b[3] * b[3] + b[2] * b[2];
  b2[3] = b[5] * b[4] + b[1] * b[3] + b[3] * b[2];
  b2[4] = b[0] * b[4] + b[5] * b[3] + b[4] * b[2];
  b2[5] = b[0] * b[5] + b[5] * b[1] + b[4] * b[3];
  double dU, d2U;
  vol_derivs(mat.vol_pot, J, dU, d2U);
  const double pJ = kap * J * dU;
#pragma unroll
  for (int i = 0; i < 6; i++) {
    o.tau[i] = G * (b2[i] - b[i]) + (i < 3 ? pJ : 0.0);
    o.s[i] = 0.0;
    o.n[i] = b[i];
    o.D[i] = 0.0;
  }
  o.a1 = -2.0 * pJ;
  o.a2 = kap * (J * dU + J * J * d2U);
  o.a4 = 0.0;
  o.a5 = 0.0;
}

}  // namespace pgb
