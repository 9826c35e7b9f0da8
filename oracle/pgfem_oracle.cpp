// pgfem_oracle.cpp -- CPU oracle (test infrastructure only; see pgfem_oracle.h).
//
// Each function states the reference file:line it restates.  Paths are
// relative to the PGFem3D source tree.
#include "pgfem_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr int DIM = 3;

// ---------------------------------------------------------------------------
// 3x3 helpers.  det3x3 / inv3x3 follow src/utils.cc:478-482 and :542-562
// (inverse refused when |det| < 1e-15); det() of FEMLIB follows
// FEMLIB/src/femlib.cc:366-390.
// ---------------------------------------------------------------------------
double det3x3(const double *m) {
  return ((m[0] * (m[4] * m[8] - m[5] * m[7])) + m[1] * (m[5] * m[6] - m[3] * m[8]) +
          m[2] * (m[3] * m[7] - m[4] * m[6]));
}

int inv3x3(const double *m, double *mi) {
  double A = det3x3(m);
  if (std::fabs(A) >= 1.0e-15) {
    mi[0] = 1 / A * (m[4] * m[8] - m[5] * m[7]);
    mi[1] = -1 / A * (m[1] * m[8] - m[2] * m[7]);
    mi[2] = 1 / A * (m[1] * m[5] - m[2] * m[4]);
    mi[3] = -1 / A * (m[3] * m[8] - m[5] * m[6]);
    mi[4] = 1 / A * (m[0] * m[8] - m[2] * m[6]);
    mi[5] = -1 / A * (m[0] * m[5] - m[2] * m[3]);
    mi[6] = 1 / A * (m[3] * m[7] - m[4] * m[6]);
    mi[7] = -1 / A * (m[0] * m[7] - m[1] * m[6]);
    mi[8] = 1 / A * (m[0] * m[4] - m[1] * m[3]);
    return 0;
  }
  return 1;
}

inline int i4(int i, int j, int k, int l) { return i * 27 + j * 9 + k * 3 + l; }

void matmul(const double *A, const double *B, double *C) {  // C = A B
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = 0;
      for (int k = 0; k < 3; k++) s += A[i * 3 + k] * B[k * 3 + j];
      C[i * 3 + j] = s;
    }
}
void matmulTN(const double *A, const double *B, double *C) {  // C = A^T B
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double s = 0;
      for (int k = 0; k < 3; k++) s += A[k * 3 + i] * B[k * 3 + j];
      C[i * 3 + j] = s;
    }
}
void transpose(const double *A, double *AT) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) AT[j * 3 + i] = A[i * 3 + j];
}
void ident(double *A) {
  for (int i = 0; i < 9; i++) A[i] = 0;
  A[0] = A[4] = A[8] = 1;
}

// ---------------------------------------------------------------------------
// FEMLIB restatement.
// Shape-function derivatives: FEMLIB/src/femlib.cc:213-333 (TETRAHEDRON,
// QTETRAHEDRON).  Quadrature: :571-588 (1-point rule for linear tets, the
// 8-digit 4-point rule for quadratic tets, which FEMLIB forces at
// intg_order 0, :1009-1016).  dN/dX: :403-470.
// ---------------------------------------------------------------------------
struct Quad {
  int nint;
  double ksi[4], eta[4], zet[4], w[4];
};

Quad quad_rule(int nne) {
  Quad q{};
  if (nne == 4) {
    q.nint = 1;
    q.ksi[0] = q.eta[0] = q.zet[0] = 1.0 / 4.0;
    q.w[0] = 1.0 / 6.0;
  } else {
    q.nint = 4;
    const double a = 0.58541020, b = 0.13819660;
    const double k[4] = {a, b, b, b}, e[4] = {b, a, b, b}, z[4] = {b, b, a, b};
    for (int i = 0; i < 4; i++) {
      q.ksi[i] = k[i];
      q.eta[i] = e[i];
      q.zet[i] = z[i];
      q.w[i] = (1.0 / 4.0) / 6.0;
    }
  }
  return q;
}

void dN_dkez(int nne, double ksi, double eta, double zet, double *dN /* nne*3 */) {
  if (nne == 4) {
    const double t[12] = {-1, -1, -1, 1, 0, 0, 0, 1, 0, 0, 0, 1};
    std::memcpy(dN, t, sizeof(t));
    return;
  }
  double *d = dN;
  d[0 * 3 + 0] = 4.0 * (ksi + eta + zet) - 3.0;
  d[0 * 3 + 1] = 4.0 * (eta + ksi + zet) - 3.0;
  d[0 * 3 + 2] = 4.0 * (zet + ksi + eta) - 3.0;
  d[1 * 3 + 0] = 4.0 * ksi - 1.0;
  d[1 * 3 + 1] = 0.0;
  d[1 * 3 + 2] = 0.0;
  d[2 * 3 + 0] = 0.0;
  d[2 * 3 + 1] = 4.0 * eta - 1.0;
  d[2 * 3 + 2] = 0.0;
  d[3 * 3 + 0] = 0.0;
  d[3 * 3 + 1] = 0.0;
  d[3 * 3 + 2] = 4.0 * zet - 1.0;
  d[4 * 3 + 0] = 4.0 * (-2.0 * ksi - eta - zet + 1.0);
  d[4 * 3 + 1] = -4.0 * ksi;
  d[4 * 3 + 2] = -4.0 * ksi;
  d[5 * 3 + 0] = 4.0 * eta;
  d[5 * 3 + 1] = 4.0 * ksi;
  d[5 * 3 + 2] = 0.0;
  d[6 * 3 + 0] = -4.0 * eta;
  d[6 * 3 + 1] = 4.0 * (-ksi - 2.0 * eta - zet + 1.0);
  d[6 * 3 + 2] = -4.0 * eta;
  d[7 * 3 + 0] = -4.0 * zet;
  d[7 * 3 + 1] = -4.0 * zet;
  d[7 * 3 + 2] = 4.0 * (-ksi - eta - 2.0 * zet + 1.0);
  d[8 * 3 + 0] = 4.0 * zet;
  d[8 * 3 + 1] = 0.0;
  d[8 * 3 + 2] = 4.0 * ksi;
  d[9 * 3 + 0] = 0.0;
  d[9 * 3 + 1] = 4.0 * zet;
  d[9 * 3 + 2] = 4.0 * eta;
}

// Returns the isoparametric Jacobian J; dNdX (nne*3).  err set when J <= 0
// (the reference aborts there, FEMLIB/src/femlib.cc:426-429).
double PGFem3D_dNdX(int nne, double ksi, double eta, double zet, const double *X /*nne*3*/,
                    double *dNdX, int *err) {
  double dNk[30];
  dN_dkez(nne, ksi, eta, zet, dNk);
  double dX[9] = {0};
  for (int ib = 0; ib < 3; ++ib)
    for (int ic = 0; ic < 3; ++ic)
      for (int ia = 0; ia < nne; ++ia) dX[ib * 3 + ic] += dNk[ia * 3 + ic] * X[ia * 3 + ib];
  double J = dX[0] * (dX[4] * dX[8] - dX[5] * dX[7]) + dX[1] * (dX[5] * dX[6] - dX[3] * dX[8]) +
             dX[2] * (dX[3] * dX[7] - dX[4] * dX[6]);
  if (J <= 0.0) {
    *err += 1;
    J = 1.0;  // keep going without NaNs; the caller stops on err
  }
  double dXI[9];
  dXI[0] = dX[4] * dX[8] - dX[5] * dX[7];
  dXI[1] = dX[2] * dX[7] - dX[1] * dX[8];
  dXI[2] = dX[1] * dX[5] - dX[2] * dX[4];
  dXI[3] = dX[5] * dX[6] - dX[3] * dX[8];
  dXI[4] = dX[0] * dX[8] - dX[2] * dX[6];
  dXI[5] = dX[2] * dX[3] - dX[0] * dX[5];
  dXI[6] = dX[3] * dX[7] - dX[4] * dX[6];
  dXI[7] = dX[1] * dX[6] - dX[0] * dX[7];
  dXI[8] = dX[0] * dX[4] - dX[1] * dX[3];
  for (int ia = 0; ia < nne; ++ia)
    for (int ib = 0; ib < 3; ++ib) {
      double s = 0.0;
      for (int ic = 0; ic < 3; ++ic) s += 1.0 / J * dNk[ia * 3 + ic] * dXI[ic * 3 + ib];
      dNdX[ia * 3 + ib] = s;
    }
  return J;
}

// F = I + sum_a u_a (x) dN_a: FEMLIB/src/femlib.cc:1289-1325.
void deformation_gradient(int nne, const double *u, const double *dN, double *F) {
  ident(F);
  for (int ia = 0; ia < nne; ia++)
    for (int ib = 0; ib < 3; ++ib)
      for (int ic = 0; ic < 3; ++ic) F[ib * 3 + ic] += u[ia * 3 + ib] * dN[ia * 3 + ic];
}

// ---------------------------------------------------------------------------
// Hyperelasticity.  Deviatoric Mooney-Rivlin stress and stiffness
// (src/new_potentials.cc:333-362, 377-432), U_Common volumetric potential
// (:553-558, 578-583, 599-604) combined as in get_material_stress /
// get_material_stiffness (src/displacement_based_element.cc:1368-1445):
//   S = S_dev + kappa J U'(J) C^-1
//   L = L_dev + kappa (J U' + J^2 U'') C^-1 (x) C^-1 - 2 kappa J U' C^-1_ik C^-1_lj
// Material constants as mapped by src/homogen.cc:176-191 for an isotropic
// neo-Hookean solid: m10 = G/2, m01 = 0, kappa from src/hommat.cc:58-61.
// ---------------------------------------------------------------------------
struct Elast {
  double G, nu, m10, m01, kappa;
  int dev_pot, vol_pot;
};

// U'(J), U''(J) of the volumetric potentials (src/new_potentials.cc:553-622).
void vol_derivs(int vol_pot, double J, double &dU, double &d2U) {
  switch (vol_pot) {
    case 2:  // U_Doll_Schweizerhof_7 = 0.5 (exp(J-1) - ln J - 1)
      dU = (std::exp(-1 + J) - 1. / J) * .5;
      d2U = (std::exp(-1 + J) + 1. / (J * J)) * .5;
      break;
    case 3:  // U_Doll_Schweizerhof_8 = 0.5 (J-1) ln J
      dU = (-1 + J) / (2. * J) + std::log(J) * .5;
      d2U = 1. / J - (-1 + J) / (2. * J * J);
      break;
    default:  // 99: U_Common = 0.5 (J-1)^2
      dU = J - 1.0;
      d2U = 1.0;
  }
}

Elast make_elast(const orc_material *m) {
  Elast e;
  e.G = m->E / (2.0 * (1.0 + m->nu));
  e.nu = m->nu;
  e.m10 = 0.5 * e.G;
  e.m01 = 0.0;
  e.kappa = (2 * e.G * (1 + e.nu)) / (3 * (1 - 2 * e.nu));
  e.dev_pot = m->dev_pot == 2 ? 2 : 1;
  e.vol_pot = (m->vol_pot == 2 || m->vol_pot == 3) && m->model != 2 ? m->vol_pot : 99;
  return e;
}

void he_stress_stiffness(const Elast &el, const double *C, double J, double *S, double *L) {
  double invC[9], I[9];
  inv3x3(C, invC);
  ident(I);
  const double detC = det3x3(C);
  const double trC = C[0] + C[4] + C[8];
  double CC = 0;
  for (int i = 0; i < 9; i++) CC += C[i] * C[i];
  double dUdJ, d2UdJ2;
  vol_derivs(el.vol_pot, J, dUdJ, d2UdJ2);
  if (el.dev_pot == 2) {  // devStress_Linear / matStiff_Linear, src/new_potentials.cc:364-375, 434-452
    for (int i = 0; i < 9; i++) S[i] = el.G * (C[i] - I[i]) + el.kappa * J * dUdJ * invC[i];
    if (!L) return;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        for (int k = 0; k < 3; k++)
          for (int l = 0; l < 3; l++)
            L[i4(i, j, k, l)] = 2 * el.G * I[i * 3 + k] * I[j * 3 + l] +
                                el.kappa * (J * dUdJ + J * J * d2UdJ2) * invC[i * 3 + j] * invC[k * 3 + l] -
                                2.0 * el.kappa * J * dUdJ * invC[i * 3 + k] * invC[l * 3 + j];
    return;
  }
  for (int i = 0; i < 9; i++) {
    S[i] = ((2 * el.m10 * std::pow(detC, -1. / 3.) * (I[i] - 1. / 3. * trC * invC[i])) +
            (2 * el.m01 * std::pow(detC, -2. / 3.) *
             (trC * I[i] - C[i] + 1. / 3. * (CC - trC * trC) * invC[i])));
    S[i] += el.kappa * J * dUdJ * invC[i];
  }
  if (!L) return;
  const double detC1 = std::pow(detC, -1. / 3.), detC2 = detC1 * detC1;
  auto id2 = [](int r, int c) { return r * 3 + c; };
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) {
          double Ld =
              (4 * el.m10 * detC1 *
               ((1. / 9. * trC * invC[id2(i, j)] - 1. / 3. * I[id2(i, j)]) * invC[id2(k, l)] +
                1. / 3. *
                    (trC * invC[id2(i, k)] * invC[id2(l, j)] - I[id2(k, l)] * invC[id2(i, j)]))) +
              (4 * el.m01 * detC2 *
               (I[id2(i, j)] * I[id2(k, l)] - I[id2(i, k)] * I[id2(l, j)] +
                2. / 3. * ((C[id2(i, j)] - trC * I[id2(i, j)]) * invC[id2(k, l)]) -
                ((CC - trC * trC) * (2. / 9. * invC[id2(i, j)] * invC[id2(k, l)] +
                                      1. / 3. * invC[id2(i, k)] * invC[id2(l, j)])) +
                2. / 3. * ((C[id2(k, l)] - trC * I[id2(k, l)]) * invC[id2(i, j)])));
          L[i4(i, j, k, l)] = Ld + el.kappa * (J * dUdJ + J * J * d2UdJ2) * invC[id2(i, j)] * invC[id2(k, l)] -
                              2.0 * el.kappa * J * dUdJ * invC[id2(i, k)] * invC[id2(l, j)];
        }
}

// ---------------------------------------------------------------------------
// Finite-strain J2 plasticity with linear isotropic hardening.
//
// PARITY UNPINNED: the reference's J2 model (src/cm_j2_plasticity.cc:184-214,
// 287-382) calls J2_plasticity_integration_alg / compute_S0_Sbar_public /
// compute_Lbar_public of an external constitutive library that is absent
// from the reference tree.  This is a restatement of the published
// isochoric-split return map of Simo (1988), Simo & Hughes "Computational
// Inelasticity" (1998) Box 9.1, written in the material description with the
// state (Cp^-1, eqps): b_e_trial = J^{-2/3} F Cp^-1 F^T, radial return of
// s = mu dev(b_e), b_e_{n+1} = s/mu + (tr b_e_trial / 3) 1.  The volumetric
// part is kappa J U'(J) C^-1 with the material's potential (vol_derivs).  The
// tangent L = 2 dS/dC is the exact derivative of this update (the published
// Box 9.2 tangent is its symmetrised form); it is checked against central
// differences in tests/.
// ---------------------------------------------------------------------------
void j2_update(const Elast &el, double sy, double Hh, const double *F, const double *state_n,
               double *state_np1, double *S, double *L) {
  const double mu = el.G, kap = el.kappa;
  double C[9], Ci[9];
  matmulTN(F, F, C);
  inv3x3(C, Ci);
  const double J = det3x3(F);
  const double *A = state_n;  // Cp^-1 at n
  const double alpha_n = state_n[9];
  const double J23 = std::pow(J, -2.0 / 3.0);
  double T = 0;
  for (int i = 0; i < 9; i++) T += C[i] * A[i];
  double Str[9];
  for (int i = 0; i < 9; i++) Str[i] = mu * J23 * (A[i] - T / 3.0 * Ci[i]);
  double CA[9], CACA[9], ACA[9], tmp[9];
  matmul(C, A, CA);
  matmul(CA, CA, CACA);
  matmul(A, C, tmp);
  matmul(tmp, A, ACA);
  double Q = CACA[0] + CACA[4] + CACA[8] - T * T / 3.0;
  if (Q < 0) Q = 0;
  const double q = mu * J23 * std::sqrt(Q);
  const double mubar = mu * J23 * T / 3.0;
  const double kn = std::sqrt(2.0 / 3.0) * (sy + Hh * alpha_n);
  const double f = q - kn;
  const bool plastic = f > 0.0;

  double r = 1.0, beta0 = 1.0, dgam = 0.0;
  if (plastic) {
    beta0 = 1.0 + Hh / (3.0 * mubar);
    dgam = f / (2.0 * mubar * beta0);
    r = 1.0 - f / (beta0 * q);
  }
  double dU, d2U;
  vol_derivs(el.vol_pot, J, dU, d2U);
  const double pJ = kap * J * dU;
  for (int i = 0; i < 9; i++) S[i] = pJ * Ci[i] + r * Str[i];

  if (state_np1) {
    if (plastic) {
      const double J2_3 = std::pow(J, 2.0 / 3.0);
      for (int i = 0; i < 9; i++)
        state_np1[i] = J2_3 * (r * Str[i] / mu + (T * J23 / 3.0) * Ci[i]);
      state_np1[9] = alpha_n + std::sqrt(2.0 / 3.0) * dgam;
    } else {
      for (int i = 0; i < 10; i++) state_np1[i] = state_n[i];
    }
  }
  if (!L) return;
  // L_vol in the reference's DISP form (C^-1_ik C^-1_lj product).
  const double cvol1 = kap * (J * dU + J * J * d2U), cvol2 = 2.0 * kap * J * dU;
  double dq[9] = {0}, dr[9] = {0};
  if (plastic) {
    const double c = mu * mu * J23 * J23 / (2.0 * q);
    for (int i = 0; i < 9; i++)
      dq[i] = c * (-(4.0 / 3.0) * Q * Ci[i] + 4.0 * ACA[i] - (4.0 / 3.0) * T * A[i]);
    const double c1 = -kn / (beta0 * q * q);
    const double c2 = -(1.0 - kn / q) * Hh / (3.0 * beta0 * beta0 * mubar * mubar) * (2.0 / 3.0);
    for (int i = 0; i < 9; i++) dr[i] = c1 * dq[i] + c2 * Str[i];
  }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) {
          const int ij = i * 3 + j, kl = k * 3 + l;
          double Lv = cvol1 * Ci[ij] * Ci[kl] - cvol2 * Ci[i * 3 + k] * Ci[l * 3 + j];
          double Isym = 0.5 * (Ci[i * 3 + k] * Ci[j * 3 + l] + Ci[i * 3 + l] * Ci[j * 3 + k]);
          double dS = -(2.0 / 3.0) * Str[ij] * Ci[kl] - (2.0 / 3.0) * mu * J23 * Ci[ij] * A[kl] +
                      (2.0 / 3.0) * mu * J23 * T * Isym;
          L[i4(i, j, k, l)] = Lv + r * dS + Str[ij] * dr[kl];
        }
}

// ---------------------------------------------------------------------------
// Element integrals of the constitutive-model 1-field path, total
// Lagrangian, no thermal coupling:
//   residual:  src/constitutive_model.cc:3322-3539 -> compute_residual_vector :1628-1662
//   stiffness: src/constitutive_model.cc:2474-2692 -> compute_stiffness_matrix :1520-1616
// Shape tensor ST[a][b][i][j] = dN(a,j) delta(b,i): FEMLIB/src/femlib.cc:47-70.
// ---------------------------------------------------------------------------
void compute_residual_vector(double *f, int nne, const double *dN, double detJxW, const double *Fr,
                             const double *eFnMT, const double *eFnM, const double *S,
                             double one_over_Jn) {
  for (int a = 0; a < nne; a++)
    for (int b = 0; b < DIM; b++) {
      double ST[9] = {0};
      for (int j = 0; j < 3; j++) ST[b * 3 + j] = dN[a * 3 + j];
      double AA[9], sAA[9], t1[9], t2[9];
      matmulTN(Fr, ST, AA);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) sAA[i * 3 + j] = 0.5 * (AA[i * 3 + j] + AA[j * 3 + i]);
      matmul(eFnMT, sAA, t1);
      matmul(t1, eFnM, t2);
      double v = 0;
      for (int i = 0; i < 9; i++) v += t2[i] * S[i];
      f[a * DIM + b] += one_over_Jn * detJxW * v;
    }
}

void compute_stiffness_matrix(double *lk, int nne, const double *dN, double detJxW,
                              const double *Fr, const double *eFnMT, const double *eFn,
                              const double *M, const double *FrTFr, const double *eFnM,
                              const double *S, const double *L, const double *dMdu_all,
                              double one_over_Jn) {
  double MI[9];
  inv3x3(M, MI);
  const int nd = nne * DIM;
  for (int a = 0; a < nne; a++)
    for (int b = 0; b < DIM; b++) {
      double STab[9] = {0};
      for (int j = 0; j < 3; j++) STab[b * 3 + j] = dN[a * 3 + j];
      double AA[9], sAA[9], t[9], MTsAAeFn[9], MTsAAeFnM[9];
      matmulTN(Fr, STab, AA);
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) sAA[i * 3 + j] = 0.5 * (AA[i * 3 + j] + AA[j * 3 + i]);
      matmul(eFnMT, sAA, t);
      matmul(t, eFn, MTsAAeFn);
      matmul(MTsAAeFn, M, MTsAAeFnM);
      double MTsAAeFnMS = 0;
      for (int i = 0; i < 9; i++) MTsAAeFnMS += MTsAAeFnM[i] * S[i];
      for (int w = 0; w < nne; w++)
        for (int g = 0; g < DIM; g++) {
          double STwg[9] = {0};
          for (int j = 0; j < 3; j++) STwg[g * 3 + j] = dN[w * 3 + j];
          const double *dMdu = dMdu_all + (w * 3 + g) * 9;
          double BB[9], sBB[9], CC[9], sCC[9];
          matmulTN(Fr, STwg, BB);
          matmulTN(STab, STwg, CC);
          for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
              sBB[i * 3 + j] = 0.5 * (BB[i * 3 + j] + BB[j * 3 + i]);
              sCC[i * 3 + j] = 0.5 * (CC[i * 3 + j] + CC[j * 3 + i]);
            }
          double x1[9], x2[9], X[9], y1[9], y2[9], dCdu[9];
          matmul(eFnMT, FrTFr, x1);
          matmul(x1, eFn, x2);
          matmul(x2, dMdu, X);
          matmul(eFnMT, sBB, y1);
          matmul(y1, eFnM, y2);
          for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
              dCdu[i * 3 + j] = 0.5 * (X[i * 3 + j] + X[j * 3 + i]) + y2[i * 3 + j];
          double LdC[9];
          for (int ij = 0; ij < 9; ij++) {
            double s = 0;
            for (int kl = 0; kl < 9; kl++) s += L[ij * 9 + kl] * dCdu[kl];
            LdC[ij] = s;
          }
          double t1 = 0;
          for (int i = 0; i < 9; i++) t1 += MTsAAeFnM[i] * LdC[i];
          double z1[9], z2[9];
          matmul(eFnMT, sCC, z1);
          matmul(z1, eFnM, z2);
          double t3 = 0;
          for (int i = 0; i < 9; i++) t3 += z2[i] * S[i];
          double Y[9];
          matmul(MTsAAeFn, dMdu, Y);
          double t2 = 0;
          for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) t2 += 0.5 * (Y[i * 3 + j] + Y[j * 3 + i]) * S[i * 3 + j];
          double DpJ = 0;
          for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) DpJ -= MI[j * 3 + i] * dMdu[i * 3 + j];
          const int idx = ((a * DIM + b) * nd) + w * DIM + g;
          lk[idx] += one_over_Jn * detJxW * (t1 + 2.0 * t2 + t3 + DpJ * MTsAAeFnMS);
        }
    }
}

// ---------------------------------------------------------------------------
// Neumann (surface-load) terms of one element, quasi-static:
// compute_Neumann_boundary_conditions (src/fd_residuals.cc:123-273) and
// compute_Neumann_boundary_conditions_stiffnes_mat (src/stiffmat_fd.cc:
// 359-500), both run at the end of the element routine (:439-440 and :602-604).
// The boundary FEMLIB (FEMLIB/src/femlib.cc): face node lists Tet2Tri /
// QTet2QTri (:85-86), the volume-coordinate maps kez_map_Tet (:97-100) and
// set_tet2tri (:796-815), the triangle rules TriIntegrationPoints1/3 (:619-635;
// the boundary takes the volume element's integration order, which FEMLIB
// raises to 1 for quadratic tets: 1 point on linear faces, 3 on quadratic),
// elem_basis_S (:1578-1612: volume N and dN/dX at the point) and
// PGFem3D_dNdX_Vol2Bnd (:486-541: face Jacobian |dX/dxi_1 x dX/dxi_2| and unit
// normal from the face's own basis, compute_dN_dkez :229-246, evaluated at the
// volume coordinates picked through kez_map).
//
// Residual, per point and face node a (volume node V2B[a]), component i:
//   f[a,i] += N_a w (-1) J (F^-T PN)_i,  PN = p n (pressure), t (traction)
// Stiffness, only the component-diagonal entries (a,d; c,d):
//   k[a,d; c,d] += N_a w (-1) J FIT_d,
//   FIT_i = (tr(F^-1 ST) F^-1_ji - dFIdF_ijkl ST_kl) PN'_j,
//   dFIdF_ijkl = -F^-1_jk F^-1_li,  ST_kl = delta_dk dN/dX_{c',l}
// which is 2 g_d (F^-T PN')_d with g_m = sum_l F^-1_lm dN/dX_{c',l}.  As in the
// reference, the shape tensor is taken at volume node c' = c (the face-local
// index, src/stiffmat_fd.cc:486-488), and for a pressure PN' = (p n_0, 0, p n_2)
// (only load value 0 is read and copied to component 2, :419-423, then
// multiplied component-wise by n, :442-445).  Face 3 of the tet: the table maps
// its points onto the plane zet = 0 (face 0's plane) while its nodes are
// {0, 3, 2}; the restatement keeps that.
// ---------------------------------------------------------------------------
const int kTet2Tri[4][3] = {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {0, 3, 2}};
const int kQTet2QTri[4][6] = {{0, 2, 1, 6, 5, 4}, {0, 1, 3, 4, 8, 7}, {1, 2, 3, 5, 9, 8}, {0, 3, 2, 7, 9, 6}};
const int kKezMapTet[4][3] = {{1, 0, 2}, {0, 2, 1}, {0, 1, 2}, {0, 1, 2}};

// Volume shape functions, PGFem3D_N (FEMLIB/src/femlib.cc:158-177).
void shape_N(int nne, double ksi, double eta, double zet, double *N) {
  const double l0 = 1.0 - ksi - eta - zet;
  if (nne == 4) {
    N[0] = l0;
    N[1] = ksi;
    N[2] = eta;
    N[3] = zet;
    return;
  }
  N[0] = (2.0 * l0 - 1.0) * l0;
  N[1] = (2.0 * ksi - 1.0) * ksi;
  N[2] = (2.0 * eta - 1.0) * eta;
  N[3] = (2.0 * zet - 1.0) * zet;
  N[4] = 4.0 * l0 * ksi;
  N[5] = 4.0 * ksi * eta;
  N[6] = 4.0 * l0 * eta;
  N[7] = 4.0 * l0 * zet;
  N[8] = 4.0 * ksi * zet;
  N[9] = 4.0 * eta * zet;
}

// Face basis derivatives (nb x 2), compute_dN_dkez for TRIANGLE / QTRIANGLE.
void face_dN(int nb, double ksi, double eta, double *d) {
  if (nb == 3) {
    const double t[6] = {-1, -1, 1, 0, 0, 1};
    std::memcpy(d, t, sizeof(t));
    return;
  }
  d[0] = 4.0 * eta + 4.0 * ksi - 3.0;
  d[1] = 4.0 * eta + 4.0 * ksi - 3.0;
  d[2] = 4.0 * ksi - 1.0;
  d[3] = 0.0;
  d[4] = 0.0;
  d[5] = 4.0 * eta - 1.0;
  d[6] = 4.0 - 8.0 * ksi - 4.0 * eta;
  d[7] = -4.0 * ksi;
  d[8] = 4.0 * eta;
  d[9] = 4.0 * ksi;
  d[10] = -4.0 * eta;
  d[11] = 4.0 - 4.0 * ksi - 8.0 * eta;
}

void neumann_faces(const orc_problem *P, long e, const double *Xe, const double *u_e, double *fe,
                   double *lk) {
  const int nne = P->nne, nd = nne * 3, nb = nne == 10 ? 6 : 3;
  const int npt = nne == 10 ? 3 : 1;
  const double gk1[1] = {1.0 / 3.0}, ge1[1] = {1.0 / 3.0}, w1[1] = {0.5};
  const double gk3[3] = {2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0}, ge3[3] = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};
  const double w3[3] = {1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0};
  const double *gk = npt == 3 ? gk3 : gk1, *ge = npt == 3 ? ge3 : ge1, *wt = npt == 3 ? w3 : w1;
  for (long k = P->nbc_off[e]; k < P->nbc_off[e + 1]; k++) {
    const int f = P->nbc_face[k], type = P->nbc_type[k];
    const int *v2b = nne == 10 ? kQTet2QTri[f] : kTet2Tri[f];
    const int *km = kKezMapTet[f];
    double Pv[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < type && i < 3; i++) Pv[i] = P->nbc_load[k * 3 + i];
    if (type == 1) Pv[2] = Pv[0];  // Pv[1] stays 0
    for (int ip = 0; ip < npt; ip++) {
      double kez[3] = {0.0, 0.0, 0.0};
      kez[km[0]] = gk[ip];
      kez[km[1]] = ge[ip];
      if (f == 2) kez[km[2]] = 1.0 - gk[ip] - ge[ip];
      double N[10], dN[30];
      shape_N(nne, kez[0], kez[1], kez[2], N);
      int terr = 0;
      PGFem3D_dNdX(nne, kez[0], kez[1], kez[2], Xe, dN, &terr);
      double db[12];
      face_dN(nb, kez[km[0]], kez[km[1]], db);
      double dX[6] = {0, 0, 0, 0, 0, 0};  // dX(ib, ic), ic = 0, 1
      for (int ib = 0; ib < 3; ib++)
        for (int ic = 0; ic < 2; ic++)
          for (int ia = 0; ia < nb; ia++) dX[ib * 2 + ic] += db[ia * 2 + ic] * Xe[v2b[ia] * 3 + ib];
      const double v0 = dX[2] * dX[5] - dX[3] * dX[4];
      const double v1 = dX[1] * dX[4] - dX[0] * dX[5];
      const double v2 = dX[0] * dX[3] - dX[1] * dX[2];
      const double Jf = std::sqrt(v0 * v0 + v1 * v1 + v2 * v2);
      const double n[3] = {v0 / Jf, v1 / Jf, v2 / Jf};
      const double detJxW = Jf * wt[ip];
      double F[9], FI[9];
      deformation_gradient(nne, u_e, dN, F);
      const double J = det3x3(F);
      inv3x3(F, FI);
      double PN[3], PNk[3];
      for (int i = 0; i < 3; i++) {
        PN[i] = type == 1 ? Pv[0] * n[i] : Pv[i];
        PNk[i] = type == 1 ? Pv[i] * n[i] : Pv[i];
      }
      double FTP[3], FTPk[3];  // F^-T PN
      for (int i = 0; i < 3; i++) {
        FTP[i] = FI[0 * 3 + i] * PN[0] + FI[1 * 3 + i] * PN[1] + FI[2 * 3 + i] * PN[2];
        FTPk[i] = FI[0 * 3 + i] * PNk[0] + FI[1 * 3 + i] * PNk[1] + FI[2 * 3 + i] * PNk[2];
      }
      for (int ia = 0; ia < nb; ia++) {
        const int a = v2b[ia];
        const double s = N[a] * detJxW * (-1.0) * J;
        for (int i = 0; i < 3; i++) fe[a * 3 + i] += s * FTP[i];
        if (!lk) continue;
        for (int ic = 0; ic < nb; ic++) {
          const int c = v2b[ic];
          for (int d = 0; d < 3; d++) {
            double g = 0.0;  // shape tensor of volume node ic
            for (int l = 0; l < 3; l++) g += FI[l * 3 + d] * dN[ic * 3 + l];
            lk[(a * 3 + d) * nd + c * 3 + d] += s * 2.0 * g * FTPk[d];
          }
        }
      }
    }
  }
}

// Surface loads of the transient element (compute_Neumann_boundary_conditions
// and compute_Neumann_boundary_conditions_stiffnes_mat with include_inertia,
// src/fd_residuals.cc:123-273, src/stiffmat_fd.cc:359-500): with the load
// values P at t_{n+1}, t_n, t_{n-1} (pressure: (p, 0, p), as above) and the
// displacements at the mid points U_{n+a} = mid(U_n, U_{n+1}),
// U_{n-1+a} = mid(U_{n-1}, U_n), mid(a, b) = (1 - alpha) a + alpha b,
//   f[a,i] += N_a w (dt_np1 (1 - alpha) J_{n+a} (F_{n+a}^-T PN_{n+a})_i
//                    + dt_n alpha J_{n-1+a} (F_{n-1+a}^-T PN_{n-1+a})_i)
//   k[a,d; c,d] += N_a w dt_np1 alpha (1 - alpha) J_{n+a} FIT_d(PN'_{n+a})
// where, as in the reference, the mid-point load mixes the older value
// projected on the normal with the newer raw value:
//   residual   PN_{n+a} = (1 - alpha) PN_n + alpha P_{n+1},  PN_n = p_n n (pressure)
//              PN_{n-1+a} = (1 - alpha) PN_{n-1} + alpha P_n
//   stiffness  PN'_{n+a} = (1 - alpha) PN'_n + alpha P_{n+1},  PN'_n = (p_n n_0, 0, p_n n_2)
// (tractions: the plain mid points).  The stiffness's time step is the
// element's, dt_np1.
void neumann_faces_transient(const orc_problem *P, long e, const double *Xe, const double *u2, const double *u1,
                             const double *u0, double alpha, double dt_np1, double dt_n, double *fe, double *lk) {
  const int nne = P->nne, nd = nne * 3, nb = nne == 10 ? 6 : 3;
  const int npt = nne == 10 ? 3 : 1;
  const double gk1[1] = {1.0 / 3.0}, ge1[1] = {1.0 / 3.0}, w1[1] = {0.5};
  const double gk3[3] = {2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0}, ge3[3] = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};
  const double w3[3] = {1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0};
  const double *gk = npt == 3 ? gk3 : gk1, *ge = npt == 3 ? ge3 : ge1, *wt = npt == 3 ? w3 : w1;
  double Unpa[30], Unma[30];
  for (int i = 0; i < nd; i++) {
    Unpa[i] = (1.0 - alpha) * u1[i] + alpha * u2[i];
    Unma[i] = (1.0 - alpha) * u0[i] + alpha * u1[i];
  }
  for (long k = P->nbc_off[e]; k < P->nbc_off[e + 1]; k++) {
    const int f = P->nbc_face[k], type = P->nbc_type[k];
    const int *v2b = nne == 10 ? kQTet2QTri[f] : kTet2Tri[f];
    const int *km = kKezMapTet[f];
    double P2[3] = {0, 0, 0}, P1[3] = {0, 0, 0}, P0[3] = {0, 0, 0};
    for (int i = 0; i < type && i < 3; i++) {
      P2[i] = P->nbc_load[k * 3 + i];
      P1[i] = P->nbc_load_n[k * 3 + i];
      P0[i] = P->nbc_load_nm1[k * 3 + i];
    }
    if (type == 1) {
      P2[2] = P2[0];
      P1[2] = P1[0];
      P0[2] = P0[0];
    }
    for (int ip = 0; ip < npt; ip++) {
      double kez[3] = {0.0, 0.0, 0.0};
      kez[km[0]] = gk[ip];
      kez[km[1]] = ge[ip];
      if (f == 2) kez[km[2]] = 1.0 - gk[ip] - ge[ip];
      double N[10], dN[30];
      shape_N(nne, kez[0], kez[1], kez[2], N);
      int terr = 0;
      PGFem3D_dNdX(nne, kez[0], kez[1], kez[2], Xe, dN, &terr);
      double db[12];
      face_dN(nb, kez[km[0]], kez[km[1]], db);
      double dX[6] = {0, 0, 0, 0, 0, 0};
      for (int ib = 0; ib < 3; ib++)
        for (int ic = 0; ic < 2; ic++)
          for (int ia = 0; ia < nb; ia++) dX[ib * 2 + ic] += db[ia * 2 + ic] * Xe[v2b[ia] * 3 + ib];
      const double v0 = dX[2] * dX[5] - dX[3] * dX[4];
      const double v1 = dX[1] * dX[4] - dX[0] * dX[5];
      const double v2 = dX[0] * dX[3] - dX[1] * dX[2];
      const double Jf = std::sqrt(v0 * v0 + v1 * v1 + v2 * v2);
      const double n[3] = {v0 / Jf, v1 / Jf, v2 / Jf};
      const double detJxW = Jf * wt[ip];
      double PNn[3], PNnm1[3], PNk[3], PNnpa[3], PNnma[3], PNknpa[3];
      for (int i = 0; i < 3; i++) {
        PNn[i] = type == 1 ? P1[0] * n[i] : P1[i];
        PNnm1[i] = type == 1 ? P0[0] * n[i] : P0[i];
        PNk[i] = type == 1 ? P1[i] * n[i] : P1[i];
        PNnpa[i] = (1.0 - alpha) * PNn[i] + alpha * P2[i];
        PNnma[i] = (1.0 - alpha) * PNnm1[i] + alpha * P1[i];
        PNknpa[i] = (1.0 - alpha) * PNk[i] + alpha * P2[i];
      }
      double Fa[9], Fb[9], FIa[9], FIb[9];
      deformation_gradient(nne, Unpa, dN, Fa);
      deformation_gradient(nne, Unma, dN, Fb);
      const double Ja = det3x3(Fa), Jb = det3x3(Fb);
      inv3x3(Fa, FIa);
      inv3x3(Fb, FIb);
      double Ta[3], Tb[3], Tk[3];
      for (int i = 0; i < 3; i++) {
        Ta[i] = FIa[0 * 3 + i] * PNnpa[0] + FIa[1 * 3 + i] * PNnpa[1] + FIa[2 * 3 + i] * PNnpa[2];
        Tb[i] = FIb[0 * 3 + i] * PNnma[0] + FIb[1 * 3 + i] * PNnma[1] + FIb[2 * 3 + i] * PNnma[2];
        Tk[i] = FIa[0 * 3 + i] * PNknpa[0] + FIa[1 * 3 + i] * PNknpa[1] + FIa[2 * 3 + i] * PNknpa[2];
      }
      for (int ia = 0; ia < nb; ia++) {
        const int a = v2b[ia];
        for (int i = 0; i < 3; i++)
          fe[a * 3 + i] += N[a] * detJxW * (dt_np1 * (1.0 - alpha) * Ja * Ta[i] + dt_n * alpha * Jb * Tb[i]);
        if (!lk) continue;
        const double s = N[a] * detJxW * dt_np1 * alpha * (1.0 - alpha) * Ja;
        for (int ic = 0; ic < nb; ic++) {
          const int c = v2b[ic];
          for (int d = 0; d < 3; d++) {
            double g = 0.0;
            for (int l = 0; l < 3; l++) g += FIa[l * 3 + d] * dN[ic * 3 + l];
            lk[(a * 3 + d) * nd + c * 3 + d] += s * 2.0 * g * Tk[d];
          }
        }
      }
    }
  }
}

}  // namespace

// ===========================================================================
// Crystal plasticity (declared in orc_cp.inc, defined after the helpers).
// ===========================================================================
namespace {
#include "orc_cp.inc"
#include "orc_cp_ref_tangent.inc"
}

extern "C" {

int orc_nint(int nne) { return nne == 10 ? 4 : 1; }

int orc_state_size(int model) {
  switch (model) {
    case ORC_MODEL_J2: return 10;
    case ORC_MODEL_CP: return 10;
    default: return 0;
  }
}

int orc_cm_update(const orc_material *mat, const double *F, double dt, const double *Rcp,
                  const double *state_n, double *state_np1, double *S, double *L, int *iters) {
  Elast el = make_elast(mat);
  if (iters) *iters = 0;
  switch (mat->model) {
    case ORC_MODEL_HE: {
      double C[9];
      matmulTN(F, F, C);
      he_stress_stiffness(el, C, det3x3(F), S, L);
      return 0;
    }
    case ORC_MODEL_J2:
      j2_update(el, mat->sigma_y, mat->H, F, state_n, state_np1, S, L);
      return 0;
    case ORC_MODEL_CP: {
      CpResult res;
      int err = cp_update(mat, el, F, dt, Rcp, state_n, res);
      if (iters) *iters = res.iters;
      if (state_np1) {
        for (int i = 0; i < 9; i++) state_np1[i] = res.pFnp1[i];
        state_np1[9] = res.g;
      }
      for (int i = 0; i < 9; i++) S[i] = res.S[i];
      if (L)
        for (int i = 0; i < 81; i++) L[i] = res.L[i];
      return err;
    }
  }
  return 1;
}

int orc_element(const orc_problem *P, const orc_material *mat, long e, const double *u_e,
                double dt, const double *state_n, double *state_np1, double *fe, double *lk) {
  const int nne = P->nne;
  const int nd = nne * 3;
  const int ns = orc_state_size(mat->model);
  Quad qr = quad_rule(nne);
  double Xe[30];
  for (int a = 0; a < nne; a++)
    for (int i = 0; i < 3; i++) Xe[a * 3 + i] = P->X[(long)P->conn[e * nne + a] * 3 + i];
  Elast el = make_elast(mat);
  int err = 0;
  for (int i = 0; i < nd; i++) fe[i] = 0.0;
  if (lk)
    for (int i = 0; i < nd * nd; i++) lk[i] = 0.0;
  std::vector<double> dMdu_all(nd * 9, 0.0);
  for (int ip = 0; ip < qr.nint; ip++) {
    double dN[30];
    int terr = 0;
    double detJ = PGFem3D_dNdX(nne, qr.ksi[ip], qr.eta[ip], qr.zet[ip], Xe, dN, &terr);
    if (terr) { err += terr; break; }
    const double detJxW = detJ * qr.w[ip];
    double Fr[9];
    deformation_gradient(nne, u_e, dN, Fr);
    if (P->F0)  // cm_add_macro_F, src/constitutive_model.cc:247-252
      for (int i = 0; i < 9; i++) Fr[i] += P->F0[i];
    if (det3x3(Fr) <= 0.0) { err += 1; break; }  // getJacobian, src/utils.cc:513-527

    const double *sn = state_n ? state_n + (long)ip * ns : nullptr;
    double *snp1 = state_np1 ? state_np1 + (long)ip * ns : nullptr;
    double S[9], L[81], M[9], pFnp1[9];
    ident(M);
    ident(pFnp1);
    std::fill(dMdu_all.begin(), dMdu_all.end(), 0.0);
    if (mat->model == ORC_MODEL_CP) {
      CpResult res;
      const double *Rcp = P->R_cp ? P->R_cp + e * 9 : nullptr;
      int cerr = cp_update(mat, el, Fr, dt, Rcp, sn, res);
      if (cerr) { err += cerr; break; }
      if (snp1) {
        for (int i = 0; i < 9; i++) snp1[i] = res.pFnp1[i];
        snp1[9] = res.g;
      }
      for (int i = 0; i < 9; i++) { S[i] = res.S[i]; pFnp1[i] = res.pFnp1[i]; }
      for (int i = 0; i < 81; i++) L[i] = res.L[i];
      if (inv3x3(pFnp1, M)) { err += 1; break; }
      if (lk) cp_dMdu(res, nne, dN, dMdu_all.data());
    } else {
      double stmp[10];
      int cerr = orc_cm_update(mat, Fr, dt, nullptr, sn, snp1 ? snp1 : stmp, S, lk ? L : nullptr, nullptr);
      if (cerr) { err += cerr; break; }
    }
    const double pJ = det3x3(pFnp1);
    double MT[9];
    transpose(M, MT);
    compute_residual_vector(fe, nne, dN, detJxW, Fr, MT, M, S, pJ);
    if (lk) {
      double eFn[9], FrTFr[9];
      ident(eFn);
      matmulTN(Fr, Fr, FrTFr);
      compute_stiffness_matrix(lk, nne, dN, detJxW, Fr, MT, eFn, M, FrTFr, M, S, L,
                               dMdu_all.data(), pJ);
    }
  }
  // diagonal check of the stiffness (src/constitutive_model.cc:2682-2687)
  if (lk && !err)
    for (int a = 0; a < nd; a++)
      if (!std::isnormal(lk[a * nd + a])) err++;
  // surface loads after the element integrals (src/fd_residuals.cc:439,
  // src/stiffmat_fd.cc:602)
  if (!err && P->nbc_off) neumann_faces(P, e, Xe, u_e, fe, lk);
  return err;
}

long orc_generate_dof_ids(long nn, long ne, int nne, const int *conn, const long *Pr, long *id) {
  std::vector<char> visited(nn * 3, 0);
  long ndof = 1;
  for (long e = 0; e < ne; e++) {
    long id_adder = 0;
    for (int i = 0; i < nne; i++) {
      const long n = conn[e * nne + i];
      for (int j = 0; j < 3; j++) {
        const long di = n * 3 + j;
        if (visited[di]) continue;
        if (id[di] < 0) {
          visited[di] = 1;
        } else if (id[di] == 1) {
          id[di] = 0;
          visited[di] = 1;
        } else {
          if (Pr && Pr[n] != -1) {
            const long pdi = Pr[n] * 3 + j;
            if (!visited[pdi]) {
              id[pdi] = ndof + id_adder;
              visited[pdi] = 1;
              id_adder++;
            }
            id[di] = id[pdi];
            visited[di] = 1;
          } else {
            id[di] = ndof + id_adder;
            id_adder++;
            visited[di] = 1;
          }
        }
      }
    }
    ndof += id_adder;
  }
  // periodic nodes outside every element (src/generate_dof_ids.cc:120-150)
  for (long n = 0; n < nn; n++)
    for (int j = 0; j < 3; j++)
      if (!visited[n * 3 + j] && Pr && Pr[n] != -1) {
        id[n * 3 + j] = id[Pr[n] * 3 + j];
        visited[n * 3 + j] = 1;
      }
  return ndof - 1;
}

long orc_psparse_apai(long ne, int nne, const int *conn, const long *id, long ndof, int *Ap,
                      int *Ai) {
  // countDof: ncols[lid] += number of free dofs of the element
  std::vector<long> ncols(ndof, 0);
  std::vector<long> lids;
  for (long e = 0; e < ne; e++) {
    lids.clear();
    for (int a = 0; a < nne; a++)
      for (int j = 0; j < 3; j++) {
        long lid = id[(long)conn[e * nne + a] * 3 + j];
        if (lid > 0) lids.push_back(lid - 1);
      }
    for (long l : lids) ncols[l] += (long)lids.size();
  }
  std::vector<std::vector<long>> AA(ndof);
  for (long r = 0; r < ndof; r++) AA[r].reserve(ncols[r]);
  for (long e = 0; e < ne; e++) {
    lids.clear();
    for (int a = 0; a < nne; a++)
      for (int j = 0; j < 3; j++) {
        long lid = id[(long)conn[e * nne + a] * 3 + j];
        if (lid > 0) lids.push_back(lid - 1);
      }
    for (long l : lids)
      for (long g : lids) AA[l].push_back(g);  // gid == lid on one rank
  }
  long nnz = 0;
  Ap[0] = 0;
  for (long r = 0; r < ndof; r++) {
    std::sort(AA[r].begin(), AA[r].end());
    long cnt = 0;
    for (size_t j = 0; j < AA[r].size(); j++)
      if (j + 1 == AA[r].size() || AA[r][j] < AA[r][j + 1]) {
        if (Ai) Ai[nnz + cnt] = (int)AA[r][j];
        cnt++;
      }
    nnz += cnt;
    Ap[r + 1] = (int)nnz;
    std::vector<long>().swap(AA[r]);
  }
  return nnz;
}

}  // extern "C"

namespace {

// Element displacement gather: def_elem_total, src/utils.cc:1391-1412 (with
// u_np1 + d_u merged into one free-DOF vector u).
void gather_u(const orc_problem *P, long e, const double *u, const double *u_presc, double *ue) {
  for (int a = 0; a < P->nne; a++)
    for (int j = 0; j < 3; j++) {
      const long id = P->id[(long)P->conn[e * P->nne + a] * 3 + j];
      ue[a * 3 + j] = id == 0 ? 0.0 : (id > 0 ? u[id - 1] : (u_presc ? u_presc[-id - 1] : 0.0));
    }
}

// PLoc_Sparse restated for one rank (src/PLoc_Sparse.cc:50-125): rows and
// columns with a non-free DOF are dropped, the rest is added into the CSR
// values at (row, col) found by binary search in the row's sorted columns.
void scatter(const orc_problem *P, long e, const double *fe, const double *lk, double *R,
             double *K) {
  const int nd = P->nne * 3;
  long gid[30];
  for (int a = 0; a < P->nne; a++)
    for (int j = 0; j < 3; j++) gid[a * 3 + j] = P->id[(long)P->conn[e * P->nne + a] * 3 + j] - 1;
  for (int i = 0; i < nd; i++) {
    if (gid[i] < 0) continue;
    if (R) R[gid[i]] += fe[i];  // fd_res_assemble, src/fd_residuals.cc:58-73
    if (!K || !lk) continue;
    const int *row = P->Ai + P->Ap[gid[i]];
    const int len = P->Ap[gid[i] + 1] - P->Ap[gid[i]];
    for (int j = 0; j < nd; j++) {
      if (gid[j] < 0) continue;
      const int *pos = std::lower_bound(row, row + len, (int)gid[j]);
      K[P->Ap[gid[i]] + (pos - row)] += lk[i * nd + j];
    }
  }
}

// Greedy element colouring: no two elements of one colour share a free DOF
// (the rows of R and K they add into).  Sharing a node implies sharing its
// DOFs, and on periodic meshes distinct slave and master nodes share DOF ids,
// so the test is on DOF ids, not node ids.
std::vector<std::vector<long>> colour_elements(const orc_problem *P, long e0, long e1) {
  std::vector<std::vector<long>> colours;
  std::vector<std::vector<char>> used;  // per colour: free-DOF mask (lazy)
  auto touches = [&](long e, const std::vector<char> &mask) {
    for (int a = 0; a < P->nne; a++)
      for (int c = 0; c < 3; c++) {
        const long id = P->id[(long)P->conn[e * P->nne + a] * 3 + c];
        if (id > 0 && mask[id - 1]) return true;
      }
    return false;
  };
  for (long e = e0; e < e1; e++) {
    size_t c = 0;
    for (; c < colours.size(); c++)
      if (!touches(e, used[c])) break;
    if (c == colours.size()) {
      colours.emplace_back();
      used.emplace_back(std::max<long>(P->ndof, 1), 0);
    }
    colours[c].push_back(e);
    for (int a = 0; a < P->nne; a++)
      for (int k = 0; k < 3; k++) {
        const long id = P->id[(long)P->conn[e * P->nne + a] * 3 + k];
        if (id > 0) used[c][id - 1] = 1;
      }
  }
  return colours;
}

template <class Body>
int run_elements(const orc_problem *P, long e0, long e1, int nthreads, Body body) {
  if (nthreads <= 1) {
    int err = 0;
    for (long e = e0; e < e1; e++) err += body(e);
    return err;
  }
  auto colours = colour_elements(P, e0, e1);
  std::atomic<int> err{0};
  for (auto &col : colours) {
    std::atomic<long> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++)
      th.emplace_back([&]() {
        int lerr = 0;
        for (;;) {
          long k = next.fetch_add(64);
          if (k >= (long)col.size()) break;
          long kend = std::min<long>(k + 64, col.size());
          for (long i = k; i < kend; i++) lerr += body(col[i]);
        }
        err += lerr;
      });
    for (auto &t : th) t.join();
  }
  return err.load();
}

}  // namespace

// The crystal-plasticity tangent dM/dF (M = pF_n pF_{n+1}^-1) at F_{n+1} from
// the state at t_n (pF_n 9, g_n) two ways: the oracle's implicit derivative of
// its Newton system (CpResult::dMdF) and the reference's own formula
// (cp_ref_dMdF) fed with the converged state, eF_n = F_n pF_n^-1 and
// eF_{n+1} = F_{n+1} pF_{n+1}^-1.  Test hook.
extern "C" int orc_cp_tangent_pair(const orc_material *mat, const double *Fn, const double *Fnp1, double dt,
                                   const double *Rcp, const double *state_n, double *dMdF_newton,
                                   double *dMdF_ref) {
  Elast el = make_elast(mat);
  CpResult res;
  if (cp_update(mat, el, Fnp1, dt, Rcp, state_n, res)) return 1;
  double P[kNSlip][9];
  cp_schmid(Rcp, P);
  double pFnI[9], pFnp1I[9], eFn[9], eFnp1[9], C[9], S[9], CS[9];
  if (inv3x3(state_n, pFnI) || inv3x3(res.pFnp1, pFnp1I)) return 1;
  matmul(Fn, pFnI, eFn);
  matmul(Fnp1, pFnp1I, eFnp1);
  matmulTN(eFnp1, eFnp1, C);
  he_stress_stiffness(el, C, det3x3(eFnp1), S, nullptr);
  matmul(C, S, CS);
  double tau[kNSlip], gd[kNSlip];
  for (int a = 0; a < kNSlip; a++) {
    double t = 0.0;
    for (int i = 0; i < 9; i++) t += CS[i] * P[a][i];
    tau[a] = t;
    gd[a] = res.dgam[a] / dt;
  }
  for (int i = 0; i < 81; i++) dMdF_newton[i] = res.dMdF[i];
  return cp_ref_dMdF(mat, el, eFn, eFnp1, res.M, state_n[9], res.g, tau, gd, P, dt, dMdF_ref);
}

extern "C" int orc_assemble(const orc_problem *P, const orc_material *mat, const double *u,
                            const double *u_presc, double dt, const double *state_n,
                            double *state_np1, double *R, double *K, long e0, long e1,
                            int nthreads, int *iters) {
  const int nd = P->nne * 3;
  const int nint = orc_nint(P->nne);
  const int ns = orc_state_size(mat->model);
  return run_elements(P, e0, e1, nthreads, [&](long e) -> int {
    double ue[30], fe[30];
    std::vector<double> lk(K ? nd * nd : 0);
    gather_u(P, e, u, u_presc, ue);
    const double *sn = ns ? state_n + e * nint * ns : nullptr;
    double *snp1 = ns && state_np1 ? state_np1 + e * nint * ns : nullptr;
    int err = orc_element(P, mat, e, ue, dt, sn, snp1, fe, K ? lk.data() : nullptr);
    if (iters && mat->model == ORC_MODEL_CP) {
      // iteration counts are recomputed cheaply by a separate call (rare, tests)
    }
    if (!err) scatter(P, e, fe, K ? lk.data() : nullptr, R, K);
    return err;
  });
}

#include "orc_bform.inc"

// ---------------------------------------------------------------------------
// Three-field (CM3F) element of the hyperelastic model (and of this library's
// J2 model, whose isochoric return map gives the deviatoric S, L from the
// state at t_n, the state at t_{n+1} written to state_np1; the integration's
// volume factor (theta / J)^(1/3), src/constitutive_model.cc:813-816, leaves an
// isochoric update unchanged), quasi-static, total Lagrangian, one rank: the element loop of src/constitutive_model.cc:
// 695-881 with CM_ThreeField (src/constitutive_model_3f.cc:47-491) and the
// condensation condense_K_3F_to_1F / condense_F_3F_to_1F
// (src/condense.cc:300-385).  CM3F carries one pressure P and one volume
// theta per element (get_3f_pressure_volume_number,
// src/three_field_element.cc:1399-1409), so Np = Nt = 1.  For HE, M = pF^-1
// = I, eF = F, eFn = I, dM/du = dM/dtheta = 0, theta_n = tJn = Jn = 1, and
// set_scalars' default dt_alpha_1_minus_alpha = -1
// (include/constitutive_model_3f.h:58-65).  eSd, Ld: the deviatoric PK2 and
// tangent of the elasticity (update_elasticity_dev, include/
// constitutive_model.h:413-435: the material's potential without its
// volumetric part); dU = kappa U'(theta), ddU = kappa U''(theta)
// (include/constitutive_model.h:319-383).  Per point, with G the shape tensor
// of (a, b), Psi = sym(G^T F), w = detJxW:
//   Ru  += (Psi:eSd + P J tr(G F^-1)) w            Rp += (J - theta) w
//   Rt  += (dU - P) w
//   Kuu -= -w (Psi_ab:Ld:Psi_wg + P J (tr(G_ab F^-1) tr(G_wg F^-1)
//             - tr(G_ab F^-1 G_wg F^-1)) + sym(G_ab^T G_wg):eSd)
//   Kup -= -w J tr(F^-1 G)   Ktp -= w   Ktt -= -w ddU   (Kut = Ktu = 0)
// then, with Kpu = Kup^T and Kpt = Ktp^T:
//   K = Kuu - Kup Ktp^-1 Ktu + Kup Ktp^-1 Ktt Kpt^-1 Kpu - Kut Kpt^-1 Kpu
//   f = fu + Kup Ktp^-1 Ktt Kpt^-1 fp - Kup Ktp^-1 ft - Kut Kpt^-1 fp.
// blk (may be NULL) receives fp, ft, Ktp, Ktt and Kup[nd].
// ---------------------------------------------------------------------------
// The uncondensed blocks of one three-field element: fu (nd), Kuu (nd*nd, may
// be null), and in blk fp, ft, Ktp, Ktt, Kup (nd).
int element_3f_blocks(const orc_problem *P, const orc_material *mat, long e, const double *u_e, double Pe,
                      double theta, const double *state_n, double *state_np1, double *fu_out, double *lk,
                      double *blk) {
  if (mat->model != ORC_MODEL_HE && mat->model != ORC_MODEL_J2) return 1;
  if (mat->model == ORC_MODEL_J2 && !state_n) return 1;
  const int ns = orc_state_size(mat->model);
  const int nne = P->nne, nd = nne * 3;
  Quad qr = quad_rule(nne);
  double Xe[30];
  for (int a = 0; a < nne; a++)
    for (int i = 0; i < 3; i++) Xe[a * 3 + i] = P->X[(long)P->conn[e * nne + a] * 3 + i];
  Elast el = make_elast(mat);
  Elast dev = el;
  dev.kappa = 0.0;  // the deviatoric part alone
  double dUs, d2Us;
  vol_derivs(el.vol_pot, theta, dUs, d2Us);
  const double dU = el.kappa * dUs, ddU = el.kappa * d2Us;
  std::vector<double> fu(nd, 0.0), Kup(nd, 0.0), Kuu(lk ? nd * nd : 0, 0.0);
  double fp = 0.0, ft = 0.0, Ktp = 0.0, Ktt = 0.0;
  int err = 0;
  for (int ip = 0; ip < qr.nint; ip++) {
    double dN[30];
    int terr = 0;
    const double detJ = PGFem3D_dNdX(nne, qr.ksi[ip], qr.eta[ip], qr.zet[ip], Xe, dN, &terr);
    if (terr) { err += terr; break; }
    const double w = detJ * qr.w[ip];
    double F[9], Fi[9], C[9], S[9], L[81];
    deformation_gradient(nne, u_e, dN, F);
    if (P->F0)
      for (int i = 0; i < 9; i++) F[i] += P->F0[i];
    const double J = det3x3(F);
    if (J <= 0.0 || inv3x3(F, Fi)) { err += 1; break; }
    if (mat->model == ORC_MODEL_J2) {
      double stmp[10];
      j2_update(dev, mat->sigma_y, mat->H, F, state_n + (long)ip * ns,
                state_np1 ? state_np1 + (long)ip * ns : stmp, S, lk ? L : nullptr);
    } else {
      matmulTN(F, F, C);
      he_stress_stiffness(dev, C, J, S, lk ? L : nullptr);
    }
    // per (a, b): Psi = sym(G^T F) and tr(G F^-1), G_ij = delta_ib dN_a,j
    std::vector<double> Psi(nd * 9), trGFi(nd), GFi(nd * 9);
    for (int a = 0; a < nne; a++)
      for (int b = 0; b < 3; b++) {
        const int r = a * 3 + b;
        double G[9] = {0}, A[9], X[9];
        for (int j = 0; j < 3; j++) G[b * 3 + j] = dN[a * 3 + j];
        matmulTN(G, F, A);
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) Psi[r * 9 + i * 3 + j] = 0.5 * (A[i * 3 + j] + A[j * 3 + i]);
        matmul(G, Fi, X);
        for (int i = 0; i < 9; i++) GFi[r * 9 + i] = X[i];
        trGFi[r] = X[0] + X[4] + X[8];
        double PsiS = 0.0;
        for (int i = 0; i < 9; i++) PsiS += Psi[r * 9 + i] * S[i];
        fu[r] += (PsiS + Pe * J * trGFi[r]) * w;
        Kup[r] -= -w * J * trGFi[r];
      }
    fp += (J - theta) * w;
    ft += (dU - Pe) * w;
    Ktp -= w;
    Ktt -= -w * ddU;
    if (!lk) continue;
    for (int r = 0; r < nd; r++) {
      const int a = r / 3, b = r % 3;
      double PsiL[9];
      for (int ij = 0; ij < 9; ij++) {
        double v = 0.0;
        for (int kl = 0; kl < 9; kl++) v += Psi[r * 9 + kl] * L[kl * 9 + ij];
        PsiL[ij] = v;
      }
      for (int c = 0; c < nd; c++) {
        const int wn = c / 3, g = c % 3;
        double PLP = 0.0;
        for (int ij = 0; ij < 9; ij++) PLP += PsiL[ij] * Psi[c * 9 + ij];
        double tr2 = 0.0;  // tr(G_ab F^-1 G_wg F^-1)
        for (int i = 0; i < 3; i++)
          for (int k = 0; k < 3; k++) tr2 += GFi[r * 9 + i * 3 + k] * GFi[c * 9 + k * 3 + i];
        // sym(G_ab^T G_wg):eSd, (G_ab^T G_wg)_ij = delta_bg dN_a,i dN_w,j
        double DPsiS = 0.0;
        if (b == g)
          for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
              DPsiS += 0.5 * (dN[a * 3 + i] * dN[wn * 3 + j] + dN[a * 3 + j] * dN[wn * 3 + i]) * S[i * 3 + j];
        Kuu[r * nd + c] -= -w * (PLP + Pe * J * (trGFi[r] * trGFi[c] - tr2) + DPsiS);
      }
    }
  }
  if (err) return err;
  for (int r = 0; r < nd; r++) fu_out[r] = fu[r];
  if (lk)
    for (int i = 0; i < nd * nd; i++) lk[i] = Kuu[i];
  blk[0] = fp;
  blk[1] = ft;
  blk[2] = Ktp;
  blk[3] = Ktt;
  for (int r = 0; r < nd; r++) blk[4 + r] = Kup[r];
  return 0;
}

// Static condensation of the element's (P, theta) for npres = nVol = 1
// (condense_F_3F_to_1F / condense_K_3F_to_1F, src/constitutive_model_3f.cc,
// with Ktu = Kut = 0): f = fu - Kup Ktp^-1 (ft - Ktt Kpt^-1 fp),
// k = Kuu + Kup Ktp^-1 Ktt Kpt^-1 Kpu.
void condense_3f(int nd, const double *fu, const double *Kuu, const double *blk, double *fe, double *lk) {
  const double fp = blk[0], ft = blk[1], Ktp = blk[2], Ktt = blk[3], Kpt = Ktp;
  const double KtpI = 1.0 / Ktp, KptI = 1.0 / Kpt;
  const double *Kup = blk + 4;
  for (int r = 0; r < nd; r++) fe[r] = fu[r] + Kup[r] * KtpI * Ktt * KptI * fp - Kup[r] * KtpI * ft;
  if (lk)
    for (int r = 0; r < nd; r++)
      for (int c = 0; c < nd; c++) lk[r * nd + c] = Kuu[r * nd + c] + Kup[r] * KtpI * Ktt * KptI * Kup[c];
}

extern "C" int orc_element_3f(const orc_problem *P, const orc_material *mat, long e, const double *u_e,
                              double Pe, double theta, const double *state_n, double *state_np1, double *fe,
                              double *lk, double *blk) {
  const int nd = P->nne * 3;
  std::vector<double> fu(nd), Kuu(lk ? nd * nd : 0), b(4 + nd);
  const int err = element_3f_blocks(P, mat, e, u_e, Pe, theta, state_n, state_np1, fu.data(),
                                    lk ? Kuu.data() : nullptr, b.data());
  if (err) return err;
  condense_3f(nd, fu.data(), lk ? Kuu.data() : nullptr, b.data(), fe, lk);
  if (blk)
    for (int i = 0; i < 4 + nd; i++) blk[i] = b[i];
  if (P->nbc_off) {
    double Xe[30];
    for (int a = 0; a < P->nne; a++)
      for (int i = 0; i < 3; i++) Xe[a * 3 + i] = P->X[(long)P->conn[e * P->nne + a] * 3 + i];
    neumann_faces(P, e, Xe, u_e, fe, lk);
  }
  return 0;
}

// Global assembly of the three-field element: P_e, theta_e per element.
extern "C" int orc_assemble_3f(const orc_problem *P, const orc_material *mat, const double *u,
                               const double *u_presc, const double *Pe, const double *theta,
                               const double *state_n, double *state_np1, double *R, double *K) {
  const int nd = P->nne * 3;
  const int nint = orc_nint(P->nne), ns = orc_state_size(mat->model);
  return run_elements(P, 0, P->ne, 1, [&](long e) -> int {
    double ue[30], fe[30];
    std::vector<double> lk(K ? nd * nd : 0);
    gather_u(P, e, u, u_presc, ue);
    const double *sn = state_n ? state_n + e * nint * ns : nullptr;
    double *snp1 = state_np1 ? state_np1 + e * nint * ns : nullptr;
    int err = orc_element_3f(P, mat, e, ue, Pe[e], theta[e], sn, snp1, fe, K ? lk.data() : nullptr, nullptr);
    if (!err) scatter(P, e, fe, K ? lk.data() : nullptr, R, K);
    return err;
  });
}

// Increments of the element pressure and volume after a displacement
// increment du (free-DOF vector; prescribed values unchanged):
// compute_d_theta_dP (src/constitutive_model_3f.cc:494-549) with the blocks
// at u, Ktu = 0 for HE:
//   d_theta = -Kpt^-1 (Kpu du + fp),  dP = -Ktp^-1 (ft + Ktu du + Ktt d_theta).
extern "C" int orc_update_3f(const orc_problem *P, const orc_material *mat, const double *u,
                             const double *u_presc, const double *du, const double *Pe, const double *theta,
                             const double *state_n, double *dP, double *dtheta) {
  const int nd = P->nne * 3;
  const int nint = orc_nint(P->nne), ns = orc_state_size(mat->model);
  int err = 0;
  for (long e = 0; e < P->ne; e++) {
    double ue[30], due[30], fe[30], blk[4 + 30];
    gather_u(P, e, u, u_presc, ue);
    gather_u(P, e, du, nullptr, due);
    const double *sn = state_n ? state_n + e * nint * ns : nullptr;
    const int r = orc_element_3f(P, mat, e, ue, Pe[e], theta[e], sn, nullptr, fe, nullptr, blk);
    if (r) { err += r; continue; }
    const double fp = blk[0], ft = blk[1], Ktp = blk[2], Ktt = blk[3], Kpt = Ktp;
    double Kpu_du = 0.0;
    for (int i = 0; i < nd; i++) Kpu_du += blk[4 + i] * due[i];
    dtheta[e] = -(1.0 / Kpt) * (Kpu_du + fp);
    dP[e] = -(1.0 / Ktp) * ft - (1.0 / Ktp) * Ktt * dtheta[e];
  }
  return err;
}

// ---------------------------------------------------------------------------
// Transient (inertia) 1-field element of the hyperelastic model, one rank:
// residual_with_inertia / stiffness_with_inertia (src/dynamics.cc:183-432),
// which PGFem3D runs instead of the quasi-static element whenever the
// material density exceeds 1e-16 (src/stiffmat_fd.cc:549-565,
// src/fd_residuals.cc:494-500), with the constitutive-model parts
// residuals_el_constitutive_model_w_inertia_1f (src/constitutive_model.cc:
// 2803-2958), residuals_el_constitutive_model_n_plus_alpha (:1905-1978) and
// stiffness_el_constitutive_model_w_inertia_1f (:2024-2170).  For HE the
// plastic parts are the identity (HE_PARAM::get_pF,
// src/plasticity_model_none.cc:282-291), and F at t_n, t_{n-1} are those of the
// given displacements.  mid(a, b) = (1 - alpha) a + alpha b (mid_point_rule,
// src/utils.cc:3213-3223).
//   f  = -dt_np1 (1 - alpha) r(F(n+alpha)) - dt_n alpha r(F(n-1+alpha)) - f_i
//   f_i[a,b] = rho / (dt_np1 dt_n) sum_q N_a du_b w,
//       du = sum_c N_c (dt_n u_np1 - (dt_np1 + dt_n) u_n + dt_np1 u_nm1)_c
//   k  = -rho / dt_np1 sum_q N_a N_c w delta_bd - alpha (1 - alpha) dt_np1 k(F(n+alpha))
// with r, k the quasi-static element integrals at the given F (M = I); the
// body force of the manufactured-solution tests is zero here.
//
// Crystal plasticity (orc_assemble_transient_state): the point update runs at
// F_{n+1} from the state at t_n (run_integration_algorithm, :2886-2888), then
// each mid point takes the mid-point plastic part, pF(n+alpha) =
// mid(pF_n, pF_{n+1}) and pF(n-1+alpha) = mid(pF_{n-1}, pF_n) (get_pF at
// levels 2, 1, 0, :2893-2895), M = pF^-1, eF = F M, the elastic stress at eF
// and the factor det pF (residuals_el_constitutive_model_n_plus_alpha,
// :1926-1975).  The stiffness is compute_stiffness_matrix at n+alpha with
// M(n+alpha) (:2120-2156) and dM/du the derivative of M(n+alpha) through
// pF_{n+1}, divided by alpha (the blend's alpha (1 - alpha) carries it):
//   dM(n+alpha)/du / alpha = M(n+alpha) pF_{n+1} d(pF_{n+1}^-1)/du pF_{n+1} M(n+alpha),
// with d(pF_{n+1}^-1)/du the consistent derivative of the local update (the
// reference evaluates its own compute_dMdu formula at the mid-point values
// instead, plasticity_compute_dMdu_npa, src/plasticity_model.cc:779-866).
// ---------------------------------------------------------------------------
extern "C" int orc_assemble_transient_state(const orc_problem *P, const orc_material *mat, const double *u_np1,
                                            const double *u_n, const double *u_nm1, const double *p_np1,
                                            const double *p_n, const double *p_nm1, double alpha, double dt_np1,
                                            double dt_n, double rho, const double *state_nm1,
                                            const double *state_n, double *state_np1, double *R, double *K) {
  const bool cp = mat->model == ORC_MODEL_CP;
  if (mat->model != ORC_MODEL_HE && !(cp && state_nm1 && state_n)) return 1;
  const int nne = P->nne, nd = nne * 3;
  int err = 0;
  Quad qr = quad_rule(nne);
  Elast el = make_elast(mat);
  for (long e = 0; e < P->ne; e++) {
    double u2[30], u1[30], u0[30], Xe[30];
    gather_u(P, e, u_np1, p_np1, u2);
    gather_u(P, e, u_n, p_n, u1);
    gather_u(P, e, u_nm1, p_nm1, u0);
    for (int a = 0; a < nne; a++)
      for (int i = 0; i < 3; i++) Xe[a * 3 + i] = P->X[(long)P->conn[e * nne + a] * 3 + i];
    std::vector<double> fe(nd, 0.0), fi(nd, 0.0), lk(K ? nd * nd : 0, 0.0), kI(K ? nd * nd : 0, 0.0),
        lk1(K ? nd * nd : 0, 0.0);
    double I3[9];
    ident(I3);
    int eerr = 0;
    for (int ip = 0; ip < qr.nint && !eerr; ip++) {
      double dN[30], N[10];
      int terr = 0;
      const double detJ = PGFem3D_dNdX(nne, qr.ksi[ip], qr.eta[ip], qr.zet[ip], Xe, dN, &terr);
      if (terr) { eerr += terr; break; }
      const double w = detJ * qr.w[ip];
      shape_N(nne, qr.ksi[ip], qr.eta[ip], qr.zet[ip], N);
      double F2[9], F1[9], F0[9], Fnpa[9], Fnma[9];
      deformation_gradient(nne, u2, dN, F2);
      deformation_gradient(nne, u1, dN, F1);
      deformation_gradient(nne, u0, dN, F0);
      for (int i = 0; i < 9; i++) {
        Fnpa[i] = (1.0 - alpha) * F1[i] + alpha * F2[i];
        Fnma[i] = (1.0 - alpha) * F0[i] + alpha * F1[i];
      }
      if (det3x3(Fnpa) <= 0.0 || det3x3(Fnma) <= 0.0) { eerr += 1; break; }  // getJacobian
      if (!cp) {
        double S[9], L[81], st[10];
        if (orc_cm_update(mat, Fnpa, 0.0, nullptr, nullptr, st, S, K ? L : nullptr, nullptr)) { eerr++; break; }
        compute_residual_vector(fe.data(), nne, dN, w, Fnpa, I3, I3, S, -dt_np1 * (1.0 - alpha));
        if (K) {
          double FrTFr[9];
          matmulTN(Fnpa, Fnpa, FrTFr);
          std::vector<double> dMdu(nd * 9, 0.0);
          compute_stiffness_matrix(lk1.data(), nne, dN, w, Fnpa, I3, I3, I3, FrTFr, I3, S, L, dMdu.data(), 1.0);
        }
        double S0[9];
        if (orc_cm_update(mat, Fnma, 0.0, nullptr, nullptr, st, S0, nullptr, nullptr)) { eerr++; break; }
        compute_residual_vector(fe.data(), nne, dN, w, Fnma, I3, I3, S0, -dt_n * alpha);
      } else {
        const long q = e * qr.nint + ip;
        const double *s0 = state_nm1 + q * 10, *s1 = state_n + q * 10;
        CpResult res;
        if (cp_update(mat, el, F2, dt_np1, P->R_cp ? P->R_cp + e * 9 : nullptr, s1, res)) { eerr++; break; }
        if (state_np1) {
          for (int i = 0; i < 9; i++) state_np1[q * 10 + i] = res.pFnp1[i];
          state_np1[q * 10 + 9] = res.g;
        }
        double pFa[9], pFb[9], Ma[9], Mb[9];
        for (int i = 0; i < 9; i++) {
          pFa[i] = (1.0 - alpha) * s1[i] + alpha * res.pFnp1[i];
          pFb[i] = (1.0 - alpha) * s0[i] + alpha * s1[i];
        }
        if (inv3x3(pFa, Ma) || inv3x3(pFb, Mb)) { eerr++; break; }
        // one mid point: S at eF = F M, residual with the factor det pF
        auto mid_point = [&](const double *Fm, const double *Mm, const double *pFm, double coef, double *Sm,
                             double *Lm) {
          double eF[9], Ce[9], MT[9];
          matmul(Fm, Mm, eF);
          matmulTN(eF, eF, Ce);
          he_stress_stiffness(el, Ce, det3x3(eF), Sm, Lm);
          transpose(Mm, MT);
          compute_residual_vector(fe.data(), nne, dN, w, Fm, MT, Mm, Sm, coef * det3x3(pFm));
        };
        double Sa[9], La[81], Sb[9];
        mid_point(Fnpa, Ma, pFa, -dt_np1 * (1.0 - alpha), Sa, K ? La : nullptr);
        mid_point(Fnma, Mb, pFb, -dt_n * alpha, Sb, nullptr);
        if (K) {
          std::vector<double> dMtl(nd * 9, 0.0), dMa(nd * 9, 0.0);
          cp_dMdu(res, nne, dN, dMtl.data());
          for (int k = 0; k < nd; k++) {  // M(n+a) pF_{n+1} d(pF_{n+1}^-1) pF_{n+1} M(n+a)
            double t1[9], t2[9], t3[9];
            matmul(Ma, res.pFnp1, t1);
            matmul(t1, dMtl.data() + k * 9, t2);
            matmul(t2, res.pFnp1, t3);
            matmul(t3, Ma, dMa.data() + k * 9);
          }
          double MaT[9], FrTFr[9];
          transpose(Ma, MaT);
          matmulTN(Fnpa, Fnpa, FrTFr);
          compute_stiffness_matrix(lk1.data(), nne, dN, w, Fnpa, MaT, I3, Ma, FrTFr, Ma, Sa, La, dMa.data(),
                                   det3x3(pFa));
        }
      }
      // inertia (DISP_resid_w_inertia_el, src/dynamics.cc:78-181; mass of
      // stiffness_with_inertia, :383-396)
      double du[3] = {0.0, 0.0, 0.0};
      for (int a = 0; a < nne; a++)
        for (int b = 0; b < 3; b++)
          du[b] += N[a] * (dt_n * u2[a * 3 + b] - (dt_np1 + dt_n) * u1[a * 3 + b] + dt_np1 * u0[a * 3 + b]);
      for (int a = 0; a < nne; a++)
        for (int b = 0; b < 3; b++) fi[a * 3 + b] += rho / dt_np1 / dt_n * N[a] * du[b] * w;
      if (K)
        for (int a = 0; a < nne; a++)
          for (int c = 0; c < nne; c++)
            for (int b = 0; b < 3; b++) kI[(a * 3 + b) * nd + c * 3 + b] += rho / dt_np1 * N[a] * N[c] * w;
    }
    if (eerr) { err += eerr; continue; }
    for (int i = 0; i < nd; i++) fe[i] -= fi[i];
    if (K)
      for (int i = 0; i < nd * nd; i++) lk[i] = -kI[i] - alpha * (1.0 - alpha) * dt_np1 * lk1[i];
    if (P->nbc_off) {  // surface loads at the mid points (needs the values at t_n, t_{n-1})
      if (!P->nbc_load_n || !P->nbc_load_nm1) { err++; continue; }
      neumann_faces_transient(P, e, Xe, u2, u1, u0, alpha, dt_np1, dt_n, fe.data(), K ? lk.data() : nullptr);
    }
    scatter(P, e, fe.data(), K ? lk.data() : nullptr, R, K);
  }
  return err;
}

// ---------------------------------------------------------------------------
// Transient three-field element of the hyperelastic model, one rank:
// residuals_el_constitutive_model_w_inertia_3f (src/constitutive_model.cc:
// 2960-3229) and stiffness_el_constitutive_model_w_inertia_3f (:2190-2395),
// combined with the inertia terms by residual_with_inertia /
// stiffness_with_inertia (src/dynamics.cc:183-447, case CM3F).  With
// mid(a, b) = (1 - alpha) a + alpha b, the newer mid point takes u_{n+alpha},
// theta = mid(theta_n, theta_{n+1}), P = mid(P_n, P_{n+1}) and the older one
// the same from t_{n-1}, t_n:
//   R_x = -dt_np1 (1 - alpha) R_x(n+alpha) - dt_n alpha R_x(n-1+alpha)   (x = u, p, t)
//   K_xy = -dt_np1 alpha (1 - alpha) K_xy(n+alpha)   (dt_alpha_1_minus_alpha of
//        the blocks, src/constitutive_model_3f.cc:297-470)
//   f = condense(R, K) - f_i,   k = condense(K) - M / dt_np1.
// Pe3 / th3: per element the values at t_{n+1}, t_n, t_{n-1} (ne x 3).
// ---------------------------------------------------------------------------
namespace {
struct Blocks3fTr {
  std::vector<double> fu, Kuu, blk;  // combined (scaled) blocks of one element
};

int element_3f_transient(const orc_problem *P, const orc_material *mat, long e, const double *u2, const double *u1,
                         const double *u0, const double *Pe3, const double *th3, double alpha, double dt_np1,
                         double dt_n, bool wantK, Blocks3fTr &B) {
  const int nd = P->nne * 3;
  double ua[30], ub[30];
  for (int i = 0; i < nd; i++) {
    ua[i] = (1.0 - alpha) * u1[i] + alpha * u2[i];
    ub[i] = (1.0 - alpha) * u0[i] + alpha * u1[i];
  }
  const double *pe = Pe3 + e * 3, *te = th3 + e * 3;
  const double Pa = (1.0 - alpha) * pe[1] + alpha * pe[0], ta = (1.0 - alpha) * te[1] + alpha * te[0];
  const double Pb = (1.0 - alpha) * pe[2] + alpha * pe[1], tb = (1.0 - alpha) * te[2] + alpha * te[1];
  std::vector<double> fua(nd), fub(nd), Kuu(wantK ? nd * nd : 0), ba(4 + nd), bb(4 + nd);
  int err = element_3f_blocks(P, mat, e, ua, Pa, ta, nullptr, nullptr, fua.data(), wantK ? Kuu.data() : nullptr,
                              ba.data());
  if (!err) err = element_3f_blocks(P, mat, e, ub, Pb, tb, nullptr, nullptr, fub.data(), nullptr, bb.data());
  if (err) return err;
  const double cA = -dt_np1 * (1.0 - alpha), cB = -dt_n * alpha, kK = -dt_np1 * alpha * (1.0 - alpha);
  B.fu.assign(nd, 0.0);
  B.blk.assign(4 + nd, 0.0);
  for (int r = 0; r < nd; r++) B.fu[r] = cA * fua[r] + cB * fub[r];
  B.blk[0] = cA * ba[0] + cB * bb[0];  // Rp
  B.blk[1] = cA * ba[1] + cB * bb[1];  // Rt
  B.blk[2] = kK * ba[2];               // Ktp
  B.blk[3] = kK * ba[3];               // Ktt
  for (int r = 0; r < nd; r++) B.blk[4 + r] = kK * ba[4 + r];  // Kup
  if (wantK) {
    B.Kuu.resize(nd * nd);
    for (int i = 0; i < nd * nd; i++) B.Kuu[i] = kK * Kuu[i];
  }
  return 0;
}
}  // namespace

extern "C" int orc_assemble_3f_transient(const orc_problem *P, const orc_material *mat, const double *u_np1,
                                         const double *u_n, const double *u_nm1, const double *p_np1,
                                         const double *p_n, const double *p_nm1, const double *Pe3,
                                         const double *th3, double alpha, double dt_np1, double dt_n, double rho,
                                         double *R, double *K) {
  if (mat->model != ORC_MODEL_HE) return 1;
  const int nne = P->nne, nd = nne * 3;
  Quad qr = quad_rule(nne);
  int err = 0;
  for (long e = 0; e < P->ne; e++) {
    double u2[30], u1[30], u0[30], Xe[30];
    gather_u(P, e, u_np1, p_np1, u2);
    gather_u(P, e, u_n, p_n, u1);
    gather_u(P, e, u_nm1, p_nm1, u0);
    for (int a = 0; a < nne; a++)
      for (int i = 0; i < 3; i++) Xe[a * 3 + i] = P->X[(long)P->conn[e * nne + a] * 3 + i];
    Blocks3fTr B;
    int r = element_3f_transient(P, mat, e, u2, u1, u0, Pe3, th3, alpha, dt_np1, dt_n, K != nullptr, B);
    if (r) { err += r; continue; }
    std::vector<double> fe(nd), lk(K ? nd * nd : 0);
    condense_3f(nd, B.fu.data(), K ? B.Kuu.data() : nullptr, B.blk.data(), fe.data(), K ? lk.data() : nullptr);
    // inertia (DISP_resid_w_inertia_el, src/dynamics.cc:78-181; mass of
    // stiffness_with_inertia, :378-392)
    for (int ip = 0; ip < qr.nint; ip++) {
      double dN[30], N[10];
      int terr = 0;
      const double detJ = PGFem3D_dNdX(nne, qr.ksi[ip], qr.eta[ip], qr.zet[ip], Xe, dN, &terr);
      if (terr) { err += terr; break; }
      const double w = detJ * qr.w[ip];
      shape_N(nne, qr.ksi[ip], qr.eta[ip], qr.zet[ip], N);
      double du[3] = {0.0, 0.0, 0.0};
      for (int a = 0; a < nne; a++)
        for (int b = 0; b < 3; b++)
          du[b] += N[a] * (dt_n * u2[a * 3 + b] - (dt_np1 + dt_n) * u1[a * 3 + b] + dt_np1 * u0[a * 3 + b]);
      for (int a = 0; a < nne; a++)
        for (int b = 0; b < 3; b++) fe[a * 3 + b] -= rho / dt_np1 / dt_n * N[a] * du[b] * w;
      if (K)
        for (int a = 0; a < nne; a++)
          for (int c = 0; c < nne; c++)
            for (int b = 0; b < 3; b++) lk[(a * 3 + b) * nd + c * 3 + b] -= rho / dt_np1 * N[a] * N[c] * w;
    }
    if (P->nbc_off) {
      if (!P->nbc_load_n || !P->nbc_load_nm1) { err++; continue; }
      neumann_faces_transient(P, e, Xe, u2, u1, u0, alpha, dt_np1, dt_n, fe.data(), K ? lk.data() : nullptr);
    }
    scatter(P, e, fe.data(), K ? lk.data() : nullptr, R, K);
  }
  return err;
}

// Increments of the element pressure and volume in the transient
// (update_3f_state_variables_w_inertia, src/constitutive_model.cc:3880-3898,
// with compute_d_theta_dP, src/constitutive_model_3f.cc:494-549, Ktu = 0):
// the combined blocks above, d_theta = -Kpt^-1 (Kpu du + Rp),
// dP = -Ktp^-1 (Rt + Ktt d_theta).
extern "C" int orc_update_3f_transient(const orc_problem *P, const orc_material *mat, const double *u_np1,
                                       const double *u_n, const double *u_nm1, const double *p_np1,
                                       const double *p_n, const double *p_nm1, const double *du,
                                       const double *Pe3, const double *th3, double alpha, double dt_np1,
                                       double dt_n, double *dP, double *dtheta) {
  if (mat->model != ORC_MODEL_HE) return 1;
  const int nd = P->nne * 3;
  int err = 0;
  for (long e = 0; e < P->ne; e++) {
    double u2[30], u1[30], u0[30], due[30];
    gather_u(P, e, u_np1, p_np1, u2);
    gather_u(P, e, u_n, p_n, u1);
    gather_u(P, e, u_nm1, p_nm1, u0);
    gather_u(P, e, du, nullptr, due);
    Blocks3fTr B;
    int r = element_3f_transient(P, mat, e, u2, u1, u0, Pe3, th3, alpha, dt_np1, dt_n, false, B);
    if (r) { err += r; continue; }
    const double Rp = B.blk[0], Rt = B.blk[1], Ktp = B.blk[2], Ktt = B.blk[3], Kpt = Ktp;
    double Kpu_du = 0.0;
    for (int i = 0; i < nd; i++) Kpu_du += B.blk[4 + i] * due[i];
    dtheta[e] = -(Kpu_du + Rp) / Kpt;
    dP[e] = -(Rt + Ktt * dtheta[e]) / Ktp;
  }
  return err;
}

extern "C" int orc_assemble_transient(const orc_problem *P, const orc_material *mat, const double *u_np1,
                                      const double *u_n, const double *u_nm1, const double *p_np1,
                                      const double *p_n, const double *p_nm1, double alpha, double dt_np1,
                                      double dt_n, double rho, double *R, double *K) {
  return orc_assemble_transient_state(P, mat, u_np1, u_n, u_nm1, p_np1, p_n, p_nm1, alpha, dt_np1, dt_n, rho,
                                      nullptr, nullptr, nullptr, R, K);
}

extern "C" long orc_cp_update_batch(const orc_material *mat, long nqp, const double *F, double dt,
                                    const double *Rcp, const double *state_n, const double *M0,
                                    const double *g_guess, double *state_np1, int *iters, double *dgam,
                                    int *converged, int warm_k, int *fallback) {
  Elast el = make_elast(mat);
  long bad = 0;
  for (long q = 0; q < nqp; q++) {
    CpResult res;
    int err = cp_update_guess(mat, el, F + q * 9, dt, Rcp ? Rcp + q * 9 : nullptr, state_n + q * 10,
                              M0 ? M0 + q * 9 : nullptr, g_guess ? g_guess[q] : -1.0, res, warm_k);
    if (fallback) fallback[q] = res.fallback;
    if (state_np1) {
      for (int i = 0; i < 9; i++) state_np1[q * 10 + i] = res.pFnp1[i];
      state_np1[q * 10 + 9] = res.g;
    }
    if (iters) iters[q] = res.iters;
    if (dgam)
      for (int a = 0; a < kNSlip; a++) dgam[q * kNSlip + a] = res.dgam[a];
    if (converged) converged[q] = !err;
    bad += err != 0;
  }
  return bad;
}
