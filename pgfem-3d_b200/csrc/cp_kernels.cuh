// cp_kernels.cuh -- crystal plasticity (CP_PARAM) on the device.
//
// Constitutive law (the reference's CM crystal plasticity, src/plasticity_model.cc,
// with the flow and hardening laws of src/TA_GA.cc:8-41 and
// src/integration.cc:378-423): FCC {111}<110> slip, resolved shear
// tau_a = s_a . (Ce S) n_a, gamma_dot_a = gamma_dot_0 sgn(tau_a)|tau_a/g|^(1/m),
// M = pF_n pF_{n+1}^-1 = I - dt sum gamma_dot_a P_a, saturation hardening
// g - g_n - dt G0 gamma_dot (gs - g)/(gs - g0) = 0 with the rate-dependent
// saturation stress gs = gs_0 (gamma_dot / gamma_dot_s)^w (src/integration.cc:
// 394-402; gs = gs_0 for w = 0), neo-Hookean + U_Common elasticity at
// Ce = M^T Ce' M.  The local problem in x = (M, g) is
// solved by Newton with backtracking from the elastic predictor or from a
// supplied initial guess; at convergence the consistent dM/dF is formed.
//
// k_cp_update is persistent: every lane owns one quadrature point at a time
// and takes a new one from a global counter as soon as its Newton converges,
// so lanes with 2 and 15 iterations do not idle each other.  The 10x10
// Jacobian of each lane lives in shared memory (lane-strided, bank-conflict
// free).  Slip systems are evaluated in the crystal frame: the Mandel product
// is rotated once per evaluation, the slip directions/normals are constants.
#pragma once
#include <cuda_runtime.h>

#include "cm_models.cuh"

namespace pgb {

constexpr int kSlip = 12;
constexpr int kCpOut = 9 + 81 + 1 + 12;  // M (UL), dM/dF, g, dt*gamma_dot_a  (per point, SoA)

// FCC slip directions (unnormalised <110>) and normals (unnormalised {111})
__constant__ double c_slip_s[kSlip][3] = {{0, 1, -1}, {1, 0, -1}, {1, -1, 0}, {0, 1, -1}, {1, 0, 1}, {1, 1, 0},
                                          {0, 1, 1},  {1, 0, -1}, {1, 1, 0},  {0, 1, 1},  {1, 0, 1}, {1, -1, 0}};
__constant__ double c_slip_n[kSlip][3] = {{1, 1, 1},  {1, 1, 1},  {1, 1, 1},  {-1, 1, 1}, {-1, 1, 1}, {-1, 1, 1},
                                          {1, -1, 1}, {1, -1, 1}, {1, -1, 1}, {1, 1, -1}, {1, 1, -1}, {1, 1, -1}};

__device__ __forceinline__ void mm3(const double *A, const double *B, double *C) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      C[i * 3 + j] = A[i * 3] * B[j] + A[i * 3 + 1] * B[3 + j] + A[i * 3 + 2] * B[6 + j];
}
__device__ __forceinline__ void mm3tn(const double *A, const double *B, double *C) {  // A^T B
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) C[i * 3 + j] = A[i] * B[j] + A[3 + i] * B[3 + j] + A[6 + i] * B[6 + j];
}
__device__ __forceinline__ void mm3nt(const double *A, const double *B, double *C) {  // A B^T
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      C[i * 3 + j] = A[i * 3] * B[j * 3] + A[i * 3 + 1] * B[j * 3 + 1] + A[i * 3 + 2] * B[j * 3 + 2];
}

// Neo-Hookean (Mooney-Rivlin m01 = 0) + U_Common PK2 stress at C and its
// directional derivative dS[X] for symmetric X (= 1/2 L : X).
struct NeoHooke {
  double Ci[9], S[9], J, J23, trC;
};

__device__ __forceinline__ bool nh_stress(const Mat &mat, const double *C, NeoHooke &h) {
  const double detC = det3(C);
  if (!(detC > 0.0)) return false;
  inv3(C, h.Ci);
  h.J = sqrt(detC);
  h.J23 = 1.0 / cbrt(detC);  // detC^{-1/3}
  h.trC = C[0] + C[4] + C[8];
  const double a = mat.mu * h.J23, pv = mat.kappa * h.J * (h.J - 1.0);
#pragma unroll
  for (int i = 0; i < 9; i++) h.S[i] = a * ((i % 4 == 0 ? 1.0 : 0.0) - h.trC / 3.0 * h.Ci[i]) + pv * h.Ci[i];
  return true;
}

__device__ __forceinline__ void nh_dS(const Mat &mat, const NeoHooke &h, const double *X, double *dS) {
  // S = mu detC^{-1/3} (I - trC/3 Ci) + kappa J(J-1) Ci
  double CiX = 0, trX = X[0] + X[4] + X[8];
#pragma unroll
  for (int i = 0; i < 9; i++) CiX += h.Ci[i] * X[i];
  double t[9], CXC[9];
  mm3(h.Ci, X, t);
  mm3(t, h.Ci, CXC);
  const double a = mat.mu * h.J23;
  const double dpv = mat.kappa * (2.0 * h.J - 1.0) * 0.5 * h.J * CiX;
  const double pv = mat.kappa * h.J * (h.J - 1.0);
#pragma unroll
  for (int i = 0; i < 9; i++) {
    const double d = (i % 4 == 0 ? 1.0 : 0.0);
    dS[i] = a * (-CiX / 3.0 * (d - h.trC / 3.0 * h.Ci[i]) - trX / 3.0 * h.Ci[i] + h.trC / 3.0 * CXC[i]) +
            dpv * h.Ci[i] - pv * CXC[i];
  }
}

// Sample-frame Schmid tensor of system a from the crystal rotation R.
__device__ __forceinline__ void schmid(const double *R, int a, double *P) {
  const double is2 = 0.70710678118654752440, is3 = 0.57735026918962576451;
  double s[3], n[3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    s[i] = (R[i * 3] * c_slip_s[a][0] + R[i * 3 + 1] * c_slip_s[a][1] + R[i * 3 + 2] * c_slip_s[a][2]) * is2;
    n[i] = (R[i * 3] * c_slip_n[a][0] + R[i * 3 + 1] * c_slip_n[a][1] + R[i * 3 + 2] * c_slip_n[a][2]) * is3;
  }
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) P[i * 3 + j] = s[i] * n[j];
}

// |tau/g|^(1/m - 1) of the power-law flow rule.  When the exponent is a small
// non-negative integer (m = 0.05 gives 19) it is formed by binary
// exponentiation (repeated squaring: seven multiplies for 19, a few ulp from
// the correctly rounded power); otherwise pow.  The exponent is the same for
// every lane, so the branch does not diverge.
__device__ __forceinline__ double flow_pow(double r, double e) {
  const int n = (int)e;
  if ((double)n == e && n >= 0 && n <= 64) {
    double x = r, y = 1.0;
    for (int k = n; k; k >>= 1) {
      if (k & 1) y *= x;
      x *= x;
    }
    return y;
  }
  return pow(r, e);
}

// Residual of the local problem at (M, g).  Returns false on an invalid state.
struct CpPoint {
  double Cep[9], R[9];  // trial Ce' and crystal rotation
  double g_n, dt;
};

// Saturation stress gs(gamma_dot) and dRg = d R_g / d gamma_dot (through gs as
// well): -dt G0 [(gs - g)/(gs - g0) + w gs (g - g0)/(gs - g0)^2].
struct CpHard {
  double gs, dRg;
};
__device__ __forceinline__ CpHard cp_hardening(const Mat &mat, double gdot, double g, double dt) {
  CpHard h;
  const bool rate = mat.w > 0.0 && gdot > 0.0;
  h.gs = rate ? mat.gs0 * pow(gdot / mat.gdots, mat.w) : mat.gs0;
  const double d = h.gs - mat.g0;
  h.dRg = -dt * mat.G0 * ((h.gs - g) / d + (rate ? mat.w * h.gs * (g - mat.g0) / (d * d) : 0.0));
  return h;
}

__device__ __forceinline__ bool cp_residual(const Mat &mat, const CpPoint &pt, const double *M, double g,
                                            double *Res, NeoHooke &h, double *gd, double *dgd, double &gdot) {
  double t[9], Ce[9];
  mm3(pt.Cep, M, t);
  mm3tn(M, t, Ce);
  if (!(g > 0.0) || !nh_stress(mat, Ce, h)) return false;
  double CS[9];
  mm3(Ce, h.S, CS);
  const double im = 1.0 / mat.m;
  gdot = 0.0;
#pragma unroll
  for (int i = 0; i < 9; i++) Res[i] = M[i] - (i % 4 == 0 ? 1.0 : 0.0);
  for (int a = 0; a < kSlip; a++) {
    double P[9];
    schmid(pt.R, a, P);
    double tau = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) tau += CS[i] * P[i];
    const double pw = flow_pow(fabs(tau / g), im - 1.0);
    gd[a] = mat.gdot0 * (tau / g) * pw;
    dgd[a] = mat.gdot0 * im / g * pw;
    gdot += fabs(gd[a]);
#pragma unroll
    for (int i = 0; i < 9; i++) Res[i] += pt.dt * gd[a] * P[i];
  }
  const double gs = cp_hardening(mat, gdot, g, pt.dt).gs;
  Res[9] = g - pt.g_n - pt.dt * mat.G0 * gdot * (gs - g) / (gs - mat.g0);
  return true;
}

__device__ __forceinline__ double cp_norm(const double *R, double g0) {
  double m = 0;
#pragma unroll
  for (int i = 0; i < 9; i++) m = fmax(m, fabs(R[i]));
  return fmax(m, fabs(R[9]) / g0);
}

// Ysym_a = sym(P_a S + dS[sym(Ce P_a)]): d tau_a = dCe : Ysym_a.
__device__ __forceinline__ void ysym(const Mat &mat, const NeoHooke &h, const double *Ce, const double *P,
                                     double *Y) {
  double PS[9], CP[9], X[9], dS[9];
  mm3(P, h.S, PS);
  mm3(Ce, P, CP);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) X[i * 3 + j] = 0.5 * (CP[i * 3 + j] + CP[j * 3 + i]);
  nh_dS(mat, h, X, dS);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const double y1 = PS[i * 3 + j] + dS[i * 3 + j], y2 = PS[j * 3 + i] + dS[j * 3 + i];
      Y[i * 3 + j] = 0.5 * (y1 + y2);
    }
}

// Lane-strided dense 10 x nc block in shared memory: element (r, c) at
// base[(r * nc + c) * 32].
__device__ __forceinline__ double &lm(double *base, int nc, int r, int c) { return base[(r * nc + c) * 32]; }

// Gaussian elimination with partial pivoting, n x n matrix A with nrhs
// right-hand sides B (both lane-strided).  false if singular.
__device__ bool lane_solve(double *A, int n, double *B, int nrhs) {
  for (int k = 0; k < n; k++) {
    int p = k;
    double best = fabs(lm(A, n, k, k));
    for (int i = k + 1; i < n; i++) {
      const double v = fabs(lm(A, n, i, k));
      if (v > best) {
        best = v;
        p = i;
      }
    }
    if (!(best > 0.0)) return false;
    if (p != k) {
      for (int j = 0; j < n; j++) {
        const double t = lm(A, n, k, j);
        lm(A, n, k, j) = lm(A, n, p, j);
        lm(A, n, p, j) = t;
      }
      for (int j = 0; j < nrhs; j++) {
        const double t = lm(B, nrhs, k, j);
        lm(B, nrhs, k, j) = lm(B, nrhs, p, j);
        lm(B, nrhs, p, j) = t;
      }
    }
    const double inv = 1.0 / lm(A, n, k, k);
    for (int i = k + 1; i < n; i++) {
      const double f = lm(A, n, i, k) * inv;
      if (f == 0.0) continue;
      for (int j = k; j < n; j++) lm(A, n, i, j) -= f * lm(A, n, k, j);
      for (int j = 0; j < nrhs; j++) lm(B, nrhs, i, j) -= f * lm(B, nrhs, k, j);
    }
  }
  for (int k = n - 1; k >= 0; k--) {
    const double inv = 1.0 / lm(A, n, k, k);
    for (int j = 0; j < nrhs; j++) {
      double v = lm(B, nrhs, k, j);
      for (int i = k + 1; i < n; i++) v -= lm(A, n, k, i) * lm(B, nrhs, i, j);
      lm(B, nrhs, k, j) = v * inv;
    }
  }
  return true;
}

// Jacobian dR/dx (10 x 10, lane-strided) at an evaluated point.
__device__ void cp_jacobian(const Mat &mat, const CpPoint &pt, const double *M, double g, const NeoHooke &h,
                            const double *gd, const double *dgd, double gdot, double *Jm) {
  double t[9], Ce[9], CepM[9];
  mm3(pt.Cep, M, CepM);
  mm3tn(M, CepM, Ce);
  const CpHard hd = cp_hardening(mat, gdot, g, pt.dt);
  const double c = pt.dt * mat.G0 / (hd.gs - mat.g0);
  for (int r = 0; r < 10; r++)
    for (int q = 0; q < 10; q++) lm(Jm, 10, r, q) = (r == q && r < 9) ? 1.0 : 0.0;
  double dgdM[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int a = 0; a < kSlip; a++) {
    double P[9], Y[9], dtau[9];
    schmid(pt.R, a, P);
    ysym(mat, h, Ce, P, Y);
    mm3(CepM, Y, t);
#pragma unroll
    for (int i = 0; i < 9; i++) dtau[i] = 2.0 * t[i];
    const double sg = gd[a] < 0 ? -1.0 : 1.0;
    const double cf = pt.dt * dgd[a], cg = pt.dt * (-gd[a] / (mat.m * g));
    for (int i = 0; i < 9; i++) {
      const double Pi = P[i];
      for (int j = 0; j < 9; j++) lm(Jm, 10, i, j) += cf * Pi * dtau[j];
      lm(Jm, 10, i, 9) += cg * Pi;
    }
#pragma unroll
    for (int j = 0; j < 9; j++) dgdM[j] += sg * dgd[a] * dtau[j];
  }
  for (int j = 0; j < 9; j++) lm(Jm, 10, 9, j) = hd.dRg * dgdM[j];
  lm(Jm, 10, 9, 9) = 1.0 + c * gdot - hd.dRg * gdot / (mat.m * g);
}

struct CpArgs {
  long nqp;
  const double *F;        // 9*nqp (SoA)
  const double *Rcp;      // 9*nelem (SoA, per element; qp -> element = qp / nqp_e)
  int nqp_e;
  long ne;
  const double *state_n;  // 10*nqp SoA
  double *state_np1;      // 10*nqp SoA
  const double *guess;    // 10*nqp SoA (M0 9, g0) or nullptr
  double *out;            // kCpOut*nqp SoA: M (UL) 9, dM/dF 81, g
  int *iters;             // nqp or nullptr
  unsigned *counter;
  unsigned long long *status;
  Mat mat;
  double dt;
  int warm_k;                     // Newton iterations from the guess before the cold restart (0: max_iter)
  unsigned long long *fallbacks;  // cold restarts (or nullptr)
  uint8_t *conv;                  // nqp: 1 when the point converged with an invertible M (or nullptr)
};

constexpr int kCpWarps = 4;      // warps per CTA of k_cp_update
constexpr int kCpTanWarps = 2;   // warps per CTA of k_cp_tangent

__global__ void __launch_bounds__(32 * kCpWarps) k_cp_update(const CpArgs A) {
  extern __shared__ double smem_cp[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double *Jm = smem_cp + warp * (100 + 10) * 32 + lane;  // 10x10 Jacobian
  double *Bm = Jm + 100 * 32;                            // right-hand side
  const unsigned FULL = 0xffffffffu;
  const long S = A.nqp;
  const double tol = A.mat.tol;
  long qp = -1;
  bool done = false;
  CpPoint pt;
  double M[9], g = 0, Res[10], nr = 0, gd[kSlip], dgd[kSlip], gdot = 0, Fq[9], pFni[9];
  int it = 0, it0 = 0;  // total iterations; iterations before the current start
  bool warm = false;    // Newton running from the caller's guess
  NeoHooke h;
  for (;;) {
    // refill lanes without a point (warp-aggregated tickets)
    const unsigned need = __ballot_sync(FULL, qp < 0 && !done);
    if (need) {
      unsigned base = 0;
      const int leader = __ffs(need) - 1;
      if (lane == leader) base = atomicAdd(A.counter, (unsigned)__popc(need));
      base = __shfl_sync(FULL, base, leader);
      if (qp < 0 && !done) {
        const long cand = (long)base + __popc(need & ((1u << lane) - 1u));
        if (cand < S) {
          qp = cand;
          // point set-up: trial Ce', rotation, initial guess, first residual
          const long e = qp / A.nqp_e;
#pragma unroll
          for (int i = 0; i < 9; i++) {
            Fq[i] = A.F[i * S + qp];
            pt.R[i] = A.Rcp[i * A.ne + e];
          }
          double pFn[9];
#pragma unroll
          for (int i = 0; i < 9; i++) pFn[i] = A.state_n[i * S + qp];
          pt.g_n = A.state_n[9 * S + qp];
          pt.dt = A.dt;
          inv3(pFn, pFni);
          double Fe[9];
          mm3(Fq, pFni, Fe);
          mm3tn(Fe, Fe, pt.Cep);
          if (A.guess) {
#pragma unroll
            for (int i = 0; i < 9; i++) M[i] = A.guess[i * S + qp];
            g = A.guess[9 * S + qp];
          } else {
#pragma unroll
            for (int i = 0; i < 9; i++) M[i] = (i % 4 == 0) ? 1.0 : 0.0;
            g = pt.g_n;
          }
          it = it0 = 0;
          warm = A.guess != nullptr;
          if (cp_residual(A.mat, pt, M, g, Res, h, gd, dgd, gdot)) nr = cp_norm(Res, A.mat.g0);
          else nr = 1e300;
        } else {
          done = true;
        }
      }
    }
    if (__all_sync(FULL, done)) break;
    if (qp < 0) continue;
    // one Newton step (or finish)
    const int cap = warm && A.warm_k > 0 ? A.warm_k : A.mat.max_iter;
    bool finish = !(nr > tol) || it - it0 >= cap || !(nr < 1e299);
    if (!finish) {
      cp_jacobian(A.mat, pt, M, g, h, gd, dgd, gdot, Jm);
      for (int i = 0; i < 10; i++) lm(Bm, 1, i, 0) = -Res[i];
      if (!lane_solve(Jm, 10, Bm, 1)) {
        nr = 1e300;
        finish = true;
      } else {
        double dx[10];
        for (int i = 0; i < 10; i++) dx[i] = lm(Bm, 1, i, 0);
        double lam = 1.0, Mt[9], gt = g, nt = 1e300;
        double Rt[10], gdt[kSlip], dgdt[kSlip], gdott = 0;
        NeoHooke ht;
        for (int ls = 0; ls < 8; ls++) {
#pragma unroll
          for (int i = 0; i < 9; i++) Mt[i] = M[i] + lam * dx[i];
          gt = g + lam * dx[9];
          if (cp_residual(A.mat, pt, Mt, gt, Rt, ht, gdt, dgdt, gdott)) {
            nt = cp_norm(Rt, A.mat.g0);
            if (nt < nr || ls == 7) break;
          }
          lam *= 0.5;
        }
#pragma unroll
        for (int i = 0; i < 9; i++) M[i] = Mt[i];
        g = gt;
        nr = nt;
        h = ht;
        gdot = gdott;
#pragma unroll
        for (int i = 0; i < 10; i++) Res[i] = Rt[i];
#pragma unroll
        for (int a = 0; a < kSlip; a++) {
          gd[a] = gdt[a];
          dgd[a] = dgdt[a];
        }
        it++;
      }
    }
    if (finish && warm && !(nr <= tol)) {
      // the guess did not converge in cap iterations (or left the domain):
      // restart from the elastic predictor with the full iteration budget
      warm = false;
      it0 = it;
      if (A.fallbacks) atomicAdd(A.fallbacks, 1ull);
#pragma unroll
      for (int i = 0; i < 9; i++) M[i] = (i % 4 == 0) ? 1.0 : 0.0;
      g = pt.g_n;
      if (cp_residual(A.mat, pt, M, g, Res, h, gd, dgd, gdot)) nr = cp_norm(Res, A.mat.g0);
      else nr = 1e300;
      finish = false;
    }
    if (finish) {
      const bool conv = nr <= tol;
      if (!conv) atomicAdd(&A.status[1], 1ull);
      // state at n+1: pF_{n+1} = M^-1 pF_n
      double Mi[9], pFn[9], pFnp1[9];
#pragma unroll
      for (int i = 0; i < 9; i++) pFn[i] = A.state_n[i * S + qp];
      const bool okM = inv3(M, Mi);
      mm3(Mi, pFn, pFnp1);
#pragma unroll
      for (int i = 0; i < 9; i++) A.state_np1[i * S + qp] = okM ? pFnp1[i] : pFn[i];
      A.state_np1[9 * S + qp] = g;
#pragma unroll
      for (int i = 0; i < 9; i++) A.out[i * S + qp] = M[i];
      A.out[90 * S + qp] = g;
#pragma unroll
      for (int a = 0; a < kSlip; a++) A.out[(91 + a) * S + qp] = A.dt * gd[a];
      if (A.iters) A.iters[qp] = it;
      if (A.conv) A.conv[qp] = (conv && okM) ? 1 : 0;
      qp = -1;
    }
  }
}

inline size_t cp_update_smem() { return sizeof(double) * kCpWarps * (100 + 10) * 32; }

// ---- consistent tangent, four lanes per point -------------------------------

// Sample-frame slip direction and normal of system a (unit vectors).
__device__ __forceinline__ void slip_sn(const double *R, int a, double *sv, double *nv) {
  const double is2 = 0.70710678118654752440, is3 = 0.57735026918962576451;
#pragma unroll
  for (int i = 0; i < 3; i++) {
    sv[i] = (R[i * 3] * c_slip_s[a][0] + R[i * 3 + 1] * c_slip_s[a][1] + R[i * 3 + 2] * c_slip_s[a][2]) * is2;
    nv[i] = (R[i * 3] * c_slip_n[a][0] + R[i * 3 + 1] * c_slip_n[a][1] + R[i * 3 + 2] * c_slip_n[a][2]) * is3;
  }
}

// Sum of v over the four lanes of a point (every lane gets the same bits).
__device__ __forceinline__ double quad_sum(unsigned qm, double v) {
  v += __shfl_xor_sync(qm, v, 1);
  v += __shfl_xor_sync(qm, v, 2);
  return v;
}

// symmetric 3x3 in Voigt order (xx yy zz yz xz xy): y = A x
__device__ __forceinline__ void symv6(const double *A, const double *x, double *y) {
  y[0] = A[0] * x[0] + A[5] * x[1] + A[4] * x[2];
  y[1] = A[5] * x[0] + A[1] * x[1] + A[3] * x[2];
  y[2] = A[4] * x[0] + A[3] * x[1] + A[2] * x[2];
}

// Ysym of slip system (s, n) for the neo-Hookean + U_Common law from the
// shared per-point state (Ce, Ce^-1 in Voigt form; a = mu detC^-1/3, pv =
// kappa J (J - 1), trC, J), by the rank-one Schmid structure P = s n^T:
// sym(P S) = sym(s w^T) with w = S n, and dS[X] for X = sym(c n^T), c = Ce s
// (nh_dS with Ci:X = n . Ci c and Ci X Ci = sym(p q^T), p = Ci c, q = Ci n).
// The same tensor as ysym; tau = s . (Ce S) n is returned too.
__device__ __forceinline__ double ysym_sn(const Mat &mat, const double *C6, const double *Ci, double a, double pv,
                                          double trC, double J, const double *sv, const double *nv, double *Y) {
  double c[3], p[3], q[3], w[3];
  symv6(C6, sv, c);
  symv6(Ci, c, p);
  symv6(Ci, nv, q);
#pragma unroll
  for (int i = 0; i < 3; i++) w[i] = a * (nv[i] - trC / 3.0 * q[i]) + pv * q[i];
  const double sn = sv[0] * nv[0] + sv[1] * nv[1] + sv[2] * nv[2];
  const double trX = c[0] * nv[0] + c[1] * nv[1] + c[2] * nv[2];
  const double CiX = nv[0] * p[0] + nv[1] * p[1] + nv[2] * p[2];
  const double dpv = mat.kappa * (2.0 * J - 1.0) * 0.5 * J * CiX;
  const int vi[6] = {0, 1, 2, 1, 0, 0}, vj[6] = {0, 1, 2, 2, 2, 1};
#pragma unroll
  for (int v = 0; v < 6; v++) {
    const int i = vi[v], j = vj[v];
    const double d = i == j ? 1.0 : 0.0;
    const double cxc = 0.5 * (p[i] * q[j] + q[i] * p[j]);
    const double y = 0.5 * (sv[i] * w[j] + w[i] * sv[j]) +
                     a * (-CiX / 3.0 * (d - trC / 3.0 * Ci[v]) - trX / 3.0 * Ci[v] + trC / 3.0 * cxc) +
                     dpv * Ci[v] - pv * cxc;
    Y[i * 3 + j] = y;
    Y[j * 3 + i] = y;
  }
  return a * (trX - trC / 3.0 * sn) + pv * sn;  // tau
}

// Shared region of one point of k_cp_tangent (doubles): [0, 100) the
// Jacobian rows, [100, 190) the right-hand sides (10 x 9, row-major), [190,
// 234) exchange records of four slip systems, then the crystal rotation, W =
// pF_n^-1 M, F, Ce (Voigt), Ce^-1 (Voigt), Ce' M and five scalars.  The
// stride is 2 mod 16 doubles (the eight points of a warp on distinct banks).
constexpr int kCtQS = 290;
constexpr int kCtJ = 0, kCtB = 100, kCtX = 190, kCtR = 234, kCtW = 243, kCtF = 252, kCtCe = 261, kCtCi = 267,
              kCtCM = 273, kCtSc = 282;
constexpr int kCtPts = 8 * kCpTanWarps;  // points per CTA

// Consistent tangent of the converged local update, four lanes per point:
// dM/dF = -J^-1 dR/dF with d tau_a / dF = 2 F Z_a, Z_a = pF_n^-1 M Ysym_a M^T
// pF_n^-T (the role of compute_dMdu, src/plasticity_model.cc:578-881).  The
// Jacobian rows and the nine right-hand sides are built in rounds of four
// slip-system records (each lane forms the record of one system per round,
// every lane adds the four records to its rows sub, sub + 4, sub + 8), the
// pivoted elimination splits rows over the lanes, the back substitution the
// nine columns.  Points that did not converge, or whose Jacobian is singular
// (counted in status[3]), get a zero tangent.  Every point does the same work:
// a uniform grid over the points, four lanes each.
__global__ void __launch_bounds__(32 * kCpTanWarps, 6) k_cp_tangent(const CpArgs A) {
  extern __shared__ double smem_ct[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sub = lane & 3, qd = lane >> 2;
  const unsigned qm = 0xFu << (lane & ~3);
  double *reg = smem_ct + (warp * 8 + qd) * kCtQS;
  const long S = A.nqp;
  const double dt = A.dt, im = 1.0 / A.mat.m;
  const long nquads = (long)gridDim.x * kCtPts;
  for (long qp = (long)blockIdx.x * kCtPts + warp * 8 + qd; qp < S; qp += nquads) {
    bool ok = A.conv[qp] != 0;
    double g = 0.0, gsum = 0.0;
    if (ok) {
      // point set-up (every lane computes, lane 0 stores as it goes): F, W =
      // pF_n^-1 M, Ce' M, Ce, its inverse and the stress scalars
      __syncwarp(qm);  // the previous point's reads of the region are done
      const long e = qp / A.nqp_e;
      double M[9], pFni[9], C6[6];
#pragma unroll
      for (int i = 0; i < 9; i++) M[i] = A.out[i * S + qp];
      g = A.out[90 * S + qp];
      {
        double pFn[9];
#pragma unroll
        for (int i = 0; i < 9; i++) pFn[i] = A.state_n[i * S + qp];
        inv3(pFn, pFni);
      }
      {
        double W[9];
        mm3(pFni, M, W);
        if (sub == 0)
#pragma unroll
          for (int i = 0; i < 9; i++) reg[kCtW + i] = W[i];
      }
      {
        double Fq[9], Fe[9], Cep[9], CepM[9];
#pragma unroll
        for (int i = 0; i < 9; i++) Fq[i] = A.F[i * S + qp];
        if (sub == 0)
#pragma unroll
          for (int i = 0; i < 9; i++) reg[kCtF + i] = Fq[i];
        mm3(Fq, pFni, Fe);
        mm3tn(Fe, Fe, Cep);
        mm3(Cep, M, CepM);
        if (sub == 0)
#pragma unroll
          for (int i = 0; i < 9; i++) reg[kCtCM + i] = CepM[i];
        double Ce[9];
        mm3tn(M, CepM, Ce);
        C6[0] = Ce[0], C6[1] = Ce[4], C6[2] = Ce[8], C6[3] = Ce[5], C6[4] = Ce[2], C6[5] = Ce[1];
      }
      const double detC = C6[0] * (C6[1] * C6[2] - C6[3] * C6[3]) - C6[5] * (C6[5] * C6[2] - C6[3] * C6[4]) +
                          C6[4] * (C6[5] * C6[3] - C6[1] * C6[4]);
      ok = detC > 0.0 && g > 0.0;
      if (ok) {
        const double J = sqrt(detC), a = A.mat.mu / cbrt(detC), pv = A.mat.kappa * J * (J - 1.0);
        const double trC = C6[0] + C6[1] + C6[2], id = 1.0 / detC;
        if (sub == 0) {
          reg[kCtCi + 0] = (C6[1] * C6[2] - C6[3] * C6[3]) * id;
          reg[kCtCi + 1] = (C6[0] * C6[2] - C6[4] * C6[4]) * id;
          reg[kCtCi + 2] = (C6[0] * C6[1] - C6[5] * C6[5]) * id;
          reg[kCtCi + 3] = (C6[4] * C6[5] - C6[0] * C6[3]) * id;
          reg[kCtCi + 4] = (C6[5] * C6[3] - C6[1] * C6[4]) * id;
          reg[kCtCi + 5] = (C6[3] * C6[4] - C6[2] * C6[5]) * id;
#pragma unroll
          for (int i = 0; i < 6; i++) reg[kCtCe + i] = C6[i];
          reg[kCtSc] = a;
          reg[kCtSc + 1] = pv;
          reg[kCtSc + 2] = trC;
          reg[kCtSc + 3] = J;
#pragma unroll
          for (int i = 0; i < 9; i++) reg[kCtR + i] = A.Rcp[i * A.ne + e];
        }
        __syncwarp(qm);
        // the own systems' slip rates: the hardening slope needs their sum
#pragma unroll 1
        for (int k = 0; k < 3; k++) {
          double sv[3], nv[3], c[3];
          slip_sn(reg + kCtR, 4 * k + sub, sv, nv);
          symv6(C6, sv, c);
          const double sn = sv[0] * nv[0] + sv[1] * nv[1] + sv[2] * nv[2];
          const double tau = a * ((c[0] * nv[0] + c[1] * nv[1] + c[2] * nv[2]) - trC / 3.0 * sn) + pv * sn;
          gsum += fabs(A.mat.gdot0 * (tau / g) * flow_pow(fabs(tau / g), im - 1.0));
        }
      }
    }
    ok = __shfl_sync(qm, ok, lane & ~3) != 0;  // the quad agrees (identical inputs)
    if (ok) {
      gsum = quad_sum(qm, gsum);
      const CpHard hd = cp_hardening(A.mat, gsum, g, dt);
      // own rows: J identity (row 9 zero), B zero
#pragma unroll
      for (int r = 0; r < 3; r++) {
        const int i = sub + 4 * r;
        if (i < 10) {
#pragma unroll
          for (int j = 0; j < 10; j++) reg[kCtJ + i * 10 + j] = (i == j && i < 9) ? 1.0 : 0.0;
#pragma unroll
          for (int j = 0; j < 9; j++) reg[kCtB + i * 9 + j] = 0.0;
        }
      }
      __syncwarp(qm);
      const double a = reg[kCtSc], pv = reg[kCtSc + 1], trC = reg[kCtSc + 2], J = reg[kCtSc + 3];
      const double *R = reg + kCtR;
      // pass 0: Jacobian rows (records dtau, gd, dgd); pass 1: right-hand
      // sides (records 2 dtF, cf, dRg sg dgd)
#pragma unroll 1
      for (int pass = 0; pass < 2; pass++) {
#pragma unroll 1
        for (int k = 0; k < 3; k++) {
          {
            const int sa = 4 * k + sub;
            double sv[3], nv[3], Y[9], out9[9];
            slip_sn(R, sa, sv, nv);
            const double tau = ysym_sn(A.mat, reg + kCtCe, reg + kCtCi, a, pv, trC, J, sv, nv, Y);
            const double pw = flow_pow(fabs(tau / g), im - 1.0);
            const double gd = A.mat.gdot0 * (tau / g) * pw, dgd = A.mat.gdot0 * im / g * pw;
            double *x = reg + kCtX + sub * 11;
            if (pass == 0) {
              mm3(reg + kCtCM, Y, out9);  // dtau = 2 Ce'M Ysym
#pragma unroll
              for (int i = 0; i < 9; i++) x[i] = 2.0 * out9[i];
              x[9] = gd;
              x[10] = dgd;
            } else {
              double t1[9], Z[9];
              mm3(reg + kCtW, Y, t1);
              mm3nt(t1, reg + kCtW, Z);  // Z = pF_n^-1 M Ysym M^T pF_n^-T
              mm3(reg + kCtF, Z, out9);   // dtF
              const double sg = gd < 0 ? -1.0 : 1.0;
#pragma unroll
              for (int i = 0; i < 9; i++) x[i] = 2.0 * out9[i];
              x[9] = dt * dgd;            // cf
              x[10] = hd.dRg * sg * dgd;  // row 9 weight
            }
          }
          __syncwarp(qm);
          // the round's four systems into the own rows: the Schmid entries of
          // the own rows first, then one row at a time
          double Pr[4][3];
#pragma unroll 1
          for (int o = 0; o < 4; o++) {
            double sv[3], nv[3];
            slip_sn(R, 4 * k + o, sv, nv);
#pragma unroll
            for (int r = 0; r < 3; r++) {
              const int i = sub + 4 * r, ii = i / 3, jj = i - 3 * ii;  // run-time row: select, do not index
              const double Pv = (ii == 0 ? sv[0] : (ii == 1 ? sv[1] : sv[2])) *
                                (jj == 0 ? nv[0] : (jj == 1 ? nv[1] : nv[2]));
#pragma unroll
              for (int oo = 0; oo < 4; oo++)
                if (oo == o) Pr[oo][r] = Pv;
            }
          }
#pragma unroll
          for (int r = 0; r < 3; r++) {
            const int i = sub + 4 * r;
            if (i >= 10) continue;
#pragma unroll 1
            for (int o = 0; o < 4; o++) {
              const double *x = reg + kCtX + o * 11;
              const double Pi = o == 0 ? Pr[0][r] : (o == 1 ? Pr[1][r] : (o == 2 ? Pr[2][r] : Pr[3][r]));
              if (pass == 0) {
                double *row = reg + kCtJ + i * 10;
                const double gd = x[9], dgd = x[10];
                if (i == 9) {
                  const double sgd = (gd < 0 ? -1.0 : 1.0) * dgd;
#pragma unroll
                  for (int j = 0; j < 9; j++) row[j] += sgd * x[j];
                } else {
                  const double cf = dt * dgd, cg = dt * (-gd / (A.mat.m * g));
#pragma unroll
                  for (int j = 0; j < 9; j++) row[j] += cf * Pi * x[j];
                  row[9] += cg * Pi;
                }
              } else {
                double *row = reg + kCtB + i * 9;
                const double wgt = i == 9 ? x[10] : x[9] * Pi;
#pragma unroll
                for (int j = 0; j < 9; j++) row[j] -= wgt * x[j];
              }
            }
          }
          __syncwarp(qm);  // the records are read before the next round overwrites them
        }
        if (pass == 0 && sub == 1) {  // row 9 of the Jacobian
          const double c = dt * A.mat.G0 / (hd.gs - A.mat.g0);
          double *row = reg + kCtJ + 90;
#pragma unroll
          for (int j = 0; j < 9; j++) row[j] = hd.dRg * row[j];
          row[9] = 1.0 + c * gsum - hd.dRg * gsum / (A.mat.m * g);
        }
        __syncwarp(qm);
      }
      // pivoted elimination: rows i = sub (mod 4), swaps over the 19 columns
      double *Am = reg + kCtJ, *Bm = reg + kCtB;
#pragma unroll 1
      for (int k = 0; k < 10 && ok; k++) {
        double best = -1.0;
        int p = k;
        for (int i = k + ((sub - k) & 3); i < 10; i += 4) {
          const double v = fabs(Am[i * 10 + k]);
          if (v > best) {
            best = v;
            p = i;
          }
        }
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
          const double ob = __shfl_xor_sync(qm, best, o);
          const int op = __shfl_xor_sync(qm, p, o);
          if (ob > best || (ob == best && op < p)) {
            best = ob;
            p = op;
          }
        }
        if (!(best > 0.0)) {
          ok = false;
          break;
        }
        if (p != k) {
          for (int j = sub; j < 19; j += 4) {
            double *x = j < 10 ? Am + k * 10 + j : Bm + k * 9 + (j - 10);
            double *y = j < 10 ? Am + p * 10 + j : Bm + p * 9 + (j - 10);
            const double t = *x;
            *x = *y;
            *y = t;
          }
          __syncwarp(qm);
        }
        const double inv = 1.0 / Am[k * 10 + k];
        for (int i = k + 1 + ((sub - k - 1) & 3); i < 10; i += 4) {
          const double f = Am[i * 10 + k] * inv;
          if (f == 0.0) continue;
          for (int j = k; j < 10; j++) Am[i * 10 + j] -= f * Am[k * 10 + j];
          for (int j = 0; j < 9; j++) Bm[i * 9 + j] -= f * Bm[k * 9 + j];
        }
        __syncwarp(qm);
      }
      if (ok) {
        // back substitution, columns c = sub (mod 4), and the output
        for (int c = sub; c < 9; c += 4) {
          for (int k = 9; k >= 0; k--) {
            const double inv = 1.0 / Am[k * 10 + k];
            double v = Bm[k * 9 + c];
            for (int i = k + 1; i < 10; i++) v -= Am[k * 10 + i] * Bm[i * 9 + c];
            Bm[k * 9 + c] = v * inv;
          }
#pragma unroll
          for (int r = 0; r < 9; r++) A.out[(9 + r * 9 + c) * S + qp] = Bm[r * 9 + c];
        }
      } else if (sub == 0) {
        atomicAdd(&A.status[3], 1ull);
      }
    }
    if (!ok)
      for (int r = sub; r < 81; r += 4) A.out[(9 + r) * S + qp] = 0.0;
    __syncwarp(qm);
  }
}

inline size_t cp_tangent_smem() { return sizeof(double) * kCtPts * kCtQS; }

}  // namespace pgb

namespace pgb {

// Deformation gradient per point of linear tets (constant gradients); status
// (inverted elements) and detJw may be null.
__global__ void k_cp_F(const double *X, const double *unode, const int *conn, long nn, long ne,
                       const double *F0, double *F, double *detJw, unsigned long long *status) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int nd[4];
  double x[4][3], u[4][3];
#pragma unroll
  for (int a = 0; a < 4; a++) {
    nd[a] = conn[(long)a * ne + e];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      x[a][i] = X[i * nn + nd[a]];
      u[a][i] = unode[i * nn + nd[a]];
    }
  }
  double dX[9], dU[9];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      dX[i * 3 + c] = x[c + 1][i] - x[0][i];
      dU[i * 3 + c] = u[c + 1][i] - u[0][i];
    }
  double dXi[9], Fe[9];
  const double dJ = det3(dX);
  bool ok = dJ > 0.0 && inv3(dX, dXi);
  if (ok) {
    mm3(dU, dXi, Fe);
#pragma unroll
    for (int i = 0; i < 9; i++) Fe[i] += (i % 4 == 0 ? 1.0 : 0.0) + (F0 ? F0[i] : 0.0);
    ok = det3(Fe) > 0.0;
  }
  if (!ok) {
    if (status) atomicAdd(&status[0], 1ull);
#pragma unroll
    for (int i = 0; i < 9; i++) Fe[i] = (i % 4 == 0 ? 1.0 : 0.0);
  }
#pragma unroll
  for (int i = 0; i < 9; i++) F[i * ne + e] = Fe[i];
  if (detJw) detJw[e] = ok ? dJ / 6.0 : 0.0;
}

// Directional derivative of P / pJ = F M S M^T, with pJ = det pF = 1 / det M
// carried as -tr(M^-1 dM) F M S M^T, for the increments dF and dM
// (Ce = M^T F^T F M; h the stress at Ce; C = F^T F, FM = F M, FMS = F M S,
// Pk = F M S M^T, Mi = M^-1).
__device__ __forceinline__ void cp_piola_dir(const Mat &mat, const NeoHooke &h, const double *F, const double *M,
                                             const double *Mi, const double *C, const double *FM,
                                             const double *FMS, const double *Pk, const double *dF,
                                             const double *dM, double *dP) {
  // dCe = dM^T C M + M^T (dF^T F + F^T dF) M + M^T C dM
  double dC[9], a1[9], a2[9], dCe[9], CdM[9];
  mm3tn(dF, F, a1);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) dC[i * 3 + j] = a1[i * 3 + j] + a1[j * 3 + i];
  mm3(C, dM, CdM);
  mm3(dC, M, a1);
  mm3tn(M, a1, a2);  // M^T dC M
  double b1[9];
  mm3tn(M, CdM, b1);  // M^T C dM
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) dCe[i * 3 + j] = a2[i * 3 + j] + b1[i * 3 + j] + b1[j * 3 + i];
  double dS[9];
  nh_dS(mat, h, dCe, dS);
  // dF M S M^T + F dM S M^T + F M dS M^T + F M S dM^T - tr(M^-1 dM) F M S M^T
  double q1[9], q2[9], q3[9], tmp[9];
  mm3(dF, M, tmp);
  mm3(tmp, h.S, q1);
  mm3nt(q1, M, dP);
  mm3(F, dM, tmp);
  mm3(tmp, h.S, q2);
  mm3nt(q2, M, q3);
#pragma unroll
  for (int i = 0; i < 9; i++) dP[i] += q3[i];
  mm3(FM, dS, q1);
  mm3nt(q1, M, q3);
#pragma unroll
  for (int i = 0; i < 9; i++) dP[i] += q3[i];
  mm3nt(FMS, dM, q3);
  double trMdM = 0;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int k = 0; k < 3; k++) trMdM += Mi[i * 3 + k] * dM[k * 3 + i];
#pragma unroll
  for (int i = 0; i < 9; i++) dP[i] += q3[i] - trMdM * Pk[i];
}

struct CpElemArgs {
  const double *X;
  const int *conn;
  const int *dof, *rowptr0, *rowlen;
  const uint8_t *mask;
  const uint16_t *pos;  // element -> CSR node-block map
  long nn, ne;
  const double *F, *detJw;
  const double *state_n;
  const double *out;  // kCpOut * ne
  double *R, *K;
  // element level (stiffmatel_fd / resid_on_elem): the listed elements' dense
  // element vector fe[nlist][12] and matrix lk[nlist][12][12] (idx_K order,
  // every DOF of the element) instead of the CSR scatter; lk may be nullptr
  const int *elist;
  long nlist;
  double *lk_out, *fe_out;
  Mat mat;
  // transient (mid-point rule) element, k_cp_element_tr: F at t_n and
  // t_{n-1} (SoA 9*ne), the state at t_{n+1} and t_{n-1}, alpha and the two
  // mid points' residual factors; inverted mid points counted in status[0]
  const double *F_n, *F_nm1, *state_np1, *state_nm1;
  double alpha, cA, cB;
  unsigned long long *status;
};

// Element residual and tangent of the CM 1-field element with plasticity
// (compute_residual_vector / compute_stiffness_matrix,
// src/constitutive_model.cc:1520-1662, with M = pF_{n+1}^-1 and dM/du),
// written through the first Piola stress P = pJ F M S M^T of the element:
// R_a = w P grad N_a and dR_a/du = w dP grad N_a.
__global__ void __launch_bounds__(128) k_cp_element(const CpElemArgs A) {
  const long it = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const bool dense = A.elist != nullptr;
  if (it >= (dense ? A.nlist : A.ne)) return;
  const long e = dense ? (long)A.elist[it] : it;
  double *fe = dense ? A.fe_out + it * 12 : nullptr;
  double *lk = dense && A.lk_out ? A.lk_out + it * 144 : nullptr;
  if (dense) {  // zero outputs for an inverted element (counted by the F kernel)
#pragma unroll
    for (int k = 0; k < 12; k++) fe[k] = 0.0;
    if (lk)
      for (int k = 0; k < 144; k++) lk[k] = 0.0;
  }
  const long S = A.ne;
  const double w = A.detJw[e];
  if (!(w > 0.0)) return;
  int nd[4];
  double x[4][3];
#pragma unroll
  for (int a = 0; a < 4; a++) {
    nd[a] = A.conn[(long)a * A.ne + e];
#pragma unroll
    for (int i = 0; i < 3; i++) x[a][i] = A.X[i * A.nn + nd[a]];
  }
  double dX[9], dXi[9];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int c = 0; c < 3; c++) dX[i * 3 + c] = x[c + 1][i] - x[0][i];
  inv3(dX, dXi);
  double gN[4][3];  // grad_X N_a = dXi^T dN/dxi
#pragma unroll
  for (int j = 0; j < 3; j++) {
    gN[1][j] = dXi[0 * 3 + j];
    gN[2][j] = dXi[1 * 3 + j];
    gN[3][j] = dXi[2 * 3 + j];
    gN[0][j] = -(gN[1][j] + gN[2][j] + gN[3][j]);
  }
  double F[9], Mu[9], pFn[9], pFni[9], M[9];
#pragma unroll
  for (int i = 0; i < 9; i++) {
    F[i] = A.F[i * S + e];
    Mu[i] = A.out[i * S + e];
    pFn[i] = A.state_n[i * S + e];
  }
  inv3(pFn, pFni);
  mm3(pFni, Mu, M);  // M_TL = pF_{n+1}^-1
  double C[9], t[9], Ce[9];
  mm3tn(F, F, C);
  mm3(C, M, t);
  mm3tn(M, t, Ce);
  NeoHooke h;
  if (!nh_stress(A.mat, Ce, h)) return;
  const double pJ = det3(pFn) / det3(Mu);
  double Mi[9];
  inv3(M, Mi);
  double FM[9], FMS[9], Pk[9];
  mm3(F, M, FM);
  mm3(FM, h.S, FMS);
  mm3nt(FMS, M, Pk);  // F M S M^T
  // residual
  double Re[12];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int i = 0; i < 3; i++)
      Re[a * 3 + i] = w * pJ * (Pk[i * 3] * gN[a][0] + Pk[i * 3 + 1] * gN[a][1] + Pk[i * 3 + 2] * gN[a][2]);
  // dense element outputs take every DOF of the element
  const unsigned mk[4] = {dense ? 7u : A.mask[nd[0]], dense ? 7u : A.mask[nd[1]], dense ? 7u : A.mask[nd[2]],
                          dense ? 7u : A.mask[nd[3]]};
  if (dense) {
#pragma unroll
    for (int k = 0; k < 12; k++) fe[k] = Re[k];
    if (!lk) return;
  } else {
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int i = 0; i < 3; i++) {
        const int id = A.dof[i * A.nn + nd[a]];
        if (id > 0) atomicAdd(A.R + (id - 1), Re[a * 3 + i]);
      }
    if (!A.K) return;
  }
  // tangent columns (node wn, component gc)
  for (int wn = 0; wn < 4; wn++) {
    if (!mk[wn]) continue;
    for (int gc = 0; gc < 3; gc++) {
      if (!((mk[wn] >> gc) & 1u)) continue;
      double dMu[9], dM[9];
#pragma unroll
      for (int ij = 0; ij < 9; ij++)
        dMu[ij] = A.out[(9 + ij * 9 + gc * 3 + 0) * S + e] * gN[wn][0] +
                  A.out[(9 + ij * 9 + gc * 3 + 1) * S + e] * gN[wn][1] +
                  A.out[(9 + ij * 9 + gc * 3 + 2) * S + e] * gN[wn][2];
      mm3(pFni, dMu, dM);
      double dF[9];
#pragma unroll
      for (int i = 0; i < 9; i++) dF[i] = 0.0;
      dF[gc * 3 + 0] = gN[wn][0];
      dF[gc * 3 + 1] = gN[wn][1];
      dF[gc * 3 + 2] = gN[wn][2];
      double dP[9];
      cp_piola_dir(A.mat, h, F, M, Mi, C, FM, FMS, Pk, dF, dM, dP);
#pragma unroll
      for (int i = 0; i < 9; i++) dP[i] *= w * pJ;
      if (dense) {  // column (wn, gc) of the element matrix, idx_K order
        for (int a = 0; a < 4; a++)
#pragma unroll
          for (int i = 0; i < 3; i++)
            lk[(a * 3 + i) * 12 + wn * 3 + gc] =
                dP[i * 3] * gN[a][0] + dP[i * 3 + 1] * gN[a][1] + dP[i * 3 + 2] * gN[a][2];
        continue;
      }
      // scatter the column into the rows of the element's nodes
      const long pcol = (e * 4 + 0) * 4 + wn;  // pos of (a, wn) at (e*4 + a)*4 + wn
      for (int a = 0; a < 4; a++) {
        if (!mk[a]) continue;
        const long base = (long)A.rowptr0[nd[a]] + A.pos[pcol + a * 4] + rank_of(mk[wn], gc);
#pragma unroll
        for (int i = 0; i < 3; i++) {
          if (!((mk[a] >> i) & 1u)) continue;
          const double v = dP[i * 3] * gN[a][0] + dP[i * 3 + 1] * gN[a][1] + dP[i * 3 + 2] * gN[a][2];
          atomicAdd(A.K + base + (long)rank_of(mk[a], i) * A.rowlen[nd[a]], v);
        }
      }
    }
  }
}

// Transient (mid-point rule) element of crystal plasticity on linear tets
// (residuals_el_constitutive_model_n_plus_alpha and
// stiffness_el_constitutive_model_w_inertia_1f, src/constitutive_model.cc:
// 1905-2170, 2803-2958).  At a mid point F = mid(F_a, F_b), pF = mid(pF_a,
// pF_b), M = pF^-1 and P = det(pF) F M S(M^T F^T F M) M^T:
//   R += cA w P(n+alpha) grad N_a + cB w P(n-1+alpha) grad N_a
//   K += cA w dP(n+alpha) grad N_a
// where only the newer mid point depends on u_{n+1}: dF(n+alpha) = alpha dF,
// dM(n+alpha) = -M (alpha dpF_{n+1}) M and dpF_{n+1} = -pF_{n+1}
// d(pF_{n+1}^-1) pF_{n+1}, from the consistent derivative of the local
// update (pF_{n+1}^-1 = pF_n^-1 M_u, dM_u = dM/dF : dF).
__global__ void __launch_bounds__(128) k_cp_element_tr(const CpElemArgs A) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= A.ne) return;
  const long S = A.ne;
  const double w = A.detJw[e];
  if (!(w > 0.0)) return;
  int nd[4];
  double x[4][3];
#pragma unroll
  for (int a = 0; a < 4; a++) {
    nd[a] = A.conn[(long)a * A.ne + e];
#pragma unroll
    for (int i = 0; i < 3; i++) x[a][i] = A.X[i * A.nn + nd[a]];
  }
  double dX[9], dXi[9];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int c = 0; c < 3; c++) dX[i * 3 + c] = x[c + 1][i] - x[0][i];
  inv3(dX, dXi);
  double gN[4][3];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    gN[1][j] = dXi[0 * 3 + j];
    gN[2][j] = dXi[1 * 3 + j];
    gN[3][j] = dXi[2 * 3 + j];
    gN[0][j] = -(gN[1][j] + gN[2][j] + gN[3][j]);
  }
  const double al = A.alpha;
  double Fa[9], Fb[9], pFa[9], pFb[9], pF2[9], pF1[9];
#pragma unroll
  for (int i = 0; i < 9; i++) {
    const double f2 = A.F[i * S + e], f1 = A.F_n[i * S + e], f0 = A.F_nm1[i * S + e];
    pF2[i] = A.state_np1[i * S + e];
    pF1[i] = A.state_n[i * S + e];
    const double p0 = A.state_nm1[i * S + e];
    Fa[i] = (1.0 - al) * f1 + al * f2;
    Fb[i] = (1.0 - al) * f0 + al * f1;
    pFa[i] = (1.0 - al) * pF1[i] + al * pF2[i];
    pFb[i] = (1.0 - al) * p0 + al * pF1[i];
  }
  if (!(det3(Fa) > 0.0) || !(det3(Fb) > 0.0)) {  // getJacobian of each mid point
    atomicAdd(&A.status[0], 1ull);
    return;
  }
  double Ma[9], Mb[9];
  if (!inv3(pFa, Ma) || !inv3(pFb, Mb)) return;
  double Re[12];
  {  // the older mid point: residual only
    double C[9], t[9], Ce[9];
    mm3tn(Fb, Fb, C);
    mm3(C, Mb, t);
    mm3tn(Mb, t, Ce);
    NeoHooke hb;
    if (!nh_stress(A.mat, Ce, hb)) return;
    double FM[9], FMS[9], Pb[9];
    mm3(Fb, Mb, FM);
    mm3(FM, hb.S, FMS);
    mm3nt(FMS, Mb, Pb);
    const double cb = A.cB * w * det3(pFb);
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int i = 0; i < 3; i++)
        Re[a * 3 + i] = cb * (Pb[i * 3] * gN[a][0] + Pb[i * 3 + 1] * gN[a][1] + Pb[i * 3 + 2] * gN[a][2]);
  }
  double C[9], FM[9], FMS[9], Pa[9];
  NeoHooke h;
  {
    double t[9], Ce[9];
    mm3tn(Fa, Fa, C);
    mm3(C, Ma, t);
    mm3tn(Ma, t, Ce);
    if (!nh_stress(A.mat, Ce, h)) return;
  }
  mm3(Fa, Ma, FM);
  mm3(FM, h.S, FMS);
  mm3nt(FMS, Ma, Pa);
  const double ca = A.cA * w * det3(pFa);
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int i = 0; i < 3; i++)
      Re[a * 3 + i] += ca * (Pa[i * 3] * gN[a][0] + Pa[i * 3 + 1] * gN[a][1] + Pa[i * 3 + 2] * gN[a][2]);
  const unsigned mk[4] = {A.mask[nd[0]], A.mask[nd[1]], A.mask[nd[2]], A.mask[nd[3]]};
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const int id = A.dof[i * A.nn + nd[a]];
      if (id > 0) atomicAdd(A.R + (id - 1), Re[a * 3 + i]);
    }
  if (!A.K) return;
  double pF1i[9];
  inv3(pF1, pF1i);
  for (int wn = 0; wn < 4; wn++) {
    if (!mk[wn]) continue;
    for (int gc = 0; gc < 3; gc++) {
      if (!((mk[wn] >> gc) & 1u)) continue;
      double dMu[9], dMtl[9], t1[9], t2[9], dMa[9];
#pragma unroll
      for (int ij = 0; ij < 9; ij++)
        dMu[ij] = A.out[(9 + ij * 9 + gc * 3 + 0) * S + e] * gN[wn][0] +
                  A.out[(9 + ij * 9 + gc * 3 + 1) * S + e] * gN[wn][1] +
                  A.out[(9 + ij * 9 + gc * 3 + 2) * S + e] * gN[wn][2];
      mm3(pF1i, dMu, dMtl);  // d(pF_{n+1}^-1)
      mm3(pF2, dMtl, t1);
      mm3(t1, pF2, t2);      // -dpF_{n+1}
      mm3(Ma, t2, t1);
      mm3(t1, Ma, dMa);
#pragma unroll
      for (int i = 0; i < 9; i++) dMa[i] *= al;
      double dF[9];
#pragma unroll
      for (int i = 0; i < 9; i++) dF[i] = 0.0;
      dF[gc * 3 + 0] = al * gN[wn][0];
      dF[gc * 3 + 1] = al * gN[wn][1];
      dF[gc * 3 + 2] = al * gN[wn][2];
      double dP[9];
      cp_piola_dir(A.mat, h, Fa, Ma, pFa, C, FM, FMS, Pa, dF, dMa, dP);
      const long pcol = (e * 4 + 0) * 4 + wn;
      for (int a = 0; a < 4; a++) {
        if (!mk[a]) continue;
        const long base = (long)A.rowptr0[nd[a]] + A.pos[pcol + a * 4] + rank_of(mk[wn], gc);
#pragma unroll
        for (int i = 0; i < 3; i++) {
          if (!((mk[a] >> i) & 1u)) continue;
          const double v = ca * (dP[i * 3] * gN[a][0] + dP[i * 3 + 1] * gN[a][1] + dP[i * 3 + 2] * gN[a][2]);
          atomicAdd(A.K + base + (long)rank_of(mk[a], i) * A.rowlen[nd[a]], v);
        }
      }
    }
  }
}

// ---- learned warm start: features, guess, training pairs -------------------

// Unit quaternion (w, x, y, z), w >= 0, of a rotation matrix (Shepperd's
// method: branch on the largest of the trace and the diagonal).
__device__ __forceinline__ void rot_to_quat(const double *R, double *q) {
  const double tr = R[0] + R[4] + R[8];
  double w, x, y, z;
  if (tr > 0.0) {
    const double s = 2.0 * sqrt(tr + 1.0);
    w = 0.25 * s, x = (R[7] - R[5]) / s, y = (R[2] - R[6]) / s, z = (R[3] - R[1]) / s;
  } else if (R[0] > R[4] && R[0] > R[8]) {
    const double s = 2.0 * sqrt(1.0 + R[0] - R[4] - R[8]);
    w = (R[7] - R[5]) / s, x = 0.25 * s, y = (R[1] + R[3]) / s, z = (R[2] + R[6]) / s;
  } else if (R[4] > R[8]) {
    const double s = 2.0 * sqrt(1.0 + R[4] - R[0] - R[8]);
    w = (R[2] - R[6]) / s, x = (R[1] + R[3]) / s, y = 0.25 * s, z = (R[5] + R[7]) / s;
  } else {
    const double s = 2.0 * sqrt(1.0 + R[8] - R[0] - R[4]);
    w = (R[3] - R[1]) / s, x = (R[2] + R[6]) / s, y = (R[5] + R[7]) / s, z = 0.25 * s;
  }
  const double sg = w < 0.0 ? -1.0 : 1.0;
  q[0] = sg * w, q[1] = sg * x, q[2] = sg * y, q[3] = sg * z;
}

constexpr int kCpFeat = 34;

// Network features per point (row of 34 FP32), tensors in the lattice frame of
// the point's crystal (R^T A R), where the slip systems are the same for every
// grain: F F_n^-1 - I (9), pF_n - I (9), the 12 slip resistances (g_n for every
// system), lattice quaternion (4).
__global__ void k_cp_features(long nqp, const double *__restrict__ F, const double *__restrict__ Fn,
                              const double *__restrict__ state_n, const double *__restrict__ Rcp, int nqp_e,
                              long ne, float *__restrict__ x) {
  const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= nqp) return;
  double f[9], fn[9], fni[9], d[9], R[9], qt[4];
  const long e = q / nqp_e;
#pragma unroll
  for (int i = 0; i < 9; i++) {
    f[i] = F[i * nqp + q];
    fn[i] = Fn[i * nqp + q];
    R[i] = Rcp[i * ne + e];
  }
  if (!inv3(fn, fni))
#pragma unroll
    for (int i = 0; i < 9; i++) fni[i] = (i % 4 == 0) ? 1.0 : 0.0;
  mm3(f, fni, d);
  rot_to_quat(R, qt);
  double pf[9], t[9], dc[9], pc[9];
#pragma unroll
  for (int i = 0; i < 9; i++) pf[i] = state_n[i * nqp + q];
  mm3(d, R, t);  // lattice frame: R^T A R
  mm3tn(R, t, dc);
  mm3(pf, R, t);
  mm3tn(R, t, pc);
  float *o = x + q * kCpFeat;
#pragma unroll
  for (int i = 0; i < 9; i++) o[i] = (float)(dc[i] - (i % 4 == 0 ? 1.0 : 0.0));
#pragma unroll
  for (int i = 0; i < 9; i++) o[9 + i] = (float)(pc[i] - (i % 4 == 0 ? 1.0 : 0.0));
  const float gn = (float)state_n[9 * nqp + q];
#pragma unroll
  for (int a = 0; a < kSlip; a++) o[18 + a] = gn;
#pragma unroll
  for (int i = 0; i < 4; i++) o[30 + i] = (float)qt[i];
}

// Newton guess from predicted slip increments y (AoS nqp x 12):
// M0 = I - sum_a y_a P_a, and g0 from the hardening update with
// dt*gamma_dot = sum_a |y_a|:  g0 = (g_n + c gs) / (1 + c),  c = G0 sum|y| / (gs - g0).
__global__ void k_cp_guess(long nqp, const float *__restrict__ y, const double *__restrict__ Rcp, int nqp_e,
                           long ne, const double *__restrict__ state_n, const Mat mat, double *__restrict__ guess) {
  const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= nqp) return;
  double R[9], M[9];
  const long e = q / nqp_e;
#pragma unroll
  for (int i = 0; i < 9; i++) {
    R[i] = Rcp[i * ne + e];
    M[i] = (i % 4 == 0) ? 1.0 : 0.0;
  }
  double sabs = 0.0;
  for (int a = 0; a < kSlip; a++) {
    double P[9];
    schmid(R, a, P);
    const double da = (double)y[q * kSlip + a];
    sabs += fabs(da);
#pragma unroll
    for (int i = 0; i < 9; i++) M[i] -= da * P[i];
  }
  const double c = mat.G0 * sabs / (mat.gs0 - mat.g0);
  const double gn = state_n[9 * nqp + q];
#pragma unroll
  for (int i = 0; i < 9; i++) guess[i * nqp + q] = M[i];
  guess[9 * nqp + q] = (gn + c * mat.gs0) / (1.0 + c);
}

// Converged slip increments of the last local solve as FP32 training targets (AoS nqp x 12).
__global__ void k_cp_targets(long nqp, const double *__restrict__ out, float *__restrict__ t) {
  const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (q >= nqp) return;
#pragma unroll
  for (int a = 0; a < kSlip; a++) t[q * kSlip + a] = (float)out[(91 + a) * nqp + q];
}

}  // namespace pgb
