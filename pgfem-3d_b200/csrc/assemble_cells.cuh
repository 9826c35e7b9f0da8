// assemble_cells.cuh -- fused FP64 R+K assembly of quadratic tets, one Kuhn
// cell (6 elements, 24 quadrature points, 27 nodes) per CTA iteration.
//
// Same operation as k_assemble (fd_residuals_MP + stiffmat_fd_MP for the
// constitutive-model element, src/fd_residuals.cc:468-636,
// src/stiffmat_fd.cc:831-993) with a layout chosen for the FP64 pipe and the
// L2 reduction units:
//
//  L   the cell's node coordinates / displacements, CSR row metadata and
//      node-pair slot map are staged in shared memory (tile_plan.hpp, TE = 6);
//  QV  four lanes per quadrature point: each lane forms F and runs the
//      constitutive update (run_integration_algorithm,
//      src/constitutive_model.cc:1100-1129) in registers -- the four copies
//      are identical, lane 0 writes the state at t_{n+1} -- and then writes
//      the vector records of its 2-3 element nodes (no point record in
//      memory).  With p_a = F^-T grad_X N_a and the spatial tangent
//      c = a1 I + a2 1(x)1 - 2/3 (s(x)1 + 1(x)s) + a4 n(x)n + a5 n(x)dev(n^2)
//      scaled by w = det(dX/dxi) * weight:
//        right  p_b, U_b = w (a2 p_b - 2/3 s p_b), W_b = w (a4 n p_b + a5 dev(n^2) p_b),
//               T_b = w (a1/2 p_b + tau p_b)
//        left   S_a = -2/3 w s p_a, n p_a   (and p_a, shared with the right set)
//      and the residual w tau p_a goes into the cell's node accumulators
//      (compute_residual_vector, :1628-1662);
//  B   thread (element, row node a, half of the column nodes): the left
//      vectors stay in registers while five 3x3 blocks
//        K_ab += (p_b)(a1/2 w p_a)^T + p_a U_b^T + S_a p_b^T + (n p_a) W_b^T + (p_a . T_b) 1
//      accumulate over the points (compute_stiffness_matrix, :1520-1616, in
//      spatial form): 45 independent FMA chains per thread, right vectors as
//      16-byte shared loads that a warp shares across its lanes; the blocks
//      are then added into the cell's node-pair slots (shared FP64 atomics);
//  W   one warp per (node, component) row issues the cell's slots as FP64
//      reductions in CSR address order (consecutive lanes -> consecutive
//      doubles), plus the nodal residuals (fd_res_assemble,
//      src/fd_residuals.cc:58-73; PLoc_Sparse, src/PLoc_Sparse.cc:15-175).
#pragma once
#include <cstdint>

#include "assemble_tiles.cuh"

namespace pgb {

constexpr int kCellThreads = 128;
constexpr int kCellVS = 18;  // doubles per (point, element node) vector record
constexpr int kCellTE = 6, kCellNNE = 10, kCellNQP = 4;
constexpr int kCellNL = kCellTE * kCellNNE;   // local node bound (27 used)
constexpr int kCellNQ = kCellTE * kCellNQP;  // points per cell

struct CellArgs {
  const double *X, *unode;  // 3*nn SoA
  const int *conn;          // NNE*ne SoA
  long nn, ne, nqp;
  const double *F0;
  const double *state_n;
  double *state_np1;
  const int *dof, *rowptr0, *rowlen;
  const uint8_t *mask;
  // plan (tile_plan.hpp with TE = 6)
  const int *tile_nodes;
  const uint8_t *tile_nl;
  const uint8_t *elem_lnode;
  const uint16_t *elem_slot;
  const long long *slot_off;
  const uint32_t *slot_info;
  const uint16_t *aoff;
  const uint8_t *allfree;
  long ntiles;
  int nslots_max;
  double *R, *K;
  unsigned long long *status;
  Mat mat;
  ShapeTable shp;
};

inline size_t cells_smem_bytes(int nslots_max) {
  return sizeof(double) * ((size_t)kCellNL * 6 + (size_t)kCellNQ * kCellNNE * kCellVS + (size_t)kCellNL * 3 +
                           (size_t)kCellNQ + (size_t)nslots_max * 9) +
         sizeof(uint32_t) * (size_t)nslots_max;
}

template <int MODEL>
__global__ void __launch_bounds__(kCellThreads, 3) k_assemble_cells(const CellArgs A) {
  constexpr int NNE = kCellNNE, NQP = kCellNQP, TE = kCellTE, NL = kCellNL, NQ = kCellNQ, VS = kCellVS;
  constexpr bool PLASTIC = (MODEL == 1);
  extern __shared__ double sm[];
  double *sXU = sm;                      // [NL][6] local node X, u
  double *sV = sXU + NL * 6;             // [NQ][NNE][VS] vector records
  double *sR = sV + NQ * NNE * VS;       // [NL][3] nodal residuals
  double *sA1 = sR + NL * 3;             // [NQ] w a1 / 2
  double *sAcc = sA1 + NQ;               // [nslots][9] node-pair blocks
  uint32_t *s_sinfo = reinterpret_cast<uint32_t *>(sAcc + (size_t)A.nslots_max * 9);
  __shared__ int s_rp[NL], s_rl[NL], s_ndof[NL * 3];
  __shared__ uint8_t s_mask[NL];
  __shared__ uint8_t s_lnode[TE * NNE];
  __shared__ uint16_t s_aoff[NL + 1];
  __shared__ uint16_t s_eslot[TE * NNE * NNE];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  for (int i = tid; i < A.nslots_max * 9; i += kCellThreads) sAcc[i] = 0.0;
  for (int i = tid; i < NL * 3; i += kCellThreads) sR[i] = 0.0;

  for (long t = blockIdx.x; t < A.ntiles; t += gridDim.x) {
    const long e0 = t * TE;
    const int nel = (int)min((long)TE, A.ne - e0);
    const int nl = A.tile_nl[t];
    const long sbeg = A.slot_off[t];
    const int nslots = (int)(A.slot_off[t + 1] - sbeg);

    // ---- L: cell metadata ----
    for (int i = tid; i < nl; i += kCellThreads) {
      const int n = A.tile_nodes[t * NL + i];
      s_mask[i] = A.mask[n];
      s_rp[i] = A.rowptr0[n];
      s_rl[i] = A.rowlen[n];
      s_ndof[i * 3 + 0] = A.dof[n];
      s_ndof[i * 3 + 1] = A.dof[A.nn + n];
      s_ndof[i * 3 + 2] = A.dof[2 * A.nn + n];
      double *d = sXU + i * 6;
      d[0] = A.X[n];
      d[1] = A.X[A.nn + n];
      d[2] = A.X[2 * A.nn + n];
      d[3] = A.unode[n];
      d[4] = A.unode[A.nn + n];
      d[5] = A.unode[2 * A.nn + n];
    }
    for (int i = tid; i < nslots; i += kCellThreads) s_sinfo[i] = A.slot_info[sbeg + i];
    for (int i = tid; i < nel * NNE * NNE; i += kCellThreads) s_eslot[i] = A.elem_slot[e0 * NNE * NNE + i];
    for (int i = tid; i < nel * NNE; i += kCellThreads) s_lnode[i] = A.elem_lnode[e0 * NNE + i];
    for (int i = tid; i <= nl; i += kCellThreads) s_aoff[i] = A.aoff[t * (NL + 1) + i];
    __syncthreads();

    // ---- QV: four lanes per quadrature point ----
    if (tid < NQ * 4) {
      const int qi = tid >> 2, g = tid & 3;
      const int el = qi / NQP, q = qi - el * NQP;
      if (el < nel) {
        const long e = e0 + el;
        double dX[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, dU[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int b = 0; b < NNE; b++) {
          const double *xu = sXU + s_lnode[el * NNE + b] * 6;
          const double g0 = A.shp.dNxi[q][b][0], g1 = A.shp.dNxi[q][b][1], g2 = A.shp.dNxi[q][b][2];
#pragma unroll
          for (int i = 0; i < 3; i++) {
            const double x = xu[i], u = xu[3 + i];
            dX[i * 3 + 0] += g0 * x;
            dX[i * 3 + 1] += g1 * x;
            dX[i * 3 + 2] += g2 * x;
            dU[i * 3 + 0] += g0 * u;
            dU[i * 3 + 1] += g1 * u;
            dU[i * 3 + 2] += g2 * u;
          }
        }
        const double detJ = det3(dX);
        double dXi[9], F[9], Fi[9];
        bool ok = detJ > 0.0 && inv3(dX, dXi);
        if (ok) {
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
              F[i * 3 + j] = (i == j ? 1.0 : 0.0) + dU[i * 3 + 0] * dXi[0 * 3 + j] +
                             dU[i * 3 + 1] * dXi[1 * 3 + j] + dU[i * 3 + 2] * dXi[2 * 3 + j];
          if (A.F0)
#pragma unroll
            for (int i = 0; i < 9; i++) F[i] += A.F0[i];
        }
        const double J = ok ? det3(F) : -1.0;
        if (ok) ok = J > 0.0 && inv3(F, Fi);
        const long qp = e * NQP + q;
        if (!ok) {
          if (g == 0) {
            atomicAdd(&A.status[0], 1ull);
            sA1[qi] = 0.0;
          }
          for (int a = g; a < NNE; a += 4) {
            double *v = sV + (qi * NNE + a) * VS;
#pragma unroll
            for (int c = 0; c < VS; c++) v[c] = 0.0;
          }
        } else {
          double Ast[6] = {1, 1, 1, 0, 0, 0}, alpha = 0.0;
          if (PLASTIC) {
#pragma unroll
            for (int c = 0; c < 6; c++) Ast[c] = A.state_n[c * A.nqp + qp];
            alpha = A.state_n[6 * A.nqp + qp];
          }
          QpTangent tg;
          double Anp1[6], alpha_np1;
          spatial_update<PLASTIC>(A.mat, F, J, Ast, alpha, tg, Anp1, &alpha_np1);
          if (PLASTIC && A.state_np1 && g == 0) {
#pragma unroll
            for (int c = 0; c < 6; c++) A.state_np1[c * A.nqp + qp] = Anp1[c];
            A.state_np1[6 * A.nqp + qp] = alpha_np1;
          }
          double G[9];  // p_a = G^T dN_a/dxi
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
              G[i * 3 + j] = dXi[i * 3 + 0] * Fi[0 * 3 + j] + dXi[i * 3 + 1] * Fi[1 * 3 + j] +
                             dXi[i * 3 + 2] * Fi[2 * 3 + j];
          const double w = detJ * A.shp.w[q];
          const double a1h = 0.5 * tg.a1 * w, a2w = tg.a2 * w, c23 = (2.0 / 3.0) * w;
          const double a4w = tg.a4 * w, a5w = tg.a5 * w;
          if (g == 0) sA1[qi] = a1h;
          for (int a = g; a < NNE; a += 4) {
            const double d0 = A.shp.dNxi[q][a][0], d1 = A.shp.dNxi[q][a][1], d2 = A.shp.dNxi[q][a][2];
            double p[3], sp[3], tp[3], np_[3], mp[3];
#pragma unroll
            for (int j = 0; j < 3; j++) p[j] = G[0 * 3 + j] * d0 + G[1 * 3 + j] * d1 + G[2 * 3 + j] * d2;
            smv(tg.s, p, sp);
            smv(tg.tau, p, tp);
            if (PLASTIC) {
              smv(tg.n, p, np_);
              smv(tg.D, p, mp);
            }
            double *v = sV + (qi * NNE + a) * VS;
            // right set (16-byte aligned pairs): p, U, W, T
#pragma unroll
            for (int j = 0; j < 3; j++) {
              v[j] = p[j];
              v[3 + j] = a2w * p[j] - c23 * sp[j];
              v[6 + j] = PLASTIC ? a4w * np_[j] + a5w * mp[j] : 0.0;
              v[9 + j] = a1h * p[j] + w * tp[j];
              v[12 + j] = -c23 * sp[j];
              v[15 + j] = PLASTIC ? np_[j] : 0.0;
            }
            double *r = sR + s_lnode[el * NNE + a] * 3;
            atomicAdd(r + 0, w * tp[0]);
            atomicAdd(r + 1, w * tp[1]);
            atomicAdd(r + 2, w * tp[2]);
          }
        }
      }
    }
    __syncthreads();

    // ---- B: blocks of (element, row node a, five column nodes) ----
    if (tid < TE * 20) {
      const int el = tid / 20, r = tid - el * 20;
      const int h = r / 10, a = r - h * 10;
      if (el < nel) {
        double acc[5][9];
#pragma unroll
        for (int j = 0; j < 5; j++)
#pragma unroll
          for (int c = 0; c < 9; c++) acc[j][c] = 0.0;
#pragma unroll 1
        for (int q = 0; q < NQP; q++) {
          const int qi = el * NQP + q;
          const double *L = sV + (qi * NNE + a) * VS;
          const double2 l01 = *reinterpret_cast<const double2 *>(L);
          const double pa[3] = {l01.x, l01.y, L[2]};
          const double2 s01 = *reinterpret_cast<const double2 *>(L + 12);
          const double2 s2n0 = *reinterpret_cast<const double2 *>(L + 14);
          const double2 n12 = *reinterpret_cast<const double2 *>(L + 16);
          const double Sa[3] = {s01.x, s01.y, s2n0.x};
          const double na[3] = {s2n0.y, n12.x, n12.y};
          const double a1h = sA1[qi];
          const double ha[3] = {a1h * pa[0], a1h * pa[1], a1h * pa[2]};
#pragma unroll
          for (int j = 0; j < 5; j++) {
            const double *Rv = sV + (qi * NNE + 5 * h + j) * VS;
            const double2 r0 = *reinterpret_cast<const double2 *>(Rv + 0);
            const double2 r1 = *reinterpret_cast<const double2 *>(Rv + 2);
            const double2 r2 = *reinterpret_cast<const double2 *>(Rv + 4);
            const double2 r3 = *reinterpret_cast<const double2 *>(Rv + 6);
            const double2 r4 = *reinterpret_cast<const double2 *>(Rv + 8);
            const double2 r5 = *reinterpret_cast<const double2 *>(Rv + 10);
            const double pb[3] = {r0.x, r0.y, r1.x}, U[3] = {r1.y, r2.x, r2.y};
            const double W[3] = {r3.x, r3.y, r4.x}, T[3] = {r4.y, r5.x, r5.y};
            const double dg = pa[0] * T[0] + pa[1] * T[1] + pa[2] * T[2];
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
              for (int k = 0; k < 3; k++) {
                double v = acc[j][i * 3 + k];
                v = fma(pb[i], ha[k], v);
                v = fma(pa[i], U[k], v);
                v = fma(Sa[i], pb[k], v);
                if (PLASTIC) v = fma(na[i], W[k], v);
                acc[j][i * 3 + k] = v;
              }
            acc[j][0] += dg;
            acc[j][4] += dg;
            acc[j][8] += dg;
          }
        }
        const uint16_t *es = s_eslot + (el * NNE + a) * NNE + 5 * h;
#pragma unroll
        for (int j = 0; j < 5; j++) {
          const uint16_t s = es[j];
          if (s == 0xFFFF) continue;
          double *d = sAcc + s * 9;
#pragma unroll
          for (int c = 0; c < 9; c++) atomicAdd(d + c, acc[j][c]);
        }
      }
    }
    __syncthreads();

    // ---- W: one warp per (node, component) row, lanes along the row ----
    const bool allfree = A.allfree[t] != 0;
    for (int row = warp; row < nl * 3; row += kCellThreads / 32) {
      const int la = row / 3, i = row - la * 3;
      const unsigned mA = s_mask[la];
      const int a0 = s_aoff[la], m3 = 3 * (s_aoff[la + 1] - a0);
      if (allfree) {
        const long base = (long)s_rp[la] + (long)i * s_rl[la];
        for (int j = lane; j < m3; j += 32) {
          const int sl = j / 3, k = j - sl * 3, s = a0 + sl;
          double *src = sAcc + s * 9 + i * 3 + k;
          atomicAdd(A.K + base + (long)(s_sinfo[s] & 0xFFFF) + k, *src);
          *src = 0.0;
        }
        continue;
      }
      const long base = (long)s_rp[la] + (long)rank_of(mA, i) * s_rl[la];
      for (int j = lane; j < m3; j += 32) {
        const int sl = j / 3, k = j - sl * 3, s = a0 + sl;
        double *src = sAcc + s * 9 + i * 3 + k;
        const double v = *src;
        *src = 0.0;
        const uint32_t info = s_sinfo[s];
        const unsigned mB = s_mask[(info >> 16) & 0xFF];
        if (!((mA >> i) & 1u) || !((mB >> k) & 1u)) continue;
        atomicAdd(A.K + base + (long)(info & 0xFFFF) + rank_of(mB, k), v);
      }
    }
    for (int f = tid; f < nl * 3; f += kCellThreads) {
      const int id = s_ndof[f];
      const double v = sR[f];
      sR[f] = 0.0;
      if (id > 0) atomicAdd(A.R + (id - 1), v);
    }
    __syncthreads();
  }
}

}  // namespace pgb
