// assemble_p2.cuh -- FP64 R+K assembly of quadratic tets with column-split
// block rows.  Three kernels share the phases below: k_assemble_p2 (all
// threads run the phases of a tile in turn), k_assemble_p2ws (one producer
// warp runs phases 0-2 of the next tile while four consumer warps run phase 3)
// and k_assemble_p2r, the default for 10-node elements: phase 1 runs first in
// its own kernel (k_qp_update, one thread per point) and k_assemble_p2r is
// the producer/consumer pipeline from the point records.
//
// Same operation as k_assemble (fd_residuals_MP + stiffmat_fd_MP for the
// constitutive-model element, src/fd_residuals.cc:468-636,
// src/stiffmat_fd.cc:831-993), organised for the FP64 pipe and the L2
// reduction units:
//
//  0  thread (element, node): node data and CSR row metadata -> shared memory;
//  1  thread (element, point): F, the constitutive update
//     (run_integration_algorithm, src/constitutive_model.cc:1100-1129; state
//     n -> n+1) and a point record (G = (dX/dxi)^-1 F^-1, w, tau, s, n,
//     dev(n^2), tangent coefficients);
//  2  item (element, point, node): the spatial vectors of the node,
//        p = G^T dN/dxi,  U = w (a2 p - 2/3 s p),  W = w (a4 n p + a5 dev(n^2) p),
//        T = w (a1/2 p + tau p),  S = -2/3 w s p,  n p
//     (the tangent c = a1 I + a2 1(x)1 - 2/3 (s(x)1 + 1(x)s) + a4 n(x)n
//      + a5 n(x)dev(n^2) applied to p_a and p_b in closed form);
//  3  thread (element, row node a, column component k): for every column
//     node b the three entries (i = 0..2, k) of
//        K_ab = sum_q (p_b)(a1/2 w p_a)^T + p_a U_b^T + S_a p_b^T + (n p_a) W_b^T + (p_a . T_b) 1
//     (compute_stiffness_matrix, src/constitutive_model.cc:1520-1616, in
//     spatial form) with the left vectors of a held in registers, and the
//     residual w tau p_a (compute_residual_vector, :1628-1662).  The three
//     lanes k of one (element, a) are adjacent, so each FP64 reduction
//     instruction writes three consecutive doubles of a CSR row segment
//     (fd_res_assemble, src/fd_residuals.cc:58-73; PLoc_Sparse,
//     src/PLoc_Sparse.cc:15-175).
#pragma once
#include <cstdint>

#include "assemble.cuh"

namespace pgb {

constexpr int kP2TE = 8;                      // elements per CTA iteration
constexpr int kP2Threads = kP2TE * 10 * 3;    // (element, node, component)
constexpr int kP2VS = 18;                     // doubles per (point, node) vector record
constexpr int kP2Rec = 38;                    // doubles per point record
// doubles per element in the vector records: 4 points x 10 nodes x 18, padded by
// 6 so that the records of consecutive elements start 12 banks apart
constexpr int kP2ES = 4 * 10 * kP2VS + 6;

// shared memory: node data, J2 state and row metadata of two tiles (the tile
// being assembled and the prefetched next one), point records, vector records
constexpr int kP2XU = kP2TE * 10 * 6;     // doubles per node-data buffer
constexpr int kP2ST = kP2TE * 4 * 7;      // doubles per state buffer
constexpr int kP2MT = kP2TE * 10 * 7;     // ints per metadata buffer: mask word, rp, rl, dof x3, mask shift
constexpr int kP2PS = kP2TE * 10 * 10;    // uint16 per position buffer

inline size_t p2_smem_bytes() {
  return sizeof(double) * (2 * (size_t)kP2XU + 2 * (size_t)kP2ST + (size_t)kP2TE * 4 * kRec +
                           (size_t)kP2TE * kP2ES + (size_t)kP2TE * 4) +
         sizeof(int) * 2 * (size_t)kP2MT + sizeof(uint16_t) * 2 * (size_t)kP2PS;
}

__device__ __forceinline__ void cpa4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cpa8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cpa16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cpa_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ---- the three phases as device functions (shared by both kernels) ----

// Phase 1 for one quadrature point: Jacobian, F, constitutive update (state
// n -> n+1 written to global memory) and the 38-double point record.
// xu: the element's 10 nodes (x, u) in shared memory; st: 7 state doubles.
template <bool PLASTIC>
__device__ __forceinline__ void p2_point(const AsmArgs &args, const double *xu, const double *st, double *rec,
                                         long e, int q) {
  constexpr int NNE = 10, NQP = 4;
  double dX[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, dU[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int b = 0; b < NNE; b++) {
    const double g0 = args.shp.dNxi[q][b][0], g1 = args.shp.dNxi[q][b][1], g2 = args.shp.dNxi[q][b][2];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const double x = xu[b * 6 + i], u = xu[b * 6 + 3 + i];
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
        F[i * 3 + j] = (i == j ? 1.0 : 0.0) + dU[i * 3 + 0] * dXi[0 * 3 + j] + dU[i * 3 + 1] * dXi[1 * 3 + j] +
                       dU[i * 3 + 2] * dXi[2 * 3 + j];
    const double *F0 = args.elem_group ? args.F0_tab + 9 * (long)args.elem_group[e] : args.F0;
    if (F0)
#pragma unroll
      for (int i = 0; i < 9; i++) F[i] += F0[i];
  }
  const double J = ok ? det3(F) : -1.0;
  if (ok) ok = J > 0.0 && inv3(F, Fi);
  if (!ok) {
    atomicAdd(&args.status[0], 1ull);
#pragma unroll
    for (int i = 0; i < kRec; i++) rec[i] = 0.0;
    return;
  }
  const long qp = e * NQP + q;
  double Ast[6] = {1, 1, 1, 0, 0, 0}, alpha = 0.0;
  if (PLASTIC) {
#pragma unroll
    for (int c = 0; c < 6; c++) Ast[c] = st[c];
    alpha = st[6];
  }
  QpTangent t;
  double Anp1[6], alpha_np1;
  spatial_update<PLASTIC>(args.mat, F, J, Ast, alpha, t, Anp1, &alpha_np1);
  if (PLASTIC && args.state_np1) {
#pragma unroll
    for (int c = 0; c < 6; c++) args.state_np1[c * args.nqp + qp] = Anp1[c];
    args.state_np1[6 * args.nqp + qp] = alpha_np1;
  }
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      rec[i * 3 + j] =
          dXi[i * 3 + 0] * Fi[0 * 3 + j] + dXi[i * 3 + 1] * Fi[1 * 3 + j] + dXi[i * 3 + 2] * Fi[2 * 3 + j];
  rec[9] = detJ * args.shp.w[q];
#pragma unroll
  for (int i = 0; i < 6; i++) {
    rec[10 + i] = t.tau[i];
    rec[16 + i] = t.s[i];
    rec[22 + i] = t.n[i];
    rec[28 + i] = t.D[i];
  }
  rec[34] = t.a1;
  rec[35] = t.a2;
  rec[36] = t.a4;
  rec[37] = t.a5;
}

// Phase 2 for one (point, node): the 18-double vector record
// [p, U, W, T, S, n p] (16-byte aligned pairs) and, for node 0, w a1 / 2.
// RS: stride between consecutive values of the point record (1: one record
// per point, contiguous; 16: structure of arrays over a tile's 16 points)
template <bool PLASTIC, int RS = 1>
__device__ __forceinline__ void p2_vectors(const AsmArgs &args, const double *rec, int q, int a, double *v,
                                           double *a1_out) {
  const double w = rec[9 * RS];
  const double a1h = 0.5 * rec[34 * RS] * w, a2w = rec[35 * RS] * w, c23 = (2.0 / 3.0) * w;
  const double g0 = args.shp.dNxi[q][a][0], g1 = args.shp.dNxi[q][a][1], g2 = args.shp.dNxi[q][a][2];
  double p[3], sp[3], tp[3], S6[6];
#pragma unroll
  for (int j = 0; j < 3; j++)
    p[j] = rec[(0 * 3 + j) * RS] * g0 + rec[(1 * 3 + j) * RS] * g1 + rec[(2 * 3 + j) * RS] * g2;
#pragma unroll
  for (int c = 0; c < 6; c++) S6[c] = rec[(16 + c) * RS];
  smv(S6, p, sp);
#pragma unroll
  for (int c = 0; c < 6; c++) S6[c] = rec[(10 + c) * RS];
  smv(S6, p, tp);
#pragma unroll
  for (int j = 0; j < 3; j++) {
    v[j] = p[j];
    v[3 + j] = a2w * p[j] - c23 * sp[j];
    v[9 + j] = a1h * p[j] + w * tp[j];
    v[12 + j] = -c23 * sp[j];
  }
  if (PLASTIC) {
    const double a4w = rec[36 * RS] * w, a5w = rec[37 * RS] * w;
    double np_[3], mp[3];
#pragma unroll
    for (int c = 0; c < 6; c++) S6[c] = rec[(22 + c) * RS];
    smv(S6, p, np_);
#pragma unroll
    for (int c = 0; c < 6; c++) S6[c] = rec[(28 + c) * RS];
    smv(S6, p, mp);
#pragma unroll
    for (int j = 0; j < 3; j++) {
      v[6 + j] = a4w * np_[j] + a5w * mp[j];
      v[15 + j] = np_[j];
    }
  } else {
#pragma unroll
    for (int j = 0; j < 3; j++) v[6 + j] = v[15 + j] = 0.0;
  }
  if (a == 0) *a1_out = a1h;
}

// Phase 3 for one lane (row node a, column component k of one element):
// the entries (i, k) of K_ab for all b, scattered with FP64 reductions, and
// the residual component k of node a.  vec: the element's vector records;
// a1: its four w a1 / 2; meta / pos: its nodes' row metadata and positions.
// NB: column nodes per pass (5: two passes, fewer registers; 10: one pass,
// the row node's vectors loaded once per point)
// NNE, NQP: nodes and quadrature points of the element (10, 4 quadratic tets;
// 4, 1 linear tets).
template <bool PLASTIC, int NB = 5, int NNE = 10, int NQP = 4>
__device__ __forceinline__ void p2_blocks(const AsmArgs &args, const double *vec, const double *a1,
                                          const int *meta, const uint16_t *pos, int a, int k) {
  constexpr int VS = kP2VS;
  const int *mA = meta + a * 7;
  const unsigned maskA = ((unsigned)mA[0] >> mA[6]) & 0xFFu;
  if (!maskA) return;
  // the diagonal term (p_a . T_b) 1 enters entry (k, k): weights instead of
  // lane-dependent branches (the three lanes k of a warp stay converged)
  const double ek0 = k == 0 ? 1.0 : 0.0, ek1 = k == 1 ? 1.0 : 0.0, ek2 = k == 2 ? 1.0 : 0.0;
  const long rp = mA[1], rl = mA[2];
  const uint16_t *posrow = pos + a * NNE;
  double Rk = 0.0;
  // points outer, NB column nodes inner: 3 NB independent accumulators per pass
#pragma unroll 1
  for (int hb = 0; hb < NNE / NB; hb++) {
    double acc[NB][3];
#pragma unroll
    for (int j = 0; j < NB; j++) acc[j][0] = acc[j][1] = acc[j][2] = 0.0;
#pragma unroll 1
    for (int q = 0; q < NQP; q++) {
      const double *base = vec + q * NNE * VS;
      const double *L = base + a * VS;
      const double2 l01 = *reinterpret_cast<const double2 *>(L);
      const double pa0 = l01.x, pa1 = l01.y, pa2 = L[2];
      const double2 s01 = *reinterpret_cast<const double2 *>(L + 12);
      const double2 s2n0 = *reinterpret_cast<const double2 *>(L + 14);
      const double2 n12 = *reinterpret_cast<const double2 *>(L + 16);
      const double pak = L[k];
      const double ha = a1[q] * pak;
      if (hb == 0) Rk += L[9 + k] - ha;  // w tau p_a = T_a - a1/2 w p_a
#pragma unroll
      for (int j = 0; j < NB; j++) {
        const double *Rv = base + (NB * hb + j) * VS;
        const double2 r0 = *reinterpret_cast<const double2 *>(Rv + 0);
        const double pb2 = Rv[2];
        const double pbk = Rv[k], Uk = Rv[3 + k], Wk = PLASTIC ? Rv[6 + k] : 0.0;
        const double2 t01 = *reinterpret_cast<const double2 *>(Rv + 10);
        const double dg = pa0 * Rv[9] + pa1 * t01.x + pa2 * t01.y;
        double x0 = acc[j][0], x1 = acc[j][1], x2 = acc[j][2];
        x0 = fma(r0.x, ha, x0);
        x1 = fma(r0.y, ha, x1);
        x2 = fma(pb2, ha, x2);
        x0 = fma(pa0, Uk, x0);
        x1 = fma(pa1, Uk, x1);
        x2 = fma(pa2, Uk, x2);
        x0 = fma(s01.x, pbk, x0);
        x1 = fma(s01.y, pbk, x1);
        x2 = fma(s2n0.x, pbk, x2);
        if (PLASTIC) {
          x0 = fma(s2n0.y, Wk, x0);
          x1 = fma(n12.x, Wk, x1);
          x2 = fma(n12.y, Wk, x2);
        }
        acc[j][0] = fma(ek0, dg, x0);
        acc[j][1] = fma(ek1, dg, x1);
        acc[j][2] = fma(ek2, dg, x2);
      }
    }
#pragma unroll
    for (int j = 0; j < NB; j++) {
      const int b = NB * hb + j;
      const int *mB = meta + b * 7;
      const unsigned maskB = ((unsigned)mB[0] >> mB[6]) & 0xFFu;
      if (!((maskB >> k) & 1u)) continue;
      const long col = rp + posrow[b] + rank_of(maskB, k);
#pragma unroll
      for (int i = 0; i < 3; i++) {
        if (!((maskA >> i) & 1u)) continue;
        atomicAdd(&args.K[col + (long)rank_of(maskA, i) * rl], acc[j][i]);
      }
    }
  }
  const int id = mA[3 + k];
  if (id > 0) atomicAdd(&args.R[id - 1], Rk);
}

// asynchronous copy of one element node's data and row metadata
__device__ __forceinline__ void p2_fetch_meta(const AsmArgs &args, long e, int a, int node, int *m,
                                              uint16_t *sp) {
  constexpr int NNE = 10;
  cpa4(m + 0, args.mask + (node & ~3));  // the aligned word holding the mask byte
  cpa4(m + 1, args.rowptr0 + node);
  cpa4(m + 2, args.rowlen + node);
  cpa4(m + 3, args.dof + node);
  cpa4(m + 4, args.dof + args.nn + node);
  cpa4(m + 5, args.dof + 2 * args.nn + node);
  m[6] = (node & 3) * 8;
  const uint16_t *pr = args.pos + (e * NNE + a) * NNE;
#pragma unroll
  for (int j = 0; j < NNE; j += 2) cpa4(sp + j, pr + j);
}

__device__ __forceinline__ void p2_fetch_node(const AsmArgs &args, long e, int a, int node, double *d, int *m,
                                              uint16_t *sp) {
  cpa8(d + 0, args.X + node);
  cpa8(d + 1, args.X + args.nn + node);
  cpa8(d + 2, args.X + 2 * args.nn + node);
  cpa8(d + 3, args.unode + node);
  cpa8(d + 4, args.unode + args.nn + node);
  cpa8(d + 5, args.unode + 2 * args.nn + node);
  p2_fetch_meta(args, e, a, node, m, sp);
}

template <int MODEL>
__global__ void __launch_bounds__(kP2Threads, 2) k_assemble_p2(const AsmArgs args) {
  constexpr int NNE = 10, NQP = 4, TE = kP2TE, VS = kP2VS;
  constexpr bool PLASTIC = (MODEL == 1);
  extern __shared__ double smem[];
  double *sXUb = smem;                         // [2][TE][NNE][6]
  double *sStb = sXUb + 2 * kP2XU;             // [2][TE][NQP][7] state at t_n
  double *sRec = sStb + 2 * kP2ST;             // [TE][NQP][kRec]
  double *sVec = sRec + TE * NQP * kRec;       // [TE][kP2ES]: [NQP][NNE][VS] per element
  double *sA1 = sVec + TE * kP2ES;             // [TE][NQP]  w a1 / 2
  int *sMetab = reinterpret_cast<int *>(sA1 + TE * NQP);                // [2][TE*NNE][7]
  uint16_t *sPosb = reinterpret_cast<uint16_t *>(sMetab + 2 * kP2MT);  // [2][TE*NNE][NNE]
  const int tid = threadIdx.x;
  const long ne = args.ne;
  const long stride = (long)gridDim.x * TE;

  // asynchronous copy of tile t1's node data, row metadata and state into
  // buffer `buf` (node = this thread's element node of that tile)
  auto prefetch = [&](long t1, int buf, int node) {
    if (tid < TE * NNE) {
      const int el = tid / NNE, a = tid - el * NNE;
      const long e = t1 + el;
      if (e < ne && node >= 0)
        p2_fetch_node(args, e, a, node, sXUb + buf * kP2XU + tid * 6, sMetab + buf * kP2MT + tid * 7,
                      sPosb + buf * kP2PS + tid * NNE);
    }
    if (PLASTIC && tid < TE * NQP) {
      const int el = tid / NQP, q = tid - el * NQP;
      const long e = t1 + el;
      if (e < ne) {
        const long qp = e * NQP + q;
        double *st = sStb + buf * kP2ST + tid * 7;
#pragma unroll
        for (int c = 0; c < 7; c++) cpa8(st + c, args.state_n + c * args.nqp + qp);
      }
    }
    cpa_commit();
  };
  auto node_of = [&](long t1) -> int {
    if (tid >= TE * NNE) return -1;
    const int el = tid / NNE, a = tid - el * NNE;
    const long e = t1 + el;
    return (t1 < ne && e < ne) ? args.conn[(long)a * ne + e] : -1;
  };

  long tile0 = (long)blockIdx.x * TE;
  int buf = 0;
  if (tile0 < ne) prefetch(tile0, 0, node_of(tile0));
  int next_node = node_of(tile0 + stride);
  cpa_wait_all();
  __syncthreads();

  for (; tile0 < ne; tile0 += stride, buf ^= 1) {
    const double *sXU = sXUb + buf * kP2XU;
    const double *sSt = sStb + buf * kP2ST;
    const int *sMeta = sMetab + buf * kP2MT;
    const uint16_t *sPos = sPosb + buf * kP2PS;

    // ---------------- 1: quadrature points ----------------
    if (tid < TE * NQP) {
      const int el = tid / NQP, q = tid - el * NQP;
      const long e = tile0 + el;
      if (e < ne) p2_point<PLASTIC>(args, sXU + el * NNE * 6, sSt + tid * 7, sRec + tid * kRec, e, q);
    }
    __syncthreads();

    // ---------------- 2: node vectors per point ----------------
    for (int it = tid; it < TE * NQP * NNE; it += kP2Threads) {
      const int eq = it / NNE, a = it - eq * NNE;  // eq = el * NQP + q
      p2_vectors<PLASTIC>(args, sRec + eq * kRec, eq % NQP, a,
                          sVec + (eq / NQP) * kP2ES + ((eq % NQP) * NNE + a) * VS, sA1 + eq);
    }
    __syncthreads();

    // the next tile's data lands while this tile's blocks are formed
    if (tile0 + stride < ne) prefetch(tile0 + stride, buf ^ 1, next_node);
    next_node = node_of(tile0 + 2 * stride);

    // ---------------- 3: column-split block rows + scatter ----------------
    {
      const int el = tid / 30, r = tid - el * 30;
      const int a = r / 3, k = r - a * 3;
      if (tile0 + el < ne)
        p2_blocks<PLASTIC>(args, sVec + el * kP2ES, sA1 + el * NQP, sMeta + el * NNE * 7, sPos + el * NNE * NNE,
                           a, k);
    }
    cpa_wait_all();
    __syncthreads();
  }
}


// ---- warp-specialised variant ---------------------------------------------
//
// Producer / consumer pipeline over tiles of 4 elements.  Warp 4 (producer)
// runs the serial, latency-bound phases of tile i+1 -- the point updates
// (lanes 0-15) and the vector records -- and issues the cp.async prefetch of
// tile i+2's node data, while warps 0-3 (consumers) run the issue-bound block
// phase and the reductions of tile i.  Hand-off through two mbarriers per
// vector buffer (full: produced; empty: consumed), every wait bounded: a wait
// that runs out sets status[3] and both roles leave the loop (their next
// waits run out too), so a fault cannot hang the GPU.
constexpr int kWTE = 4;                   // elements per tile
constexpr int kWCons = 128;               // consumer threads (120 form blocks)
constexpr int kWThreads = kWCons + 32;    // + one producer warp
constexpr int kWXU = kWTE * 10 * 6, kWST = kWTE * 4 * 7, kWMT = kWTE * 10 * 7, kWPS = kWTE * 10 * 10;
constexpr unsigned long long kWWaitNs = 2000000000ull;

inline size_t p2ws_smem_bytes() {
  return 64 + sizeof(double) * (2 * (size_t)kWXU + 2 * (size_t)kWST + (size_t)kWTE * 4 * kRec +
                                2 * (size_t)kWTE * kP2ES + 2 * (size_t)kWTE * 4) +
         sizeof(int) * 3 * (size_t)kWMT + sizeof(uint16_t) * 3 * (size_t)kWPS;
}

__device__ __forceinline__ unsigned long long w_gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void w_mb_init(uint64_t *b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(b)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void w_mb_arrive(uint64_t *b) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(
                   (unsigned)__cvta_generic_to_shared(b))
               : "memory");
}
// bounded wait for the completion of the phase with the given parity
__device__ __forceinline__ bool w_mb_wait(uint64_t *b, unsigned parity) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(b);
  const unsigned long long t0 = w_gtimer();
  for (;;) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
    if (w_gtimer() - t0 > kWWaitNs) return false;
  }
}

template <int MODEL>
__global__ void __launch_bounds__(kWThreads, 3) k_assemble_p2ws(const AsmArgs args) {
  constexpr int NNE = 10, NQP = 4, TE = kWTE, VS = kP2VS;
  constexpr bool PLASTIC = (MODEL == 1);
  extern __shared__ __align__(16) unsigned char wsm[];
  uint64_t *full = reinterpret_cast<uint64_t *>(wsm);       // [2]
  uint64_t *empty = full + 2;                                // [2]
  double *sXU = reinterpret_cast<double *>(wsm + 64);        // [2][TE][NNE][6]
  double *sSt = sXU + 2 * kWXU;                              // [2][TE][NQP][7]
  double *sRec = sSt + 2 * kWST;                             // [TE][NQP][kRec]
  double *sVec = sRec + TE * NQP * kRec;                     // [2][TE][kP2ES]
  double *sA1 = sVec + 2 * TE * kP2ES;                       // [2][TE][NQP]
  int *sMeta = reinterpret_cast<int *>(sA1 + 2 * TE * NQP);  // [3][TE*NNE][7]
  uint16_t *sPos = reinterpret_cast<uint16_t *>(sMeta + 3 * kWMT);  // [3][TE*NNE][NNE]
  const int tid = threadIdx.x;
  const long ne = args.ne;
  auto tile_e0 = [&](long i) -> long { return ((long)blockIdx.x + i * (long)gridDim.x) * TE; };
  if (tid == 0) {
    w_mb_init(&full[0], 32);
    w_mb_init(&full[1], 32);
    w_mb_init(&empty[0], kWCons);
    w_mb_init(&empty[1], kWCons);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  bool fail = false;
  if (tid >= kWCons) {
    // ------------------------------ producer ------------------------------
    const int pl = tid - kWCons;
    auto load_nodes = [&](long i, int *nd) {
      const long e0 = tile_e0(i);
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int slot = pl + 32 * j;
        nd[j] = -1;
        if (slot < TE * NNE && e0 < ne) {
          const int el = slot / NNE, a = slot - el * NNE;
          const long e = e0 + el;
          if (e < ne) nd[j] = args.conn[(long)a * ne + e];
        }
      }
    };
    auto issue = [&](long i, const int *nd) {
      const long e0 = tile_e0(i);
      const int bx = (int)(i & 1), bm = (int)(i % 3);
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int slot = pl + 32 * j;
        if (slot < TE * NNE && nd[j] >= 0) {
          const int el = slot / NNE, a = slot - el * NNE;
          p2_fetch_node(args, e0 + el, a, nd[j], sXU + bx * kWXU + slot * 6, sMeta + bm * kWMT + slot * 7,
                        sPos + bm * kWPS + slot * NNE);
        }
      }
      if (PLASTIC && pl < TE * NQP) {
        const int el = pl / NQP, q = pl - el * NQP;
        const long e = e0 + el;
        if (e < ne) {
          const long qp = e * NQP + q;
          double *st = sSt + bx * kWST + pl * 7;
#pragma unroll
          for (int c = 0; c < 7; c++) cpa8(st + c, args.state_n + c * args.nqp + qp);
        }
      }
      cpa_commit();
    };
    int nd[2], nd_next[2];
    if (tile_e0(0) < ne) {
      load_nodes(0, nd);
      issue(0, nd);
    }
    load_nodes(1, nd_next);
    for (long i = 0; tile_e0(i) < ne; i++) {
      const int bx = (int)(i & 1);
      if (i >= 2) {
        const bool ok = w_mb_wait(&empty[bx], (unsigned)(((i - 2) >> 1) & 1));
        if (__any_sync(0xffffffffu, !ok)) {
          fail = true;
          break;
        }
      }
      cpa_wait_all();  // tile i's node data and state have landed
      __syncwarp();
      if (tile_e0(i + 1) < ne) issue(i + 1, nd_next);
      load_nodes(i + 2, nd_next);
      const long e0 = tile_e0(i);
      if (pl < TE * NQP) {
        const int el = pl / NQP, q = pl - el * NQP;
        const long e = e0 + el;
        if (e < ne) p2_point<PLASTIC>(args, sXU + bx * kWXU + el * NNE * 6, sSt + bx * kWST + pl * 7,
                                      sRec + pl * kRec, e, q);
      }
      __syncwarp();
      for (int it = pl; it < TE * NQP * NNE; it += 32) {
        const int eq = it / NNE, a = it - eq * NNE;
        const int el = eq / NQP, q = eq - el * NQP;
        if (e0 + el < ne)
          p2_vectors<PLASTIC>(args, sRec + eq * kRec, q, a, sVec + (bx * TE + el) * kP2ES + (q * NNE + a) * VS,
                              sA1 + bx * TE * NQP + eq);
      }
      w_mb_arrive(&full[bx]);  // release: this lane's records are visible to the consumers
    }
    cpa_wait_all();
  } else {
    // ------------------------------ consumers ------------------------------
    const int el = tid / 30, r = tid - el * 30;
    const int a = r / 3, k = r - a * 3;
    for (long i = 0; tile_e0(i) < ne; i++) {
      const int bx = (int)(i & 1), bm = (int)(i % 3);
      if (!w_mb_wait(&full[bx], (unsigned)((i >> 1) & 1))) {
        fail = true;
        break;
      }
      if (tid < TE * 30 && tile_e0(i) + el < ne)
        p2_blocks<PLASTIC>(args, sVec + (bx * TE + el) * kP2ES, sA1 + bx * TE * NQP + el * NQP,
                           sMeta + bm * kWMT + el * NNE * 7, sPos + bm * kWPS + el * NNE * NNE, a, k);
      w_mb_arrive(&empty[bx]);
    }
  }
  if (fail && (tid & 31) == 0) atomicAdd(&args.status[3], 1ull);
}


// ---- two-kernel variant: point records from HBM --------------------------
//
// The point updates run first in their own kernel (k_qp_update, one thread
// per point at full occupancy, records as structure of arrays).  This kernel
// is the pipeline above without them: the producer warp copies a tile's 16
// point records (38 x 16 doubles, 16-byte cp.async chunks) and its CSR row
// metadata two tiles ahead and builds the vector records of tile i+1 while the
// consumer warps run the blocks and reductions of tile i.  Same hand-off and
// bounded waits as k_assemble_p2ws.
constexpr int kRRT = kWTE * 4;  // points per tile

inline size_t p2r_smem_bytes() {
  return 64 + sizeof(double) * (2 * (size_t)kRec * kRRT + 2 * (size_t)kWTE * kP2ES + 2 * (size_t)kRRT) +
         sizeof(int) * 3 * (size_t)kWMT + sizeof(uint16_t) * 3 * (size_t)kWPS;
}

template <int MODEL>
__global__ void __launch_bounds__(kWThreads, 3) k_assemble_p2r(const AsmArgs args) {
  constexpr int NNE = 10, NQP = 4, TE = kWTE, VS = kP2VS, RT = kRRT;
  constexpr bool PLASTIC = (MODEL == 1);
  extern __shared__ __align__(16) unsigned char wsm[];
  uint64_t *full = reinterpret_cast<uint64_t *>(wsm);       // [2]
  uint64_t *empty = full + 2;                                // [2]
  double *sRec = reinterpret_cast<double *>(wsm + 64);       // [2][kRec][RT]
  double *sVec = sRec + 2 * kRec * RT;                       // [2][TE][kP2ES]
  double *sA1 = sVec + 2 * TE * kP2ES;                       // [2][TE][NQP]
  int *sMeta = reinterpret_cast<int *>(sA1 + 2 * RT);        // [3][TE*NNE][7]
  uint16_t *sPos = reinterpret_cast<uint16_t *>(sMeta + 3 * kWMT);  // [3][TE*NNE][NNE]
  const int tid = threadIdx.x;
  const long ne = args.ne;
  auto tile_e0 = [&](long i) -> long { return ((long)blockIdx.x + i * (long)gridDim.x) * TE; };
  if (tid == 0) {
    w_mb_init(&full[0], 32);
    w_mb_init(&full[1], 32);
    w_mb_init(&empty[0], kWCons);
    w_mb_init(&empty[1], kWCons);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  bool fail = false;
  if (tid >= kWCons) {
    // ------------------------------ producer ------------------------------
    const int pl = tid - kWCons;
    auto load_nodes = [&](long i, int *nd) {
      const long e0 = tile_e0(i);
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int slot = pl + 32 * j;
        nd[j] = -1;
        if (slot < TE * NNE && e0 < ne) {
          const int el = slot / NNE, a = slot - el * NNE;
          const long e = e0 + el;
          if (e < ne) nd[j] = args.conn[(long)a * ne + e];
        }
      }
    };
    auto issue = [&](long i, const int *nd) {
      const long e0 = tile_e0(i);
      const int bx = (int)(i & 1), bm = (int)(i % 3);
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const int slot = pl + 32 * j;
        if (slot < TE * NNE && nd[j] >= 0) {
          const int el = slot / NNE, a = slot - el * NNE;
          p2_fetch_meta(args, e0 + el, a, nd[j], sMeta + bm * kWMT + slot * 7, sPos + bm * kWPS + slot * NNE);
        }
      }
      // records: kRec rows of RT consecutive points, in 16-byte chunks (two
      // points of one element each; nqp = 4 ne keeps every chunk aligned)
      const long qp0 = e0 * NQP;
      for (int ch = pl; ch < kRec * RT / 2; ch += 32) {
        const int c = ch / (RT / 2), part = ch - c * (RT / 2);
        if (e0 + part / 2 < ne)
          cpa16(sRec + (bx * kRec + c) * RT + part * 2, args.qrec + (long)c * args.nqp + qp0 + part * 2);
      }
      cpa_commit();
    };
    int nd[2], nd_next[2];
    if (tile_e0(0) < ne) {
      load_nodes(0, nd);
      issue(0, nd);
    }
    load_nodes(1, nd_next);
    for (long i = 0; tile_e0(i) < ne; i++) {
      const int bx = (int)(i & 1);
      if (i >= 2) {
        const bool ok = w_mb_wait(&empty[bx], (unsigned)(((i - 2) >> 1) & 1));
        if (__any_sync(0xffffffffu, !ok)) {
          fail = true;
          break;
        }
      }
      cpa_wait_all();  // tile i's records and metadata have landed
      __syncwarp();
      if (tile_e0(i + 1) < ne) issue(i + 1, nd_next);
      load_nodes(i + 2, nd_next);
      const long e0 = tile_e0(i);
      for (int it = pl; it < RT * NNE; it += 32) {
        const int eq = it / NNE, a = it - eq * NNE;
        const int el = eq / NQP, q = eq - el * NQP;
        if (e0 + el < ne)
          p2_vectors<PLASTIC, RT>(args, sRec + bx * kRec * RT + eq, q, a,
                                  sVec + (bx * TE + el) * kP2ES + (q * NNE + a) * VS, sA1 + bx * RT + eq);
      }
      w_mb_arrive(&full[bx]);  // release: this lane's vectors are visible to the consumers
    }
    cpa_wait_all();
  } else {
    // ------------------------------ consumers ------------------------------
    // one warp per element (lanes 30 and 31 idle): the column-node loads of
    // a warp are broadcasts from a single record
    const int el = tid >> 5, r = tid & 31;
    const int a = r / 3, k = r - a * 3;
    for (long i = 0; tile_e0(i) < ne; i++) {
      const int bx = (int)(i & 1), bm = (int)(i % 3);
      if (!w_mb_wait(&full[bx], (unsigned)((i >> 1) & 1))) {
        fail = true;
        break;
      }
      if (r < 30 && tile_e0(i) + el < ne)
        p2_blocks<PLASTIC, 10>(args, sVec + (bx * TE + el) * kP2ES, sA1 + bx * RT + el * NQP,
                           sMeta + bm * kWMT + el * NNE * 7, sPos + bm * kWPS + el * NNE * NNE, a, k);
      w_mb_arrive(&empty[bx]);
    }
  }
  if (fail && (tid & 31) == 0) atomicAdd(&args.status[3], 1ull);
}


// ---- linear tets: column-split assembly from point records ----------------
//
// The linear-tet counterpart of k_assemble_p2r for the default R+K path
// (configs 1 and 5): the point updates run first in k_qp_update<4, 1, MODEL>
// (one thread per point, records in HBM); this kernel takes tiles of TE
// elements -- claimed `grab` tiles at a time from a ticket when a work-stealing
// schedule is set, else grid-stride -- and runs in turn
//   0  the tile's point records (structure of arrays, coalesced) and the CSR
//      metadata of its (element, node) pairs into shared memory;
//   2  item (element, node): the vector record (p, U, W, T, S, n p);
//   3  thread (element, row node a, column component k): the entries
//      (a, i; b, k) of K_ab for i = 0..2 and the four column nodes b, and the
//      residual; the three lanes k of one (element, a) are adjacent, so each
//      FP64 reduction instruction writes three consecutive doubles of a CSR
//      row segment (the per-node kernel writes one double per sector).
constexpr int kP1ES = 4 * kP2VS + 2;  // doubles per element of vector records (even, bank-spread)

inline size_t p1r_smem_bytes(int TE) {
  return sizeof(double) * ((size_t)kRec * TE + (size_t)TE * kP1ES + TE) + sizeof(int) * (size_t)TE * 4 * 7 +
         sizeof(uint16_t) * (size_t)TE * 16;
}

template <int MODEL, int TE>
__global__ void __launch_bounds__(TE * 12) k_assemble_p1r(const AsmArgs args) {
  constexpr int NNE = 4, VS = kP2VS, NT = TE * 12;
  constexpr bool PLASTIC = (MODEL == 1);
  extern __shared__ __align__(16) double p1s[];
  double *sRec = p1s;                                                   // [kRec][TE]
  double *sVec = sRec + kRec * TE;                                      // [TE][kP1ES]
  double *sA1 = sVec + TE * kP1ES;                                      // [TE]
  int *sMeta = reinterpret_cast<int *>(sA1 + TE);                       // [TE][NNE][7]
  uint16_t *sPos = reinterpret_cast<uint16_t *>(sMeta + TE * NNE * 7);  // [TE][NNE][NNE]
  const int tid = threadIdx.x;
  const long ne = args.ne;
  __shared__ long s_claim;
  long claim_end = 0;
  long tile0 = (long)blockIdx.x * TE;
  if (args.ticket) {
    if (tid == 0) s_claim = (long)atomicAdd(args.ticket, (unsigned)args.grab) * TE;
    __syncthreads();
    tile0 = s_claim;
    claim_end = tile0 + (long)args.grab * TE;
    __syncthreads();
  }
  while (tile0 < ne) {
    // phase 0: records and metadata
    for (int t = tid; t < kRec * TE; t += NT) {
      const int c = t / TE, el = t - c * TE;
      const long e = tile0 + el;
      sRec[t] = e < ne ? args.qrec[(long)c * args.nqp + e] : 0.0;  // one point per element
    }
    if (tid < TE * NNE) {
      const int el = tid / NNE, a = tid - el * NNE;
      const long e = tile0 + el;
      if (e < ne) {
        const int node = args.conn[(long)a * ne + e];
        int *m = sMeta + tid * 7;
        m[0] = args.mask[node];
        m[1] = args.rowptr0[node];
        m[2] = args.rowlen[node];
        m[3] = args.dof[node];
        m[4] = args.dof[args.nn + node];
        m[5] = args.dof[2 * args.nn + node];
        m[6] = 0;
        const uint16_t *pr = args.pos + (e * NNE + a) * NNE;
#pragma unroll
        for (int b = 0; b < NNE; b++) sPos[tid * NNE + b] = pr[b];
      }
    }
    __syncthreads();
    // phase 2: vector records
    if (tid < TE * NNE) {
      const int el = tid / NNE, a = tid - el * NNE;
      if (tile0 + el < ne) p2_vectors<PLASTIC, TE>(args, sRec + el, 0, a, sVec + el * kP1ES + a * VS, sA1 + el);
    }
    __syncthreads();
    // phase 3: column-split blocks and reductions
    {
      const int el = tid / 12, r = tid - el * 12;
      const int a = r / 3, k = r - a * 3;
      if (tile0 + el < ne)
        p2_blocks<PLASTIC, 4, 4, 1>(args, sVec + el * kP1ES, sA1 + el, sMeta + el * NNE * 7,
                                    sPos + el * NNE * NNE, a, k);
    }
    __syncthreads();
    if (args.ticket) {
      tile0 += TE;
      if (tile0 >= claim_end) {
        if (tid == 0) s_claim = (long)atomicAdd(args.ticket, (unsigned)args.grab) * TE;
        __syncthreads();
        tile0 = s_claim;
        claim_end = tile0 + (long)args.grab * TE;
        __syncthreads();
      }
    } else {
      tile0 += (long)gridDim.x * TE;
    }
  }
}


// ---- linear tets: warp-specialised column-split assembly (default) ---------
//
// k_assemble_p1r as a producer/consumer pipeline: the last warp (producer)
// claims tiles of TE elements (from the ticket, `grab` at a time, when a
// work-stealing schedule is set; else grid-stride), copies a tile's point
// records and CSR metadata with cp.async one tile ahead, builds its vector
// records and hands it over with the tile's first element in shared memory
// (-1: no more tiles); TE/2 consumer warps (16 lanes per element, 12 used)
// form the column-split blocks and issue the reductions.  Hand-off through the
// bounded mbarrier waits of k_assemble_p2ws (a wait that runs out sets
// status[3] and ends the loops).  Records are copied 8 bytes at a time: with
// an odd element count a 16-byte chunk of a record row would be misaligned.
template <int TE>
constexpr int p1ws_threads() { return TE * 16 + 32; }

inline size_t p1ws_smem_bytes(int TE) {
  return 64 + sizeof(double) * (2 * (size_t)kRec * TE + 2 * (size_t)TE * kP1ES + 2 * (size_t)TE) +
         sizeof(int) * 3 * (size_t)TE * 4 * 7 + sizeof(uint16_t) * 3 * (size_t)TE * 16;
}

__device__ __forceinline__ void p1_fetch_meta(const AsmArgs &args, long e, int a, int node, int *m,
                                              uint16_t *sp) {
  cpa4(m + 0, args.mask + (node & ~3));  // the aligned word holding the mask byte
  cpa4(m + 1, args.rowptr0 + node);
  cpa4(m + 2, args.rowlen + node);
  cpa4(m + 3, args.dof + node);
  cpa4(m + 4, args.dof + args.nn + node);
  cpa4(m + 5, args.dof + 2 * args.nn + node);
  m[6] = (node & 3) * 8;
  cpa8(sp, args.pos + (e * 4 + a) * 4);  // the four uint16 column positions of (e, a)
}

template <int MODEL, int TE>
__global__ void __launch_bounds__(p1ws_threads<TE>()) k_assemble_p1ws(const AsmArgs args) {
  constexpr int NNE = 4, VS = kP2VS, NC = TE * 16;
  constexpr bool PLASTIC = (MODEL == 1);
  extern __shared__ __align__(16) unsigned char p1w[];
  uint64_t *full = reinterpret_cast<uint64_t *>(p1w);     // [2]
  uint64_t *empty = full + 2;                              // [2]
  long *sTile = reinterpret_cast<long *>(p1w + 32);        // [2] first element of the handed-over tile
  double *sRec = reinterpret_cast<double *>(p1w + 64);     // [2][kRec][TE]
  double *sVec = sRec + 2 * kRec * TE;                     // [2][TE][kP1ES]
  double *sA1 = sVec + 2 * TE * kP1ES;                     // [2][TE]
  int *sMeta = reinterpret_cast<int *>(sA1 + 2 * TE);      // [3][TE][NNE][7]
  uint16_t *sPos = reinterpret_cast<uint16_t *>(sMeta + 3 * TE * NNE * 7);  // [3][TE][NNE][NNE]
  const int tid = threadIdx.x;
  const long ne = args.ne;
  if (tid == 0) {
    w_mb_init(&full[0], 32);
    w_mb_init(&full[1], 32);
    w_mb_init(&empty[0], NC);
    w_mb_init(&empty[1], NC);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  bool fail = false;
  if (tid >= NC) {
    // ------------------------------ producer ------------------------------
    const int pl = tid - NC;
    long claim_next = 0, claim_end = 0, grid_next = (long)blockIdx.x * TE;
    auto next_tile = [&]() -> long {  // first element of the next tile (>= ne: none)
      if (!args.ticket) {
        const long t = grid_next;
        grid_next += (long)gridDim.x * TE;
        return t;
      }
      if (claim_next >= claim_end) {
        unsigned c = 0;
        if (pl == 0) c = atomicAdd(args.ticket, (unsigned)args.grab);
        c = __shfl_sync(0xffffffffu, c, 0);
        claim_next = (long)c * TE;
        claim_end = claim_next + (long)args.grab * TE;
      }
      const long t = claim_next;
      claim_next += TE;
      return t;
    };
    auto issue = [&](long t0, int slot, int bm) {
      for (int u = pl; u < TE * NNE; u += 32) {
        const int el = u / NNE, a = u - el * NNE;
        const long e = t0 + el;
        if (e < ne) {
          const int node = args.conn[(long)a * ne + e];
          p1_fetch_meta(args, e, a, node, sMeta + (bm * TE * NNE + u) * 7, sPos + (bm * TE * NNE + u) * NNE);
        }
      }
      for (int u = pl; u < kRec * TE; u += 32) {
        const int c = u / TE, el = u - c * TE;
        const long e = t0 + el;
        if (e < ne) cpa8(sRec + (slot * kRec + c) * TE + el, args.qrec + (long)c * args.nqp + e);
      }
      cpa_commit();
    };
    long t_cur = next_tile();
    if (t_cur < ne) issue(t_cur, 0, 0);
    for (long i = 0;; i++) {
      const int bx = (int)(i & 1);
      if (i >= 2) {
        const bool ok = w_mb_wait(&empty[bx], (unsigned)(((i - 2) >> 1) & 1));
        if (__any_sync(0xffffffffu, !ok)) {
          fail = true;
          break;
        }
      }
      if (t_cur >= ne) {  // no more tiles: tell the consumers
        if (pl == 0) sTile[bx] = -1;
        w_mb_arrive(&full[bx]);
        break;
      }
      cpa_wait_all();  // tile i's records and metadata have landed
      __syncwarp();
      const long t_nxt = next_tile();
      if (t_nxt < ne) issue(t_nxt, (int)((i + 1) & 1), (int)((i + 1) % 3));
      for (int u = pl; u < TE * NNE; u += 32) {
        const int el = u / NNE, a = u - el * NNE;
        if (t_cur + el < ne)
          p2_vectors<PLASTIC, TE>(args, sRec + bx * kRec * TE + el, 0, a,
                                  sVec + (bx * TE + el) * kP1ES + a * VS, sA1 + bx * TE + el);
      }
      if (pl == 0) sTile[bx] = t_cur;
      w_mb_arrive(&full[bx]);  // release: vectors and the tile index are visible to the consumers
      t_cur = t_nxt;
    }
    cpa_wait_all();
  } else {
    // ------------------------------ consumers ------------------------------
    const int el = tid >> 4, r = tid & 15;
    const int a = r / 3, k = r - a * 3;
    for (long i = 0;; i++) {
      const int bx = (int)(i & 1), bm = (int)(i % 3);
      if (!w_mb_wait(&full[bx], (unsigned)((i >> 1) & 1))) {
        fail = true;
        break;
      }
      const long t0 = sTile[bx];
      if (t0 < 0) break;
      if (r < 12 && t0 + el < ne)
        p2_blocks<PLASTIC, 4, 4, 1>(args, sVec + (bx * TE + el) * kP1ES, sA1 + bx * TE + el,
                                    sMeta + (bm * TE + el) * NNE * 7, sPos + (bm * TE + el) * NNE * NNE, a, k);
      w_mb_arrive(&empty[bx]);
    }
  }
  if (fail && (tid & 31) == 0) atomicAdd(&args.status[3], 1ull);
}

}  // namespace pgb
