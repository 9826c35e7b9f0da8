// assemble_tiles.cuh -- FP64 R+K assembly in two kernels:
//
//  k_qp_update  (one thread per quadrature point): gathers the element's node
//      coordinates and displacements, forms the isoparametric Jacobian and F,
//      runs the constitutive update (run_integration_algorithm,
//      src/constitutive_model.cc:1100-1129; state n -> n+1) and writes a
//      compact point record (structure of arrays): G = (dX/dxi)^-1 F^-1 (so
//      that p_a = F^-T grad_X N_a = G^T dN_a/dxi), w = det(dX/dxi) * weight,
//      the Kirchhoff stress tau and the coefficients of the spatial tangent.
//
//  k_assemble_tiles  (persistent; tiles of TE consecutive elements taken from
//      a global ticket counter in increasing order):
//   Z  zero-fill the CSR rows the tile touches first (one contiguous K range,
//      tile_plan.hpp) and publish a per-tile flag; the lines stay in L2,
//   L  load the tile's point records, build the Voigt tangents D (6x6,
//      engineering shear) and the spatial gradients p_a; sum w tau p_a per
//      tile node (compute_residual_vector, src/constitutive_model.cc:1628-1662),
//   B  thread (element, column node b, row component i) forms w D B_b (the
//      three rows that row i needs) and rows i of K_ab = B_a^T w D B_b +
//      w (p_a . tau p_b) 1 for all a, summed over the points in registers
//      (compute_stiffness_matrix, :1520-1616, in B-matrix form), and adds them
//      into the tile's node-pair accumulators (shared FP64 atomics),
//   W  after the tiles that first touched its rows have published their flags
//      (bounded wait), one warp per (node, component) row issues the tile's
//      blocks as FP64 reductions in CSR address order -- consecutive lanes hit
//      consecutive doubles -- plus the nodal residuals
//      (fd_res_assemble, src/fd_residuals.cc:58-73; PLoc_Sparse,
//      src/PLoc_Sparse.cc:15-175).
#pragma once
#include <cstdint>

#include "assemble.cuh"

namespace pgb {

constexpr int kQRec = 38;  // point record: G 9, w 1, tau 6, s 6, n 6, dev(n^2) 6, a1 a2 a4 a5

struct QpArgs {
  const double *X;      // 3*nn
  const double *unode;  // 3*nn
  const int *conn;      // NNE*ne (SoA)
  long nn, ne, nqp;
  const double *F0;
  const int *elem_group;  // FE2 batches: element -> group (or nullptr)
  const double *F0_tab;   // group -> macro deformation (9)
  const double *state_n;
  double *state_np1;
  double *qrec;         // kQRec*nqp (SoA)
  unsigned long long *status;
  Mat mat;
  ShapeTable shp;
};

template <int NNE, int NQP, int MODEL>
__global__ void __launch_bounds__(128) k_qp_update(const QpArgs A) {
  constexpr bool PLASTIC = (MODEL == 1);
  const long qp = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (qp >= A.nqp) return;
  const long e = qp / NQP;
  const int q = (int)(qp - e * NQP);
  double dX[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, dU[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int b = 0; b < NNE; b++) {
    const int n = A.conn[(long)b * A.ne + e];
    const double g0 = A.shp.dNxi[q][b][0], g1 = A.shp.dNxi[q][b][1], g2 = A.shp.dNxi[q][b][2];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const double x = A.X[i * A.nn + n], u = A.unode[i * A.nn + n];
      dX[i * 3 + 0] += g0 * x;
      dX[i * 3 + 1] += g1 * x;
      dX[i * 3 + 2] += g2 * x;
      dU[i * 3 + 0] += g0 * u;
      dU[i * 3 + 1] += g1 * u;
      dU[i * 3 + 2] += g2 * u;
    }
  }
  double *rec = A.qrec;
  const long S = A.nqp;
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
    const double *F0 = A.elem_group ? A.F0_tab + 9 * (long)A.elem_group[e] : A.F0;
    if (F0)
#pragma unroll
      for (int i = 0; i < 9; i++) F[i] += F0[i];
  }
  const double J = ok ? det3(F) : -1.0;
  if (ok) ok = J > 0.0 && inv3(F, Fi);
  if (!ok) {
    atomicAdd(&A.status[0], 1ull);
#pragma unroll
    for (int c = 0; c < kQRec; c++) rec[c * S + qp] = 0.0;
    return;
  }
  double Ast[6] = {1, 1, 1, 0, 0, 0}, alpha = 0.0;
  if (PLASTIC) {
#pragma unroll
    for (int c = 0; c < 6; c++) Ast[c] = A.state_n[c * S + qp];
    alpha = A.state_n[6 * S + qp];
  }
  QpTangent t;
  double Anp1[6], alpha_np1;
  spatial_update<PLASTIC>(A.mat, F, J, Ast, alpha, t, Anp1, &alpha_np1);
  if (PLASTIC && A.state_np1) {
#pragma unroll
    for (int c = 0; c < 6; c++) A.state_np1[c * S + qp] = Anp1[c];
    A.state_np1[6 * S + qp] = alpha_np1;
  }
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      rec[(i * 3 + j) * S + qp] =
          dXi[i * 3 + 0] * Fi[0 * 3 + j] + dXi[i * 3 + 1] * Fi[1 * 3 + j] + dXi[i * 3 + 2] * Fi[2 * 3 + j];
  rec[9 * S + qp] = detJ * A.shp.w[q];
#pragma unroll
  for (int c = 0; c < 6; c++) {
    rec[(10 + c) * S + qp] = t.tau[c];
    rec[(16 + c) * S + qp] = t.s[c];
    rec[(22 + c) * S + qp] = t.n[c];
    rec[(28 + c) * S + qp] = t.D[c];
  }
  rec[34 * S + qp] = t.a1;
  rec[35 * S + qp] = t.a2;
  rec[36 * S + qp] = t.a4;
  rec[37 * S + qp] = t.a5;
}

struct TileArgs {
  const int *dof;         // 3*nn
  const int *rowptr0;     // nn
  const int *rowlen;      // nn
  const uint8_t *mask;    // nn
  long nn, ne, nqp;
  const double *qrec;     // kQRec*nqp
  // tile plan
  const int *tile_nodes;       // ntiles*NLMAX
  const uint8_t *tile_nl;      // ntiles
  const uint8_t *elem_lnode;   // ne*NNE
  const uint16_t *elem_slot;   // ne*NNE*NNE
  const long long *slot_off;   // ntiles+1
  const uint32_t *slot_info;
  const uint16_t *aoff;        // ntiles*(NLMAX+1)
  const long long *zlo, *zhi;  // ntiles
  const int *deps;             // ntiles*kDepMax
  const uint8_t *allfree;      // ntiles
  unsigned *flags;             // ntiles
  unsigned *ticket;
  unsigned epoch;
  int zero_mode;               // 1: first-touch zeroing + dependency waits
  int zahead;                  // tiles between a tile and the one whose rows it zeroes
  long ntiles;
  int nslots_max;
  // outputs
  double *R;
  double *K;
  unsigned long long *status;
  ShapeTable shp;
};

template <int NNE>
struct TileCfg;
template <>
struct TileCfg<10> {
  static constexpr int TE = 6;  // one Kuhn cell of quadratic tets
};
template <>
struct TileCfg<4> {
  static constexpr int TE = 24;  // four Kuhn cells of linear tets
};

// Threads of a tile CTA: three groups (row component i = 0, 1, 2), each a
// whole number of warps covering the TE*NNE (element, column node) pairs, so
// every warp executes a single row component.
template <int NNE>
__host__ __device__ constexpr int tile_group() {
  return ((TileCfg<NNE>::TE * NNE + 31) / 32) * 32;
}
template <int NNE>
__host__ __device__ constexpr int tile_threads() {
  return 3 * tile_group<NNE>();
}

template <int NNE, int NQP>
inline size_t tiles_smem_bytes(int nslots_max) {
  constexpr int TE = TileCfg<NNE>::TE;
  constexpr int NL = TE * NNE;
  const size_t nq = (size_t)TE * NQP;
  return sizeof(double) * (nq * kQRec + nq * 36 + nq * NNE * 4 + (size_t)NL * 3 + (size_t)nslots_max * 9) +
         sizeof(uint32_t) * (size_t)nslots_max;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Zero-fill the K range of the rows tile u touches first and publish its flag.
template <int T>
__device__ __forceinline__ void zero_tile_rows(const TileArgs &A, long u, int tid) {
  const long long lo = A.zlo[u], hi = A.zhi[u];
  if (hi > lo) {
    const long long alo = (lo + 1) & ~1ll, ahi = hi & ~1ll;  // 16-byte aligned interior
    if (tid == 0 && alo > lo) A.K[lo] = 0.0;
    if (tid == 1 && ahi < hi && ahi >= alo) A.K[ahi] = 0.0;
    const double2 z2 = make_double2(0.0, 0.0);
    for (long long k = alo + 2 * tid; k < ahi; k += 2 * T) *reinterpret_cast<double2 *>(A.K + k) = z2;
  }
  __syncthreads();
  if (tid == 0) {
    __threadfence();
    st_release(&A.flags[u], A.epoch);
  }
}

// Rows i of the node blocks K_ab (all a) for one column node b, summed over
// the quadrature points; I is the row component (compile time).
template <int NNE, int NQP, int I>
__device__ __forceinline__ void block_rows(const double *sQ, const double *sD, const double *sP, int el, int b,
                                           double (&acc)[NNE][3]) {
  // column I of B_a: rows (I, I1, I2) of the Voigt strain with coefficients p_(I, C1, C2)
  constexpr int I1 = (I == 0) ? 4 : 3, I2 = (I == 2) ? 4 : 5;
  constexpr int C1 = (I == 2) ? 1 : 2, C2 = (I == 0) ? 1 : 0;
#pragma unroll 1
  for (int q = 0; q < NQP; q++) {
    const int qi = el * NQP + q;
    const double *Q = sQ + qi * kQRec;
    const double *D = sD + qi * 36;  // w D
    const double *P = sP + qi * NNE * 4;
    const double w = Q[9];
    const double2 pb01 = *reinterpret_cast<const double2 *>(P + b * 4);
    const double pb0 = pb01.x, pb1 = pb01.y, pb2 = P[b * 4 + 2];
    double db[3][3];
    const int Is[3] = {I, I1, I2};
#pragma unroll
    for (int m = 0; m < 3; m++) {
      const double *Dr = D + Is[m] * 6;
      const double2 d01 = *reinterpret_cast<const double2 *>(Dr);
      const double2 d23 = *reinterpret_cast<const double2 *>(Dr + 2);
      const double2 d45 = *reinterpret_cast<const double2 *>(Dr + 4);
      db[m][0] = d01.x * pb0 + d45.x * pb2 + d45.y * pb1;
      db[m][1] = d01.y * pb1 + d23.y * pb2 + d45.y * pb0;
      db[m][2] = d23.x * pb2 + d23.y * pb1 + d45.x * pb0;
    }
    // w tau p_b
    const double *ta = Q + 10;
    const double t0 = w * (ta[0] * pb0 + ta[5] * pb1 + ta[4] * pb2);
    const double t1 = w * (ta[5] * pb0 + ta[1] * pb1 + ta[3] * pb2);
    const double t2 = w * (ta[4] * pb0 + ta[3] * pb1 + ta[2] * pb2);
#pragma unroll
    for (int a = 0; a < NNE; a++) {
      const double2 pa01 = *reinterpret_cast<const double2 *>(P + a * 4);
      const double pa[3] = {pa01.x, pa01.y, P[a * 4 + 2]};
      const double g = pa[0] * t0 + pa[1] * t1 + pa[2] * t2;
      const double x0 = pa[I], x1 = pa[C1], x2 = pa[C2];
      acc[a][0] += x0 * db[0][0] + x1 * db[1][0] + x2 * db[2][0];
      acc[a][1] += x0 * db[0][1] + x1 * db[1][1] + x2 * db[2][1];
      acc[a][2] += x0 * db[0][2] + x1 * db[1][2] + x2 * db[2][2];
      acc[a][I] += g;
    }
  }
}

template <int NNE, int NQP, int MODEL>
__global__ void __launch_bounds__(tile_threads<NNE>(), NNE == 10 ? 2 : 3) k_assemble_tiles(const TileArgs A) {
  constexpr int TE = TileCfg<NNE>::TE;
  constexpr int NL = TE * NNE;
  constexpr int T = tile_threads<NNE>();
  constexpr int NQ = TE * NQP;
  constexpr bool PLASTIC = (MODEL == 1);
  extern __shared__ double sm[];
  double *sQ = sm;                  // [NQ][kQRec]: G 9, w, tau 6, s 6, n 6, dev n^2 6, a1 a2 a4 a5
  double *sD = sQ + NQ * kQRec;     // [NQ][36]
  double *sP = sD + NQ * 36;        // [NQ][NNE][4] (padded for 16-byte loads)
  double *sR = sP + NQ * NNE * 4;   // [NL][3]
  double *sAcc = sR + NL * 3;       // [nslots][9]
  uint32_t *s_sinfo = reinterpret_cast<uint32_t *>(sAcc + A.nslots_max * 9);  // [nslots]
  __shared__ int s_tile;
  __shared__ int s_nodes[NL];
  __shared__ int s_rp[NL], s_rl[NL], s_ndof[NL * 3];
  __shared__ uint8_t s_mask[NL];
  __shared__ uint8_t s_lnode[TE * NNE];
  __shared__ uint16_t s_aoff[NL + 1];
  __shared__ uint16_t s_eslot[TE * NNE * NNE];
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;

  // accumulators start at zero; phase W zeroes every entry it consumes
  for (int i = tid; i < A.nslots_max * 9; i += T) sAcc[i] = 0.0;
  for (int i = tid; i < NL * 3; i += T) sR[i] = 0.0;
  // prologue: the rows first touched by the first zahead tiles
  if (A.zero_mode)
    for (long u = blockIdx.x; u < min((long)A.zahead, A.ntiles); u += gridDim.x) zero_tile_rows<T>(A, u, tid);
  if (tid == 0) s_tile = (int)atomicAdd(A.ticket, 1u);
  __syncthreads();
  for (;;) {
    const long t = s_tile;
    if (t >= A.ntiles) break;
    // next ticket, requested now and consumed at the end of this tile
    int next_ticket = 0;
    if (tid == 0) next_ticket = (int)atomicAdd(A.ticket, 1u);
    const long e0 = t * TE;
    const int nel = (int)min((long)TE, A.ne - e0);
    const int nq = nel * NQP;
    const long q0 = e0 * NQP;
    const int nl = A.tile_nl[t];
    const long sbeg = A.slot_off[t];
    const int nslots = (int)(A.slot_off[t + 1] - sbeg);

    // ---- Z: zero the rows first touched by the tile A.zahead tickets ahead ----
    if (A.zero_mode && t + A.zahead < A.ntiles) zero_tile_rows<T>(A, t + A.zahead, tid);

    // ---- L: tile metadata and point records ----
    for (int i = tid; i < nl; i += T) {
      const int n = A.tile_nodes[t * NL + i];
      s_nodes[i] = n;
      s_mask[i] = A.mask[n];
      s_rp[i] = A.rowptr0[n];
      s_rl[i] = A.rowlen[n];
      s_ndof[i * 3 + 0] = A.dof[n];
      s_ndof[i * 3 + 1] = A.dof[A.nn + n];
      s_ndof[i * 3 + 2] = A.dof[2 * A.nn + n];
    }
    for (int i = tid; i < nslots; i += T) s_sinfo[i] = A.slot_info[sbeg + i];
    for (int i = tid; i < nel * NNE * NNE; i += T) s_eslot[i] = A.elem_slot[e0 * NNE * NNE + i];
    for (int i = tid; i < nel * NNE; i += T) s_lnode[i] = A.elem_lnode[e0 * NNE + i];
    for (int i = tid; i <= nl; i += T) s_aoff[i] = A.aoff[t * (NL + 1) + i];
    for (int i = tid; i < kQRec * NQ; i += T) {
      const int c = i / NQ, q = i - c * NQ;
      if (q < nq) sQ[q * kQRec + c] = A.qrec[c * A.nqp + q0 + q];
    }
    __syncthreads();
    // Voigt tangent rows w D[I][:] (xx, yy, zz, yz, xz, xy; engineering shear):
    // c = a1 I + a2 1(x)1 - 2/3 (s(x)1 + 1(x)s) + a4 n(x)n + a5 n(x)dev(n^2)
    for (int i = tid; i < nq * 6; i += T) {
      const int q = i / 6, I = i - q * 6;
      const double *Q = sQ + q * kQRec;
      const double w = Q[9], a1 = Q[34], a2 = Q[35];
      const double eI = I < 3 ? 1.0 : 0.0, sI = Q[16 + I];
      const double nI4 = PLASTIC ? Q[22 + I] * Q[36] : 0.0, nI5 = PLASTIC ? Q[22 + I] * Q[37] : 0.0;
      double *Dr = sD + q * 36 + I * 6;
#pragma unroll
      for (int J = 0; J < 6; J++) {
        const double eJ = J < 3 ? 1.0 : 0.0;
        double v = a2 * eI * eJ - (2.0 / 3.0) * (sI * eJ + eI * Q[16 + J]);
        if (PLASTIC) v += nI4 * Q[22 + J] + nI5 * Q[28 + J];
        if (I == J) v += I < 3 ? a1 : 0.5 * a1;
        Dr[J] = w * v;
      }
    }
    // spatial gradients p_a and the residual w tau p_a
    for (int i = tid; i < nq * NNE; i += T) {
      const int q = i / NNE, a = i - q * NNE;
      const int qq = q % NQP;
      const double *G = sQ + q * kQRec;
      const double g0 = A.shp.dNxi[qq][a][0], g1 = A.shp.dNxi[qq][a][1], g2 = A.shp.dNxi[qq][a][2];
      double p[3], tp[3];
#pragma unroll
      for (int j = 0; j < 3; j++) p[j] = G[0 * 3 + j] * g0 + G[1 * 3 + j] * g1 + G[2 * 3 + j] * g2;
      double *pp = sP + (q * NNE + a) * 4;
      pp[0] = p[0];
      pp[1] = p[1];
      pp[2] = p[2];
      pp[3] = 0.0;
      smv(G + 10, p, tp);
      const double w = G[9];
      double *r = sR + s_lnode[(q / NQP) * NNE + a] * 3;
      atomicAdd(r + 0, w * tp[0]);
      atomicAdd(r + 1, w * tp[1]);
      atomicAdd(r + 2, w * tp[2]);
    }
    __syncthreads();

    // ---- B: node-block rows ----
    constexpr int GRP = tile_group<NNE>();
    const int i = tid / GRP, jj = tid - i * GRP;
    if (jj < nel * NNE) {
      const int el = jj / NNE, b = jj - el * NNE;
      double acc[NNE][3];
#pragma unroll
      for (int a = 0; a < NNE; a++) acc[a][0] = acc[a][1] = acc[a][2] = 0.0;
      if (i == 0) block_rows<NNE, NQP, 0>(sQ, sD, sP, el, b, acc);
      else if (i == 1) block_rows<NNE, NQP, 1>(sQ, sD, sP, el, b, acc);
      else block_rows<NNE, NQP, 2>(sQ, sD, sP, el, b, acc);
      const uint16_t *es = s_eslot + el * NNE * NNE;
#pragma unroll
      for (int a = 0; a < NNE; a++) {
        const uint16_t s = es[a * NNE + b];
        if (s == 0xFFFF) continue;
        double *d = sAcc + s * 9 + i * 3;
        atomicAdd(d + 0, acc[a][0]);
        atomicAdd(d + 1, acc[a][1]);
        atomicAdd(d + 2, acc[a][2]);
      }
    }

    // ---- wait for the tiles that zeroed the other rows we write ----
    if (A.zero_mode && tid <= kDepMax) {
      const int d = tid == kDepMax ? (int)t : A.deps[t * kDepMax + tid];
      if (d >= 0) {
        unsigned spins = 0;
        while (ld_acquire(&A.flags[d]) != A.epoch) {
          if (++spins > (1u << 22)) {
            atomicAdd(&A.status[3], 1ull);
            break;
          }
          __nanosleep(64);
        }
      }
    }
    __syncthreads();

    // ---- W: one warp per (node, component) row, lanes along the row ----
    const bool allfree = A.allfree[t] != 0;
    for (int row = warp; row < nl * 3; row += T / 32) {
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
    for (int f = tid; f < nl * 3; f += T) {
      const int id = s_ndof[f];
      const double v = sR[f];
      sR[f] = 0.0;
      if (id > 0) atomicAdd(A.R + (id - 1), v);
    }
    __syncthreads();
    if (tid == 0) s_tile = next_ticket;
    __syncthreads();
  }
}

}  // namespace pgb
