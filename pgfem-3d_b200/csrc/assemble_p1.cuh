// assemble_p1.cuh -- FP64 R+K assembly of linear tets (configs 1 and 5) with
// column-split block rows, the default R+K path for 4-node elements.  The
// point updates run first in k_qp_update<4, 1, MODEL> (assemble_mma.cuh: one
// thread per point, records in HBM); k_assemble_p1ws is a producer/consumer
// pipeline over tiles of elements.
//
// Same operation as k_assemble (fd_residuals_MP + stiffmat_fd_MP for the
// constitutive-model element, src/fd_residuals.cc:468-636,
// src/stiffmat_fd.cc:831-993), organised for the FP64 pipe and the L2
// reduction units:
//
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

constexpr int kP2VS = 18;                     // doubles per (point, node) vector record

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

// ---- bounded mbarrier hand-off between the producer and consumer warps ----
//
// Every wait is bounded: a wait that runs out sets status[3] and both roles
// leave their loops (their next waits run out too), so a fault cannot hang
// the GPU.
constexpr unsigned long long kWWaitNs = 2000000000ull;  // default bound of a hand-off wait

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
__device__ __forceinline__ bool w_mb_wait(uint64_t *b, unsigned parity, unsigned long long limit) {
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
    if (w_gtimer() - t0 > limit) return false;
  }
}

// ---- linear tets: column-split assembly from point records ----------------
//
// Point records come from k_qp_update<4, 1, MODEL> (one thread per point);
// the vector records of an element are its four nodes' (p, U, W, T, S, n p).
constexpr int kP1ES = 4 * kP2VS + 2;  // doubles per element of vector records (even, bank-spread)

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
        const bool ok = w_mb_wait(&empty[bx], (unsigned)(((i - 2) >> 1) & 1), args.wait_ns);
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
      // release: vectors and the tile index are visible to the consumers (the
      // failure-path test withholds lane 0's first arrive: the phase never completes)
      if (!(args.stall && i == 0 && pl == 0)) w_mb_arrive(&full[bx]);
      t_cur = t_nxt;
    }
    cpa_wait_all();
  } else {
    // ------------------------------ consumers ------------------------------
    const int el = tid >> 4, r = tid & 15;
    const int a = r / 3, k = r - a * 3;
    for (long i = 0;; i++) {
      const int bx = (int)(i & 1), bm = (int)(i % 3);
      if (!w_mb_wait(&full[bx], (unsigned)((i >> 1) & 1), args.wait_ns)) {
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
