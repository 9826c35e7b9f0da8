// assemble_mma.cuh -- FP64 R+K assembly of quadratic tets with the element
// contraction on the FP64 tensor cores (mma.sync .m8n8k4 .f64).
//
// Same operation as the other assembly kernels (fd_residuals_MP +
// stiffmat_fd_MP for the constitutive-model element, src/fd_residuals.cc:
// 468-636, src/stiffmat_fd.cc:831-993), in two kernels:
//
//  k_qp_update<..., YREC = true>  one thread per quadrature point: F, the
//      constitutive update (run_integration_algorithm,
//      src/constitutive_model.cc:1100-1129; state n -> n+1) and a 26-double
//      point record (structure of arrays) from which the assembly forms the
//      matrices of the element contraction:
//        G = (dX/dxi)^-1 F^-1      (p_a = G^T dN_a/dxi = F^-T grad_X N_a)
//        T' = a1 w/2 1 + w tau,  s'' = -2/3 w s,  U' = w a2 1 + s'',
//        W' = w (a4 n + a5 dev(n^2)),  h = a1 w / 2
//      for the spatial tangent c = a1 I + a2 1(x)1 - 2/3 (s(x)1 + 1(x)s)
//      + a4 n(x)n + a5 n(x)dev(n^2) (cm_models.cuh) and w = det(dX/dxi) x weight.
//      At a plastic point s = |s| n (radial return), so the record holds
//      V = n and s'' = c V with c = -2/3 w (s : n); elsewhere V = s,
//      c = -2/3 w and a4 = a5 = 0.
//
//  k_assemble_p2m  persistent grid over tiles of 4 consecutive elements, four
//      warps per CTA, one element per warp in the contraction.  With the
//      vectors p, T = T'p, U = U'p, W = W'p, h p of node b at point q, the
//      element block K_ab[i][k] (compute_stiffness_matrix,
//      src/constitutive_model.cc:1520-1616, in spatial form) is
//        K_ab[i][k] = sum_q sum_j p_a[j] Y_q[j][(b,i,k)],
//        Y_q[j][(b,i,k)] = d_jk h p_b[i] + d_ij U_b[k] + s''_ij p_b[k]
//                          + n_ij W_b[k] + d_ik T_b[j],
//      and the residual R_a[i] = sum_q sum_j p_a[j] w tau_ij
//      (compute_residual_vector, :1628-1662): one GEMM per element,
//        C (96 x 10) = Y^T (96 x 12) P (12 x 10),  P[(q,j)][a] = p_qa[j],
//      whose 96 rows are (i, b, k) in blocks of 32 per i (30 K columns, the
//      residual, one pad) and whose 12-deep contraction runs over (q, j).
//   Y  all threads: item (element, point, column node b) builds its 27 Y
//      values and its p into shared memory (Y in the A-fragment order of the
//      mma, so that each fragment load is 32 consecutive doubles), and the
//      column offsets of node b's block in the rows of the element's nodes;
//   C  warp per element: 36 mma.m8n8k4 for row nodes a = 0..7 and 36 more on
//      the same A fragments for row nodes 8 and 9 (B columns p_8, p_9
//      repeated, so that every lane holds its row tiles' results);
//   S  FP64 reductions of the 900 K entries and 30 R entries into the CSR
//      through the node-block map (fd_res_assemble, src/fd_residuals.cc:58-73;
//      PLoc_Sparse, src/PLoc_Sparse.cc:15-175).  Per reduction instruction a
//      warp writes eight consecutive entries of four CSR rows.
#pragma once
#include <cstdint>

#include "assemble.cuh"
#include "assemble_p1.cuh"  // bounded mbarrier waits

namespace pgb {

constexpr int kQRec = kRec;  // point record of the linear-tet path: G 9, w, tau 6, s 6, n 6, dev(n^2) 6, a1 a2 a4 a5
// point record of the tensor-core path: G 9, T' 6, V 6, w a2, c, w a4, w a5, h
constexpr int kYRec = 26;
// the three-field (CM3F) element adds w J, w and the element's theta and P
constexpr int kYRecTF = 30;
__host__ __device__ constexpr int yrec_fields(bool tf) { return tf ? kYRecTF : kYRec; }
constexpr int kMPtsT = 16;  // points per record tile (the assembly tile: 4 elements x 4 points)

// index of field c of record slot qs in the tiled layout of the tensor-core path
template <int NRF = kYRec>
__host__ __device__ __forceinline__ long yrec_idx(long qs, int c) {
  return ((qs >> 4) * NRF + c) * kMPtsT + (qs & (kMPtsT - 1));
}

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
  double *qrec;         // kQRec*nqp (SoA) or, for 10-node elements, kYRec doubles per point in
                        // tiles of kMPtsT points ([tile][field][point], padded to whole tiles)
  unsigned long long *status;
  // processing order: record slot e' holds element perm[e'] (nullptr: e' = e);
  // the state stays in element order
  const int *perm;
  Mat mat;
  ShapeTable shp;
  // three-field element (10-node records, hyperelastic and J2 models): the
  // pressure and the volume of each element (element order)
  const double *tf_P, *tf_theta;
};

template <int NNE, int NQP, int MODEL, bool YREC = false, bool TF = false>
__global__ void __launch_bounds__(128) k_qp_update(const QpArgs A) {
  constexpr bool PLASTIC = (MODEL == 1);
  constexpr int NRF = yrec_fields(TF);
  constexpr int NR = YREC ? NRF : kQRec;
  const long qs = blockIdx.x * (long)blockDim.x + threadIdx.x;  // record slot
  if (qs >= A.nqp) return;
  const long es = qs / NQP;
  const int q = (int)(qs - es * NQP);
  const long e = A.perm ? (long)A.perm[es] : es;
  const long qp = e * NQP + q;  // state index
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
    for (int c = 0; c < NR; c++) rec[YREC ? yrec_idx<NRF>(qs, c) : c * S + qs] = 0.0;
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
  double tfP = 0.0, tfTh = 0.0;
  if (TF) {
    // three-field element: the volumetric stress is the element pressure,
    // P J 1, at fixed P (no kappa J^2 U'' term in the tangent)
    tfP = A.tf_P[e];
    tfTh = A.tf_theta[e];
    double dU, d2U;
    vol_derivs(A.mat.vol_pot, J, dU, d2U);
    const double pJ = A.mat.kappa * J * dU, PJ = tfP * J;
#pragma unroll
    for (int c = 0; c < 3; c++) t.tau[c] += PJ - pJ;
    t.a1 += 2.0 * (pJ - PJ);
    t.a2 += PJ - A.mat.kappa * (J * dU + J * J * d2U);
  }
  if (PLASTIC && A.state_np1) {
#pragma unroll
    for (int c = 0; c < 6; c++) A.state_np1[c * S + qp] = Anp1[c];
    A.state_np1[6 * S + qp] = alpha_np1;
  }
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      rec[YREC ? yrec_idx<NRF>(qs, i * 3 + j) : (i * 3 + j) * S + qs] =
          dXi[i * 3 + 0] * Fi[0 * 3 + j] + dXi[i * 3 + 1] * Fi[1 * 3 + j] + dXi[i * 3 + 2] * Fi[2 * 3 + j];
  const double w = detJ * A.shp.w[q];
  if (YREC) {
    const double h = 0.5 * t.a1 * w, c23 = (2.0 / 3.0) * w;
    // plastic point: n != 0 (the unit flow direction, s = (s : n) n)
    const bool pl = PLASTIC && (t.n[0] != 0.0 || t.n[1] != 0.0 || t.n[2] != 0.0 || t.n[3] != 0.0 ||
                                t.n[4] != 0.0 || t.n[5] != 0.0);
#pragma unroll
    for (int c = 0; c < 6; c++) {
      rec[yrec_idx<NRF>(qs, 9 + c)] = h * (c < 3 ? 1.0 : 0.0) + w * t.tau[c];
      rec[yrec_idx<NRF>(qs, 15 + c)] = pl ? t.n[c] : t.s[c];
    }
    rec[yrec_idx<NRF>(qs, 21)] = w * t.a2;
    rec[yrec_idx<NRF>(qs, 22)] = pl ? -c23 * sdot(t.s, t.n) : -c23;
    rec[yrec_idx<NRF>(qs, 23)] = w * t.a4;
    rec[yrec_idx<NRF>(qs, 24)] = w * t.a5;
    rec[yrec_idx<NRF>(qs, 25)] = h;
    if (TF) {
      rec[yrec_idx<NRF>(qs, 26)] = w * J;
      rec[yrec_idx<NRF>(qs, 27)] = w;
      rec[yrec_idx<NRF>(qs, 28)] = tfTh;
      rec[yrec_idx<NRF>(qs, 29)] = tfP;
    }
  } else {
    rec[9 * S + qs] = w;
#pragma unroll
    for (int c = 0; c < 6; c++) {
      rec[(10 + c) * S + qs] = t.tau[c];
      rec[(16 + c) * S + qs] = t.s[c];
      rec[(22 + c) * S + qs] = t.n[c];
      rec[(28 + c) * S + qs] = t.D[c];
    }
    rec[34 * S + qs] = t.a1;
    rec[35 * S + qs] = t.a2;
    rec[36 * S + qs] = t.a4;
    rec[37 * S + qs] = t.a5;
  }
}

// ---- tensor-core element assembly ------------------------------------------

constexpr int kMTE = 4;                 // elements per tile (one per warp)
constexpr int kMThreads = 32 * kMTE;    // 128
constexpr int kMPts = kMTE * 4;         // points per tile
// Y doubles per element: [kstep 3][row tile 12][lane 32], and P doubles per
// element: [a 10][t 12]; both padded so that the item stores of a half-warp
// (four column-node pairs x four points, possibly of two elements) hit 16
// distinct banks
constexpr int kMY = 3 * 12 * 32 + 12;
constexpr int kMP = 10 * 12 + 4;
constexpr int kMCS = 36;                // column-table row stride (words): lane loads hit 32 banks
// column table per element: [a 10][rr = 3 b + k, 30 -> R, 31 -> pad], element stride padded by three
// words so that the item stores (element, column-node pair, point) spread over the banks
constexpr int kMCol = 10 * kMCS + 3;
constexpr int kMMeta = kMTE * 10;       // (element, node) pairs per tile
constexpr int kMColR = -2;              // column-table marker of the residual row
// Per-element scatter block (int32 words, 464 bytes so that it copies in 16-byte chunks):
//   [0, 30)    row base of (node a, component i): CSR offset of the row, -1 if not free
//   [30, 60)   residual index of (a, i): free DOF id - 1, -1 if not free
//   [60, 110)  node-pair positions pos[a][b] (uint16, column offset of b's block in a's rows)
//   [110, 113) free-component masks of the ten nodes (bytes)
constexpr int kEBW = 116;
constexpr int kEBPos = 60, kEBMask = 110;

inline size_t p2m_smem_bytes(bool tf = false) {
  return sizeof(double) * ((size_t)kMTE * kMY + (size_t)kMTE * kMP + (size_t)yrec_fields(tf) * kMPts) +
         sizeof(int) * (size_t)kMTE * kMCol + sizeof(int) * 2 * (size_t)kMTE * kEBW + 2 * sizeof(uint64_t) +
         2 * sizeof(long);
}

// bytes of one tile's copies: its point records and its elements' scatter blocks
__host__ __device__ constexpr unsigned tile_bytes(bool tf) {
  return (unsigned)(sizeof(double) * yrec_fields(tf) * kMPtsT + sizeof(int) * kMTE * kEBW);
}

// one-dimensional bulk copy global -> shared through the tensor memory
// accelerator, completing on an mbarrier (16-byte aligned, size a multiple of 16)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          (unsigned)__cvta_generic_to_shared(dst)),
      "l"(src), "r"(bytes), "r"((unsigned)__cvta_generic_to_shared(bar))
      : "memory");
}
__device__ __forceinline__ void mb_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(bar)),
               "r"(bytes)
               : "memory");
}

// Builds the scatter blocks of all 10-node elements from the node arrays and
// the element->CSR node-block map (thread per element).
// Block slot e' holds element perm[e'] (the processing order).
__global__ void k_build_eblock(const int *conn, long ne, const int *dof, long nn, const int *rowptr0,
                               const int *rowlen, const uint8_t *mask, const uint16_t *pos, const int *perm,
                               int *eb) {
  const long es = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (es >= ne) return;
  const long e = perm ? (long)perm[es] : es;
  int *o = eb + es * kEBW;
  uint16_t *o16 = reinterpret_cast<uint16_t *>(o + kEBPos);
  uint8_t *o8 = reinterpret_cast<uint8_t *>(o + kEBMask);
  for (int a = 0; a < 10; a++) {
    const int n = conn[(long)a * ne + e];
    const unsigned mk = mask[n];
    for (int i = 0; i < 3; i++) {
      const bool fr = (mk >> i) & 1u;
      o[a * 3 + i] = fr ? rowptr0[n] + __popc(mk & ((1u << i) - 1u)) * rowlen[n] : -1;
      o[30 + a * 3 + i] = fr ? dof[i * nn + n] - 1 : -1;
    }
    for (int b = 0; b < 10; b++) o16[a * 10 + b] = pos[(e * 10 + a) * 10 + b];
    o8[a] = (uint8_t)mk;
  }
  o8[10] = o8[11] = 0;
  o[113] = o[114] = o[115] = 0;
}

// index of Y[t][r] (t = 3q + j, r = 32 i + 3 b + k) in the fragment-ordered buffer
__device__ __forceinline__ int y_idx(int t, int r) {
  return (((t >> 2) * 12 + (r >> 3)) << 5) + ((r & 7) << 2) + (t & 3);
}

// D (8x8) += A (8x4, row) B (4x8, col), FP64.  Lane l holds A[l/4][l%4],
// B[l%4][l/4], and C[l/4][2 (l%4) + c] in c<c>.
__device__ __forceinline__ void dmma884(double &c0, double &c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}


// Item (point q, column nodes b0 and b0 + 5) of one element: p_b into P, the
// 27 values Y_q[j][(b, i, k)] of each column node and, for b0 = 0, the
// residual rows Y_q[j][32 i + 30] = w tau_ij.  rec: the point's record fields
// with stride RS (the element's other points at rec - q + q'); shp: the
// shape-function derivatives.
// TF (three-field element, one pressure P and one volume theta per element):
// the static condensation of (P, theta) adds c Kup Kup^T to the element's K and
// s Kup to its R, with Kup_b = sum_q w J p_qb (the derivative of the volume
// constraint), W = sum_q w, fp = sum_q w J - theta W, c = kappa U''(theta) / W
// and s = c fp + kappa U'(theta) - P -- in the contraction, w J c Kup_b[k] is
// added to U_b[k] and w J s delta_ij to the residual rows (the pressure part
// of the point's stress is P J 1 already, from the point kernel).
// Y[t][r] sits at y_idx(t, r) = tb(t) + 128 i + gk(3 b + k) for r = 32 i + 3 b + k.
template <bool PLASTIC, int RS, bool TF = false>
__device__ __forceinline__ void p2m_item(const double *rec, const ShapeTable &shp, int q, int b0, double *Y,
                                         double *P, const Mat &mat) {
  const double(*dN)[3] = shp.dNxi[q];
  double G[9], Tm[6], Um[6], Wm[6], s2[6], nn[6];
#pragma unroll
  for (int c = 0; c < 9; c++) G[c] = rec[c * RS];
  const double wa2 = rec[21 * RS], cs = rec[22 * RS], h = rec[25 * RS];
#pragma unroll
  for (int c = 0; c < 6; c++) {
    Tm[c] = rec[(9 + c) * RS];
    nn[c] = rec[(15 + c) * RS];
    s2[c] = cs * nn[c];
    Um[c] = s2[c] + (c < 3 ? wa2 : 0.0);
  }
  if (PLASTIC) {
    // W' = w a4 n + w a5 dev(n^2) (zero at elastic points: w a4 = w a5 = 0)
    const double w4 = rec[23 * RS], w5 = rec[24 * RS];
    const double *n = nn;
    double n2[6];
    n2[0] = n[0] * n[0] + n[5] * n[5] + n[4] * n[4];
    n2[1] = n[5] * n[5] + n[1] * n[1] + n[3] * n[3];
    n2[2] = n[4] * n[4] + n[3] * n[3] + n[2] * n[2];
    n2[3] = n[5] * n[4] + n[1] * n[3] + n[3] * n[2];
    n2[4] = n[0] * n[4] + n[5] * n[3] + n[4] * n[2];
    n2[5] = n[0] * n[5] + n[5] * n[1] + n[4] * n[3];
    const double t3 = (n2[0] + n2[1] + n2[2]) * (1.0 / 3.0);
#pragma unroll
    for (int c = 0; c < 6; c++) Wm[c] = w4 * n[c] + w5 * (n2[c] - (c < 3 ? t3 : 0.0));
  } else {
#pragma unroll
    for (int c = 0; c < 6; c++) Wm[c] = nn[c] = 0.0;
  }
  double wJq = 0.0, tfc = 0.0, tfs = 0.0;
  if (TF) {
    const double *r0 = rec - q;  // point 0 of the element
    double W = 0.0, SJ = 0.0;
#pragma unroll
    for (int qq = 0; qq < 4; qq++) {
      SJ += r0[26 * RS + qq];
      W += r0[27 * RS + qq];
    }
    wJq = rec[26 * RS];
    const double th = rec[28 * RS], Pe = rec[29 * RS];
    double dU, d2U;
    vol_derivs(mat.vol_pot, th, dU, d2U);
    tfc = mat.kappa * d2U / W;
    tfs = tfc * (SJ - th * W) + mat.kappa * dU - Pe;
  }
  int tb[3];
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const int t = 3 * q + j;
    tb[j] = (t >> 2) * 384 + (t & 3);
  }
  // full 3x3 index of a Voigt-stored symmetric matrix (xx yy zz yz xz xy)
  auto vo = [](int i, int j) { return i == j ? i : 6 - i - j; };
#pragma unroll
  for (int half = 0; half < 2; half++) {
    const int b = b0 + 5 * half;
    const double g0 = dN[b][0], g1 = dN[b][1], g2 = dN[b][2];
    double p[3], T[3], U[3], W[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int j = 0; j < 3; j++) p[j] = G[j] * g0 + G[3 + j] * g1 + G[6 + j] * g2;
    smv(Tm, p, T);
    smv(Um, p, U);
    if (PLASTIC) smv(Wm, p, W);
    if (TF) {
      // Kup_b = sum over the element's points of w J G^T dN_b
      const double *r0 = rec - q;
      double v[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int qq = 0; qq < 4; qq++) {
        const double *rq = r0 + qq;
        const double d0 = shp.dNxi[qq][b][0], d1 = shp.dNxi[qq][b][1], d2 = shp.dNxi[qq][b][2];
        const double wj = rq[26 * RS];
#pragma unroll
        for (int j = 0; j < 3; j++) v[j] = fma(wj, rq[j * RS] * d0 + rq[(3 + j) * RS] * d1 + rq[(6 + j) * RS] * d2, v[j]);
      }
#pragma unroll
      for (int k = 0; k < 3; k++) U[k] = fma(wJq * tfc, v[k], U[k]);
    }
    int gk[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const int x = 3 * b + k;
      gk[k] = ((x >> 3) << 5) + ((x & 7) << 2);
    }
#pragma unroll
    for (int j = 0; j < 3; j++) {
#pragma unroll
      for (int k = 0; k < 3; k++) {
        double *Yjk = Y + tb[j] + gk[k];
#pragma unroll
        for (int i = 0; i < 3; i++) {
          double y = s2[vo(i, j)] * p[k];
          if (PLASTIC) y = fma(nn[vo(i, j)], W[k], y);
          if (j == k) y = fma(h, p[i], y);
          if (i == j) y += U[k];
          if (i == k) y += T[j];
          Yjk[128 * i] = y;
        }
      }
      P[b * 12 + 3 * q + j] = p[j];
    }
  }
  if (b0 == 0) {
    // w tau = T' - h 1 (row r = 32 i + 30: offset 128 i + 120)
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
      for (int i = 0; i < 3; i++) Y[tb[j] + 128 * i + 120] = Tm[vo(i, j)] - (i == j ? h - wJq * tfs : 0.0);
  }
}

template <int MODEL, bool TF = false>
__global__ void __launch_bounds__(kMThreads, 4) k_assemble_p2m(const AsmArgs args) {
  constexpr int NNE = 10, NQP = 4, TE = kMTE, NT = kMThreads;
  constexpr bool PLASTIC = (MODEL == 1);
  constexpr int NRF = yrec_fields(TF);
  extern __shared__ __align__(16) double msm[];
  double *sY = msm;                                          // [TE][kMY]
  double *sP = sY + TE * kMY;                                // [TE][kMP]
  double *sRec = sP + TE * kMP;                              // [NRF][kMPts]
  int *sCol = reinterpret_cast<int *>(sRec + NRF * kMPts);    // [TE][10][kMCS]
  int *sEB = sCol + TE * kMCol;                              // [2][TE][kEBW]
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sEB + 2 * TE * kEBW);  // [2]: tile copies landed
  long *sTile = reinterpret_cast<long *>(mbar + 2);                    // [2]: the tile of each buffer
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long ne = args.ne;
  const long ntiles = (ne + TE - 1) / TE;
  // pad rows r = 32 i + 31 of Y stay zero; the column table marks the
  // residual row (rr = 30) and the pad row (rr = 31)
  for (int x = tid; x < TE * 12; x += NT) {
    const int el = x / 12, t = x - el * 12;
#pragma unroll
    for (int i = 0; i < 3; i++) sY[el * kMY + y_idx(t, 32 * i + 31)] = 0.0;
  }
  for (int x = tid; x < TE * 10; x += NT) {
    int *row = sCol + (x / 10) * kMCol + (x % 10) * kMCS;
    row[30] = kMColR;
    row[31] = -1;
  }

  // one tile's point records (5120 contiguous bytes of the tiled layout) and
  // its elements' scatter blocks (1856 contiguous bytes) by two bulk copies of
  // the tensor memory accelerator, completing on mbar[buf]; the buffers are
  // padded to whole tiles, so a partial last tile copies whole too
  if (tid == 0) {
    w_mb_init(&mbar[0], 1);
    w_mb_init(&mbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // Tiles are claimed in order from a global counter (zeroed before the
  // launch), one tile ahead: all CTAs then work on neighbouring tiles of the
  // processing order, and the CSR rows they reduce into stay in L2 between
  // the contributions of neighbouring elements.  Thread 0 claims, records the
  // tile in sTile[buf] and issues its copies; with no tile left it completes
  // the buffer's phase by a plain arrive.
  auto claim = [&](int buf) {  // thread 0
    const long t = (long)atomicAdd(args.ticket, 1u);
    sTile[buf] = t;
    if (t < ntiles) {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // after the generic reads of the buffers
      mb_expect_tx(&mbar[buf], tile_bytes(TF));
      bulk_g2s(sRec, args.qrec + t * (long)(NRF * kMPtsT), sizeof(double) * NRF * kMPtsT, &mbar[buf]);
      bulk_g2s(sEB + buf * TE * kEBW, args.eblk + t * TE * kEBW, sizeof(int) * TE * kEBW, &mbar[buf]);
    } else {
      w_mb_arrive(&mbar[buf]);
    }
  };
  if (tid == 0) claim(0);

  for (int it = 0;; it++) {
    const int mb = it & 1;
    // this tile's copies landed (bounded wait: a wait that runs out is
    // counted in status[3] and every thread leaves, after waiting -- again
    // bounded -- for the copies still in flight)
    const bool landed = w_mb_wait(&mbar[mb], (unsigned)((it >> 1) & 1), args.wait_ns);
    if (__syncthreads_or(!landed)) {  // also: previous tile's C/S done
      if (tid == 0) {
        atomicAdd(&args.status[3], 1ull);
        w_mb_wait(&mbar[mb], (unsigned)((it >> 1) & 1), args.wait_ns);
      }
      break;
    }
    const long e0 = sTile[mb] * TE;  // written before the barrier above
    if (e0 >= ne) break;
    // ---- Y: items (element, column-node pair, point), point fastest ----
    if (tid < TE * 20) {
      const int el = tid / 20, rem = tid - el * 20;
      const int bp = rem >> 2, q = rem & 3;
      if (e0 + el < ne) {
        p2m_item<PLASTIC, kMPts, TF>(sRec + el * NQP + q, args.shp, q, bp, sY + el * kMY, sP + el * kMP,
                                     args.mat);
        // column offsets of node b's block inside the rows of nodes a = q, q+4, q+8
        const int *eb = sEB + (mb * TE + el) * kEBW;
        const uint16_t *pos16 = reinterpret_cast<const uint16_t *>(eb + kEBPos);
        const uint8_t *mk8 = reinterpret_cast<const uint8_t *>(eb + kEBMask);
#pragma unroll
        for (int half = 0; half < 2; half++) {
          const int b = bp + 5 * half;
          const unsigned maskB = mk8[b];
          int *ct = sCol + el * kMCol + 3 * b;
#pragma unroll
          for (int x4 = 0; x4 < 3; x4++) {
            const int a = q + 4 * x4;
            if (a < NNE) {
              const int pab = pos16[a * 10 + b];
#pragma unroll
              for (int k = 0; k < 3; k++)
                ct[a * kMCS + k] = ((maskB >> k) & 1u) ? pab + rank_of(maskB, k) : -1;
            }
          }
        }
      }
    }
    __syncthreads();  // Y, P and column offsets complete; the record buffer is free
    // ---- claim the next tile, prefetch its records and scatter blocks ----
    if (tid == 0) claim(mb ^ 1);
    // ---- C: the element's GEMM on the FP64 tensor cores ----
    // m8n8k4 for row nodes a = 0..7 (12 row tiles of 8 Y rows, 3 steps over
    // the contraction) and, on the same A fragments, for row nodes 8 and 9
    // with B columns (p_8, p_9) repeated four times: lane (rho, u) then holds
    // C[8 m + rho][8 + c] of every row tile m in a89[m][c], and no lane
    // exchange is needed to spread rows 8, 9 over the warp for the scatter
    const int el = warp;
    if (e0 + el >= ne) continue;
    const double *Y = sY + el * kMY;
    const double *P = sP + el * kMP;
    const int rho = lane >> 2, u = lane & 3;
    double acc[12][2], a89[12][2];
#pragma unroll
    for (int m = 0; m < 12; m++) acc[m][0] = acc[m][1] = a89[m][0] = a89[m][1] = 0.0;
#pragma unroll
    for (int s = 0; s < 3; s++) {
      const double bf = P[rho * 12 + 4 * s + u];
      const double b89 = P[(8 + (rho & 1)) * 12 + 4 * s + u];
#pragma unroll
      for (int m = 0; m < 12; m++) {
        const double af = Y[(s * 12 + m) * 32 + lane];
        dmma884(acc[m][0], acc[m][1], af, bf);
        dmma884(a89[m][0], a89[m][1], af, b89);
      }
    }
    // ---- S: reductions into the CSR ----
    // C[r][a], r = 8 m + rho = 32 i + rr: K entry (row i of node a, column rr
    // of the column table) or, for rr = 30, the residual of (a, i); one
    // reduction instruction per value, its target selected.
    const int *eb = sEB + (mb * TE + el) * kEBW;
    const int *ct = sCol + el * kMCol;
    // the target of value v: K entry (row base rb, column offset cv >= 0) or,
    // for the residual row (cv = kMColR), the residual entry rd; nothing when
    // component i of node a is not free (rb < 0) or the column is (cv = -1)
    auto red = [&](int rb, int rd, int cv, double v) {
      const bool kk = cv >= 0;
      if (rb >= 0 && (kk || cv == kMColR)) atomicAdd(kk ? args.K + (rb + cv) : args.R + rd, v);
    };
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const int a = 2 * u + c;
      int rb[3], rd[3], cv[4];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        rb[i] = eb[a * 3 + i];
        rd[i] = eb[30 + a * 3 + i];
      }
#pragma unroll
      for (int mq = 0; mq < 4; mq++) cv[mq] = ct[a * kMCS + 8 * mq + rho];
#pragma unroll
      for (int m = 0; m < 12; m++) red(rb[m >> 2], rd[m >> 2], cv[m & 3], acc[m][c]);
    }
    {
      // lane u of a row group takes the row tile m = 4 mm + u (row i = mm)
      const int rr = 8 * u + rho;
      const int cv8 = ct[8 * kMCS + rr], cv9 = ct[9 * kMCS + rr];
#pragma unroll
      for (int mm = 0; mm < 3; mm++) {
        double v8 = a89[4 * mm][0], v9 = a89[4 * mm][1];
#pragma unroll
        for (int x = 1; x < 4; x++) {
          v8 = u == x ? a89[4 * mm + x][0] : v8;
          v9 = u == x ? a89[4 * mm + x][1] : v9;
        }
        red(eb[24 + mm], eb[54 + mm], cv8, v8);
        red(eb[27 + mm], eb[57 + mm], cv9, v9);
      }
    }
  }
}

// Three-field element (one pressure P and one volume theta per element,
// quadratic tets, hyperelastic and J2 models): the local update after a displacement
// increment du (compute_d_theta_dP, src/constitutive_model_3f.cc:494-549, with
// the blocks at u; thread per element): with W = sum_q w, fp = sum_q w J -
// theta W and Kpu du = sum_q w J tr(Grad(du) F^-1),
//   d_theta = (Kpu du + fp) / W,  dP = kappa U'(theta) - P + kappa U''(theta) d_theta.
// An element with an inverted point gets zero increments and is counted.
__global__ void k_tf_update(const QpArgs A, const double *dunode, double *dP, double *dtheta) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= A.ne) return;
  double W = 0.0, SJ = 0.0, Kdu = 0.0;
  bool ok = true;
  for (int q = 0; q < 4 && ok; q++) {
    double dX[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, dU[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0},
           dD[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = 0; b < 10; b++) {
      const int n = A.conn[(long)b * A.ne + e];
      const double g0 = A.shp.dNxi[q][b][0], g1 = A.shp.dNxi[q][b][1], g2 = A.shp.dNxi[q][b][2];
      for (int i = 0; i < 3; i++) {
        const double x = A.X[i * A.nn + n], u = A.unode[i * A.nn + n], d = dunode[i * A.nn + n];
        dX[i * 3 + 0] += g0 * x;
        dX[i * 3 + 1] += g1 * x;
        dX[i * 3 + 2] += g2 * x;
        dU[i * 3 + 0] += g0 * u;
        dU[i * 3 + 1] += g1 * u;
        dU[i * 3 + 2] += g2 * u;
        dD[i * 3 + 0] += g0 * d;
        dD[i * 3 + 1] += g1 * d;
        dD[i * 3 + 2] += g2 * d;
      }
    }
    const double detJ = det3(dX);
    double dXi[9], F[9], Fi[9], L[9];
    ok = detJ > 0.0 && inv3(dX, dXi);
    if (!ok) break;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        F[i * 3 + j] = (i == j ? 1.0 : 0.0) + dU[i * 3 + 0] * dXi[0 * 3 + j] + dU[i * 3 + 1] * dXi[1 * 3 + j] +
                       dU[i * 3 + 2] * dXi[2 * 3 + j];
        L[i * 3 + j] = dD[i * 3 + 0] * dXi[0 * 3 + j] + dD[i * 3 + 1] * dXi[1 * 3 + j] + dD[i * 3 + 2] * dXi[2 * 3 + j];
      }
    if (A.F0)
      for (int i = 0; i < 9; i++) F[i] += A.F0[i];
    const double J = det3(F);
    ok = J > 0.0 && inv3(F, Fi);
    if (!ok) break;
    const double w = detJ * A.shp.w[q];
    double tr = 0.0;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) tr += L[i * 3 + j] * Fi[j * 3 + i];
    W += w;
    SJ += w * J;
    Kdu += w * J * tr;
  }
  if (!ok) {
    atomicAdd(&A.status[0], 1ull);
    dP[e] = dtheta[e] = 0.0;
    return;
  }
  const double th = A.tf_theta[e], P = A.tf_P[e];
  double dUv, d2U;
  vol_derivs(A.mat.vol_pot, th, dUv, d2U);
  const double dth = (Kdu + SJ - th * W) / W;
  dtheta[e] = dth;
  dP[e] = A.mat.kappa * dUv - P + A.mat.kappa * d2U * dth;
}

// The three-field element in the transient (quadratic tets, hyperelastic):
// the corrections that turn the two condensed quasi-static assemblies at the
// mid points into the reference's transient condensation
// (residuals_el_constitutive_model_w_inertia_3f, src/constitutive_model.cc:
// 2960-3229).  With the blocks of the newer mid point a scaled by
// kK = -dt_np1 alpha (1 - alpha) and the residuals combined as
// R_x = cA R_x(a) + cB R_x(b), the condensed residual is
//   f = cA (fu_a + s_a Kup_a) + cB (fu_b + s_b Kup_b) - cB s_b Kup_b + d Kup_a,
//   d = cB (c_a fp_b + kappa U'(theta_b) - P_b),
// c = kappa U''(theta) / W, fp = sum w J - theta W, s = c fp + kappa U'(theta) - P
// (the first two terms are the condensed assemblies at a and at b): this
// kernel adds d Kup_a - cB s_b Kup_b into R.  With dunode set it instead
// forms the local update (compute_d_theta_dP with the combined blocks,
// :3880-3898): d_theta = (kK Kup_a du + Rp) / (kK W),
// dP = (Rt + kK W kappa U''(theta_a) d_theta) / (kK W).
struct TfTrArgs {
  QpArgs A;               // X, conn, shp, mat, status; unode = u_{n+alpha}
  const double *unode_b;  // u_{n-1+alpha} at the nodes (SoA 3*nn)
  const double *mid;      // 4*ne: P_a, theta_a, P_b, theta_b
  const int *dof;         // 3*nn SoA, 1-based free DOF ids
  double *R;
  const double *dunode;   // update mode: du at the nodes
  double *dP, *dtheta;
  double cA, cB, kK;
};

__global__ void k_tf_transient(const TfTrArgs T) {
  const QpArgs &A = T.A;
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= A.ne) return;
  const bool upd = T.dunode != nullptr;
  int nd[10];
  for (int b = 0; b < 10; b++) nd[b] = A.conn[(long)b * A.ne + e];
  // point q: reference gradient inverse, w, and F, F^-1, J at both mid points
  auto point = [&](int q, double *dXi, double &w, double *Fa, double *Fia, double &Ja, double *Fb, double *Fib,
                   double &Jb, double *Ld) -> bool {
    double dX[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, da[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0},
           db[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, dd[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = 0; b < 10; b++) {
      const int n = nd[b];
      const double g[3] = {A.shp.dNxi[q][b][0], A.shp.dNxi[q][b][1], A.shp.dNxi[q][b][2]};
      for (int i = 0; i < 3; i++) {
        const double x = A.X[i * A.nn + n], ua = A.unode[i * A.nn + n], ub = T.unode_b[i * A.nn + n];
        const double d = upd ? T.dunode[i * A.nn + n] : 0.0;
        for (int c = 0; c < 3; c++) {
          dX[i * 3 + c] += g[c] * x;
          da[i * 3 + c] += g[c] * ua;
          db[i * 3 + c] += g[c] * ub;
          dd[i * 3 + c] += g[c] * d;
        }
      }
    }
    const double detJ = det3(dX);
    if (!(detJ > 0.0) || !inv3(dX, dXi)) return false;
    w = detJ * A.shp.w[q];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        double fa = (i == j ? 1.0 : 0.0), fb = fa, l = 0.0;
        for (int c = 0; c < 3; c++) {
          fa += da[i * 3 + c] * dXi[c * 3 + j];
          fb += db[i * 3 + c] * dXi[c * 3 + j];
          l += dd[i * 3 + c] * dXi[c * 3 + j];
        }
        Fa[i * 3 + j] = fa;
        Fb[i * 3 + j] = fb;
        Ld[i * 3 + j] = l;
      }
    Ja = det3(Fa);
    Jb = det3(Fb);
    return Ja > 0.0 && Jb > 0.0 && inv3(Fa, Fia) && inv3(Fb, Fib);
  };
  double W = 0.0, SJa = 0.0, SJb = 0.0, Kdu = 0.0;
  bool ok = true;
  for (int q = 0; q < 4 && ok; q++) {
    double dXi[9], w, Fa[9], Fia[9], Ja, Fb[9], Fib[9], Jb, Ld[9];
    ok = point(q, dXi, w, Fa, Fia, Ja, Fb, Fib, Jb, Ld);
    if (!ok) break;
    W += w;
    SJa += w * Ja;
    SJb += w * Jb;
    if (upd) {
      double tr = 0.0;
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) tr += Ld[i * 3 + j] * Fia[j * 3 + i];
      Kdu += w * Ja * tr;
    }
  }
  if (!ok) {
    atomicAdd(&A.status[0], 1ull);
    if (upd) T.dP[e] = T.dtheta[e] = 0.0;
    return;
  }
  const double Pa = T.mid[e], tha = T.mid[A.ne + e], Pb = T.mid[2 * A.ne + e], thb = T.mid[3 * A.ne + e];
  const double kap = A.mat.kappa;
  double dUa, d2Ua, dUb, d2Ub;
  vol_derivs(A.mat.vol_pot, tha, dUa, d2Ua);
  vol_derivs(A.mat.vol_pot, thb, dUb, d2Ub);
  if (upd) {
    const double Rp = T.cA * (SJa - tha * W) + T.cB * (SJb - thb * W);
    const double Rt = W * (T.cA * (kap * dUa - Pa) + T.cB * (kap * dUb - Pb));
    const double dth = (T.kK * Kdu + Rp) / (T.kK * W);
    T.dtheta[e] = dth;
    T.dP[e] = (Rt + T.kK * W * kap * d2Ua * dth) / (T.kK * W);
    return;
  }
  const double ca = kap * d2Ua / W, cb = kap * d2Ub / W, fpb = SJb - thb * W;
  const double sb = cb * fpb + kap * dUb - Pb;
  const double da_ = T.cB * (ca * fpb + kap * dUb - Pb), db_ = -T.cB * sb;
  double out[10][3];
  for (int b = 0; b < 10; b++) out[b][0] = out[b][1] = out[b][2] = 0.0;
  for (int q = 0; q < 4; q++) {
    double dXi[9], w, Fa[9], Fia[9], Ja, Fb[9], Fib[9], Jb, Ld[9];
    point(q, dXi, w, Fa, Fia, Ja, Fb, Fib, Jb, Ld);
    for (int b = 0; b < 10; b++) {
      double gX[3];  // dN_b / dX
      for (int j = 0; j < 3; j++)
        gX[j] = A.shp.dNxi[q][b][0] * dXi[0 * 3 + j] + A.shp.dNxi[q][b][1] * dXi[1 * 3 + j] +
                A.shp.dNxi[q][b][2] * dXi[2 * 3 + j];
      for (int k = 0; k < 3; k++) {
        const double ta = gX[0] * Fia[0 * 3 + k] + gX[1] * Fia[1 * 3 + k] + gX[2] * Fia[2 * 3 + k];
        const double tb = gX[0] * Fib[0 * 3 + k] + gX[1] * Fib[1 * 3 + k] + gX[2] * Fib[2 * 3 + k];
        out[b][k] += w * (da_ * Ja * ta + db_ * Jb * tb);
      }
    }
  }
  for (int b = 0; b < 10; b++)
    for (int k = 0; k < 3; k++) {
      const int id = T.dof[k * A.nn + nd[b]];
      if (id > 0) atomicAdd(T.R + (id - 1), out[b][k]);
    }
}

// Residual of the condensed three-field element from its point records alone
// (quadratic tets; the residual rows of k_assemble_p2m without its stiffness):
// R_bi = sum_q sum_j (w tau_ij + w J s delta_ij) p_qb,j with p_qb = G_q^T dN_b/dxi,
// s = c (sum w J - theta W) + kappa U'(theta) - P, c = kappa U''(theta) / W;
// w tau = record fields 9..14 minus the geometric term h on the diagonal.
// One thread per record slot (element perm[es]); inverted elements have zeroed
// records (W = 0) and are skipped, as the assembly skips them.
__global__ void k_tf_residual(const QpArgs A, const int *dof, double *R) {
  constexpr int NRF = kYRecTF;
  const long es = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (es >= A.ne) return;
  const long e = A.perm ? (long)A.perm[es] : es;
  const double *rec = A.qrec;
  double W = 0.0, SJ = 0.0;
  for (int q = 0; q < 4; q++) {
    SJ += rec[yrec_idx<NRF>(es * 4 + q, 26)];
    W += rec[yrec_idx<NRF>(es * 4 + q, 27)];
  }
  if (!(W > 0.0)) return;
  const double th = rec[yrec_idx<NRF>(es * 4, 28)], Pe = rec[yrec_idx<NRF>(es * 4, 29)];
  double dU, d2U;
  vol_derivs(A.mat.vol_pot, th, dU, d2U);
  const double c = A.mat.kappa * d2U / W;
  const double sc = c * (SJ - th * W) + A.mat.kappa * dU - Pe;
  double out[10][3];
  for (int b = 0; b < 10; b++) out[b][0] = out[b][1] = out[b][2] = 0.0;
  for (int q = 0; q < 4; q++) {
    const long qs = es * 4 + q;
    double G[9], T[3][3];
    for (int k = 0; k < 9; k++) G[k] = rec[yrec_idx<NRF>(qs, k)];
    const double h = rec[yrec_idx<NRF>(qs, 25)], wJs = rec[yrec_idx<NRF>(qs, 26)] * sc;
    double wt[6];
    for (int k = 0; k < 6; k++) wt[k] = rec[yrec_idx<NRF>(qs, 9 + k)] - (k < 3 ? h : 0.0);
    // Voigt order xx yy zz yz xz xy
    T[0][0] = wt[0] + wJs; T[1][1] = wt[1] + wJs; T[2][2] = wt[2] + wJs;
    T[1][2] = T[2][1] = wt[3];
    T[0][2] = T[2][0] = wt[4];
    T[0][1] = T[1][0] = wt[5];
    for (int b = 0; b < 10; b++) {
      const double g0 = A.shp.dNxi[q][b][0], g1 = A.shp.dNxi[q][b][1], g2 = A.shp.dNxi[q][b][2];
      double p[3];
      for (int j = 0; j < 3; j++) p[j] = G[j] * g0 + G[3 + j] * g1 + G[6 + j] * g2;
      for (int i = 0; i < 3; i++) out[b][i] += T[i][0] * p[0] + T[i][1] * p[1] + T[i][2] * p[2];
    }
  }
  for (int b = 0; b < 10; b++) {
    const int n = A.conn[(long)b * A.ne + e];
    for (int i = 0; i < 3; i++) {
      const int id = dof[i * A.nn + n];
      if (id > 0) atomicAdd(R + (id - 1), out[b][i]);
    }
  }
}

}  // namespace pgb
