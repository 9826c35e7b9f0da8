// assemble.cuh -- fused FP64 R+K element-assembly kernel.
//
// One pass does what fd_residuals_MP + stiffmat_fd_MP do for the
// constitutive-model element (src/fd_residuals.cc:468-636,
// src/stiffmat_fd.cc:831-993): element gather, F per quadrature point, the
// constitutive update (run_integration_algorithm, src/constitutive_model.cc:
// 1100-1129) with the state written at t_{n+1}, the element residual
// (compute_residual_vector, :1628-1662) and tangent (compute_stiffness_matrix,
// :1520-1616) and their scatter into R and the CSR values (fd_res_assemble,
// src/fd_residuals.cc:58-73; PLoc_Sparse, src/PLoc_Sparse.cc:15-175).
//
// The element integrals are evaluated in the algebraically identical spatial
// B-matrix form (M = I, dM/du = 0 for HE and J2):
//   R_ai   = w (tau p_a)_i,                 p_a = F^-T grad_X N_a
//   K_aibk = w [ p_a,j c_ijkl p_b,l + (p_a . tau p_b) d_ik ]
// with w = det(dX/dxi) * weight.
//
// Thread mapping: a CTA holds TE elements and TE*NNE threads.  Phase 0: node
// threads stage X and u of their node in shared memory.  Phase 1: one thread
// per quadrature point computes the isoparametric Jacobian, F, the
// constitutive update and the per-point tangent record.  Phase 2: node
// threads form their node's spatial vectors per point and scatter R.
// Phase 3: node thread a forms the 3x3 blocks K_ab for b = 0..NNE-1, summed
// over the points, and scatters them through the element->CSR node-block map.
//
// MODEL: 0 HE (neo-Hookean), 1 J2, 3 HE with the linear deviatoric potential,
// whose tangent adds w G [b_ik (p_a . b p_b) + (b p_b)_i (b p_a)_k] to K_ab
// (b = F F^T in the record's n slot, b p_a in the vector record's n p slot).
#pragma once
#include <cstdint>

#include "cm_models.cuh"

namespace pgb {

constexpr int kRec = 38;  // doubles per quadrature-point record
constexpr int kVec = 15;  // doubles per (point, node) vector record

struct ShapeTable {
  double dNxi[4][10][3];  // dN/dxi at the quadrature points
  double w[4];            // quadrature weights
  double N[4][10];        // shape functions at the quadrature points
};

struct AsmArgs {
  // mesh (SoA)
  const double *X;       // 3*nn
  const int *conn;       // NNE*ne  (conn[a*ne + e])
  const int *dof;        // 3*nn    (reference id convention)
  const int *rowptr0;    // nn: CSR offset of the node's first free row, -1 if none
  const int *rowlen;     // nn: length of the node's rows
  const uint8_t *mask;   // nn: bit c set when component c is free
  const uint16_t *pos;   // ne*NNE*NNE: column position of node b's block in node a's rows
  long nn, ne;
  // displacement expanded per node (SoA, 3*nn)
  const double *unode;
  const double *F0;      // 9 or nullptr
  // state SoA [comp][nqp]
  const double *state_n;
  double *state_np1;
  long nqp;
  // outputs
  double *R;             // ndof
  double *K;             // nnz
  unsigned long long *status;  // [4]
  // element list (colour mode, element-level calls) or nullptr for 0..ne-1
  const int *elist;
  long nlist;
  // dense element outputs (element-level entry points): lk[nlist][nd][nd], fe[nlist][nd]
  double *lk_out;
  double *fe_out;
  // batches of independent meshes (FE2 micro-structures): element -> group,
  // group -> macro deformation F0 (9); nullptr = the single F0 above
  const int *elem_group;
  const double *F0_tab;
  // work stealing: tiles are claimed `grab` at a time from *ticket (zeroed
  // before the launch); nullptr = static grid-stride order
  unsigned *ticket;
  int grab;
  // point records written by the point-update kernel (kRec x nqp, structure
  // of arrays), read by the two-kernel quadratic-tet assembly
  const double *qrec;
  // per-element scatter blocks of the tensor-core quadratic-tet kernel
  // (kEBW int32 words per element: row bases, residual indices, node-pair
  // positions, free masks)
  const int *eblk;
  // bound of the pipelined kernels' hand-off waits (ns), and the failure-path
  // test switch: the producer withholds its first hand-off
  unsigned long long wait_ns;
  int stall;
  Mat mat;
  ShapeTable shp;
};

template <int NNE>
struct Tile;
template <>
struct Tile<4> {
  static constexpr int TE = 32;
};
template <>
struct Tile<10> {
  static constexpr int TE = 12;
};

__device__ __forceinline__ int rank_of(unsigned mask, int c) {
  return __popc(mask & ((1u << c) - 1u));
}

template <bool ATOMIC>
__device__ __forceinline__ void add_to(double *p, double v) {
  if (ATOMIC)
    atomicAdd(p, v);
  else
    *p += v;
}

template <int NNE, int NQP, int MODEL, bool ATOMIC, bool WANT_K, bool DENSE, int TEP = Tile<NNE>::TE>
__global__ void __launch_bounds__(TEP *NNE)
    k_assemble(const AsmArgs args) {
  constexpr int TE = TEP;
  constexpr bool PLASTIC = (MODEL == 1);
  extern __shared__ double smem[];
  double *sXU = smem;                             // [TE][NNE][6]
  double *sRec = sXU + TE * NNE * 6;              // [TE][NQP][kRec]
  double *sVec = sRec + TE * NQP * kRec;          // [TE][NQP][NNE][kVec]
  // per (element, node) metadata staged once per tile, so that the block and
  // scatter phases issue no dependent global loads
  int *sMeta = reinterpret_cast<int *>(sVec + TE * NQP * NNE * kVec);  // [TE*NNE][6]: mask, rp, rl, dof x3
  uint16_t *sPos = reinterpret_cast<uint16_t *>(sMeta + TE * NNE * 6);  // [TE*NNE][NNE]

  const long ntot = args.elist ? args.nlist : args.ne;
  const int tid = threadIdx.x;
  __shared__ long s_claim;
  long claim_end = 0;  // work stealing: end of the current claim of tiles
  long tile0 = (long)blockIdx.x * TE;
  if (args.ticket) {
    if (tid == 0) s_claim = (long)atomicAdd(args.ticket, (unsigned)args.grab) * TE;
    __syncthreads();
    tile0 = s_claim;
    claim_end = tile0 + (long)args.grab * TE;
    __syncthreads();
  }
  while (tile0 < ntot) {
    // ---------------- phase 0: stage node data ----------------
    const int el = tid / NNE, a = tid % NNE;
    const long ei = tile0 + el;
    const bool valid = ei < ntot;
    const long e = valid ? (args.elist ? (long)args.elist[ei] : ei) : 0;
    int node = -1;
    if (valid) {
      node = args.conn[(long)a * args.ne + e];
      double *d = sXU + (el * NNE + a) * 6;
      d[0] = args.X[node];
      d[1] = args.X[args.nn + node];
      d[2] = args.X[2 * args.nn + node];
      d[3] = args.unode[node];
      d[4] = args.unode[args.nn + node];
      d[5] = args.unode[2 * args.nn + node];
      int *m = sMeta + (el * NNE + a) * 6;
      if (DENSE) {
        m[0] = 7;
      } else {
        m[0] = args.mask[node];
        m[1] = args.rowptr0[node];
        m[2] = args.rowlen[node];
        m[3] = args.dof[node];
        m[4] = args.dof[args.nn + node];
        m[5] = args.dof[2 * args.nn + node];
        const uint16_t *pr = args.pos + (e * NNE + a) * NNE;
        uint16_t *sp = sPos + (el * NNE + a) * NNE;
#pragma unroll
        for (int b = 0; b < NNE; b++) sp[b] = pr[b];
      }
    }
    __syncthreads();

    // ---------------- phase 1: quadrature-point work ----------------
    if (tid < TE * NQP) {
      const int qe = tid / NQP, q = tid % NQP;
      const long qei = tile0 + qe;
      if (qei < ntot) {
        const long qel = args.elist ? (long)args.elist[qei] : qei;
        const double *xu = sXU + qe * NNE * 6;
        double dX[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, dU[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int b = 0; b < NNE; b++) {
          const double g0 = args.shp.dNxi[q][b][0], g1 = args.shp.dNxi[q][b][1],
                       g2 = args.shp.dNxi[q][b][2];
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
        double *rec = sRec + (qe * NQP + q) * kRec;
        const double detJ = det3(dX);
        double dXi[9];
        bool ok = detJ > 0.0 && inv3(dX, dXi);
        double F[9];
        if (ok) {
          // F = I + dU dXi   (dU_ic = sum_a u_a,i dN_a/dxi_c)
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
              F[i * 3 + j] = (i == j ? 1.0 : 0.0) + dU[i * 3 + 0] * dXi[0 * 3 + j] +
                             dU[i * 3 + 1] * dXi[1 * 3 + j] + dU[i * 3 + 2] * dXi[2 * 3 + j];
          const double *F0 = args.elem_group ? args.F0_tab + 9 * (long)args.elem_group[qel] : args.F0;
          if (F0)
#pragma unroll
            for (int i = 0; i < 9; i++) F[i] += F0[i];
        }
        const double J = ok ? det3(F) : -1.0;
        double Fi[9];
        if (ok) ok = J > 0.0 && inv3(F, Fi);
        if (!ok) {
          atomicAdd(&args.status[0], 1ull);
#pragma unroll
          for (int i = 0; i < kRec; i++) rec[i] = 0.0;
        } else {
          const long qp = qel * NQP + q;
          double A[6] = {1, 1, 1, 0, 0, 0}, alpha = 0.0;
          if (PLASTIC) {
#pragma unroll
            for (int c = 0; c < 6; c++) A[c] = args.state_n[c * args.nqp + qp];
            alpha = args.state_n[6 * args.nqp + qp];
          }
          QpTangent t;
          double Anp1[6], alpha_np1;
          if (MODEL == 3)
            linear_dev_update(args.mat, F, J, t);
          else
            spatial_update<PLASTIC>(args.mat, F, J, A, alpha, t, Anp1, &alpha_np1);
          if (PLASTIC && args.state_np1) {
#pragma unroll
            for (int c = 0; c < 6; c++) args.state_np1[c * args.nqp + qp] = Anp1[c];
            args.state_np1[6 * args.nqp + qp] = alpha_np1;
          }
          // G = dXi Fi: p_a = G^T dN_a/dxi
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
              rec[i * 3 + j] = dXi[i * 3 + 0] * Fi[0 * 3 + j] + dXi[i * 3 + 1] * Fi[1 * 3 + j] +
                               dXi[i * 3 + 2] * Fi[2 * 3 + j];
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
      }
    }
    __syncthreads();

    // ---------------- phase 2: node vectors + residual ----------------
    unsigned maskA = 0;
    if (valid) {
      double Ra[3] = {0, 0, 0};
#pragma unroll
      for (int q = 0; q < NQP; q++) {
        const double *rec = sRec + (el * NQP + q) * kRec;
        const double g0 = args.shp.dNxi[q][a][0], g1 = args.shp.dNxi[q][a][1],
                     g2 = args.shp.dNxi[q][a][2];
        double p[3];
#pragma unroll
        for (int j = 0; j < 3; j++) p[j] = rec[0 * 3 + j] * g0 + rec[1 * 3 + j] * g1 + rec[2 * 3 + j] * g2;
        double *v = sVec + ((el * NQP + q) * NNE + a) * kVec;
        double sp[3], tp[3];
        smv(rec + 16, p, sp);
        smv(rec + 10, p, tp);
        v[0] = p[0];
        v[1] = p[1];
        v[2] = p[2];
        v[3] = sp[0];
        v[4] = sp[1];
        v[5] = sp[2];
        if (MODEL == 3) {
          double bp[3];
          smv(rec + 22, p, bp);
          v[6] = bp[0];
          v[7] = bp[1];
          v[8] = bp[2];
        }
        if (PLASTIC) {
          double np_[3], Dp[3];
          smv(rec + 22, p, np_);
          smv(rec + 28, p, Dp);
          v[6] = np_[0];
          v[7] = np_[1];
          v[8] = np_[2];
          v[9] = Dp[0];
          v[10] = Dp[1];
          v[11] = Dp[2];
        }
        v[12] = tp[0];
        v[13] = tp[1];
        v[14] = tp[2];
        const double w = rec[9];
        Ra[0] += w * tp[0];
        Ra[1] += w * tp[1];
        Ra[2] += w * tp[2];
      }
      if (DENSE) {
#pragma unroll
        for (int i = 0; i < 3; i++) args.fe_out[ei * (NNE * 3) + a * 3 + i] = Ra[i];
        maskA = 7u;
      } else {
        const int *m = sMeta + (el * NNE + a) * 6;
#pragma unroll
        for (int i = 0; i < 3; i++) {
          const int id = m[3 + i];
          if (id > 0) add_to<ATOMIC>(&args.R[id - 1], Ra[i]);
        }
        maskA = (unsigned)m[0];
      }
    }
    __syncthreads();

    // ---------------- phase 3: stiffness blocks + CSR scatter ----------------
    if (WANT_K && valid && maskA) {
      const int *mA = sMeta + (el * NNE + a) * 6;
      const long rp = DENSE ? 0 : mA[1];
      const long rl = DENSE ? 0 : mA[2];
      const uint16_t *posrow = sPos + (el * NNE + a) * NNE;
      for (int b = 0; b < NNE; b++) {
        const unsigned maskB = DENSE ? 7u : (unsigned)sMeta[(el * NNE + b) * 6];
        if (!maskB) continue;
        double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int q = 0; q < NQP; q++) {
          const double *rec = sRec + (el * NQP + q) * kRec;
          const double *va = sVec + ((el * NQP + q) * NNE + a) * kVec;
          const double *vb = sVec + ((el * NQP + q) * NNE + b) * kVec;
          const double w = rec[9];
          const double a1h = 0.5 * rec[34] * w, a2 = rec[35] * w;
          const double pa[3] = {va[0], va[1], va[2]}, spa[3] = {va[3], va[4], va[5]};
          const double pb[3] = {vb[0], vb[1], vb[2]}, spb[3] = {vb[3], vb[4], vb[5]};
          const double tpb[3] = {vb[12], vb[13], vb[14]};
          const double pr = pa[0] * pb[0] + pa[1] * pb[1] + pa[2] * pb[2];
          const double ptr = pa[0] * tpb[0] + pa[1] * tpb[1] + pa[2] * tpb[2];
          const double dg = a1h * pr + w * ptr;
          const double c23 = (2.0 / 3.0) * w;
          // x2 = a2 p_a - 2/3 sp_a,  x3 = -2/3 p_a
          double x2[3], x3[3], x1[3];
#pragma unroll
          for (int i = 0; i < 3; i++) {
            x1[i] = a1h * pa[i];
            x2[i] = a2 * pa[i] - c23 * spa[i];
            x3[i] = -c23 * pa[i];
          }
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int k = 0; k < 3; k++)
              acc[i * 3 + k] += pb[i] * x1[k] + x2[i] * pb[k] + x3[i] * spb[k];
          acc[0] += dg;
          acc[4] += dg;
          acc[8] += dg;
          if (PLASTIC) {
            const double a4 = rec[36] * w, a5 = rec[37] * w;
            const double npa[3] = {va[6], va[7], va[8]};
            const double npb[3] = {vb[6], vb[7], vb[8]}, Dpb[3] = {vb[9], vb[10], vb[11]};
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
              for (int k = 0; k < 3; k++) acc[i * 3 + k] += npa[i] * (a4 * npb[k] + a5 * Dpb[k]);
          }
          if (MODEL == 3) {
            const double wG = w * args.mat.mu;
            const double *b = rec + 22;  // Voigt xx yy zz yz xz xy
            const double bpa[3] = {va[6], va[7], va[8]}, bpb[3] = {vb[6], vb[7], vb[8]};
            const double pbb = wG * (pa[0] * bpb[0] + pa[1] * bpb[1] + pa[2] * bpb[2]);
            const double bf[9] = {b[0], b[5], b[4], b[5], b[1], b[3], b[4], b[3], b[2]};
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
              for (int k = 0; k < 3; k++) acc[i * 3 + k] += bf[i * 3 + k] * pbb + wG * bpb[i] * bpa[k];
          }
        }
        if (DENSE) {
          double *lk = args.lk_out + ei * (NNE * 3) * (NNE * 3);
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int k = 0; k < 3; k++) lk[(a * 3 + i) * (NNE * 3) + b * 3 + k] = acc[i * 3 + k];
          continue;
        }
        const long base = rp + posrow[b];
#pragma unroll
        for (int i = 0; i < 3; i++) {
          if (!(maskA >> i & 1u)) continue;
          const long rowoff = base + (long)rank_of(maskA, i) * rl;
#pragma unroll
          for (int k = 0; k < 3; k++) {
            if (!(maskB >> k & 1u)) continue;
            add_to<ATOMIC>(&args.K[rowoff + rank_of(maskB, k)], acc[i * 3 + k]);
          }
        }
      }
    }
    __syncthreads();
    // next tile: the rest of this claim, then a new claim
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

template <int NNE, int NQP, int TEP = Tile<NNE>::TE>
constexpr size_t asm_smem_bytes() {
  return sizeof(double) * (size_t)TEP * (NNE * 6 + NQP * kRec + NQP * NNE * kVec) +
         (size_t)TEP * NNE * (6 * sizeof(int) + NNE * sizeof(uint16_t));
}

}  // namespace pgb
