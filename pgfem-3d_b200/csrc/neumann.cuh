// neumann.cuh -- surface loads (Neumann boundary conditions) on element faces.
//
// The quasi-static terms that the reference adds at the end of each element's
// residual and stiffness routines: compute_Neumann_boundary_conditions
// (src/fd_residuals.cc:123-273) and
// compute_Neumann_boundary_conditions_stiffnes_mat (src/stiffmat_fd.cc:
// 359-500), with the boundary FEMLIB of FEMLIB/src/femlib.cc (face node lists
// Tet2Tri / QTet2QTri :85-86, volume-coordinate maps kez_map_Tet :97-100 and
// set_tet2tri :796-815, triangle rules :619-635, elem_basis_S :1578-1612,
// PGFem3D_dNdX_Vol2Bnd :486-541).
//
// Per face point (1 on a linear face, 3 on a quadratic one: the boundary takes
// the volume element's integration order, raised to 1 for quadratic tets):
// volume N and dN/dX at the point's volume coordinates, the face Jacobian
// |dX/dxi_1 x dX/dxi_2| and unit normal n from the face's own basis, F = I +
// sum u_a (x) dN_a/dX, J = det F.  Then, for face node a (volume node V2B[a]):
//   R[a,i]     += -N_a w J (F^-T PN)_i,          PN = p n or the traction t
//   K[a,d;c,d] += -N_a w J 2 g_d (F^-T PN')_d,   g_m = sum_l F^-1_lm dN_c/dX_l
// The stiffness keeps the reference's form: only component-diagonal entries,
// the shape tensor of volume node c (the face-local index), and for a pressure
// PN' = (p n_0, 0, p n_2) (src/stiffmat_fd.cc:419-445); on face 3 the points
// lie on the plane zet = 0 as the reference's table puts them.
//
// One thread per face (global assembly, FP64 atomics into R and the CSR
// values through the element's node-block map) or per listed element
// (element-level calls: dense blocks, no atomics).  Faces are few next to the
// volume elements (a surface against a volume), so this is a short kernel that
// runs after the element kernel on the same stream.
#pragma once
#include <cstdint>

namespace pgb {

// Per-feature load descriptor: PN = c n + t (residual), PN'_i = c'_i n_i + t'_i
// (stiffness), stored as (c, t[3], c'[3], t'[3]).
constexpr int kNbcDesc = 10;

// The load values as the reference reads them: the first `type` values, and
// for a pressure (type 1) value 0 copied to component 2 (component 1 stays 0),
// src/fd_residuals.cc:199-203.
inline void nbc_raw(int type, const double *L, double *P) {
  P[0] = P[1] = P[2] = 0.0;
  for (int i = 0; i < type && i < 3; i++) P[i] = L[i];
  if (type == 1) P[2] = P[0];
}

// Quasi-static: pressure PN = p n, PN' = (p n_0, 0, p n_2); traction PN = PN' = t.
inline void nbc_desc_static(int type, const double *L, double *d) {
  double P[3];
  nbc_raw(type, L, P);
  for (int i = 0; i < kNbcDesc; i++) d[i] = 0.0;
  if (type == 1) {
    d[0] = P[0];
    for (int i = 0; i < 3; i++) d[4 + i] = P[i];
  } else {
    for (int i = 0; i < 3; i++) d[1 + i] = d[7 + i] = P[i];
  }
}

// A mid point of the transient element (older values Lo, newer Ln):
// PN = (1 - a) PN_o + a P_n, PN' = (1 - a) PN'_o + a P_n, the newer value taken
// raw as the reference does (src/fd_residuals.cc:238-239, src/stiffmat_fd.cc:465).
inline void nbc_desc_mid(int type, const double *Lo, const double *Ln, double a, double *d) {
  double Po[3], Pn[3];
  nbc_raw(type, Lo, Po);
  nbc_raw(type, Ln, Pn);
  for (int i = 0; i < kNbcDesc; i++) d[i] = 0.0;
  if (type == 1) {
    d[0] = (1.0 - a) * Po[0];
    for (int i = 0; i < 3; i++) {
      d[1 + i] = d[7 + i] = a * Pn[i];
      d[4 + i] = (1.0 - a) * Po[i];
    }
  } else {
    for (int i = 0; i < 3; i++) d[1 + i] = d[7 + i] = (1.0 - a) * Po[i] + a * Pn[i];
  }
}

struct NbcArgs {
  const double *X;         // 3*nn SoA
  const int *conn;         // NNE*ne  (conn[a*ne + e])
  const int *dof;          // 3*nn SoA, reference id convention
  const int *rowptr0;      // nn
  const int *rowlen;       // nn
  const uint8_t *mask;     // nn
  const uint16_t *pos;     // ne*NNE*NNE
  long nn, ne;
  const double *unode;     // 3*nn SoA
  long nface;
  const int *face_elem;    // nface, sorted by element
  const uint8_t *face_id;  // nface: local face 0..3
  const int *face_feat;    // nface: feature (load) index
  // kNbcDesc doubles per feature: the load of the residual PN = c n + t and
  // of the stiffness PN'_i = c'_i n_i + t'_i, as (c, t[3], c'[3], t'[3])
  const double *feat_desc;
  const int *elem_face_off;  // ne+1: faces of element e (element-level calls)
  double *R;               // ndof or nullptr
  double *K;               // nnz or nullptr
  // element-level calls: listed elements and their dense outputs
  const int *elist;
  long nlist;
  double *lk_out;          // nlist*(3NNE)^2 or nullptr
  double *fe_out;          // nlist*3NNE
};

__constant__ int c_tet2tri[4][3] = {{0, 2, 1}, {0, 1, 3}, {1, 2, 3}, {0, 3, 2}};
__constant__ int c_qtet2qtri[4][6] = {{0, 2, 1, 6, 5, 4}, {0, 1, 3, 4, 8, 7}, {1, 2, 3, 5, 9, 8}, {0, 3, 2, 7, 9, 6}};
__constant__ int c_kezmap[4][3] = {{1, 0, 2}, {0, 2, 1}, {0, 1, 2}, {0, 1, 2}};

template <int NNE>
__device__ __forceinline__ void nbc_shape(double k, double e, double z, double *N, double (*dk)[3]) {
  const double l0 = 1.0 - k - e - z;
  if (NNE == 4) {
    N[0] = l0, N[1] = k, N[2] = e, N[3] = z;
    const double t[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int i = 0; i < 3; i++) dk[a][i] = t[a][i];
    return;
  }
  N[0] = (2.0 * l0 - 1.0) * l0;
  N[1] = (2.0 * k - 1.0) * k;
  N[2] = (2.0 * e - 1.0) * e;
  N[3] = (2.0 * z - 1.0) * z;
  N[4] = 4.0 * l0 * k;
  N[5] = 4.0 * k * e;
  N[6] = 4.0 * l0 * e;
  N[7] = 4.0 * l0 * z;
  N[8] = 4.0 * k * z;
  N[9] = 4.0 * e * z;
  const double s = 4.0 * (k + e + z) - 3.0;
  const double d[10][3] = {{s, s, s},
                           {4.0 * k - 1.0, 0.0, 0.0},
                           {0.0, 4.0 * e - 1.0, 0.0},
                           {0.0, 0.0, 4.0 * z - 1.0},
                           {4.0 * (1.0 - 2.0 * k - e - z), -4.0 * k, -4.0 * k},
                           {4.0 * e, 4.0 * k, 0.0},
                           {-4.0 * e, 4.0 * (1.0 - k - 2.0 * e - z), -4.0 * e},
                           {-4.0 * z, -4.0 * z, 4.0 * (1.0 - k - e - 2.0 * z)},
                           {4.0 * z, 0.0, 4.0 * k},
                           {0.0, 4.0 * z, 4.0 * e}};
#pragma unroll
  for (int a = 0; a < 10; a++)
#pragma unroll
    for (int i = 0; i < 3; i++) dk[a][i] = d[a][i];
}

// Face basis derivatives: TRIANGLE (3 nodes) or QTRIANGLE (6).
template <int NB>
__device__ __forceinline__ void nbc_face_dN(double k, double e, double (*d)[2]) {
  if (NB == 3) {
    d[0][0] = -1.0, d[0][1] = -1.0, d[1][0] = 1.0, d[1][1] = 0.0, d[2][0] = 0.0, d[2][1] = 1.0;
    return;
  }
  d[0][0] = 4.0 * e + 4.0 * k - 3.0, d[0][1] = 4.0 * e + 4.0 * k - 3.0;
  d[1][0] = 4.0 * k - 1.0, d[1][1] = 0.0;
  d[2][0] = 0.0, d[2][1] = 4.0 * e - 1.0;
  d[3][0] = 4.0 - 8.0 * k - 4.0 * e, d[3][1] = -4.0 * k;
  d[4][0] = 4.0 * e, d[4][1] = 4.0 * k;
  d[5][0] = -4.0 * e, d[5][1] = 4.0 - 4.0 * k - 8.0 * e;
}

// The terms of one face.  xe/ue: element node coordinates and displacements;
// addR(a, i, v) and addK(a, c, d, v) receive R[a,i] and K[a,d; c,d] (volume
// node numbers).
template <int NNE, bool WANT_K, class AddR, class AddK>
__device__ void nbc_face_terms(const double (*xe)[3], const double (*ue)[3], int f, const double *desc,
                               AddR addR, AddK addK) {
  constexpr int NB = NNE == 10 ? 6 : 3;
  constexpr int NPT = NNE == 10 ? 3 : 1;
  const int *v2b = NNE == 10 ? c_qtet2qtri[f] : c_tet2tri[f];
  const int *km = c_kezmap[f];
#pragma unroll 1
  for (int ip = 0; ip < NPT; ip++) {
    const double gk = NPT == 1 ? 1.0 / 3.0 : (ip == 0 ? 2.0 / 3.0 : 1.0 / 6.0);
    const double ge = NPT == 1 ? 1.0 / 3.0 : (ip == 2 ? 2.0 / 3.0 : 1.0 / 6.0);
    const double wt = NPT == 1 ? 0.5 : 1.0 / 6.0;
    double kez[3] = {0.0, 0.0, 0.0};
    kez[km[0]] = gk;
    kez[km[1]] = ge;
    if (f == 2) kez[km[2]] = 1.0 - gk - ge;
    double N[NNE], dk[NNE][3];
    nbc_shape<NNE>(kez[0], kez[1], kez[2], N, dk);
    // volume Jacobian dX/dxi, its adjugate, dN/dX
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int a = 0; a < NNE; a++)
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int c = 0; c < 3; c++) J[i * 3 + c] += dk[a][c] * xe[a][i];
    const double det = J[0] * (J[4] * J[8] - J[5] * J[7]) + J[1] * (J[5] * J[6] - J[3] * J[8]) +
                       J[2] * (J[3] * J[7] - J[4] * J[6]);
    const double ai[9] = {J[4] * J[8] - J[5] * J[7], J[2] * J[7] - J[1] * J[8], J[1] * J[5] - J[2] * J[4],
                          J[5] * J[6] - J[3] * J[8], J[0] * J[8] - J[2] * J[6], J[2] * J[3] - J[0] * J[5],
                          J[3] * J[7] - J[4] * J[6], J[1] * J[6] - J[0] * J[7], J[0] * J[4] - J[1] * J[3]};
    const double rdet = 1.0 / det;
    double dN[NNE][3];
    double F[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
#pragma unroll
    for (int a = 0; a < NNE; a++) {
#pragma unroll
      for (int b = 0; b < 3; b++)
        dN[a][b] = rdet * dk[a][0] * ai[0 * 3 + b] + rdet * dk[a][1] * ai[1 * 3 + b] + rdet * dk[a][2] * ai[2 * 3 + b];
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int c = 0; c < 3; c++) F[i * 3 + c] += ue[a][i] * dN[a][c];
    }
    // face Jacobian and unit normal
    double db[NB][2];
    nbc_face_dN<NB>(kez[km[0]], kez[km[1]], db);
    double dX[3][2] = {{0, 0}, {0, 0}, {0, 0}};
#pragma unroll
    for (int a = 0; a < NB; a++) {
      const int n = v2b[a];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        dX[i][0] += db[a][0] * xe[n][i];
        dX[i][1] += db[a][1] * xe[n][i];
      }
    }
    const double v0 = dX[1][0] * dX[2][1] - dX[1][1] * dX[2][0];
    const double v1 = dX[0][1] * dX[2][0] - dX[0][0] * dX[2][1];
    const double v2 = dX[0][0] * dX[1][1] - dX[0][1] * dX[1][0];
    const double jf = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
    const double nrm[3] = {v0 / jf, v1 / jf, v2 / jf};
    const double detJxW = jf * wt;
    // J = det F and F^-1
    const double Jd = F[0] * (F[4] * F[8] - F[5] * F[7]) + F[1] * (F[5] * F[6] - F[3] * F[8]) +
                      F[2] * (F[3] * F[7] - F[4] * F[6]);
    const double rJ = 1.0 / Jd;
    const double FI[9] = {rJ * (F[4] * F[8] - F[5] * F[7]), rJ * (F[2] * F[7] - F[1] * F[8]),
                          rJ * (F[1] * F[5] - F[2] * F[4]), rJ * (F[5] * F[6] - F[3] * F[8]),
                          rJ * (F[0] * F[8] - F[2] * F[6]), rJ * (F[2] * F[3] - F[0] * F[5]),
                          rJ * (F[3] * F[7] - F[4] * F[6]), rJ * (F[1] * F[6] - F[0] * F[7]),
                          rJ * (F[0] * F[4] - F[1] * F[3])};
    double ftp[3], ftk[3];  // F^-T PN, F^-T PN'
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const double pn0 = desc[0] * nrm[0] + desc[1];
      const double pn1 = desc[0] * nrm[1] + desc[2];
      const double pn2 = desc[0] * nrm[2] + desc[3];
      ftp[i] = FI[0 * 3 + i] * pn0 + FI[1 * 3 + i] * pn1 + FI[2 * 3 + i] * pn2;
      const double pk0 = desc[4] * nrm[0] + desc[7];
      const double pk1 = desc[5] * nrm[1] + desc[8];
      const double pk2 = desc[6] * nrm[2] + desc[9];
      ftk[i] = FI[0 * 3 + i] * pk0 + FI[1 * 3 + i] * pk1 + FI[2 * 3 + i] * pk2;
    }
#pragma unroll 1
    for (int ia = 0; ia < NB; ia++) {
      const int a = v2b[ia];
      const double s = N[a] * detJxW * (-1.0) * Jd;
#pragma unroll
      for (int i = 0; i < 3; i++) addR(a, i, s * ftp[i]);
      if (!WANT_K) continue;
#pragma unroll 1
      for (int ic = 0; ic < NB; ic++) {
        const int c = v2b[ic];
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const double g = FI[0 * 3 + d] * dN[ic][0] + FI[1 * 3 + d] * dN[ic][1] + FI[2 * 3 + d] * dN[ic][2];
          addK(a, c, d, s * 2.0 * g * ftk[d]);
        }
      }
    }
  }
}

template <int NNE>
__device__ __forceinline__ void nbc_gather(const NbcArgs &A, long e, int *nd, double (*xe)[3], double (*ue)[3]) {
#pragma unroll
  for (int a = 0; a < NNE; a++) {
    const int n = A.conn[(long)a * A.ne + e];
    nd[a] = n;
#pragma unroll
    for (int i = 0; i < 3; i++) {
      xe[a][i] = A.X[i * A.nn + n];
      ue[a][i] = A.unode[i * A.nn + n];
    }
  }
}

// Global assembly: one thread per face, FP64 atomics into R and K.
template <int NNE, bool WANT_K>
__global__ void __launch_bounds__(128) k_neumann(const NbcArgs A) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= A.nface) return;
  const long e = A.face_elem[k];
  const int feat = A.face_feat[k];
  int nd[NNE];
  double xe[NNE][3], ue[NNE][3];
  nbc_gather<NNE>(A, e, nd, xe, ue);
  auto addR = [&](int a, int i, double v) {
    const int id = A.dof[i * A.nn + nd[a]];
    if (A.R && id > 0) atomicAdd(&A.R[id - 1], v);
  };
  auto addK = [&](int a, int c, int d, double v) {
    const int na = nd[a], nc = nd[c];
    const unsigned ma = A.mask[na], mc = A.mask[nc];
    if (!((ma >> d) & 1u) || !((mc >> d) & 1u)) return;
    const long off = (long)A.rowptr0[na] + (long)__popc(ma & ((1u << d) - 1u)) * A.rowlen[na] +
                     A.pos[(e * NNE + a) * NNE + c] + __popc(mc & ((1u << d) - 1u));
    atomicAdd(&A.K[off], v);
  };
  nbc_face_terms<NNE, WANT_K>(xe, ue, A.face_id[k], A.feat_desc + kNbcDesc * feat, addR, addK);
}

// Element-level calls: one thread per listed element, its faces added into
// the element's dense residual and stiffness (all components, as the element
// kernels write them).
template <int NNE, bool WANT_K>
__global__ void __launch_bounds__(128) k_neumann_dense(const NbcArgs A) {
  const long ei = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (ei >= A.nlist) return;
  const long e = A.elist[ei];
  const int k0 = A.elem_face_off[e], k1 = A.elem_face_off[e + 1];
  if (k0 == k1) return;
  constexpr int ND = 3 * NNE;
  int nd[NNE];
  double xe[NNE][3], ue[NNE][3];
  nbc_gather<NNE>(A, e, nd, xe, ue);
  double *fe = A.fe_out + ei * ND;
  double *lk = WANT_K ? A.lk_out + ei * ND * ND : nullptr;
  auto addR = [&](int a, int i, double v) { fe[a * 3 + i] += v; };
  auto addK = [&](int a, int c, int d, double v) { lk[(a * 3 + d) * ND + c * 3 + d] += v; };
  for (int k = k0; k < k1; k++) {
    const int feat = A.face_feat[k];
    nbc_face_terms<NNE, WANT_K>(xe, ue, A.face_id[k], A.feat_desc + kNbcDesc * feat, addR, addK);
  }
}

}  // namespace pgb
