// transient.cuh -- the inertia (mid-point rule) form of the 1-field element.
//
// PGFem3D runs it instead of the quasi-static element whenever the material
// density exceeds 1e-16 (src/stiffmat_fd.cc:549-565, src/fd_residuals.cc:
// 494-500): residual_with_inertia / stiffness_with_inertia (src/dynamics.cc:
// 183-432) with the constitutive-model parts of src/constitutive_model.cc:
// 1905-2170 and 2803-2958.  For the hyperelastic model (identity plastic
// parts, HE_PARAM::get_pF) it is a combination of quasi-static assemblies at
// the mid-point displacements plus the inertia terms:
//   R = -dt_np1 (1 - a) R(u_{n+a}) - dt_n a R(u_{n-1+a}) - f_i
//   K = -M / dt_np1 - a (1 - a) dt_np1 K(u_{n+a})
//   f_i[A,b] = rho / (dt_np1 dt_n) sum_q N_A du_b w,  du = sum_C N_C v_C,
//   v = dt_n u_{n+1} - (dt_np1 + dt_n) u_n + dt_np1 u_{n-1}
//   M[A b; C b] = rho sum_q N_A N_C w
// (u_{n+a} = (1 - a) u_n + a u_{n+1}, mid_point_rule of src/utils.cc:
// 3213-3223).  The quasi-static parts run through the context's assembly
// kernels; this file holds the blends and the inertia kernel.
#pragma once
#include "assemble.cuh"

namespace pgb {

// out = (1 - a) x + a y
__global__ void k_blend(double *out, const double *x, const double *y, double a, long n) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = (1.0 - a) * x[i] + a * y[i];
}

// out = cx x + cy y + cz z (the inertia combination v)
__global__ void k_comb3(double *out, const double *x, double cx, const double *y, double cy, const double *z,
                        double cz, long n) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = cx * x[i] + cy * y[i] + cz * z[i];
}

// y = a y + b x (x may be null: y = a y)
__global__ void k_scale_add(double *y, double a, const double *x, double b, long n) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) y[i] = x ? a * y[i] + b * x[i] : a * y[i];
}

struct InertiaArgs {
  const double *X;       // 3*nn SoA
  const int *conn;       // NNE*ne
  const int *dof;        // 3*nn SoA
  const int *rowptr0, *rowlen;
  const uint8_t *mask;
  const uint16_t *pos;   // ne*NNE*NNE
  long nn, ne;
  const double *vnode;   // 3*nn SoA: v of the element nodes
  double cR;             // rho / (dt_np1 dt_n): f_i scale
  double cK;             // rho / dt_np1: mass scale
  double *R, *K;         // either may be null
  ShapeTable shp;
};

// One thread per element: f_i into R (subtracted) and/or the mass into the
// component-diagonal K entries (subtracted), FP64 atomics through the
// element's node-block map.  The transient call forms the mass once (K alone,
// cK = 1, into a cached CSR-aligned array) and then runs this kernel for R.
template <int NNE, int NQP>
__global__ void __launch_bounds__(128) k_inertia(const InertiaArgs A) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= A.ne) return;
  int nd[NNE];
  double xe[NNE][3], ve[NNE][3];
#pragma unroll
  for (int a = 0; a < NNE; a++) {
    const int n = A.conn[(long)a * A.ne + e];
    nd[a] = n;
#pragma unroll
    for (int i = 0; i < 3; i++) {
      xe[a][i] = A.X[i * A.nn + n];
      ve[a][i] = A.vnode[i * A.nn + n];
    }
  }
  double fi[NNE][3], mm[NNE][NNE];
#pragma unroll
  for (int a = 0; a < NNE; a++) {
    fi[a][0] = fi[a][1] = fi[a][2] = 0.0;
#pragma unroll
    for (int c = 0; c < NNE; c++) mm[a][c] = 0.0;
  }
  bool bad = false;
#pragma unroll
  for (int q = 0; q < NQP; q++) {
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int a = 0; a < NNE; a++)
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int c = 0; c < 3; c++) J[i * 3 + c] += A.shp.dNxi[q][a][c] * xe[a][i];
    const double det = J[0] * (J[4] * J[8] - J[5] * J[7]) + J[1] * (J[5] * J[6] - J[3] * J[8]) +
                       J[2] * (J[3] * J[7] - J[4] * J[6]);
    if (!(det > 0.0)) bad = true;  // the quasi-static kernels count such elements
    const double w = det * A.shp.w[q];
    double du[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int a = 0; a < NNE; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) du[b] += A.shp.N[q][a] * ve[a][b];
#pragma unroll
    for (int a = 0; a < NNE; a++) {
      const double Na = A.shp.N[q][a];
#pragma unroll
      for (int b = 0; b < 3; b++) fi[a][b] += A.cR * Na * du[b] * w;
#pragma unroll
      for (int c = 0; c < NNE; c++) mm[a][c] += A.cK * Na * A.shp.N[q][c] * w;
    }
  }
  if (bad) return;
#pragma unroll
  for (int a = 0; a < NNE; a++) {
    const unsigned ma = A.mask[nd[a]];
#pragma unroll
    for (int b = 0; b < 3; b++) {
      if (!((ma >> b) & 1u)) continue;
      if (A.R) atomicAdd(&A.R[A.dof[b * A.nn + nd[a]] - 1], -fi[a][b]);
      if (!A.K) continue;
      const long row = (long)A.rowptr0[nd[a]] + (long)__popc(ma & ((1u << b) - 1u)) * A.rowlen[nd[a]];
#pragma unroll
      for (int c = 0; c < NNE; c++) {
        const unsigned mc = A.mask[nd[c]];
        if (!((mc >> b) & 1u)) continue;
        atomicAdd(&A.K[row + A.pos[(e * NNE + a) * NNE + c] + __popc(mc & ((1u << b) - 1u))], -mm[a][c]);
      }
    }
  }
}

}  // namespace pgb
