// pgfem_gpu.cu -- C ABI of the sm_100a assembly path (include/pgfem_gpu.h).
//
// The context keeps every array of the path resident in HBM in
// structure-of-arrays form: node coordinates X[3][nn], connectivity
// conn[nne][ne] (int32), DOF ids dof[3][nn], the element->CSR node-block map
// (pos[ne][nne][nne], uint16 column offsets inside the rows of the block's
// first node), the per-node row offsets/lengths and free-component masks, and
// the per-quadrature-point state at t_n and t_{n+1} as [comp][nqp].  No call
// falls back to a CPU path: without an sm_100 device every entry point
// returns PGFEM_GPU_ENODEV.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "assemble.cuh"
#include "assemble_mma.cuh"
#include "assemble_p1.cuh"
#include "cm_integrate.cuh"
#include "cp_kernels.cuh"
#include "neumann.cuh"
#include "transient.cuh"
#include "peak_probe.cuh"
#include "pgfem_gpu.h"

using namespace pgb;

struct pgfem_gpu_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int nne = 0, nqp_e = 0;
  long nn = 0, ne = 0, ndof = 0, npres = 0, nnz = 0, nqp = 0;
  int model = 0, nstate = 0;  // device state components per qp
  Mat mat{};
  ShapeTable shp{};
  // device arrays
  double *X = nullptr;
  int *conn = nullptr;
  int *dof = nullptr;
  int *rowptr0 = nullptr;
  int *rowlen = nullptr;
  uint8_t *mask = nullptr;
  uint16_t *pos = nullptr;
  double *unode = nullptr;
  double *F0 = nullptr;
  double *state_n = nullptr, *state_np1 = nullptr;
  double *state_nm1 = nullptr;  // crystal plasticity: the state at t_{n-1} (transient element)
  unsigned long long *status = nullptr;
  // scratch for host-buffer calls
  double *d_u = nullptr, *d_presc = nullptr, *d_R = nullptr, *d_K = nullptr;
  // colour mode
  int scatter_mode = PGFEM_SCATTER_ATOMIC;
  std::vector<long> colour_off;  // offsets into colour element list
  int *colour_elems = nullptr;
  long bytes = 0;
  double *qrec = nullptr;  // point records (kYRec x nqp for 10-node elements, kQRec x nqp for 4-node)
  int *eblk = nullptr;     // scatter blocks of 10-node elements (kEBW words each), processing order
  // tensor-core quadratic-tet path: processing order (slot -> element), and a
  // second stream with fork/join events on which K is zeroed while the point
  // kernel runs
  int *perm = nullptr;
  cudaStream_t zstream = nullptr;
  cudaEvent_t zfork = nullptr, zjoin = nullptr;
  // crystal plasticity
  double *cp_R = nullptr, *cp_F = nullptr, *cp_detJw = nullptr, *cp_out = nullptr, *cp_guess = nullptr;
  int *cp_iters = nullptr;
  unsigned *cp_counter = nullptr;
  uint8_t *cp_conv = nullptr;  // per point: converged (the tangent kernel's input)
  bool cp_use_guess = false;
  // learned warm start: F at t_n, network features / predictions, cold restarts
  double *cp_Fn = nullptr;
  float *cp_feat = nullptr, *cp_pred = nullptr;
  pgfem_mlp *cp_net = nullptr;
  int cp_warm_k = 0;
  unsigned long long *cp_fallbacks = nullptr;
  // batches of independent meshes and the work-stealing schedule
  int *elem_group = nullptr;
  double *F0_tab = nullptr;
  int ngroups = 0;
  unsigned *sched_ticket = nullptr;
  unsigned *p2m_ticket = nullptr;  // tile counter of the quadratic-tet assembly
  // three-field (CM3F) element: pressure and volume per element (element
  // order), the expanded displacement increment of the local update, and the
  // record width the point records were allocated with
  int three_field = 0;
  double *tf_P = nullptr, *tf_theta = nullptr, *tf_dunode = nullptr, *tf_inc = nullptr;
  int qrec_fields = 0;
  int sched_epb = 0, sched_grab = 0;  // elements per block (0: default), tiles per steal (0: static)
  // failure-path tests: bound of the hand-off waits, one-shot withheld hand-off
  unsigned long long wait_ns = 2000000000ull;
  int stall_next = 0;
  // surface loads: faces sorted by element, their features' load type and
  // values, per-element face offsets (ne+1)
  long nbc_nface = 0, nbc_bytes = 0;
  int nbc_nfeat = 0;
  int *nbc_elem = nullptr, *nbc_feat = nullptr, *nbc_type = nullptr, *nbc_off = nullptr;
  uint8_t *nbc_face = nullptr;
  double *nbc_load = nullptr;  // load descriptors (kNbcDesc per feature) at t_{n+1}
  // host copies of the types and values (t_{n+1}; t_n, t_{n-1} for the
  // transient element), the transient call's two mid-point descriptor sets,
  // and the set the next assembly reads (nullptr: nbc_load)
  std::vector<int> nbc_type_h;
  std::vector<double> nbc_load_h, nbc_hist_n, nbc_hist_nm1;
  double *nbc_desc_tr = nullptr;
  const double *nbc_desc_cur = nullptr;
  // transient calls: u and prescribed values at t_{n+1}, t_n, t_{n-1}, a
  // mid-point / combination vector of each, the second residual
  double *tr_buf = nullptr;
  double *tr_F = nullptr;  // crystal plasticity: F at t_n and t_{n-1} per element (SoA 2 x 9*ne)
  // three-field transient: P_n, theta_n, P_{n-1}, theta_{n-1} per element
  // (4*ne), and scratch for the mid-point P, theta (4*ne) and u_{n-1+a} at
  // the nodes (3*nn)
  double *tf_hist = nullptr, *tf_mid = nullptr;
  // transient calls: minus the consistent mass of unit density, CSR-aligned
  // (nnz; geometry only, formed on the first transient R+K call)
  double *mass_csr = nullptr;
  // kernel timing
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
};

namespace {

#define CK(x)                                                                            \
  do {                                                                                   \
    cudaError_t _e = (x);                                                                \
    if (_e != cudaSuccess) {                                                             \
      std::fprintf(stderr, "pgfem_gpu: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(_e), \
                   __FILE__, __LINE__);                                                  \
      return PGFEM_GPU_ECUDA;                                                            \
    }                                                                                    \
  } while (0)

template <class T>
int dalloc(pgfem_gpu_ctx *c, T **p, size_t n) {
  if (n == 0) n = 1;
  if (cudaMalloc((void **)p, n * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return PGFEM_GPU_ENOMEM;
  }
  c->bytes += (long)(n * sizeof(T));
  return PGFEM_GPU_OK;
}

int check_device() {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return PGFEM_GPU_ENODEV;
  }
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return PGFEM_GPU_ENODEV;
  if (p.major != 10) return PGFEM_GPU_ENODEV;
  return PGFEM_GPU_OK;
}

// Quadrature tables with the reference constants (FEMLIB/src/femlib.cc:571-588,
// shape-function derivatives :213-333); evaluated on the host in FP64.
ShapeTable make_shape(int nne) {
  ShapeTable t{};
  if (nne == 4) {
    const double d[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int a = 0; a < 4; a++)
      for (int c = 0; c < 3; c++) t.dNxi[0][a][c] = d[a][c];
    t.w[0] = 1.0 / 6.0;
    for (int a = 0; a < 4; a++) t.N[0][a] = 0.25;  // PGFem3D_N at the centroid
    return t;
  }
  const double A = 0.58541020, B = 0.13819660;
  const double k[4] = {A, B, B, B}, e[4] = {B, A, B, B}, z[4] = {B, B, A, B};
  for (int q = 0; q < 4; q++) {
    const double ksi = k[q], eta = e[q], zet = z[q];
    double d[10][3] = {
        {4.0 * (ksi + eta + zet) - 3.0, 4.0 * (eta + ksi + zet) - 3.0, 4.0 * (zet + ksi + eta) - 3.0},
        {4.0 * ksi - 1.0, 0.0, 0.0},
        {0.0, 4.0 * eta - 1.0, 0.0},
        {0.0, 0.0, 4.0 * zet - 1.0},
        {4.0 * (-2.0 * ksi - eta - zet + 1.0), -4.0 * ksi, -4.0 * ksi},
        {4.0 * eta, 4.0 * ksi, 0.0},
        {-4.0 * eta, 4.0 * (-ksi - 2.0 * eta - zet + 1.0), -4.0 * eta},
        {-4.0 * zet, -4.0 * zet, 4.0 * (-ksi - eta - 2.0 * zet + 1.0)},
        {4.0 * zet, 0.0, 4.0 * ksi},
        {0.0, 4.0 * zet, 4.0 * eta}};
    for (int a = 0; a < 10; a++)
      for (int c = 0; c < 3; c++) t.dNxi[q][a][c] = d[a][c];
    t.w[q] = (1.0 / 4.0) / 6.0;
    // PGFem3D_N (FEMLIB/src/femlib.cc:164-177)
    const double l0 = 1.0 - ksi - eta - zet;
    const double N[10] = {(2.0 * l0 - 1.0) * l0, (2.0 * ksi - 1.0) * ksi, (2.0 * eta - 1.0) * eta,
                          (2.0 * zet - 1.0) * zet, 4.0 * l0 * ksi, 4.0 * ksi * eta, 4.0 * l0 * eta,
                          4.0 * l0 * zet, 4.0 * ksi * zet, 4.0 * eta * zet};
    for (int a = 0; a < 10; a++) t.N[q][a] = N[a];
  }
  return t;
}

Mat make_mat(const pgfem_material_desc *m) {
  Mat r{};
  r.model = m->model;
  r.dev_pot = m->model == PGFEM_MODEL_HE && m->dev_pot == 2 ? 2 : 1;
  r.vol_pot = (m->vol_pot == 2 || m->vol_pot == 3) && m->model != PGFEM_MODEL_CP ? m->vol_pot : 99;
  r.mu = m->E / (2.0 * (1.0 + m->nu));
  r.kappa = (2 * r.mu * (1 + m->nu)) / (3 * (1 - 2 * m->nu));
  r.sy = m->sigma_y;
  r.H = m->H;
  r.gdot0 = m->gamma_dot_0;
  r.m = m->m;
  r.G0 = m->G0;
  r.g0 = m->g0;
  r.gs0 = m->gs_0;
  r.gdots = m->gamma_dot_s;
  r.w = m->w;
  r.tol = m->cp_tol > 0 ? m->cp_tol : 1e-10;
  r.max_iter = m->cp_max_iter > 0 ? m->cp_max_iter : 25;
  return r;
}

int device_state_size(int model) {
  switch (model) {
    case PGFEM_MODEL_J2: return 7;   // Cp^-1 (Voigt 6) + eqps
    case PGFEM_MODEL_CP: return 10;  // pF (9) + g
    default: return 0;
  }
}

// F = I + grad_X u (+ the element group's macro F0) at every point, AoS
// [ne * nqp_e][9] (compute_deformation_gradient of the restart writer's Fn).
__global__ void k_point_F(const double *X, const int *conn, long nn, long ne, int nne, int nqp_e,
                          const double *unode, ShapeTable shp, const double *F0, const int *elem_group,
                          const double *F0_tab, double *F_out) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= ne * nqp_e) return;
  const long e = t / nqp_e;
  const int q = (int)(t % nqp_e);
  double dX[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, dU[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int a = 0; a < nne; a++) {
    const long n = conn[(long)a * ne + e];
    for (int i = 0; i < 3; i++) {
      const double x = X[i * nn + n], u = unode[i * nn + n];
      for (int c = 0; c < 3; c++) {
        dX[i * 3 + c] += shp.dNxi[q][a][c] * x;
        dU[i * 3 + c] += shp.dNxi[q][a][c] * u;
      }
    }
  }
  double dXi[9], F[9];
  const bool ok = inv3(dX, dXi);
  const double *G0 = elem_group ? F0_tab + 9 * (long)elem_group[e] : F0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      F[i * 3 + j] = ok ? (i == j ? 1.0 : 0.0) + dU[i * 3] * dXi[j] + dU[i * 3 + 1] * dXi[3 + j] +
                              dU[i * 3 + 2] * dXi[6 + j] + (G0 ? G0[i * 3 + j] : 0.0)
                        : 0.0;
  for (int k = 0; k < 9; k++) F_out[t * 9 + k] = F[k];
}

__global__ void k_expand_u(const int *dof, long nn, const double *u, const double *presc,
                           double *unode) {
  const long n = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (n >= 3 * nn) return;
  const int id = dof[n];
  unode[n] = id > 0 ? u[id - 1] : (id < 0 && presc ? presc[-id - 1] : 0.0);
}

// Element->CSR node-block map: for each element and node pair (a, b), the
// column position of node b's first free DOF inside the rows of node a,
// checked against the caller's pattern (all free columns of b present and
// consecutive).  0xFFFF marks pairs without a free row or column.
__global__ void k_build_map(const int *conn, long ne, int nne, const int *dof, long nn,
                            const int *rowptr0, const int *rowlen, const uint8_t *mask,
                            const int *Ai, uint16_t *pos, int *err) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const long npair = (long)nne * nne;
  if (t >= ne * npair) return;
  const long e = t / npair;
  const int a = (int)(t % npair) / nne, b = (int)(t % npair) % nne;
  const int A = conn[(long)a * ne + e], B = conn[(long)b * ne + e];
  const unsigned mA = mask[A], mB = mask[B];
  uint16_t out = 0xFFFF;
  if (mA && mB) {
    int first = -1;
    for (int c = 0; c < 3 && first < 0; c++)
      if (dof[c * nn + B] > 0) first = dof[c * nn + B] - 1;
    const int *row = Ai + rowptr0[A];
    int lo = 0, hi = rowlen[A];
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (row[mid] < first) lo = mid + 1;
      else hi = mid;
    }
    const int nb = __popc(mB);
    bool ok = lo + nb <= rowlen[A] && lo < 0xFFFF;
    for (int k = 0; ok && k < nb; k++) ok = row[lo + k] == first + k;
    if (ok) out = (uint16_t)lo;
    else atomicAdd(err, 1);
  }
  pos[t] = out;
}

template <class T>
int upload(pgfem_gpu_ctx *c, T **d, const T *h, size_t n) {
  int r = dalloc(c, d, n);
  if (r) return r;
  CK(cudaMemcpyAsync(*d, h, n * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  return PGFEM_GPU_OK;
}

// the free-component masks, padded to whole 4-byte words: kernels copy the
// aligned word that holds a node's byte
int upload_mask(pgfem_gpu_ctx *c, const std::vector<uint8_t> &mask) {
  std::vector<uint8_t> padded(mask);
  padded.resize((mask.size() + 3) & ~(size_t)3, 0);
  return upload(c, &c->mask, padded.data(), padded.size());
}

void drop_events(pgfem_gpu_ctx *c) {
  for (auto &p : c->events) {
    cudaEventDestroy(p.first);
    cudaEventDestroy(p.second);
  }
  c->events.clear();
}

void release(pgfem_gpu_ctx *c) {
  drop_events(c);
  void *ptrs[] = {c->X, c->conn, c->dof, c->rowptr0, c->rowlen, c->mask, c->pos, c->unode, c->F0,
                  c->state_n, c->state_np1, c->status, c->d_u, c->d_presc, c->d_R, c->d_K,
                  c->colour_elems, c->qrec, c->eblk, c->perm,
                  c->cp_R, c->cp_F, c->cp_detJw, c->cp_out, c->cp_guess, c->cp_iters, c->cp_counter,
                  c->cp_Fn, c->cp_feat, c->cp_pred, c->cp_fallbacks, c->elem_group, c->F0_tab, c->cp_conv,
                  c->sched_ticket, c->p2m_ticket, c->tf_P, c->tf_theta, c->tf_dunode, c->tf_inc, c->nbc_desc_tr, c->nbc_elem, c->nbc_feat, c->nbc_type, c->nbc_off, c->nbc_face,
                  c->nbc_load, c->tr_buf, c->state_nm1, c->tr_F, c->tf_hist, c->tf_mid, c->mass_csr};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (c->zfork) cudaEventDestroy(c->zfork);
  if (c->zjoin) cudaEventDestroy(c->zjoin);
  if (c->zstream) cudaStreamDestroy(c->zstream);
  if (c->stream) cudaStreamDestroy(c->stream);
}

AsmArgs base_args(const pgfem_gpu_ctx *c) {
  AsmArgs a{};
  a.X = c->X;
  a.conn = c->conn;
  a.dof = c->dof;
  a.rowptr0 = c->rowptr0;
  a.rowlen = c->rowlen;
  a.mask = c->mask;
  a.pos = c->pos;
  a.nn = c->nn;
  a.ne = c->ne;
  a.unode = c->unode;
  a.F0 = c->F0;
  a.state_n = c->state_n;
  a.state_np1 = c->state_np1;
  a.nqp = c->nqp;
  a.status = c->status;
  a.mat = c->mat;
  a.shp = c->shp;
  a.elem_group = c->elem_group;
  a.F0_tab = c->F0_tab;
  a.wait_ns = c->wait_ns;
  return a;
}

int g_num_sms = 0;

int grid_for(long nitems, int te, int per_sm) {
  if (!g_num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  const long tiles = (nitems + te - 1) / te;
  return (int)std::max<long>(1, std::min<long>(tiles, (long)g_num_sms * per_sm * 8));
}

template <int NNE, int NQP, int MODEL, bool ATOMIC, bool WANT_K, bool DENSE, int TEP = Tile<NNE>::TE>
int launch_asm(const AsmArgs &a, long nitems, cudaStream_t s) {
  constexpr size_t smem = asm_smem_bytes<NNE, NQP, TEP>();
  auto kern = k_assemble<NNE, NQP, MODEL, ATOMIC, WANT_K, DENSE, TEP>;
  static bool attr_set = false;
  if (!attr_set) {
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set = true;
  }
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TEP * NNE, smem));
  if (per_sm < 1) per_sm = 1;
  int grid = grid_for(nitems, TEP, per_sm);
  if (a.ticket) {  // persistent: every CTA resident, tiles claimed from the ticket
    CK(cudaMemsetAsync(a.ticket, 0, sizeof(unsigned), s));
    grid = (int)std::max<long>(1, std::min<long>((nitems + TEP - 1) / TEP, (long)g_num_sms * per_sm));
  }
  kern<<<grid, TEP * NNE, smem, s>>>(a);
  CK(cudaGetLastError());
  return PGFEM_GPU_OK;
}

// Point updates of all quadrature points into c->qrec (allocated on first use;
// 26-double records for the tensor-core quadratic-tet kernel, 30 for its
// three-field form, 38 for the linear-tet kernels).
template <int NNE, int NQP, int MODEL, bool TF = false>
int launch_qp_update(pgfem_gpu_ctx *c, cudaStream_t s) {
  constexpr bool YREC = NNE == 10;
  const int nf = YREC ? yrec_fields(TF) : kQRec;
  // the tiled layout of the 10-node records is padded to whole tiles
  const size_t npts = YREC ? (size_t)((c->nqp + kMPtsT - 1) / kMPtsT) * kMPtsT : (size_t)c->nqp;
  if (c->qrec && c->qrec_fields < nf) {  // a wider record than allocated
    cudaFree(c->qrec);
    c->bytes -= (long)(sizeof(double) * c->qrec_fields * npts);
    c->qrec = nullptr;
  }
  if (!c->qrec) {
    int r = dalloc(c, &c->qrec, (size_t)nf * npts);
    if (r) return r;
    c->qrec_fields = nf;
  }
  QpArgs q{};
  q.X = c->X;
  q.unode = c->unode;
  q.conn = c->conn;
  q.nn = c->nn;
  q.ne = c->ne;
  q.nqp = c->nqp;
  q.F0 = c->F0;
  q.elem_group = c->elem_group;
  q.F0_tab = c->F0_tab;
  q.state_n = c->state_n;
  q.state_np1 = c->state_np1;
  q.qrec = c->qrec;
  q.status = c->status;
  if (YREC) q.perm = c->perm;
  q.mat = c->mat;
  q.shp = c->shp;
  q.tf_P = c->tf_P;
  q.tf_theta = c->tf_theta;
  k_qp_update<NNE, NQP, MODEL, YREC, TF><<<(unsigned)((c->nqp + 127) / 128), 128, 0, s>>>(q);
  CK(cudaGetLastError());
  return PGFEM_GPU_OK;
}

// quadratic tets in two kernels: point updates into c->qrec (40-double
// records; K zeroed meanwhile on the context's second stream), then the
// tensor-core element assembly from the records
template <int MODEL, bool TF = false>
int launch_p2m(pgfem_gpu_ctx *c, const AsmArgs &a0, cudaStream_t s) {
  if (!TF && c->three_field) return launch_p2m<MODEL, true>(c, a0, s);
  CK(cudaEventRecord(c->zfork, s));
  CK(cudaStreamWaitEvent(c->zstream, c->zfork, 0));
  CK(cudaMemsetAsync(a0.K, 0, sizeof(double) * c->nnz, c->zstream));
  CK(cudaMemsetAsync(c->p2m_ticket, 0, sizeof(unsigned), c->zstream));
  CK(cudaEventRecord(c->zjoin, c->zstream));
  if (int r = launch_qp_update<10, 4, MODEL, TF>(c, s)) return r;
  CK(cudaStreamWaitEvent(s, c->zjoin, 0));
  AsmArgs a = a0;
  a.qrec = c->qrec;
  a.eblk = c->eblk;
  a.ticket = c->p2m_ticket;
  const size_t smem = p2m_smem_bytes(TF);
  auto kern = k_assemble_p2m<MODEL, TF>;
  static bool attr_set = false;
  if (!attr_set) {
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set = true;
  }
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kMThreads, smem));
  if (per_sm < 1) per_sm = 1;
  if (!g_num_sms) grid_for(1, 1, 1);
  const long tiles = (a.ne + kMTE - 1) / kMTE;
  const long grid = std::max<long>(1, std::min<long>(tiles, (long)g_num_sms * per_sm));
  kern<<<(unsigned)grid, kMThreads, smem, s>>>(a);
  CK(cudaGetLastError());
  return PGFEM_GPU_OK;
}

// linear tets in two kernels: point updates into c->qrec, then the column-split
// assembly from the records with the context's schedule (elements per block,
// work stealing)
template <int MODEL, int TE>
int launch_p1ws_te(pgfem_gpu_ctx *c, const AsmArgs &a0, cudaStream_t s) {
  AsmArgs a = a0;
  a.qrec = c->qrec;
  a.stall = c->stall_next;
  c->stall_next = 0;
  if (c->sched_grab > 0) {
    a.ticket = c->sched_ticket;
    a.grab = c->sched_grab;
  }
  const size_t smem = p1ws_smem_bytes(TE);
  auto kern = k_assemble_p1ws<MODEL, TE>;
  constexpr int nt = p1ws_threads<TE>();
  static bool attr_set = false;
  if (!attr_set) {
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set = true;
  }
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, nt, smem));
  if (per_sm < 1) per_sm = 1;
  if (!g_num_sms) grid_for(1, 1, 1);
  const long tiles = (a.ne + TE - 1) / TE;
  if (a.ticket) CK(cudaMemsetAsync(a.ticket, 0, sizeof(unsigned), s));
  const long grid = std::max<long>(1, std::min<long>(tiles, (long)g_num_sms * per_sm));
  kern<<<(unsigned)grid, nt, smem, s>>>(a);
  CK(cudaGetLastError());
  return PGFEM_GPU_OK;
}

// elements per block of the schedule -> the pipeline's tile: 16 -> 8, 32 (or
// unset) -> 16, 64 -> 32 elements (the consumer warps of a CTA hold two
// elements each)
template <int MODEL>
int launch_p1r(pgfem_gpu_ctx *c, const AsmArgs &a, cudaStream_t s) {
  if (int r = launch_qp_update<4, 1, MODEL>(c, s)) return r;
  if (c->sched_epb == 16) return launch_p1ws_te<MODEL, 8>(c, a, s);
  if (c->sched_epb == 64) return launch_p1ws_te<MODEL, 32>(c, a, s);
  return launch_p1ws_te<MODEL, 16>(c, a, s);
}

template <bool ATOMIC, bool WANT_K, bool DENSE>
int dispatch(pgfem_gpu_ctx *c, const AsmArgs &a, long nitems, cudaStream_t s) {
  // HE with the linear deviatoric potential: its tangent is carried by the
  // per-node kernel only (template model 3), for every call of this context
  if (c->mat.dev_pot == 2)
    return c->nne == 4 ? launch_asm<4, 1, 3, ATOMIC, WANT_K, DENSE>(a, nitems, s)
                       : launch_asm<10, 4, 3, ATOMIC, WANT_K, DENSE>(a, nitems, s);
  // quadratic tets, R+K into the CSR with atomic scatter over all elements:
  // the point kernel + the tensor-core element assembly
  if (c->nne == 10 && ATOMIC && WANT_K && !DENSE && !a.elist && a.R)
    return c->model == PGFEM_MODEL_J2 ? launch_p2m<1>(c, a, s) : launch_p2m<0>(c, a, s);
  // linear tets, R+K into the CSR with atomic scatter over all elements: the
  // point kernel + column-split assembly with the context's schedule
  if (c->nne == 4 && ATOMIC && WANT_K && !DENSE && !a.elist && a.R)
    return c->model == PGFEM_MODEL_J2 ? launch_p1r<1>(c, a, s) : launch_p1r<0>(c, a, s);
  // linear tets over all elements: the tuned schedule (elements per block,
  // work stealing)
  if (c->nne == 4 && ATOMIC && !DENSE && !a.elist && (c->sched_epb || c->sched_grab)) {
    AsmArgs b = a;
    if (c->sched_grab > 0) {
      b.ticket = c->sched_ticket;
      b.grab = c->sched_grab;
    }
    if (c->sched_epb == 16)
      return c->model == PGFEM_MODEL_J2 ? launch_asm<4, 1, 1, true, WANT_K, false, 16>(b, nitems, s)
                                        : launch_asm<4, 1, 0, true, WANT_K, false, 16>(b, nitems, s);
    if (c->sched_epb == 64)
      return c->model == PGFEM_MODEL_J2 ? launch_asm<4, 1, 1, true, WANT_K, false, 64>(b, nitems, s)
                                        : launch_asm<4, 1, 0, true, WANT_K, false, 64>(b, nitems, s);
    return c->model == PGFEM_MODEL_J2 ? launch_asm<4, 1, 1, true, WANT_K, false>(b, nitems, s)
                                      : launch_asm<4, 1, 0, true, WANT_K, false>(b, nitems, s);
  }
  if (c->nne == 4) {
    switch (c->model) {
      case PGFEM_MODEL_HE: return launch_asm<4, 1, 0, ATOMIC, WANT_K, DENSE>(a, nitems, s);
      case PGFEM_MODEL_J2: return launch_asm<4, 1, 1, ATOMIC, WANT_K, DENSE>(a, nitems, s);
    }
  } else {
    switch (c->model) {
      case PGFEM_MODEL_HE: return launch_asm<10, 4, 0, ATOMIC, WANT_K, DENSE>(a, nitems, s);
      case PGFEM_MODEL_J2: return launch_asm<10, 4, 1, ATOMIC, WANT_K, DENSE>(a, nitems, s);
    }
  }
  return PGFEM_GPU_EINVAL;
}

int ensure_K_scratch(pgfem_gpu_ctx *c) {
  if (c->d_K) return PGFEM_GPU_OK;
  return dalloc(c, &c->d_K, std::max<long>(1, c->nnz));
}

// element-level outputs of assemble_cp: the listed elements' dense blocks
struct CpElemList {
  const int *list;
  long n;
  double *lk, *fe;
};

// the transient element stage of assemble_cp (k_cp_element_tr)
struct CpTransient {
  const double *F_n, *F_nm1;
  double alpha, cA, cB;
};

// The CP path: F per element, the local Newton (optionally from the network's
// guess), the consistent tangent, then the element stage -- scattered into the
// CSR (d_R, d_K) or, with el, the listed elements' dense blocks.
int assemble_cp(pgfem_gpu_ctx *c, double *d_R, double *d_K, double dt, cudaStream_t s,
                const CpElemList *el = nullptr, const CpTransient *tr = nullptr) {
  k_cp_F<<<(unsigned)((c->ne + 127) / 128), 128, 0, s>>>(c->X, c->unode, c->conn, c->nn, c->ne, c->F0, c->cp_F,
                                                          c->cp_detJw, c->status);
  CK(cudaGetLastError());
  CK(cudaMemsetAsync(c->cp_counter, 0, sizeof(unsigned), s));
  CK(cudaMemsetAsync(c->cp_fallbacks, 0, sizeof(unsigned long long), s));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (c->timing && c->events.size() < 4096) {
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s));
  }
  const unsigned pblk = (unsigned)((c->nqp + 127) / 128);
  if (c->cp_net) {  // network guess: features -> tcgen05 forward -> M0, g0
    k_cp_features<<<pblk, 128, 0, s>>>(c->nqp, c->cp_F, c->cp_Fn, c->state_n, c->cp_R, 1, c->ne, c->cp_feat);
    CK(cudaGetLastError());
    int r = pgfem_mlp_predict_device(c->cp_net, c->nqp, c->cp_feat, c->cp_pred, s);
    if (r) return r;
    k_cp_guess<<<pblk, 128, 0, s>>>(c->nqp, c->cp_pred, c->cp_R, 1, c->ne, c->state_n, c->mat, c->cp_guess);
    CK(cudaGetLastError());
  }
  CpArgs a{};
  a.nqp = c->nqp;
  a.F = c->cp_F;
  a.Rcp = c->cp_R;
  a.nqp_e = 1;
  a.ne = c->ne;
  a.state_n = c->state_n;
  a.state_np1 = c->state_np1;
  a.guess = (c->cp_use_guess || c->cp_net) ? c->cp_guess : nullptr;
  a.warm_k = c->cp_warm_k;
  a.fallbacks = c->cp_fallbacks;
  a.conv = c->cp_conv;
  a.out = c->cp_out;
  a.iters = c->cp_iters;
  a.counter = c->cp_counter;
  a.status = c->status;
  a.mat = c->mat;
  a.dt = dt;
  const size_t smem = cp_update_smem();
  static bool attr = false;
  if (!attr) {
    CK(cudaFuncSetAttribute(k_cp_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cp_update, 32 * kCpWarps, smem));
  if (per_sm < 1) per_sm = 1;
  if (!g_num_sms) grid_for(1, 1, 1);
  const long need = (c->nqp + 32 * kCpWarps - 1) / (32 * kCpWarps);
  const long grid = std::max<long>(1, std::min<long>(need, (long)g_num_sms * per_sm));
  k_cp_update<<<(unsigned)grid, 32 * kCpWarps, smem, s>>>(a);
  CK(cudaGetLastError());
  {  // consistent tangent dM/dF of the converged points
    const size_t tsm = cp_tangent_smem();
    static bool tattr = false;
    if (!tattr) {
      CK(cudaFuncSetAttribute(k_cp_tangent, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm));
      tattr = true;
    }
    int tper = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&tper, k_cp_tangent, 32 * kCpTanWarps, tsm));
    if (tper < 1) tper = 1;
    const long tgrid = std::max<long>(1, std::min<long>((c->nqp + kCtPts - 1) / kCtPts, (long)g_num_sms * tper));
    k_cp_tangent<<<(unsigned)tgrid, 32 * kCpTanWarps, tsm, s>>>(a);
    CK(cudaGetLastError());
  }
  if (e0) {
    CK(cudaEventRecord(e1, s));
    c->events.emplace_back(e0, e1);
  }
  if (d_K || d_R || el) {
    CpElemArgs b{};
    b.X = c->X;
    b.conn = c->conn;
    b.dof = c->dof;
    b.rowptr0 = c->rowptr0;
    b.rowlen = c->rowlen;
    b.mask = c->mask;
    b.pos = c->pos;
    b.nn = c->nn;
    b.ne = c->ne;
    b.F = c->cp_F;
    b.detJw = c->cp_detJw;
    b.state_n = c->state_n;
    b.out = c->cp_out;
    b.R = d_R;
    b.K = d_K;
    b.mat = c->mat;
    if (tr) {  // mid-point rule: R into d_R, K (if any) into d_K
      b.F_n = tr->F_n;
      b.F_nm1 = tr->F_nm1;
      b.state_np1 = c->state_np1;
      b.state_nm1 = c->state_nm1;
      b.alpha = tr->alpha;
      b.cA = tr->cA;
      b.cB = tr->cB;
      b.status = c->status;
      k_cp_element_tr<<<(unsigned)((c->ne + 127) / 128), 128, 0, s>>>(b);
      CK(cudaGetLastError());
      return PGFEM_GPU_OK;
    }
    if (el) {  // element level: dense blocks of the listed elements
      b.elist = el->list;
      b.nlist = el->n;
      b.lk_out = el->lk;
      b.fe_out = el->fe;
      k_cp_element<<<(unsigned)((el->n + 127) / 128), 128, 0, s>>>(b);
      CK(cudaGetLastError());
      return PGFEM_GPU_OK;
    }
    if (!d_K) return PGFEM_GPU_EINVAL;
    k_cp_element<<<(unsigned)((c->ne + 127) / 128), 128, 0, s>>>(b);
    CK(cudaGetLastError());
  }
  return PGFEM_GPU_OK;
}

NbcArgs nbc_args(const pgfem_gpu_ctx *c) {
  NbcArgs A{};
  A.X = c->X;
  A.conn = c->conn;
  A.dof = c->dof;
  A.rowptr0 = c->rowptr0;
  A.rowlen = c->rowlen;
  A.mask = c->mask;
  A.pos = c->pos;
  A.nn = c->nn;
  A.ne = c->ne;
  A.unode = c->unode;
  A.nface = c->nbc_nface;
  A.face_elem = c->nbc_elem;
  A.face_id = c->nbc_face;
  A.face_feat = c->nbc_feat;
  A.feat_desc = c->nbc_desc_cur ? c->nbc_desc_cur : c->nbc_load;
  A.elem_face_off = c->nbc_off;
  return A;
}

// Surface-load terms after the element kernels (same stream): into R and K
// (K may be null: residual only), or into the dense blocks of listed elements.
int launch_neumann(pgfem_gpu_ctx *c, double *d_R, double *d_K, cudaStream_t s, const int *elist = nullptr,
                   long nlist = 0, double *lk = nullptr, double *fe = nullptr) {
  if (!c->nbc_nface) return PGFEM_GPU_OK;
  NbcArgs A = nbc_args(c);
  if (elist) {
    if (!nlist) return PGFEM_GPU_OK;
    A.elist = elist;
    A.nlist = nlist;
    A.lk_out = lk;
    A.fe_out = fe;
    const unsigned g = (unsigned)((nlist + 127) / 128);
    if (c->nne == 10)
      lk ? k_neumann_dense<10, true><<<g, 128, 0, s>>>(A) : k_neumann_dense<10, false><<<g, 128, 0, s>>>(A);
    else
      lk ? k_neumann_dense<4, true><<<g, 128, 0, s>>>(A) : k_neumann_dense<4, false><<<g, 128, 0, s>>>(A);
  } else {
    if (!d_R && !d_K) return PGFEM_GPU_OK;
    A.R = d_R;
    A.K = d_K;
    const unsigned g = (unsigned)((c->nbc_nface + 127) / 128);
    if (c->nne == 10)
      d_K ? k_neumann<10, true><<<g, 128, 0, s>>>(A) : k_neumann<10, false><<<g, 128, 0, s>>>(A);
    else
      d_K ? k_neumann<4, true><<<g, 128, 0, s>>>(A) : k_neumann<4, false><<<g, 128, 0, s>>>(A);
  }
  CK(cudaGetLastError());
  return PGFEM_GPU_OK;
}

// Whether an R+K call of this context runs the tensor-core quadratic-tet
// path (the branch of dispatch() for 10-node elements, atomic scatter).
bool uses_p2m(const pgfem_gpu_ctx *c) {
  return c->eblk && c->model != PGFEM_MODEL_CP && c->mat.dev_pot != 2 && c->scatter_mode == PGFEM_SCATTER_ATOMIC;
}

// One assembly on device buffers (zeroing R and K first).
int assemble_device(pgfem_gpu_ctx *c, const double *d_u, const double *d_presc, double *d_R,
                    double *d_K, cudaStream_t s, double dt = 0.0) {
  if (c->three_field) {  // the three-field element runs the tensor-core path only
    if (!d_R || !uses_p2m(c)) return PGFEM_GPU_EINVAL;
    if (!d_K) {  // residual only: the stiffness goes to a scratch K
      if (int r = ensure_K_scratch(c)) return r;
      d_K = c->d_K;
    }
  }
  if (d_R) CK(cudaMemsetAsync(d_R, 0, sizeof(double) * c->ndof, s));
  // the tensor-core quadratic-tet path zeroes K itself, beside its point kernel
  if (d_K && !(uses_p2m(c) && d_R)) CK(cudaMemsetAsync(d_K, 0, sizeof(double) * c->nnz, s));
  {
    const long n3 = 3 * c->nn;
    k_expand_u<<<(unsigned)((n3 + 255) / 256), 256, 0, s>>>(c->dof, c->nn, d_u, d_presc, c->unode);
    CK(cudaGetLastError());
  }
  if (c->model == PGFEM_MODEL_CP) {
    int r;
    if (!d_K) {  // residual only: the tangent columns are skipped by a scratch K
      r = ensure_K_scratch(c);
      if (r) return r;
      CK(cudaMemsetAsync(c->d_K, 0, sizeof(double) * c->nnz, s));
      r = assemble_cp(c, d_R, c->d_K, dt, s);
    } else {
      r = assemble_cp(c, d_R, d_K, dt, s);
    }
    return r ? r : launch_neumann(c, d_R, d_K, s);
  }
  AsmArgs a = base_args(c);
  a.R = d_R;
  a.K = d_K;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (c->timing && c->events.size() < 4096) {
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s));
  }
  int r = PGFEM_GPU_OK;
  if (c->scatter_mode == PGFEM_SCATTER_COLOUR && c->colour_elems) {
    for (size_t k = 0; k + 1 < c->colour_off.size() && !r; k++) {
      a.elist = c->colour_elems + c->colour_off[k];
      a.nlist = c->colour_off[k + 1] - c->colour_off[k];
      r = d_K ? dispatch<false, true, false>(c, a, a.nlist, s)
              : dispatch<false, false, false>(c, a, a.nlist, s);
    }
  } else {
    r = d_K ? dispatch<true, true, false>(c, a, c->ne, s) : dispatch<true, false, false>(c, a, c->ne, s);
  }
  if (e0) {
    CK(cudaEventRecord(e1, s));
    c->events.emplace_back(e0, e1);
  }
  return r ? r : launch_neumann(c, d_R, d_K, s);
}

int read_status(pgfem_gpu_ctx *c, pgfem_gpu_status *st, bool clear) {
  unsigned long long h[4];
  CK(cudaMemcpyAsync(h, c->status, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (st) {
    st->inverted = (long)h[0];
    st->nonconverged = (long)h[1];
    st->bad_diagonal = (long)h[2];
    st->other = (long)h[3];
  }
  if (clear) CK(cudaMemsetAsync(c->status, 0, sizeof(h), c->stream));
  return PGFEM_GPU_OK;
}

// Greedy colouring: elements of one colour share no node, so their R and K
// updates touch disjoint rows and need no atomics.
// Greedy element colours for the plain-add scatter: no two elements of one
// colour share a free DOF, i.e. a row of R and K.  (Periodic meshes map
// distinct slave and master nodes to one DOF, so sharing no node is not
// enough.)
void build_colours(const pgfem_mesh_desc *m, std::vector<int> &elems, std::vector<long> &off) {
  std::vector<int> colour(m->ne, -1);
  std::vector<std::vector<uint8_t>> used;
  int ncol = 0;
  auto dof_of = [&](long e, int a, int k) {  // 1-based free DOF id, 0 for fixed / prescribed
    const long id = m->dof_id[(long)m->conn[e * m->nne + a] * 3 + k];
    return id > 0 && id <= m->ndof ? id : 0L;
  };
  for (long e = 0; e < m->ne; e++) {
    int c = 0;
    for (; c < ncol; c++) {
      bool ok = true;
      for (int a = 0; a < m->nne && ok; a++)
        for (int k = 0; k < 3 && ok; k++) {
          const long id = dof_of(e, a, k);
          ok = !(id > 0 && used[c][id - 1]);
        }
      if (ok) break;
    }
    if (c == ncol) {
      used.emplace_back(std::max<long>(1, m->ndof), 0);
      ncol++;
    }
    colour[e] = c;
    for (int a = 0; a < m->nne; a++)
      for (int k = 0; k < 3; k++) {
        const long id = dof_of(e, a, k);
        if (id > 0) used[c][id - 1] = 1;
      }
  }
  off.assign(ncol + 1, 0);
  for (long e = 0; e < m->ne; e++) off[colour[e] + 1]++;
  for (int c = 0; c < ncol; c++) off[c + 1] += off[c];
  elems.resize(m->ne);
  std::vector<long> fill(off.begin(), off.end() - 1);
  for (long e = 0; e < m->ne; e++) elems[fill[colour[e]]++] = (int)e;
}

// Element processing order of the tensor-core quadratic-tet kernel: columns
// of 6 x 6 element-size bins across the two shorter axes of the bounding
// box, swept along the longest axis, bins in lexicographic order inside a
// column (element centroids from the four vertex nodes; element size h =
// (6 V / ne)^(1/3)).  Nearby elements share CSR rows, so in this order a row's
// contributions arrive within about one column layer and its cache lines stay
// in L2 between them (in the mesh's own order a whole cross-section is live).
// Any permutation gives the same sums; this one only shapes the traffic.  The
// width was measured on the 64^3-cell quadratic-tet mesh: 6 bins 6.56, 4 bins
// 6.85, 8 bins 6.87, 12 bins 7.54, 32 bins 7.67 ms per R+K iterate, one
// cross-section 8.24 ms.
std::vector<int> locality_order(const pgfem_mesh_desc *m) {
  const long ne = m->ne;
  std::vector<double> cen((size_t)3 * ne);
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (long e = 0; e < ne; e++)
    for (int d = 0; d < 3; d++) {
      double x = 0.0;
      for (int a = 0; a < 4; a++) x += m->X[(long)m->conn[e * m->nne + a] * 3 + d];
      x *= 0.25;
      cen[(size_t)3 * e + d] = x;
      lo[d] = std::min(lo[d], x);
      hi[d] = std::max(hi[d], x);
    }
  double vol = 1.0;
  for (int d = 0; d < 3; d++) vol *= std::max(hi[d] - lo[d], 1e-300);
  const double h = std::max(std::cbrt(6.0 * vol / (double)ne), 1e-300);
  int sw = 2;  // sweep axis: the longest (ties: the last)
  for (int d = 1; d >= 0; d--)
    if (hi[d] - lo[d] > hi[sw] - lo[sw]) sw = d;
  const int c1 = sw == 0 ? 1 : 0, c2 = sw == 2 ? 1 : 2;
  auto bin = [&](long e, int d) {
    const double v = (cen[(size_t)3 * e + d] - lo[d]) / h;
    return (long)std::min(std::max(v, 0.0), 1.0e6);
  };
  const long nb1 = (long)((hi[c1] - lo[c1]) / h) + 1, nb2 = (long)((hi[c2] - lo[c2]) / h) + 1;
  const long nbs = (long)((hi[sw] - lo[sw]) / h) + 1, T = 6;
  const long nc2 = (nb2 + T - 1) / T;
  std::vector<std::pair<unsigned long long, int>> key((size_t)ne);
  for (long e = 0; e < ne; e++) {
    const long b1 = bin(e, c1), b2 = bin(e, c2), bs = bin(e, sw);
    const unsigned long long col = (unsigned long long)((b1 / T) * nc2 + b2 / T);
    key[e].first = ((col * (unsigned long long)nbs + (unsigned long long)bs) * (unsigned long long)nb1 +
                    (unsigned long long)b1) * (unsigned long long)nb2 + (unsigned long long)b2;
    key[e].second = (int)e;
  }
  std::stable_sort(key.begin(), key.end(),
                   [](const std::pair<unsigned long long, int> &x, const std::pair<unsigned long long, int> &y) {
                     return x.first < y.first;
                   });
  std::vector<int> perm((size_t)ne);
  for (long e = 0; e < ne; e++) perm[e] = key[e].second;
  return perm;
}

}  // namespace

extern "C" {

int pgfem_gpu_state_size(int model) {
  switch (model) {
    case PGFEM_MODEL_J2: return 10;
    case PGFEM_MODEL_CP: return 10;
    default: return 0;
  }
}

int pgfem_gpu_create(const pgfem_mesh_desc *m, const pgfem_material_desc *mat, const int *Ap,
                     const int *Ai, long nrows, pgfem_gpu_ctx **out) {
  if (!m || !mat || !out || !m->X || !m->conn || !m->dof_id || (m->nne != 4 && m->nne != 10) ||
      m->nn <= 0 || m->ne <= 0 || nrows != m->ndof || !Ap || !Ai)
    return PGFEM_GPU_EINVAL;
  if (mat->model < 0 || mat->model > 2) return PGFEM_GPU_EINVAL;
  if (mat->dev_pot < 0 || mat->dev_pot > 2 || (mat->dev_pot == 2 && mat->model != PGFEM_MODEL_HE) ||
      !(mat->vol_pot <= 0 || mat->vol_pot == 99 || ((mat->vol_pot == 2 || mat->vol_pot == 3) && mat->model != PGFEM_MODEL_CP)))
    return PGFEM_GPU_EINVAL;
  if (mat->model == PGFEM_MODEL_CP && (m->nne != 4 || !m->R_cp || !(mat->m > 0) || !(mat->g0 > 0) ||
                                       !(mat->gs_0 > mat->g0)))
    return PGFEM_GPU_EINVAL;
  if (m->nn > 0x7fffffffL || m->ne > 0x7fffffffL) return PGFEM_GPU_ELIMIT;
  int r = check_device();
  if (r) return r;
  auto *c = new pgfem_gpu_ctx();
  c->nne = m->nne;
  c->nqp_e = m->nne == 10 ? 4 : 1;
  c->nn = m->nn;
  c->ne = m->ne;
  c->ndof = m->ndof;
  c->npres = m->npres;
  c->nnz = Ap[m->ndof];
  c->nqp = c->ne * c->nqp_e;
  c->model = mat->model;
  c->nstate = device_state_size(mat->model);
  c->mat = make_mat(mat);
  c->shp = make_shape(m->nne);
  cudaGetDevice(&c->device);
  auto fail = [&](int code) {
    cudaStreamSynchronize(c->stream);
    release(c);
    delete c;
    return code;
  };
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(PGFEM_GPU_ECUDA);

  // ---- host-side SoA + per-node row information ----
  const long nn = m->nn, ne = m->ne;
  std::vector<double> X(3 * nn);
  std::vector<int> dof(3 * nn), rowptr0(nn, -1), rowlen(nn, 0);
  std::vector<uint8_t> mask(nn, 0);
  for (long n = 0; n < nn; n++) {
    int first = -1, prev = -1;
    for (int j = 0; j < 3; j++) {
      X[j * nn + n] = m->X[n * 3 + j];
      const long id = m->dof_id[n * 3 + j];
      if (id > m->ndof || (id < 0 && -id > m->npres)) return fail(PGFEM_GPU_EINVAL);
      dof[j * nn + n] = (int)id;
      if (id > 0) {
        mask[n] |= (uint8_t)(1u << j);
        if (first < 0) first = (int)id - 1;
        else if (id - 1 != prev + 1) return fail(PGFEM_GPU_EPATTERN);
        prev = (int)id - 1;
      }
    }
    if (first >= 0) {
      rowptr0[n] = Ap[first];
      rowlen[n] = Ap[first + 1] - Ap[first];
      for (int k = 1; k < __builtin_popcount(mask[n]); k++)
        if (Ap[first + k + 1] - Ap[first + k] != rowlen[n] ||
            Ap[first + k] != rowptr0[n] + k * rowlen[n])
          return fail(PGFEM_GPU_EPATTERN);
    }
  }
  std::vector<int> conn((size_t)m->nne * ne);
  for (long e = 0; e < ne; e++)
    for (int a = 0; a < m->nne; a++) {
      const int v = m->conn[e * m->nne + a];
      if (v < 0 || v >= nn) return fail(PGFEM_GPU_EINVAL);
      conn[(size_t)a * ne + e] = v;
    }
  if ((r = upload(c, &c->X, X.data(), X.size())) || (r = upload(c, &c->dof, dof.data(), dof.size())) ||
      (r = upload(c, &c->rowptr0, rowptr0.data(), nn)) ||
      (r = upload(c, &c->rowlen, rowlen.data(), nn)) || (r = upload_mask(c, mask)) ||
      (r = upload(c, &c->conn, conn.data(), conn.size())))
    return fail(r);
  if (m->F0 && (r = upload(c, &c->F0, m->F0, 9))) return fail(r);
  if ((r = dalloc(c, &c->unode, 3 * nn)) || (r = dalloc(c, &c->status, 4)) ||
      (r = dalloc(c, &c->pos, (size_t)ne * m->nne * m->nne)))
    return fail(r);
  if (c->nstate) {
    if ((r = dalloc(c, &c->state_n, (size_t)c->nstate * c->nqp)) ||
        (r = dalloc(c, &c->state_np1, (size_t)c->nstate * c->nqp)))
      return fail(r);
    if (c->model == PGFEM_MODEL_CP && (r = dalloc(c, &c->state_nm1, (size_t)c->nstate * c->nqp))) return fail(r);
  }
  if (cudaMemsetAsync(c->status, 0, 4 * sizeof(unsigned long long), c->stream) != cudaSuccess)
    return fail(PGFEM_GPU_ECUDA);

  // ---- element->CSR map, built and validated on the device ----
  {
    int *dAi = nullptr, *derr = nullptr;
    if (cudaMalloc(&dAi, sizeof(int) * std::max<long>(1, c->nnz)) != cudaSuccess ||
        cudaMalloc(&derr, sizeof(int)) != cudaSuccess) {
      cudaGetLastError();
      if (dAi) cudaFree(dAi);
      return fail(PGFEM_GPU_ENOMEM);
    }
    cudaMemcpyAsync(dAi, Ai, sizeof(int) * c->nnz, cudaMemcpyHostToDevice, c->stream);
    cudaMemsetAsync(derr, 0, sizeof(int), c->stream);
    const long nt = ne * m->nne * m->nne;
    k_build_map<<<(unsigned)((nt + 255) / 256), 256, 0, c->stream>>>(
        c->conn, ne, m->nne, c->dof, nn, c->rowptr0, c->rowlen, c->mask, dAi, c->pos, derr);
    int herr = 0;
    cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    cudaError_t ce = cudaStreamSynchronize(c->stream);
    cudaFree(dAi);
    cudaFree(derr);
    if (ce != cudaSuccess) return fail(PGFEM_GPU_ECUDA);
    if (herr) return fail(PGFEM_GPU_EPATTERN);
  }
  // tensor-core quadratic-tet path: processing order, scatter blocks in that
  // order, the second stream that zeroes K
  if (m->nne == 10 && c->model != PGFEM_MODEL_CP && c->mat.dev_pot != 2) {
    std::vector<int> perm = locality_order(m);
    if ((r = upload(c, &c->perm, perm.data(), perm.size())) ||
        (r = dalloc(c, &c->eblk, (size_t)((ne + kMTE - 1) / kMTE) * kMTE * kEBW)) || (r = dalloc(c, &c->p2m_ticket, 1)))
      return fail(r);
    if (cudaStreamCreateWithFlags(&c->zstream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->zfork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->zjoin, cudaEventDisableTiming) != cudaSuccess)
      return fail(PGFEM_GPU_ECUDA);
    k_build_eblock<<<(unsigned)((ne + 127) / 128), 128, 0, c->stream>>>(c->conn, ne, c->dof, nn, c->rowptr0,
                                                                       c->rowlen, c->mask, c->pos, c->perm, c->eblk);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(c->stream) != cudaSuccess)
      return fail(PGFEM_GPU_ECUDA);
  }
  // crystal plasticity buffers (rotations SoA, F, point outputs)
  if (c->model == PGFEM_MODEL_CP) {
    std::vector<double> Rs((size_t)9 * ne);
    for (long e = 0; e < ne; e++)
      for (int i = 0; i < 9; i++) Rs[(size_t)i * ne + e] = m->R_cp[e * 9 + i];
    if ((r = upload(c, &c->cp_R, Rs.data(), Rs.size())) || (r = dalloc(c, &c->cp_F, (size_t)9 * ne)) ||
        (r = dalloc(c, &c->cp_detJw, ne)) || (r = dalloc(c, &c->cp_out, (size_t)kCpOut * c->nqp)) ||
        (r = dalloc(c, &c->cp_iters, c->nqp)) || (r = dalloc(c, &c->cp_counter, 1)) ||
        (r = dalloc(c, &c->cp_fallbacks, 1)) || (r = dalloc(c, &c->cp_conv, c->nqp)))
      return fail(r);
    std::vector<double> Fn((size_t)9 * c->nqp, 0.0);  // F at t_n: identity until the first commit
    for (long q = 0; q < c->nqp; q++) Fn[0 * c->nqp + q] = Fn[4 * c->nqp + q] = Fn[8 * c->nqp + q] = 1.0;
    if ((r = upload(c, &c->cp_Fn, Fn.data(), Fn.size()))) return fail(r);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(PGFEM_GPU_ECUDA);
  }
  // default state: identity Cp^-1 / pF, zero eqps, g = g0
  if (c->nstate) {
    std::vector<double> s0((size_t)c->nstate * c->nqp, 0.0);
    if (c->model == PGFEM_MODEL_J2)
      for (int k = 0; k < 3; k++) std::fill(s0.begin() + k * c->nqp, s0.begin() + (k + 1) * c->nqp, 1.0);
    if (c->model == PGFEM_MODEL_CP) {
      for (int k : {0, 4, 8}) std::fill(s0.begin() + k * c->nqp, s0.begin() + (k + 1) * c->nqp, 1.0);
      std::fill(s0.begin() + 9 * c->nqp, s0.end(), mat->g0);
    }
    cudaMemcpyAsync(c->state_n, s0.data(), s0.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(c->state_np1, s0.data(), s0.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (c->state_nm1)
      cudaMemcpyAsync(c->state_nm1, s0.data(), s0.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(PGFEM_GPU_ECUDA);
  }
  // colours for the deterministic scatter mode
  {
    std::vector<int> el;
    build_colours(m, el, c->colour_off);
    if ((r = upload(c, &c->colour_elems, el.data(), el.size()))) return fail(r);
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(PGFEM_GPU_ECUDA);
  }
  *out = c;
  return PGFEM_GPU_OK;
}

int pgfem_gpu_destroy(pgfem_gpu_ctx *c) {
  if (!c) return PGFEM_GPU_EINVAL;
  cudaStreamSynchronize(c->stream);
  release(c);
  delete c;
  return PGFEM_GPU_OK;
}

int pgfem_gpu_set_scatter_mode(pgfem_gpu_ctx *c, int mode) {
  if (!c || (mode != PGFEM_SCATTER_ATOMIC && mode != PGFEM_SCATTER_COLOUR)) return PGFEM_GPU_EINVAL;
  c->scatter_mode = mode;
  return PGFEM_GPU_OK;
}

// ---- three-field (CM3F) element -------------------------------------------

static int ensure_scratch(pgfem_gpu_ctx *c, bool wantK);

int pgfem_gpu_set_three_field(pgfem_gpu_ctx *c, const double *P, const double *theta) {
  if (!c) return PGFEM_GPU_EINVAL;
  if (!P && !theta) {
    c->three_field = 0;
    return PGFEM_GPU_OK;
  }
  if (!P || !theta) return PGFEM_GPU_EINVAL;
  if (c->nne != 10 || (c->model != PGFEM_MODEL_HE && c->model != PGFEM_MODEL_J2) || !uses_p2m(c) ||
      c->elem_group)
    return PGFEM_GPU_EINVAL;
  for (long e = 0; e < c->ne; e++)
    if (!(theta[e] > 0.0) || !std::isfinite(theta[e]) || !std::isfinite(P[e])) return PGFEM_GPU_EINVAL;
  int r;
  if (!c->tf_P && ((r = dalloc(c, &c->tf_P, c->ne)) || (r = dalloc(c, &c->tf_theta, c->ne)))) return r;
  CK(cudaMemcpyAsync(c->tf_P, P, sizeof(double) * c->ne, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->tf_theta, theta, sizeof(double) * c->ne, cudaMemcpyHostToDevice, c->stream));
  if (!c->tf_hist) {  // the history starts at the given values
    if ((r = dalloc(c, &c->tf_hist, (size_t)4 * c->ne))) return r;
    for (int k = 0; k < 2; k++) {
      CK(cudaMemcpyAsync(c->tf_hist + (size_t)2 * k * c->ne, P, sizeof(double) * c->ne, cudaMemcpyHostToDevice,
                         c->stream));
      CK(cudaMemcpyAsync(c->tf_hist + (size_t)(2 * k + 1) * c->ne, theta, sizeof(double) * c->ne,
                         cudaMemcpyHostToDevice, c->stream));
    }
  }
  CK(cudaStreamSynchronize(c->stream));
  c->three_field = 1;
  return PGFEM_GPU_OK;
}

int pgfem_gpu_set_three_field_history(pgfem_gpu_ctx *c, const double *P_n, const double *theta_n,
                                      const double *P_nm1, const double *theta_nm1) {
  if (!c || !c->three_field || !c->tf_hist || !P_n || !theta_n || !P_nm1 || !theta_nm1) return PGFEM_GPU_EINVAL;
  for (long e = 0; e < c->ne; e++)
    if (!(theta_n[e] > 0.0) || !(theta_nm1[e] > 0.0) || !std::isfinite(theta_n[e]) ||
        !std::isfinite(theta_nm1[e]) || !std::isfinite(P_n[e]) || !std::isfinite(P_nm1[e]))
      return PGFEM_GPU_EINVAL;
  const double *src[4] = {P_n, theta_n, P_nm1, theta_nm1};
  for (int k = 0; k < 4; k++)
    CK(cudaMemcpyAsync(c->tf_hist + (size_t)k * c->ne, src[k], sizeof(double) * c->ne, cudaMemcpyHostToDevice,
                       c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGFEM_GPU_OK;
}

int pgfem_gpu_three_field_enabled(const pgfem_gpu_ctx *c) { return c && c->three_field ? 1 : 0; }

// The local update on device buffers: increments into d_out (2 ne: dP then
// d_theta), or, with d_out NULL, added to the context's P and theta.
__global__ void k_tf_apply(long ne, const double *inc, double *P, double *theta) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  P[e] += inc[e];
  theta[e] += inc[ne + e];
}

int pgfem_gpu_three_field_update_device(pgfem_gpu_ctx *c, const double *d_u, const double *d_presc,
                                        const double *d_du, double *d_out, void *stream) {
  if (!c || !c->three_field || (c->ndof && (!d_u || !d_du)) || (c->npres && !d_presc)) return PGFEM_GPU_EINVAL;
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  int r;
  if (!c->tf_dunode && ((r = dalloc(c, &c->tf_dunode, 3 * c->nn)) || (r = dalloc(c, &c->tf_inc, 2 * c->ne))))
    return r;
  const long n3 = 3 * c->nn;
  k_expand_u<<<(unsigned)((n3 + 255) / 256), 256, 0, s>>>(c->dof, c->nn, d_u, d_presc, c->unode);
  k_expand_u<<<(unsigned)((n3 + 255) / 256), 256, 0, s>>>(c->dof, c->nn, d_du, nullptr, c->tf_dunode);
  QpArgs q{};
  q.X = c->X;
  q.unode = c->unode;
  q.conn = c->conn;
  q.nn = c->nn;
  q.ne = c->ne;
  q.F0 = c->F0;
  q.status = c->status;
  q.mat = c->mat;
  q.shp = c->shp;
  q.tf_P = c->tf_P;
  q.tf_theta = c->tf_theta;
  double *inc = d_out ? d_out : c->tf_inc;
  const unsigned g = (unsigned)((c->ne + 127) / 128);
  k_tf_update<<<g, 128, 0, s>>>(q, c->tf_dunode, inc, inc + c->ne);
  if (!d_out) k_tf_apply<<<g, 128, 0, s>>>(c->ne, inc, c->tf_P, c->tf_theta);
  CK(cudaGetLastError());
  return PGFEM_GPU_OK;
}

int pgfem_gpu_three_field_increments(pgfem_gpu_ctx *c, const double *u, const double *presc, const double *du,
                                     double *dP, double *dtheta, pgfem_gpu_status *st) {
  if (!c || !c->three_field || !u || !du || !dP || !dtheta || (c->npres && !presc)) return PGFEM_GPU_EINVAL;
  int r = ensure_scratch(c, false);
  if (r) return r;
  if (!c->tf_dunode && ((r = dalloc(c, &c->tf_dunode, 3 * c->nn)) || (r = dalloc(c, &c->tf_inc, 2 * c->ne))))
    return r;
  // du staged in the residual scratch
  CK(cudaMemcpyAsync(c->d_u, u, sizeof(double) * c->ndof, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_R, du, sizeof(double) * c->ndof, cudaMemcpyHostToDevice, c->stream));
  if (c->npres)
    CK(cudaMemcpyAsync(c->d_presc, presc, sizeof(double) * c->npres, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->status, 0, 4 * sizeof(unsigned long long), c->stream));
  if ((r = pgfem_gpu_three_field_update_device(c, c->d_u, c->npres ? c->d_presc : nullptr, c->d_R, c->tf_inc,
                                               c->stream)))
    return r;
  CK(cudaMemcpyAsync(dP, c->tf_inc, sizeof(double) * c->ne, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(dtheta, c->tf_inc + c->ne, sizeof(double) * c->ne, cudaMemcpyDeviceToHost, c->stream));
  return read_status(c, st, false);
}

int pgfem_gpu_get_three_field(pgfem_gpu_ctx *c, double *P, double *theta) {
  if (!c || !c->three_field || !P || !theta) return PGFEM_GPU_EINVAL;
  CK(cudaMemcpyAsync(P, c->tf_P, sizeof(double) * c->ne, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(theta, c->tf_theta, sizeof(double) * c->ne, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGFEM_GPU_OK;
}

int pgfem_gpu_set_neumann(pgfem_gpu_ctx *c, long nface, const long *elem, const int *face,
                          const int *feature, int nfeature, const int *load_type, const double *load_np1) {
  if (!c || nface < 0 || nfeature < 0 || (nface && (!elem || !face || !feature || !nfeature)) ||
      (nfeature && (!load_type || !load_np1)))
    return PGFEM_GPU_EINVAL;
  for (long k = 0; k < nface; k++)
    if (elem[k] < 0 || elem[k] >= c->ne || face[k] < 0 || face[k] > 3 || feature[k] < 0 || feature[k] >= nfeature)
      return PGFEM_GPU_EINVAL;
  for (int f = 0; f < nfeature; f++)
    if (load_type[f] < 1 || load_type[f] > 3) return PGFEM_GPU_EINVAL;
  CK(cudaStreamSynchronize(c->stream));  // earlier assemblies may still read the old lists
  int *old[] = {c->nbc_elem, c->nbc_feat, c->nbc_type, c->nbc_off};
  for (int *p : old)
    if (p) cudaFree(p);
  if (c->nbc_face) cudaFree(c->nbc_face);
  if (c->nbc_load) cudaFree(c->nbc_load);
  if (c->nbc_desc_tr) {
    cudaFree(c->nbc_desc_tr);
    c->bytes -= (long)(sizeof(double) * 2 * kNbcDesc * c->nbc_nfeat);
  }
  c->nbc_elem = c->nbc_feat = c->nbc_type = c->nbc_off = nullptr;
  c->nbc_face = nullptr;
  c->nbc_load = c->nbc_desc_tr = nullptr;
  c->nbc_desc_cur = nullptr;
  c->nbc_type_h.clear();
  c->nbc_load_h.clear();
  c->nbc_hist_n.clear();
  c->nbc_hist_nm1.clear();
  c->nbc_nface = 0;
  c->nbc_nfeat = 0;
  c->bytes -= c->nbc_bytes;
  c->nbc_bytes = 0;
  if (!nface) return PGFEM_GPU_OK;
  const long bytes0 = c->bytes;
  // faces in element order (stable), per-element offsets
  std::vector<long> order(nface);
  for (long k = 0; k < nface; k++) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](long x, long y) { return elem[x] < elem[y]; });
  std::vector<int> fe_(nface), ff(nface), off(c->ne + 1, 0);
  std::vector<uint8_t> fi(nface);
  for (long k = 0; k < nface; k++) {
    fe_[k] = (int)elem[order[k]];
    fi[k] = (uint8_t)face[order[k]];
    ff[k] = feature[order[k]];
    off[fe_[k] + 1]++;
  }
  for (long e = 0; e < c->ne; e++) off[e + 1] += off[e];
  std::vector<double> ld((size_t)kNbcDesc * nfeature);
  for (int f = 0; f < nfeature; f++) nbc_desc_static(load_type[f], load_np1 + (size_t)3 * f, &ld[(size_t)kNbcDesc * f]);
  int r;
  if ((r = upload(c, &c->nbc_elem, fe_.data(), fe_.size())) || (r = upload(c, &c->nbc_face, fi.data(), fi.size())) ||
      (r = upload(c, &c->nbc_feat, ff.data(), ff.size())) || (r = upload(c, &c->nbc_type, load_type, nfeature)) ||
      (r = upload(c, &c->nbc_load, ld.data(), ld.size())) || (r = upload(c, &c->nbc_off, off.data(), off.size()))) {
    c->nbc_bytes = c->bytes - bytes0;  // freed by the next call or at destroy
    return r;
  }
  c->nbc_bytes = c->bytes - bytes0;
  CK(cudaStreamSynchronize(c->stream));
  c->nbc_nface = nface;
  c->nbc_nfeat = nfeature;
  c->nbc_type_h.assign(load_type, load_type + nfeature);
  c->nbc_load_h.assign(load_np1, load_np1 + (size_t)3 * nfeature);
  return PGFEM_GPU_OK;
}

int pgfem_gpu_set_neumann_loads(pgfem_gpu_ctx *c, int nfeature, const double *load_np1) {
  if (!c || nfeature != c->nbc_nfeat || (nfeature && !load_np1)) return PGFEM_GPU_EINVAL;
  if (!nfeature) return PGFEM_GPU_OK;
  std::vector<double> ld((size_t)kNbcDesc * nfeature);
  for (int f = 0; f < nfeature; f++)
    nbc_desc_static(c->nbc_type_h[f], load_np1 + (size_t)3 * f, &ld[(size_t)kNbcDesc * f]);
  CK(cudaMemcpyAsync(c->nbc_load, ld.data(), sizeof(double) * ld.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->nbc_load_h.assign(load_np1, load_np1 + (size_t)3 * nfeature);
  return PGFEM_GPU_OK;
}

int pgfem_gpu_set_neumann_load_history(pgfem_gpu_ctx *c, int nfeature, const double *load_n,
                                       const double *load_nm1) {
  if (!c || nfeature != c->nbc_nfeat || (nfeature && (!load_n || !load_nm1))) return PGFEM_GPU_EINVAL;
  c->nbc_hist_n.assign(load_n, load_n + (size_t)3 * nfeature);
  c->nbc_hist_nm1.assign(load_nm1, load_nm1 + (size_t)3 * nfeature);
  return PGFEM_GPU_OK;
}

int pgfem_gpu_set_wait_test(pgfem_gpu_ctx *c, double limit_s, int stall_next_assembly) {
  if (!c || !(limit_s > 0.0) || limit_s > 60.0) return PGFEM_GPU_EINVAL;
  c->wait_ns = (unsigned long long)(limit_s * 1e9);
  c->stall_next = stall_next_assembly ? 1 : 0;
  return PGFEM_GPU_OK;
}

long pgfem_gpu_device_bytes(const pgfem_gpu_ctx *c) { return c ? c->bytes : -1; }
long pgfem_gpu_nnz(const pgfem_gpu_ctx *c) { return c ? c->nnz : -1; }

int pgfem_gpu_launches_per_assembly(const pgfem_gpu_ctx *c) {
  if (!c) return -1;
  const int nbc = c->nbc_nface ? 1 : 0;  // the surface-load kernel
  if (c->model == PGFEM_MODEL_CP)  // u expansion, F, local Newton, tangent, element (+ features, network, guess)
    return (c->cp_net ? 8 : 5) + nbc;
  if (c->mat.dev_pot == 2)  // u expansion + per-node kernel launches (one per colour in colour mode)
    return 1 + (c->scatter_mode == PGFEM_SCATTER_COLOUR ? (int)c->colour_off.size() - 1 : 1) + nbc;
  if (c->nne == 10 && c->scatter_mode == PGFEM_SCATTER_ATOMIC)
    return 3 + nbc;  // u expansion, point updates, tensor-core R+K assembly
  if (c->nne == 4 && c->scatter_mode == PGFEM_SCATTER_ATOMIC)
    return 3 + nbc;  // u expansion, point updates, column-split R+K assembly
  const int nasm = c->scatter_mode == PGFEM_SCATTER_COLOUR ? (int)c->colour_off.size() - 1 : 1;
  return 1 + nasm + nbc;  // u expansion + assembly launches (memsets are not kernels of ours)
}

int pgfem_gpu_set_cp_guess(pgfem_gpu_ctx *c, const double *guess) {
  if (!c || c->model != PGFEM_MODEL_CP) return PGFEM_GPU_EINVAL;
  if (!guess) {
    c->cp_use_guess = false;
    return PGFEM_GPU_OK;
  }
  int r;
  if (!c->cp_guess && (r = dalloc(c, &c->cp_guess, (size_t)10 * c->nqp))) return r;
  std::vector<double> soa((size_t)10 * c->nqp);
  for (long q = 0; q < c->nqp; q++)
    for (int k = 0; k < 10; k++) soa[(size_t)k * c->nqp + q] = guess[q * 10 + k];
  CK(cudaMemcpyAsync(c->cp_guess, soa.data(), soa.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->cp_use_guess = true;
  return PGFEM_GPU_OK;
}

int pgfem_gpu_get_cp_iterations(pgfem_gpu_ctx *c, int *iters, double *dgam) {
  if (!c || c->model != PGFEM_MODEL_CP || !iters) return PGFEM_GPU_EINVAL;
  CK(cudaMemcpyAsync(iters, c->cp_iters, sizeof(int) * c->nqp, cudaMemcpyDeviceToHost, c->stream));
  if (dgam) {
    std::vector<double> soa((size_t)12 * c->nqp);
    CK(cudaMemcpyAsync(soa.data(), c->cp_out + (size_t)91 * c->nqp, soa.size() * sizeof(double),
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (long q = 0; q < c->nqp; q++)
      for (int a = 0; a < 12; a++) dgam[q * 12 + a] = soa[(size_t)a * c->nqp + q];
  }
  CK(cudaStreamSynchronize(c->stream));
  return PGFEM_GPU_OK;
}

int pgfem_gpu_set_cp_warm_limit(pgfem_gpu_ctx *c, int k) {
  if (!c || c->model != PGFEM_MODEL_CP || k < 0) return PGFEM_GPU_EINVAL;
  c->cp_warm_k = k;
  return PGFEM_GPU_OK;
}

int pgfem_gpu_set_cp_surrogate(pgfem_gpu_ctx *c, pgfem_mlp *m) {
  if (!c || c->model != PGFEM_MODEL_CP) return PGFEM_GPU_EINVAL;
  if (m) {
    int r;
    if (!c->cp_guess && (r = dalloc(c, &c->cp_guess, (size_t)10 * c->nqp))) return r;
    if (!c->cp_feat && (r = dalloc(c, &c->cp_feat, (size_t)kCpFeat * c->nqp))) return r;
    if (!c->cp_pred && (r = dalloc(c, &c->cp_pred, (size_t)kSlip * c->nqp))) return r;
  }
  c->cp_net = m;
  return PGFEM_GPU_OK;
}

int pgfem_gpu_cp_training_pairs(pgfem_gpu_ctx *c, float *d_x, float *d_t) {
  if (!c || c->model != PGFEM_MODEL_CP || !d_x || !d_t) return PGFEM_GPU_EINVAL;
  const unsigned blk = (unsigned)((c->nqp + 127) / 128);
  k_cp_features<<<blk, 128, 0, c->stream>>>(c->nqp, c->cp_F, c->cp_Fn, c->state_n, c->cp_R, 1, c->ne, d_x);
  CK(cudaGetLastError());
  k_cp_targets<<<blk, 128, 0, c->stream>>>(c->nqp, c->cp_out, d_t);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return PGFEM_GPU_OK;
}

int pgfem_gpu_get_cp_fallbacks(pgfem_gpu_ctx *c, long *n) {
  if (!c || c->model != PGFEM_MODEL_CP || !n) return PGFEM_GPU_EINVAL;
  unsigned long long v = 0;
  CK(cudaMemcpyAsync(&v, c->cp_fallbacks, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *n = (long)v;
  return PGFEM_GPU_OK;
}

int pgfem_gpu_set_timing(pgfem_gpu_ctx *c, int on) {
  if (!c) return PGFEM_GPU_EINVAL;
  c->timing = on != 0;
  return PGFEM_GPU_OK;
}

int pgfem_gpu_kernel_time(pgfem_gpu_ctx *c, double *ms, long *ncalls, int reset) {
  if (!c || !ms) return PGFEM_GPU_EINVAL;
  double tot = 0.0;
  for (auto &p : c->events) {
    CK(cudaEventSynchronize(p.second));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, p.first, p.second));
    tot += t;
  }
  *ms = tot;
  if (ncalls) *ncalls = (long)c->events.size();
  if (reset) drop_events(c);
  return PGFEM_GPU_OK;
}

int pgfem_gpu_fp64_peak(double *tflops) {
  if (!tflops) return PGFEM_GPU_EINVAL;
  int r = check_device();
  if (r) return r;
  return fp64_peak_probe(tflops);
}

int pgfem_gpu_binary_version(int *version) {
  if (!version) return PGFEM_GPU_EINVAL;
  int r = check_device();
  if (r) return r;
  cudaFuncAttributes fa;
  CK(cudaFuncGetAttributes(&fa, k_expand_u));
  *version = fa.binaryVersion;
  return PGFEM_GPU_OK;
}

int pgfem_gpu_set_state(pgfem_gpu_ctx *c, const double *st) {
  if (!c || !st) return PGFEM_GPU_EINVAL;
  if (!c->nstate) return PGFEM_GPU_OK;
  const long nq = c->nqp;
  std::vector<double> soa((size_t)c->nstate * nq);
  for (long q = 0; q < nq; q++) {
    const double *s = st + q * 10;
    if (c->model == PGFEM_MODEL_J2) {
      const double v[7] = {s[0], s[4], s[8], s[5], s[2], s[1], s[9]};
      for (int k = 0; k < 7; k++) soa[k * nq + q] = v[k];
    } else {
      for (int k = 0; k < 10; k++) soa[k * nq + q] = s[k];
    }
  }
  CK(cudaMemcpyAsync(c->state_n, soa.data(), soa.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->state_np1, c->state_n, soa.size() * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  if (c->state_nm1)
    CK(cudaMemcpyAsync(c->state_nm1, c->state_n, soa.size() * sizeof(double), cudaMemcpyDeviceToDevice,
                       c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGFEM_GPU_OK;
}

int pgfem_gpu_set_state_nm1(pgfem_gpu_ctx *c, const double *st) {
  if (!c || !st) return PGFEM_GPU_EINVAL;
  if (!c->state_nm1) return PGFEM_GPU_EINVAL;  // crystal plasticity only
  const long nq = c->nqp;
  std::vector<double> soa((size_t)10 * nq);
  for (long q = 0; q < nq; q++)
    for (int k = 0; k < 10; k++) soa[k * nq + q] = st[q * 10 + k];
  CK(cudaMemcpyAsync(c->state_nm1, soa.data(), soa.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGFEM_GPU_OK;
}

int pgfem_gpu_get_state(pgfem_gpu_ctx *c, int level, double *st) {
  if (!c || !st || level < 0 || level > 2 || (level == 2 && !c->state_nm1)) return PGFEM_GPU_EINVAL;
  if (!c->nstate) return PGFEM_GPU_OK;
  const long nq = c->nqp;
  std::vector<double> soa((size_t)c->nstate * nq);
  const double *src = level == 2 ? c->state_nm1 : level ? c->state_np1 : c->state_n;
  CK(cudaMemcpyAsync(soa.data(), src, soa.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (long q = 0; q < nq; q++) {
    double *s = st + q * 10;
    if (c->model == PGFEM_MODEL_J2) {
      const double xx = soa[0 * nq + q], yy = soa[1 * nq + q], zz = soa[2 * nq + q],
                   yz = soa[3 * nq + q], xz = soa[4 * nq + q], xy = soa[5 * nq + q];
      const double v[10] = {xx, xy, xz, xy, yy, yz, xz, yz, zz, soa[6 * nq + q]};
      for (int k = 0; k < 10; k++) s[k] = v[k];
    } else {
      for (int k = 0; k < 10; k++) s[k] = soa[k * nq + q];
    }
  }
  return PGFEM_GPU_OK;
}

int pgfem_gpu_commit_state(pgfem_gpu_ctx *c) {
  if (!c) return PGFEM_GPU_EINVAL;
  if (c->state_nm1)  // n-1 <- n first
    CK(cudaMemcpyAsync(c->state_nm1, c->state_n, sizeof(double) * c->nstate * c->nqp, cudaMemcpyDeviceToDevice,
                       c->stream));
  if (c->three_field && c->tf_hist) {  // three-field P, theta: n-1 <- n <- the current values
    CK(cudaMemcpyAsync(c->tf_hist + (size_t)2 * c->ne, c->tf_hist, sizeof(double) * 2 * c->ne,
                       cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->tf_hist, c->tf_P, sizeof(double) * c->ne, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->tf_hist + c->ne, c->tf_theta, sizeof(double) * c->ne, cudaMemcpyDeviceToDevice,
                       c->stream));
  }
  if (c->nstate)
    CK(cudaMemcpyAsync(c->state_n, c->state_np1, sizeof(double) * c->nstate * c->nqp,
                       cudaMemcpyDeviceToDevice, c->stream));
  if (c->cp_Fn)  // F of the converged iterate becomes F_n (warm-start features)
    CK(cudaMemcpyAsync(c->cp_Fn, c->cp_F, sizeof(double) * 9 * c->nqp, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGFEM_GPU_OK;
}

int pgfem_gpu_reset_state(pgfem_gpu_ctx *c) {
  if (!c) return PGFEM_GPU_EINVAL;
  if (c->nstate)
    CK(cudaMemcpyAsync(c->state_np1, c->state_n, sizeof(double) * c->nstate * c->nqp,
                       cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return PGFEM_GPU_OK;
}

static int ensure_scratch(pgfem_gpu_ctx *c, bool wantK);

// Nodal totals (AoS nn*3) and point F (AoS nqp*9) of a free-DOF displacement
// and the prescribed values.
static int nodal_and_F(pgfem_gpu_ctx *c, const double *u, const double *presc, std::vector<double> &nodal,
                       std::vector<double> &F) {
  int r = ensure_scratch(c, false);
  if (r) return r;
  cudaStream_t s = c->stream;
  if (c->ndof) CK(cudaMemcpyAsync(c->d_u, u, sizeof(double) * c->ndof, cudaMemcpyHostToDevice, s));
  if (c->npres && presc) CK(cudaMemcpyAsync(c->d_presc, presc, sizeof(double) * c->npres, cudaMemcpyHostToDevice, s));
  const long n3 = 3 * c->nn;
  k_expand_u<<<(unsigned)((n3 + 255) / 256), 256, 0, s>>>(c->dof, c->nn, c->d_u, presc ? c->d_presc : nullptr,
                                                          c->unode);
  CK(cudaGetLastError());
  double *dF = nullptr;
  if (cudaMalloc(&dF, sizeof(double) * 9 * c->nqp) != cudaSuccess) {
    cudaGetLastError();
    return PGFEM_GPU_ENOMEM;
  }
  k_point_F<<<(unsigned)((c->nqp + 127) / 128), 128, 0, s>>>(c->X, c->conn, c->nn, c->ne, c->nne, c->nqp_e, c->unode,
                                                             c->shp, c->F0, c->elem_group, c->F0_tab, dF);
  std::vector<double> soa((size_t)n3);
  F.resize((size_t)9 * c->nqp);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(soa.data(), c->unode, sizeof(double) * n3, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(F.data(), dF, sizeof(double) * 9 * c->nqp, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(dF);
  if (e != cudaSuccess) return PGFEM_GPU_ECUDA;
  nodal.resize((size_t)n3);
  for (long n = 0; n < c->nn; n++)
    for (int b = 0; b < 3; b++) nodal[3 * n + b] = soa[(size_t)b * c->nn + n];
  return PGFEM_GPU_OK;
}

// Slip systems of the reference's restart output in terms of this library's
// FCC table: system a of the file is sign * (system kRefSys[a] here), as its
// own restart files show (every element of its crystal plasticity tension
// case, ref_out_tension/box_<r>_49.res).
static const int kRefSys[12] = {2, 0, 1, 5, 4, 3, 8, 6, 7, 9, 10, 11};
static const double kRefSgn[12] = {1, -1, 1, 1, 1, -1, 1, 1, -1, 1, 1, 1};
// host copies of the FCC slip table of cp_kernels.cuh (directions <110>,
// normals {111}, unnormalised) and the 3x3 helpers the host needs
static const double kHostSlipS[12][3] = {{0, 1, -1}, {1, 0, -1}, {1, -1, 0}, {0, 1, -1}, {1, 0, 1}, {1, 1, 0},
                                         {0, 1, 1},  {1, 0, -1}, {1, 1, 0},  {0, 1, 1},  {1, 0, 1}, {1, -1, 0}};
static const double kHostSlipN[12][3] = {{1, 1, 1},  {1, 1, 1},  {1, 1, 1},  {-1, 1, 1}, {-1, 1, 1}, {-1, 1, 1},
                                         {1, -1, 1}, {1, -1, 1}, {1, -1, 1}, {1, 1, -1}, {1, 1, -1}, {1, 1, -1}};
static double h_det3(const double *a) {
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) + a[2] * (a[3] * a[7] - a[4] * a[6]);
}
static bool h_inv3(const double *a, double *b) {
  const double d = h_det3(a);
  if (d == 0.0 || !std::isfinite(d)) return false;
  const double id = 1.0 / d;
  b[0] = (a[4] * a[8] - a[5] * a[7]) * id, b[1] = (a[2] * a[7] - a[1] * a[8]) * id;
  b[2] = (a[1] * a[5] - a[2] * a[4]) * id, b[3] = (a[5] * a[6] - a[3] * a[8]) * id;
  b[4] = (a[0] * a[8] - a[2] * a[6]) * id, b[5] = (a[2] * a[3] - a[0] * a[5]) * id;
  b[6] = (a[3] * a[7] - a[4] * a[6]) * id, b[7] = (a[1] * a[6] - a[0] * a[7]) * id;
  b[8] = (a[0] * a[4] - a[1] * a[3]) * id;
  return true;
}
static void h_mm3(const double *A, const double *B, double *C, bool transA) {  // C = op(A) B
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double v = 0.0;
      for (int k = 0; k < 3; k++) v += (transA ? A[k * 3 + i] : A[i * 3 + k]) * B[k * 3 + j];
      C[i * 3 + j] = v;
    }
}

static int cp_resolved_shear_mat(const Mat &m, long n, const double *F, const double *pF, const double *g,
                                 const double *R, double *tau, double *gdot) {
  for (long q = 0; q < n; q++) {
    double pFi[9], Fe[9], C[9], Ci[9];
    if (!h_inv3(pF + 9 * q, pFi)) return PGFEM_GPU_EINVAL;
    h_mm3(F + 9 * q, pFi, Fe, false);
    h_mm3(Fe, Fe, C, true);
    const double detC = h_det3(C);
    if (!(detC > 0.0) || !h_inv3(C, Ci)) return PGFEM_GPU_EINVAL;
    // neo-Hookean + U_Common: S = mu detC^-1/3 (I - trC/3 C^-1) + kappa J (J - 1) C^-1
    const double J = std::sqrt(detC), a = m.mu / std::cbrt(detC), pv = m.kappa * J * (J - 1.0);
    const double trC = C[0] + C[4] + C[8];
    double S[9], CS[9];
    for (int i = 0; i < 9; i++) S[i] = a * ((i % 4 == 0 ? 1.0 : 0.0) - trC / 3.0 * Ci[i]) + pv * Ci[i];
    h_mm3(C, S, CS, false);
    double t[12];
    const double *Rq = R + 9 * q, is2 = 0.70710678118654752440, is3 = 0.57735026918962576451;
    for (int sy = 0; sy < 12; sy++) {  // sample-frame s = R s0, n = R n0; tau = s . (C S) n
      double sv[3], nv[3];
      for (int i = 0; i < 3; i++) {
        sv[i] = (Rq[i * 3] * kHostSlipS[sy][0] + Rq[i * 3 + 1] * kHostSlipS[sy][1] + Rq[i * 3 + 2] * kHostSlipS[sy][2]) * is2;
        nv[i] = (Rq[i * 3] * kHostSlipN[sy][0] + Rq[i * 3 + 1] * kHostSlipN[sy][1] + Rq[i * 3 + 2] * kHostSlipN[sy][2]) * is3;
      }
      double v = 0.0;
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) v += CS[i * 3 + j] * (sv[i] * nv[j]);
      t[sy] = v;
    }
    for (int k = 0; k < 12; k++) {
      const double tk = kRefSgn[k] * t[kRefSys[k]];
      tau[12 * q + k] = tk;
      if (gdot) {  // the flow rule at t_n: gamma_dot_0 (tau/g) |tau/g|^(1/m - 1)
        const double r = tk / g[q];
        gdot[12 * q + k] = m.gdot0 * r * std::pow(std::fabs(r), 1.0 / m.m - 1.0);
      }
    }
  }
  return PGFEM_GPU_OK;
}

int pgfem_cp_resolved_shear(const pgfem_material_desc *mat, long n, const double *F, const double *pF,
                            const double *g, const double *R, double *tau, double *gdot) {
  if (!mat || n < 0 || (n && (!F || !pF || !g || !R || !tau))) return PGFEM_GPU_EINVAL;
  return cp_resolved_shear_mat(make_mat(mat), n, F, pF, g, R, tau, gdot);
}

int pgfem_gpu_write_restart(pgfem_gpu_ctx *c, const char *path, const double *u_nm1, const double *u_n,
                            const double *presc_nm1, const double *presc_n, const double *state_nm1) {
  if (!c || !path || (c->ndof && (!u_nm1 || !u_n)) || (c->npres && (!presc_nm1 || !presc_n)))
    return PGFEM_GPU_EINVAL;
  std::vector<double> un1, un, Fn1, Fn;
  int r;
  if ((r = nodal_and_F(c, u_nm1, presc_nm1, un1, Fn1)) || (r = nodal_and_F(c, u_n, presc_n, un, Fn))) return r;
  const int bs = pgfem_restart_block_size(c->model);
  std::vector<double> blocks((size_t)bs * c->nqp, 0.0);
  std::vector<double> st, taus, gdots;
  if (c->model == PGFEM_MODEL_CP || c->model == PGFEM_MODEL_J2) {
    st.resize((size_t)10 * c->nqp);
    if ((r = pgfem_gpu_get_state(c, 0, st.data()))) return r;
  }
  if (c->model == PGFEM_MODEL_CP) {  // resolved shears and slip rates at t_n
    std::vector<double> Rs((size_t)9 * c->ne), Rq((size_t)9 * c->nqp), pFq((size_t)9 * c->nqp), gq(c->nqp);
    CK(cudaMemcpyAsync(Rs.data(), c->cp_R, sizeof(double) * Rs.size(), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (long q = 0; q < c->nqp; q++) {
      const long e = q / c->nqp_e;
      for (int i = 0; i < 9; i++) {
        Rq[9 * q + i] = Rs[(size_t)i * c->ne + e];
        pFq[9 * q + i] = st[10 * q + i];
      }
      gq[q] = st[10 * q + 9];
    }
    taus.resize((size_t)12 * c->nqp);
    gdots.resize((size_t)12 * c->nqp);
    if ((r = cp_resolved_shear_mat(c->mat, c->nqp, Fn.data(), pFq.data(), gq.data(), Rq.data(), taus.data(),
                                   gdots.data())))
      return r;
  }
  for (long q = 0; q < c->nqp; q++) {
    double *b = blocks.data() + (size_t)bs * q;
    if (c->model == PGFEM_MODEL_J2) {
      // the reference's plastic stress pS <-> this path's Cp^-1: pS = G (I - Cp^-1)
      // (zero in the initial state, as the reference's set_init_vals); the damage
      // variables are written at their undamaged values, gam_n = sqrt(3/2)(ep_n - ep_nm1)
      const double *sn = st.data() + 10 * q, *sm = state_nm1 ? state_nm1 + 10 * q : sn;
      const double G = c->mat.mu;
      for (int k = 0; k < 9; k++) {
        const double I = (k % 4 == 0) ? 1.0 : 0.0;
        b[k] = Fn[9 * q + k];
        b[9 + k] = G * (I - sn[k]);
        b[18 + k] = Fn1[9 * q + k];
        b[27 + k] = G * (I - sm[k]);
      }
      b[42] = sn[9];
      b[43] = sm[9];
      b[44] = std::sqrt(1.5) * (sn[9] - sm[9]);
      continue;
    }
    for (int k = 0; k < 9; k++) {
      b[k] = Fn[9 * q + k];
      b[9 + k] = Fn1[9 * q + k];
    }
    if (c->model == PGFEM_MODEL_CP) {
      const double *sn = st.data() + 10 * q, *sm = state_nm1 ? state_nm1 + 10 * q : sn;
      for (int k = 0; k < 9; k++) {
        b[18 + k] = sn[k];
        b[27 + k] = sm[k];
      }
      for (int k = 0; k < 12; k++) {
        b[36 + k] = taus[(size_t)12 * q + k];
        b[48 + k] = gdots[(size_t)12 * q + k];
      }
      b[60] = sn[9];
      b[61] = sm[9];  // L_n, L_nm1 (a multiplier of the reference's integrator): 0
    }
  }
  return pgfem_restart_format(path, c->nn, c->ne, c->nqp_e, c->model, un1.data(), un.data(), blocks.data());
}

int pgfem_gpu_read_restart(pgfem_gpu_ctx *c, const char *path, double *u_nm1, double *u_n) {
  if (!c || !path || (c->ndof && (!u_nm1 || !u_n))) return PGFEM_GPU_EINVAL;
  const int bs = pgfem_restart_block_size(c->model);
  std::vector<double> un1((size_t)3 * c->nn), un((size_t)3 * c->nn), blocks((size_t)bs * c->nqp);
  int r = pgfem_restart_parse(path, c->nn, c->ne, c->nqp_e, c->model, un1.data(), un.data(), blocks.data());
  if (r) return r;
  std::vector<int> dof((size_t)3 * c->nn);
  CK(cudaMemcpyAsync(dof.data(), c->dof, sizeof(int) * dof.size(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (long n = 0; n < c->nn; n++)
    for (int b = 0; b < 3; b++) {
      const int id = dof[(size_t)b * c->nn + n];
      if (id > 0) {
        u_nm1[id - 1] = un1[3 * n + b];
        u_n[id - 1] = un[3 * n + b];
      }
    }
  if (c->model == PGFEM_MODEL_CP) {
    std::vector<double> st((size_t)10 * c->nqp), Fs((size_t)9 * c->nqp);
    for (long q = 0; q < c->nqp; q++) {
      const double *b = blocks.data() + (size_t)bs * q;
      for (int k = 0; k < 9; k++) {
        st[10 * q + k] = b[18 + k];
        Fs[(size_t)k * c->nqp + q] = b[k];
      }
      st[10 * q + 9] = b[60];
    }
    if ((r = pgfem_gpu_set_state(c, st.data()))) return r;
    for (long q = 0; q < c->nqp; q++) {  // pF_{n-1}, g_{n-1}: the state at t_{n-1}
      const double *b = blocks.data() + (size_t)bs * q;
      for (int k = 0; k < 9; k++) st[10 * q + k] = b[27 + k];
      st[10 * q + 9] = b[61];
    }
    if ((r = pgfem_gpu_set_state_nm1(c, st.data()))) return r;
    CK(cudaMemcpyAsync(c->cp_Fn, Fs.data(), sizeof(double) * Fs.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  if (c->model == PGFEM_MODEL_J2) {  // Cp^-1 = I - pS / G, eqps = ep_n
    std::vector<double> st((size_t)10 * c->nqp);
    const double G = c->mat.mu;
    for (long q = 0; q < c->nqp; q++) {
      const double *b = blocks.data() + (size_t)bs * q;
      for (int k = 0; k < 9; k++) st[10 * q + k] = ((k % 4 == 0) ? 1.0 : 0.0) - b[9 + k] / G;
      st[10 * q + 9] = b[42];
    }
    if ((r = pgfem_gpu_set_state(c, st.data()))) return r;
  }
  return PGFEM_GPU_OK;
}

static int ensure_scratch(pgfem_gpu_ctx *c, bool wantK) {
  int r;
  if (!c->d_u && (r = dalloc(c, &c->d_u, c->ndof))) return r;
  if (!c->d_presc && (r = dalloc(c, &c->d_presc, std::max<long>(1, c->npres)))) return r;
  if (!c->d_R && (r = dalloc(c, &c->d_R, c->ndof))) return r;
  if (wantK && !c->d_K && (r = dalloc(c, &c->d_K, c->nnz))) return r;
  return PGFEM_GPU_OK;
}

static int assemble_host(pgfem_gpu_ctx *c, const double *u, const double *presc, double *R,
                         double *K, pgfem_gpu_status *st, double dt) {
  if (!c || !u || !R || (c->npres && !presc)) return PGFEM_GPU_EINVAL;
  int r = ensure_scratch(c, K != nullptr);
  if (r) return r;
  CK(cudaMemcpyAsync(c->d_u, u, sizeof(double) * c->ndof, cudaMemcpyHostToDevice, c->stream));
  if (c->npres)
    CK(cudaMemcpyAsync(c->d_presc, presc, sizeof(double) * c->npres, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->status, 0, 4 * sizeof(unsigned long long), c->stream));
  r = assemble_device(c, c->d_u, c->npres ? c->d_presc : nullptr, c->d_R, K ? c->d_K : nullptr, c->stream, dt);
  if (r) return r;
  CK(cudaMemcpyAsync(R, c->d_R, sizeof(double) * c->ndof, cudaMemcpyDeviceToHost, c->stream));
  if (K) CK(cudaMemcpyAsync(K, c->d_K, sizeof(double) * c->nnz, cudaMemcpyDeviceToHost, c->stream));
  return read_status(c, st, false);
}

int pgfem_gpu_assemble_R(pgfem_gpu_ctx *c, const double *u, const double *presc, double dt,
                         double *R, pgfem_gpu_status *st) {
  return assemble_host(c, u, presc, R, nullptr, st, dt);
}

int pgfem_gpu_assemble_RK(pgfem_gpu_ctx *c, const double *u, const double *presc, double dt,
                          double *R, double *K, pgfem_gpu_status *st) {
  if (!K) return PGFEM_GPU_EINVAL;
  return assemble_host(c, u, presc, R, K, st, dt);
}

// The crystal-plasticity transient on device buffers (displacements and
// prescribed values at t_{n+1}, t_n, t_{n-1}; tua / tpa / tR2 scratch): the
// surface terms at the two mid points, scaled like the element's, F at t_n
// and t_{n-1}, then the point update at u_{n+1} and the mid-point element
// stage (k_cp_element_tr) into the context's R and K.
static int transient_cp(pgfem_gpu_ctx *c, const double *tu2, const double *tu1, const double *tu0,
                        const double *tp2, const double *tp1, const double *tp0, double *tua, double *tpa,
                        double *tR2, double alpha, double dt_np1, double dt_n, bool wantK, cudaStream_t s) {
  int r;
  const long nd = c->ndof, np = c->npres;
  const unsigned gu = (unsigned)((std::max<long>(1, nd) + 255) / 256),
                 gp = (unsigned)((std::max<long>(1, np) + 255) / 256),
                 g3 = (unsigned)((3 * c->nn + 255) / 256), ge = (unsigned)((c->ne + 127) / 128);
  double *dK = wantK ? c->d_K : nullptr;
  const double cA = -dt_np1 * (1.0 - alpha), cB = -dt_n * alpha;
  CK(cudaMemsetAsync(c->d_R, 0, sizeof(double) * nd, s));
  if (dK) CK(cudaMemsetAsync(dK, 0, sizeof(double) * c->nnz, s));
  auto expand = [&](const double *u, const double *p) {
    k_expand_u<<<g3, 256, 0, s>>>(c->dof, c->nn, u, np ? p : nullptr, c->unode);
  };
  auto blend = [&](const double *x, const double *y, const double *px, const double *py) {
    k_blend<<<gu, 256, 0, s>>>(tua, x, y, alpha, nd);
    if (np) k_blend<<<gp, 256, 0, s>>>(tpa, px, py, alpha, np);
    expand(tua, tpa);
  };
  if (c->nbc_nface) {
    // the newer mid point into R and K, scaled as the element's terms are
    blend(tu1, tu2, tp1, tp2);
    c->nbc_desc_cur = c->nbc_desc_tr;
    r = launch_neumann(c, c->d_R, dK, s);
    c->nbc_desc_cur = nullptr;
    if (r) return r;
    k_scale_add<<<gu, 256, 0, s>>>(c->d_R, cA, nullptr, 0.0, nd);
    if (dK)
      k_scale_add<<<(unsigned)((c->nnz + 255) / 256), 256, 0, s>>>(dK, -alpha * (1.0 - alpha) * dt_np1, nullptr,
                                                                     0.0, c->nnz);
    // the older mid point: residual only
    blend(tu0, tu1, tp0, tp1);
    CK(cudaMemsetAsync(tR2, 0, sizeof(double) * nd, s));
    c->nbc_desc_cur = c->nbc_desc_tr + (size_t)kNbcDesc * c->nbc_nfeat;
    r = launch_neumann(c, tR2, nullptr, s);
    c->nbc_desc_cur = nullptr;
    if (r) return r;
    k_scale_add<<<gu, 256, 0, s>>>(c->d_R, 1.0, tR2, cB, nd);
  }
  if (!c->tr_F && (r = dalloc(c, &c->tr_F, (size_t)18 * c->ne))) return r;
  expand(tu1, tp1);
  k_cp_F<<<ge, 128, 0, s>>>(c->X, c->unode, c->conn, c->nn, c->ne, nullptr, c->tr_F, nullptr, nullptr);
  expand(tu0, tp0);
  k_cp_F<<<ge, 128, 0, s>>>(c->X, c->unode, c->conn, c->nn, c->ne, nullptr, c->tr_F + (size_t)9 * c->ne, nullptr,
                            nullptr);
  expand(tu2, tp2);
  CK(cudaGetLastError());
  const CpTransient tr{c->tr_F, c->tr_F + (size_t)9 * c->ne, alpha, cA, cB};
  return assemble_cp(c, c->d_R, dK, dt_np1, s, nullptr, &tr);
}

// Mid-point P and theta of the three-field element: (P_a, theta_a) =
// mid(values at t_n, current), (P_b, theta_b) = mid(t_{n-1}, t_n).
__global__ void k_tf_mid(long ne, const double *P, const double *th, const double *hist, double a, double *mid) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const double Pn = hist[e], tn = hist[ne + e], Pm = hist[2 * ne + e], tm = hist[3 * ne + e];
  mid[e] = (1.0 - a) * Pn + a * P[e];
  mid[ne + e] = (1.0 - a) * tn + a * th[e];
  mid[2 * ne + e] = (1.0 - a) * Pm + a * Pn;
  mid[3 * ne + e] = (1.0 - a) * tm + a * tn;
}

// The three-field transient's mid points (device buffers as transient_cp):
// mid-point P and theta, u_{n-1+a} at the nodes in the scratch, and the
// correction kernel's arguments.
static int tf_transient_prep(pgfem_gpu_ctx *c, double alpha, double dt_np1, double dt_n, TfTrArgs &T) {
  int r;
  if (!c->tf_mid && (r = dalloc(c, &c->tf_mid, (size_t)4 * c->ne + 3 * c->nn))) return r;
  T = TfTrArgs{};
  T.A.X = c->X;
  T.A.unode = c->unode;
  T.A.conn = c->conn;
  T.A.nn = c->nn;
  T.A.ne = c->ne;
  T.A.status = c->status;
  T.A.mat = c->mat;
  T.A.shp = c->shp;
  T.unode_b = c->tf_mid + (size_t)4 * c->ne;
  T.mid = c->tf_mid;
  T.dof = c->dof;
  T.cA = -dt_np1 * (1.0 - alpha);
  T.cB = -dt_n * alpha;
  T.kK = -dt_np1 * alpha * (1.0 - alpha);
  return PGFEM_GPU_OK;
}

// The three-field transient (hyperelastic, quadratic tets): the condensed
// residual at the older mid point (point records + k_tf_residual), the
// condensed R+K assembly at the newer one, combined as the one-field
// transient combines them, then k_tf_transient's correction of the
// condensation.
static int transient_3f(pgfem_gpu_ctx *c, const double *tu2, const double *tu1, const double *tu0,
                        const double *tp2, const double *tp1, const double *tp0, double *tua, double *tpa,
                        double *tR2, double alpha, double dt_np1, double dt_n, bool wantK, cudaStream_t s) {
  TfTrArgs T;
  int r = tf_transient_prep(c, alpha, dt_np1, dt_n, T);
  if (r) return r;
  const long nd = c->ndof, np = c->npres;
  const unsigned gu = (unsigned)((std::max<long>(1, nd) + 255) / 256),
                 gp = (unsigned)((std::max<long>(1, np) + 255) / 256),
                 g3 = (unsigned)((3 * c->nn + 255) / 256), ge = (unsigned)((c->ne + 127) / 128);
  double *pres = np ? tpa : nullptr;
  k_tf_mid<<<ge, 128, 0, s>>>(c->ne, c->tf_P, c->tf_theta, c->tf_hist, alpha, c->tf_mid);
  double *P_cur = c->tf_P, *th_cur = c->tf_theta;
  auto restore = [&]() {
    c->tf_P = P_cur;
    c->tf_theta = th_cur;
    c->nbc_desc_cur = nullptr;
  };
  // older mid point: u_{n-1+a}, P_b, theta_b
  k_blend<<<gu, 256, 0, s>>>(tua, tu0, tu1, alpha, nd);
  if (np) k_blend<<<gp, 256, 0, s>>>(tpa, tp0, tp1, alpha, np);
  c->tf_P = c->tf_mid + (size_t)2 * c->ne;
  c->tf_theta = c->tf_mid + (size_t)3 * c->ne;
  if (c->nbc_nface) c->nbc_desc_cur = c->nbc_desc_tr + (size_t)kNbcDesc * c->nbc_nfeat;
  // residual only: the point records, then their residual rows (no stiffness)
  CK(cudaMemsetAsync(tR2, 0, sizeof(double) * nd, s));
  k_expand_u<<<g3, 256, 0, s>>>(c->dof, c->nn, tua, pres, c->unode);
  r = launch_qp_update<10, 4, PGFEM_MODEL_HE, true>(c, s);
  if (!r) {
    QpArgs q{};
    q.conn = c->conn;
    q.nn = c->nn;
    q.ne = c->ne;
    q.qrec = c->qrec;
    q.perm = c->perm;
    q.mat = c->mat;
    q.shp = c->shp;
    k_tf_residual<<<ge, 128, 0, s>>>(q, c->dof, tR2);
    CK(cudaGetLastError());
    r = launch_neumann(c, tR2, nullptr, s);
  }
  if (r) {
    restore();
    return r;
  }
  k_expand_u<<<g3, 256, 0, s>>>(c->dof, c->nn, tua, pres, c->tf_mid + (size_t)4 * c->ne);
  // newer mid point: u_{n+a}, P_a, theta_a
  k_blend<<<gu, 256, 0, s>>>(tua, tu1, tu2, alpha, nd);
  if (np) k_blend<<<gp, 256, 0, s>>>(tpa, tp1, tp2, alpha, np);
  c->tf_P = c->tf_mid;
  c->tf_theta = c->tf_mid + c->ne;
  c->nbc_desc_cur = c->nbc_nface ? c->nbc_desc_tr : nullptr;
  r = assemble_device(c, tua, pres, c->d_R, wantK ? c->d_K : nullptr, s, dt_np1);
  restore();
  if (r) return r;
  k_scale_add<<<gu, 256, 0, s>>>(c->d_R, T.cA, tR2, T.cB, nd);
  T.R = c->d_R;
  k_tf_transient<<<ge, 128, 0, s>>>(T);  // c->unode holds u_{n+a}
  CK(cudaGetLastError());
  return PGFEM_GPU_OK;
}

// The transient element on device buffers (displacements and prescribed
// values at the three times), into the context's R and K buffers (K when
// wantK): the surface-load descriptors, the mid-point assemblies and their
// combination, and the inertia kernel.
static int transient_core(pgfem_gpu_ctx *c, const double *tu2, const double *tu1, const double *tu0,
                          const double *tp2, const double *tp1, const double *tp0, double alpha, double dt_np1,
                          double dt_n, double rho, bool wantK, cudaStream_t s) {
  int r;
  const long nd = std::max<long>(1, c->ndof), np = std::max<long>(1, c->npres);
  if (!c->tr_buf && (r = dalloc(c, &c->tr_buf, (size_t)5 * nd + 4 * np))) return r;
  double *tua = c->tr_buf + 3 * nd, *tR2 = tua + nd, *tpa = c->tr_buf + 5 * nd + 3 * np;
  const unsigned gu = (unsigned)((nd + 255) / 256), gp = (unsigned)((np + 255) / 256);
  double *pres = c->npres ? tpa : nullptr;
  if (c->nbc_nface) {
    // the surface loads' mid points: the first set for u_{n+a}, the second
    // for u_{n-1+a}
    const int nf = c->nbc_nfeat;
    std::vector<double> d((size_t)2 * kNbcDesc * nf);
    for (int f = 0; f < nf; f++) {
      const size_t o = (size_t)3 * f;
      nbc_desc_mid(c->nbc_type_h[f], &c->nbc_hist_n[o], &c->nbc_load_h[o], alpha, &d[(size_t)kNbcDesc * f]);
      nbc_desc_mid(c->nbc_type_h[f], &c->nbc_hist_nm1[o], &c->nbc_hist_n[o], alpha,
                   &d[(size_t)kNbcDesc * (nf + f)]);
    }
    if (!c->nbc_desc_tr && (r = dalloc(c, &c->nbc_desc_tr, d.size()))) return r;
    CK(cudaMemcpyAsync(c->nbc_desc_tr, d.data(), sizeof(double) * d.size(), cudaMemcpyHostToDevice, s));
    c->nbc_desc_cur = c->nbc_desc_tr;
  }
  if (c->three_field) {
    r = transient_3f(c, tu2, tu1, tu0, tp2, tp1, tp0, tua, tpa, tR2, alpha, dt_np1, dt_n, wantK, s);
    c->nbc_desc_cur = nullptr;
    if (r) return r;
  } else if (c->model == PGFEM_MODEL_CP) {
    r = transient_cp(c, tu2, tu1, tu0, tp2, tp1, tp0, tua, tpa, tR2, alpha, dt_np1, dt_n, wantK, s);
    c->nbc_desc_cur = nullptr;
    if (r) return r;
  } else {
    // quasi-static R and K at u_{n+a}
    k_blend<<<gu, 256, 0, s>>>(tua, tu1, tu2, alpha, c->ndof);
    if (c->npres) k_blend<<<gp, 256, 0, s>>>(tpa, tp1, tp2, alpha, c->npres);
    CK(cudaGetLastError());
    r = assemble_device(c, tua, pres, c->d_R, wantK ? c->d_K : nullptr, s, dt_np1);
    if (r) {
      c->nbc_desc_cur = nullptr;
      return r;
    }
    if (c->nbc_nface) c->nbc_desc_cur = c->nbc_desc_tr + (size_t)kNbcDesc * c->nbc_nfeat;
    // quasi-static R at u_{n-1+a}
    k_blend<<<gu, 256, 0, s>>>(tua, tu0, tu1, alpha, c->ndof);
    if (c->npres) k_blend<<<gp, 256, 0, s>>>(tpa, tp0, tp1, alpha, c->npres);
    CK(cudaGetLastError());
    r = assemble_device(c, tua, pres, tR2, nullptr, s, dt_n);
    c->nbc_desc_cur = nullptr;
    if (r) return r;
    // the mid-point combination
    k_scale_add<<<gu, 256, 0, s>>>(c->d_R, -dt_np1 * (1.0 - alpha), tR2, -dt_n * alpha, c->ndof);
  }
  // inertia: v = dt_n u_{n+1} - (dt_np1 + dt_n) u_n + dt_np1 u_{n-1} at the nodes
  k_comb3<<<gu, 256, 0, s>>>(tua, tu2, dt_n, tu1, -(dt_np1 + dt_n), tu0, dt_np1, c->ndof);
  if (c->npres) k_comb3<<<gp, 256, 0, s>>>(tpa, tp2, dt_n, tp1, -(dt_np1 + dt_n), tp0, dt_np1, c->npres);
  {
    const long n3 = 3 * c->nn;
    k_expand_u<<<(unsigned)((n3 + 255) / 256), 256, 0, s>>>(c->dof, c->nn, tua, pres, c->unode);
  }
  InertiaArgs ia{};
  ia.X = c->X;
  ia.conn = c->conn;
  ia.dof = c->dof;
  ia.rowptr0 = c->rowptr0;
  ia.rowlen = c->rowlen;
  ia.mask = c->mask;
  ia.pos = c->pos;
  ia.nn = c->nn;
  ia.ne = c->ne;
  ia.vnode = c->unode;
  ia.cR = rho / (dt_np1 * dt_n);
  ia.cK = rho / dt_np1;
  ia.R = c->d_R;
  ia.K = nullptr;  // the mass enters K below, from the cached CSR-aligned array
  ia.shp = c->shp;
  const unsigned ge = (unsigned)((c->ne + 127) / 128);
  if (c->nne == 10) k_inertia<10, 4><<<ge, 128, 0, s>>>(ia);
  else k_inertia<4, 1><<<ge, 128, 0, s>>>(ia);
  if (wantK) {
    // K = kscale K - rho / dt_np1 M: the mid-point stiffness factor (the CP
    // element applies its own) and the consistent mass, in one pass
    if (!c->mass_csr) {
      if ((r = dalloc(c, &c->mass_csr, std::max<long>(1, c->nnz)))) return r;
      CK(cudaMemsetAsync(c->mass_csr, 0, sizeof(double) * c->nnz, s));
      InertiaArgs im = ia;
      im.R = nullptr;
      im.K = c->mass_csr;
      im.cK = 1.0;
      if (c->nne == 10) k_inertia<10, 4><<<ge, 128, 0, s>>>(im);
      else k_inertia<4, 1><<<ge, 128, 0, s>>>(im);
    }
    const double kscale = c->model == PGFEM_MODEL_CP && !c->three_field ? 1.0 : -alpha * (1.0 - alpha) * dt_np1;
    k_scale_add<<<(unsigned)((c->nnz + 255) / 256), 256, 0, s>>>(c->d_K, kscale, c->mass_csr, rho / dt_np1,
                                                                   c->nnz);
  }
  CK(cudaGetLastError());
  return PGFEM_GPU_OK;
}

// Context and time parameters a transient call accepts.
static bool transient_ok(const pgfem_gpu_ctx *c, double alpha, double dt_np1, double dt_n, double rho) {
  if ((c->model != PGFEM_MODEL_HE && c->model != PGFEM_MODEL_CP) || c->F0 || c->elem_group) return false;
  // the three-field transient divides by alpha (1 - alpha) in its local update
  if (c->three_field && (!c->tf_hist || !(alpha > 0.0 && alpha < 1.0))) return false;
  // surface loads need their values at t_n and t_{n-1}
  if (c->nbc_nface && c->nbc_hist_n.size() != (size_t)3 * c->nbc_nfeat) return false;
  if (!(alpha >= 0.0 && alpha <= 1.0) || !(dt_np1 > 0.0) || !(dt_n > 0.0) || !std::isfinite(rho))
    return false;
  return true;
}

int pgfem_gpu_assemble_RK_transient(pgfem_gpu_ctx *c, const double *u_np1, const double *u_n,
                                    const double *u_nm1, const double *presc_np1, const double *presc_n,
                                    const double *presc_nm1, double alpha, double dt_np1, double dt_n, double rho,
                                    double *R, double *K, pgfem_gpu_status *st) {
  if (!c || !u_np1 || !u_n || !u_nm1 || !R || (c->npres && (!presc_np1 || !presc_n || !presc_nm1)))
    return PGFEM_GPU_EINVAL;
  if (!transient_ok(c, alpha, dt_np1, dt_n, rho)) return PGFEM_GPU_EINVAL;
  // below the reference's density threshold the element is the quasi-static one
  if (std::fabs(rho) < 1.0e-16) return assemble_host(c, u_np1, presc_np1, R, K, st, dt_np1);
  int r = ensure_scratch(c, K != nullptr);
  if (r) return r;
  const long nd = std::max<long>(1, c->ndof), np = std::max<long>(1, c->npres);
  if (!c->tr_buf && (r = dalloc(c, &c->tr_buf, (size_t)5 * nd + 4 * np))) return r;
  double *tu2 = c->tr_buf, *tu1 = tu2 + nd, *tu0 = tu1 + nd;
  double *tp2 = c->tr_buf + 5 * nd, *tp1 = tp2 + np, *tp0 = tp1 + np;
  cudaStream_t s = c->stream;
  const size_t bu = sizeof(double) * c->ndof, bp = sizeof(double) * c->npres;
  CK(cudaMemcpyAsync(tu2, u_np1, bu, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(tu1, u_n, bu, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(tu0, u_nm1, bu, cudaMemcpyHostToDevice, s));
  if (c->npres) {
    CK(cudaMemcpyAsync(tp2, presc_np1, bp, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(tp1, presc_n, bp, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(tp0, presc_nm1, bp, cudaMemcpyHostToDevice, s));
  }
  CK(cudaMemsetAsync(c->status, 0, 4 * sizeof(unsigned long long), s));
  r = transient_core(c, tu2, tu1, tu0, tp2, tp1, tp0, alpha, dt_np1, dt_n, rho, K != nullptr, s);
  if (r) return r;
  CK(cudaMemcpyAsync(R, c->d_R, bu, cudaMemcpyDeviceToHost, s));
  if (K) CK(cudaMemcpyAsync(K, c->d_K, sizeof(double) * c->nnz, cudaMemcpyDeviceToHost, s));
  return read_status(c, st, false);
}

int pgfem_gpu_assemble_RK_transient_device(pgfem_gpu_ctx *c, const double *d_u_np1, const double *d_u_n,
                                           const double *d_u_nm1, const double *d_presc_np1,
                                           const double *d_presc_n, const double *d_presc_nm1, double alpha,
                                           double dt_np1, double dt_n, double rho, double *d_R, double *d_K,
                                           void *stream) {
  if (!c || !d_u_np1 || !d_u_n || !d_u_nm1 || !d_R || (c->npres && (!d_presc_np1 || !d_presc_n || !d_presc_nm1)))
    return PGFEM_GPU_EINVAL;
  if (!transient_ok(c, alpha, dt_np1, dt_n, rho)) return PGFEM_GPU_EINVAL;
  cudaStream_t s = (cudaStream_t)stream;  // as assemble_RK_device: 0 is the default stream
  if (std::fabs(rho) < 1.0e-16) return assemble_device(c, d_u_np1, d_presc_np1, d_R, d_K, s, dt_np1);
  int r = ensure_scratch(c, false);
  if (r) return r;
  // the core writes the context's R and K buffers: point them at the caller's
  double *R0 = c->d_R, *K0 = c->d_K;
  c->d_R = d_R;
  if (d_K) c->d_K = d_K;
  r = transient_core(c, d_u_np1, d_u_n, d_u_nm1, d_presc_np1, d_presc_n, d_presc_nm1, alpha, dt_np1, dt_n, rho,
                     d_K != nullptr, s);
  c->d_R = R0;
  if (d_K) c->d_K = K0;
  return r;
}

int pgfem_gpu_assemble_RK_device(pgfem_gpu_ctx *c, const double *d_u, const double *d_presc,
                                 double dt, double *d_R, double *d_K, void *stream) {
  if (!c || !d_u || !d_R || !d_K) return PGFEM_GPU_EINVAL;
  return assemble_device(c, d_u, d_presc, d_R, d_K, (cudaStream_t)stream, dt);
}

int pgfem_gpu_three_field_increments_transient(pgfem_gpu_ctx *c, const double *u_np1, const double *u_n,
                                               const double *u_nm1, const double *presc_np1,
                                               const double *presc_n, const double *presc_nm1, const double *du,
                                               double alpha, double dt_np1, double dt_n, double *dP,
                                               double *dtheta, pgfem_gpu_status *st) {
  if (!c || !c->three_field || !c->tf_hist || c->model != PGFEM_MODEL_HE || !u_np1 || !u_n || !u_nm1 || !du ||
      !dP || !dtheta || (c->npres && (!presc_np1 || !presc_n || !presc_nm1)))
    return PGFEM_GPU_EINVAL;
  if (!(alpha > 0.0 && alpha < 1.0) || !(dt_np1 > 0.0) || !(dt_n > 0.0)) return PGFEM_GPU_EINVAL;
  int r = ensure_scratch(c, false);
  if (r) return r;
  const long nd = std::max<long>(1, c->ndof), np = std::max<long>(1, c->npres);
  if (!c->tr_buf && (r = dalloc(c, &c->tr_buf, (size_t)5 * nd + 4 * np))) return r;
  if (!c->tf_dunode && ((r = dalloc(c, &c->tf_dunode, 3 * c->nn)) || (r = dalloc(c, &c->tf_inc, 2 * c->ne))))
    return r;
  double *tu2 = c->tr_buf, *tu1 = tu2 + nd, *tu0 = tu1 + nd, *tua = tu0 + nd, *tdu = tua + nd;
  double *tp2 = tdu + nd, *tp1 = tp2 + np, *tp0 = tp1 + np, *tpa = tp0 + np;
  cudaStream_t s = c->stream;
  const size_t bu = sizeof(double) * c->ndof, bp = sizeof(double) * c->npres;
  CK(cudaMemcpyAsync(tu2, u_np1, bu, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(tu1, u_n, bu, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(tu0, u_nm1, bu, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(tdu, du, bu, cudaMemcpyHostToDevice, s));
  if (c->npres) {
    CK(cudaMemcpyAsync(tp2, presc_np1, bp, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(tp1, presc_n, bp, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(tp0, presc_nm1, bp, cudaMemcpyHostToDevice, s));
  }
  CK(cudaMemsetAsync(c->status, 0, 4 * sizeof(unsigned long long), s));
  TfTrArgs T;
  if ((r = tf_transient_prep(c, alpha, dt_np1, dt_n, T))) return r;
  const unsigned gu = (unsigned)((nd + 255) / 256), gp = (unsigned)((np + 255) / 256),
                 g3 = (unsigned)((3 * c->nn + 255) / 256), ge = (unsigned)((c->ne + 127) / 128);
  double *pres = c->npres ? tpa : nullptr;
  k_tf_mid<<<ge, 128, 0, s>>>(c->ne, c->tf_P, c->tf_theta, c->tf_hist, alpha, c->tf_mid);
  k_blend<<<gu, 256, 0, s>>>(tua, tu0, tu1, alpha, c->ndof);
  if (c->npres) k_blend<<<gp, 256, 0, s>>>(tpa, tp0, tp1, alpha, c->npres);
  k_expand_u<<<g3, 256, 0, s>>>(c->dof, c->nn, tua, pres, c->tf_mid + (size_t)4 * c->ne);
  k_blend<<<gu, 256, 0, s>>>(tua, tu1, tu2, alpha, c->ndof);
  if (c->npres) k_blend<<<gp, 256, 0, s>>>(tpa, tp1, tp2, alpha, c->npres);
  k_expand_u<<<g3, 256, 0, s>>>(c->dof, c->nn, tua, pres, c->unode);
  k_expand_u<<<g3, 256, 0, s>>>(c->dof, c->nn, tdu, nullptr, c->tf_dunode);
  T.dunode = c->tf_dunode;
  T.dP = c->tf_inc;
  T.dtheta = c->tf_inc + c->ne;
  k_tf_transient<<<ge, 128, 0, s>>>(T);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(dP, c->tf_inc, sizeof(double) * c->ne, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(dtheta, c->tf_inc + c->ne, sizeof(double) * c->ne, cudaMemcpyDeviceToHost, s));
  return read_status(c, st, false);
}

int pgfem_gpu_read_status(pgfem_gpu_ctx *c, pgfem_gpu_status *st, int clear) {
  if (!c) return PGFEM_GPU_EINVAL;
  return read_status(c, st, clear != 0);
}

static int element_level(pgfem_gpu_ctx *c, long nel, const long *elems, const double *u,
                         const double *presc, double dt, double *lk, double *fe, pgfem_gpu_status *st) {
  if (!c || nel < 0 || (nel && (!elems || !fe)) || !u || (c->npres && !presc)) return PGFEM_GPU_EINVAL;
  if (c->three_field) return PGFEM_GPU_EINVAL;  // the element-level kernels are one-field
  if (nel == 0) return PGFEM_GPU_OK;
  for (long i = 0; i < nel; i++)
    if (elems[i] < 0 || elems[i] >= c->ne) return PGFEM_GPU_EINVAL;
  int r = ensure_scratch(c, false);
  if (r) return r;
  const int nd = c->nne * 3;
  std::vector<int> el(elems, elems + nel);
  int *d_el = nullptr;
  double *d_lk = nullptr, *d_fe = nullptr;
  auto cleanup = [&]() {
    if (d_el) cudaFree(d_el);
    if (d_lk) cudaFree(d_lk);
    if (d_fe) cudaFree(d_fe);
  };
  if (cudaMalloc(&d_el, sizeof(int) * nel) != cudaSuccess ||
      cudaMalloc(&d_fe, sizeof(double) * nel * nd) != cudaSuccess ||
      (lk && cudaMalloc(&d_lk, sizeof(double) * nel * nd * nd) != cudaSuccess)) {
    cudaGetLastError();
    cleanup();
    return PGFEM_GPU_ENOMEM;
  }
  cudaMemcpyAsync(d_el, el.data(), sizeof(int) * nel, cudaMemcpyHostToDevice, c->stream);
  cudaMemcpyAsync(c->d_u, u, sizeof(double) * c->ndof, cudaMemcpyHostToDevice, c->stream);
  if (c->npres) cudaMemcpyAsync(c->d_presc, presc, sizeof(double) * c->npres, cudaMemcpyHostToDevice, c->stream);
  cudaMemsetAsync(c->status, 0, 4 * sizeof(unsigned long long), c->stream);
  const long n3 = 3 * c->nn;
  k_expand_u<<<(unsigned)((n3 + 255) / 256), 256, 0, c->stream>>>(c->dof, c->nn, c->d_u,
                                                                   c->npres ? c->d_presc : nullptr, c->unode);
  if (c->model == PGFEM_MODEL_CP) {
    // the local update runs for every point of the context (its state at
    // t_{n+1} is that of an assembly at u), then the listed elements' blocks
    CpElemList L{d_el, nel, d_lk, d_fe};
    r = assemble_cp(c, nullptr, nullptr, dt, c->stream, &L);
  } else {
    AsmArgs a = base_args(c);
    a.elist = d_el;
    a.nlist = nel;
    a.lk_out = d_lk;
    a.fe_out = d_fe;
    r = lk ? dispatch<false, true, true>(c, a, nel, c->stream) : dispatch<false, false, true>(c, a, nel, c->stream);
  }
  if (!r) r = launch_neumann(c, nullptr, nullptr, c->stream, d_el, nel, d_lk, d_fe);
  if (!r) {
    cudaMemcpyAsync(fe, d_fe, sizeof(double) * nel * nd, cudaMemcpyDeviceToHost, c->stream);
    if (lk) cudaMemcpyAsync(lk, d_lk, sizeof(double) * nel * nd * nd, cudaMemcpyDeviceToHost, c->stream);
    r = read_status(c, st, false);
  }
  cudaStreamSynchronize(c->stream);
  cleanup();
  return r;
}

int pgfem_gpu_stiffmatel_fd(pgfem_gpu_ctx *c, long nel, const long *elems, const double *u,
                            const double *presc, double dt, double *lk, double *fe,
                            pgfem_gpu_status *st) {
  if (!lk) return PGFEM_GPU_EINVAL;
  return element_level(c, nel, elems, u, presc, dt, lk, fe, st);
}

int pgfem_gpu_resid_on_elem(pgfem_gpu_ctx *c, long nel, const long *elems, const double *u,
                            const double *presc, double dt, double *fe, pgfem_gpu_status *st) {
  return element_level(c, nel, elems, u, presc, dt, nullptr, fe, st);
}

int pgfem_gpu_cm_integrate(const pgfem_material_desc *mat, long nqp, const double *F, double dt,
                           const double *R_cp, const double *state_n, double *state_np1, double *S,
                           double *L, int *qp_status) {
  if (!mat || nqp < 0 || (nqp && (!F || !S))) return PGFEM_GPU_EINVAL;
  if (mat->model != PGFEM_MODEL_HE && mat->model != PGFEM_MODEL_J2) return PGFEM_GPU_EINVAL;
  if (mat->dev_pot < 0 || mat->dev_pot > 2 || (mat->dev_pot == 2 && mat->model != PGFEM_MODEL_HE) ||
      !(mat->vol_pot <= 0 || mat->vol_pot == 99 || ((mat->vol_pot == 2 || mat->vol_pot == 3) && mat->model != PGFEM_MODEL_CP)))
    return PGFEM_GPU_EINVAL;
  if (mat->model == PGFEM_MODEL_J2 && nqp && (!state_n || !state_np1)) return PGFEM_GPU_EINVAL;
  int r = check_device();
  if (r) return r;
  if (nqp == 0) return PGFEM_GPU_OK;
  return cm_integrate_host(make_mat(mat), nqp, F, dt, state_n, state_np1, S, L, qp_status);
}


// ---- batches of independent meshes, schedule, graph capture, autotuner ----

int pgfem_gpu_set_mesh_groups(pgfem_gpu_ctx *c, int ngroups, const long *elem_off, const double *F0) {
  if (!c || ngroups < 1 || !elem_off || !F0 || c->model == PGFEM_MODEL_CP) return PGFEM_GPU_EINVAL;
  if (elem_off[0] != 0 || elem_off[ngroups] != c->ne) return PGFEM_GPU_EINVAL;
  std::vector<int> grp(c->ne);
  for (int g = 0; g < ngroups; g++) {
    if (elem_off[g + 1] < elem_off[g]) return PGFEM_GPU_EINVAL;
    for (long e = elem_off[g]; e < elem_off[g + 1]; e++) grp[e] = g;
  }
  if (c->elem_group) cudaFree(c->elem_group);
  if (c->F0_tab) cudaFree(c->F0_tab);
  c->elem_group = nullptr;
  c->F0_tab = nullptr;
  int r;
  if ((r = upload(c, &c->elem_group, grp.data(), grp.size())) ||
      (r = upload(c, &c->F0_tab, F0, (size_t)9 * ngroups)))
    return r;
  CK(cudaStreamSynchronize(c->stream));
  c->ngroups = ngroups;
  return PGFEM_GPU_OK;
}

int pgfem_gpu_set_schedule(pgfem_gpu_ctx *c, int elems_per_block, int grab) {
  if (!c || grab < 0 || (elems_per_block != 0 && elems_per_block != 16 && elems_per_block != 32 &&
                         elems_per_block != 64))
    return PGFEM_GPU_EINVAL;
  if ((elems_per_block || grab) && c->nne != 4) return PGFEM_GPU_EINVAL;
  if (grab > 0 && !c->sched_ticket) {
    int r = dalloc(c, &c->sched_ticket, 1);
    if (r) return r;
  }
  c->sched_epb = elems_per_block;
  c->sched_grab = grab;
  return PGFEM_GPU_OK;
}

int pgfem_gpu_get_schedule(const pgfem_gpu_ctx *c, int *elems_per_block, int *grab) {
  if (!c) return PGFEM_GPU_EINVAL;
  if (elems_per_block) *elems_per_block = c->sched_epb;
  if (grab) *grab = c->sched_grab;
  return PGFEM_GPU_OK;
}

struct pgfem_gpu_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

int pgfem_gpu_graph_create(pgfem_gpu_ctx *c, const double *d_u, const double *d_presc, double dt, double *d_R,
                           double *d_K, pgfem_gpu_graph **out) {
  if (!c || !d_u || !d_R || !d_K || !out) return PGFEM_GPU_EINVAL;
  *out = nullptr;
  const bool timing = c->timing;
  c->timing = false;  // no event bookkeeping inside the captured work
  // one uncaptured call sets the kernels' attributes before capture
  int r = assemble_device(c, d_u, d_presc, d_R, d_K, c->stream, dt);
  if (!r && cudaStreamSynchronize(c->stream) != cudaSuccess) r = PGFEM_GPU_ECUDA;
  pgfem_gpu_graph *g = nullptr;
  if (!r) {
    g = new pgfem_gpu_graph();
    if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) r = PGFEM_GPU_ECUDA;
    if (!r) {
      const int ra = assemble_device(c, d_u, d_presc, d_R, d_K, c->stream, dt);
      const cudaError_t ce = cudaStreamEndCapture(c->stream, &g->graph);
      r = ra ? ra : (ce != cudaSuccess ? PGFEM_GPU_ECUDA : PGFEM_GPU_OK);
    }
    if (!r && cudaGraphInstantiate(&g->exec, g->graph, 0) != cudaSuccess) r = PGFEM_GPU_ECUDA;
  }
  c->timing = timing;
  if (r) {
    cudaGetLastError();
    if (g) {
      if (g->exec) cudaGraphExecDestroy(g->exec);
      if (g->graph) cudaGraphDestroy(g->graph);
      delete g;
    }
    return r;
  }
  *out = g;
  return PGFEM_GPU_OK;
}

int pgfem_gpu_graph_launch(pgfem_gpu_graph *g, void *stream) {
  if (!g || !g->exec) return PGFEM_GPU_EINVAL;
  CK(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
  return PGFEM_GPU_OK;
}

int pgfem_gpu_graph_destroy(pgfem_gpu_graph *g) {
  if (!g) return PGFEM_GPU_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return PGFEM_GPU_OK;
}

int pgfem_gpu_autotune(pgfem_gpu_ctx *c, const double *d_u, const double *d_presc, double dt, double *d_R,
                       double *d_K, int reps, int *best_epb, int *best_grab, double *best_ms) {
  if (!c || c->nne != 4 || reps < 1) return PGFEM_GPU_EINVAL;
  const int epbs[] = {16, 32, 64};
  const int grabs[] = {1, 2, 4, 8, 16};
  double bms = 1e300;
  int be = 32, bg = 1;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  int r = PGFEM_GPU_OK;
  for (int ie = 0; ie < 3 && !r; ie++)
    for (int ig = 0; ig < 5 && !r; ig++) {
      if ((r = pgfem_gpu_set_schedule(c, epbs[ie], grabs[ig]))) break;
      pgfem_gpu_graph *g = nullptr;
      if ((r = pgfem_gpu_graph_create(c, d_u, d_presc, dt, d_R, d_K, &g))) break;
      for (int w = 0; w < 2 && !r; w++) r = pgfem_gpu_graph_launch(g, c->stream);
      if (!r && (cudaEventRecord(e0, c->stream) != cudaSuccess)) r = PGFEM_GPU_ECUDA;
      for (int k = 0; k < reps && !r; k++) r = pgfem_gpu_graph_launch(g, c->stream);
      float ms = 0.f;
      if (!r && (cudaEventRecord(e1, c->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
                 cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess))
        r = PGFEM_GPU_ECUDA;
      pgfem_gpu_graph_destroy(g);
      if (!r && ms / reps < bms) {
        bms = ms / reps;
        be = epbs[ie];
        bg = grabs[ig];
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r) return r;
  if ((r = pgfem_gpu_set_schedule(c, be, bg))) return r;
  if (best_epb) *best_epb = be;
  if (best_grab) *best_grab = bg;
  if (best_ms) *best_ms = bms;
  return PGFEM_GPU_OK;
}

}  // extern "C"

// ---- crystal plasticity point update without device allocation ------------
//
// For callers that may not call cudaMalloc: code that runs inside another
// framework's memory pool (the pool owns the device memory and a raw
// cudaMalloc would bypass its accounting or fail), callbacks on a time-
// critical path where cudaMalloc's implicit device synchronisation is not
// acceptable, and host runtimes whose policy forbids allocation after start-
// up.  The caller owns every input and output; the work record of the local
// Newton (M, dM/dF, g, slip increments per point), the work-stealing ticket
// counter and the failure counters live in the file-scope array below, which
// every GPU that loads this library holds until the process exits.
//
// Host code must not pass `pgfem_cp_scratch` itself to a kernel: on the host
// that name is only a stand-in for the device array.  The device address is
// taken with cudaGetSymbolAddress once per device, with that device current.

#define PGFEM_CP_NOALLOC_MAX_POINTS 4096L
namespace {
constexpr long kNaHeader = 32;  // doubles: ticket counter (word 0), 4 failure counters (words 1-4), pad to 256 B
constexpr long kNaWords = kNaHeader + (long)pgb::kCpOut * PGFEM_CP_NOALLOC_MAX_POINTS;
}  // namespace
static __device__ __align__(256) double pgfem_cp_scratch[kNaWords];

namespace {
struct NaDevice {
  double *scratch = nullptr;  // device address of pgfem_cp_scratch on this device
  int grid_cap = 0;           // SMs x resident CTAs of k_cp_update
  bool ready = false;
};
constexpr int kNaMaxDevices = 64;
NaDevice g_na[kNaMaxDevices];
std::mutex g_na_mu;

// One-time set-up on the current device: the scratch address, the dynamic
// shared-memory opt-in of k_cp_update and its persistent grid size.
int noalloc_setup(int dev, NaDevice **out) {
  std::lock_guard<std::mutex> lk(g_na_mu);
  NaDevice &d = g_na[dev];
  if (!d.ready) {
    void *p = nullptr;
    CK(cudaGetSymbolAddress(&p, pgfem_cp_scratch));
    if (!p || ((uintptr_t)p & 255u)) return PGFEM_GPU_ECUDA;
    const size_t smem = pgb::cp_update_smem();
    CK(cudaFuncSetAttribute(pgb::k_cp_update, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0, sms = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pgb::k_cp_update, 32 * pgb::kCpWarps, smem));
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    d.scratch = (double *)p;
    d.grid_cap = std::max(1, per_sm) * std::max(1, sms);
    d.ready = true;
  }
  *out = &d;
  return PGFEM_GPU_OK;
}
}  // namespace

extern "C" {

int pgfem_gpu_cp_integrate_noalloc(const pgfem_material_desc *mat, long nqp, const double *d_F,
                                   const double *d_R_cp, const double *d_state_n, double dt,
                                   double *d_state_np1, double *d_dgam, int *d_iters,
                                   pgfem_gpu_status *st, void *stream) {
  if (!mat || nqp < 0 || (nqp && (!d_F || !d_R_cp || !d_state_n || !d_state_np1))) return PGFEM_GPU_EINVAL;
  if (mat->model != PGFEM_MODEL_CP || !(mat->m > 0) || !(mat->g0 > 0) || !(mat->gs_0 > mat->g0))
    return PGFEM_GPU_EINVAL;
  if (nqp > PGFEM_CP_NOALLOC_MAX_POINTS) {
    std::fprintf(stderr,
                 "pgfem_gpu_cp_integrate_noalloc: %ld points exceed the fixed maximum of %ld per call; "
                 "split the batch\n",
                 nqp, PGFEM_CP_NOALLOC_MAX_POINTS);
    return PGFEM_GPU_ELIMIT;
  }
  int r = check_device();
  if (r) return r;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNaMaxDevices) return PGFEM_GPU_ENODEV;
  cudaStream_t s = (cudaStream_t)stream;
  if (st) {  // reading the counts back waits for the stream: not allowed while it is captured
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(s, &cs));
    if (cs != cudaStreamCaptureStatusNone) return PGFEM_GPU_EINVAL;
  }
  NaDevice *d = nullptr;
  if ((r = noalloc_setup(dev, &d))) return r;
  if (st) *st = pgfem_gpu_status{};
  if (nqp == 0) return PGFEM_GPU_OK;
  // the ticket counter and the failure counters must start at zero; the work
  // record is written in full for every point before it is read
  CK(cudaMemsetAsync(d->scratch, 0, sizeof(double) * kNaHeader, s));
  pgb::CpArgs a{};
  a.nqp = nqp;
  a.F = d_F;
  a.Rcp = d_R_cp;
  a.nqp_e = 1;
  a.ne = nqp;
  a.state_n = d_state_n;
  a.state_np1 = d_state_np1;
  a.guess = nullptr;
  a.out = d->scratch + kNaHeader;
  a.iters = d_iters;
  a.counter = (unsigned *)d->scratch;
  a.status = (unsigned long long *)(d->scratch + 1);
  a.mat = make_mat(mat);
  a.dt = dt;
  const long need = (nqp + 32 * pgb::kCpWarps - 1) / (32 * pgb::kCpWarps);
  const long grid = std::max<long>(1, std::min<long>(need, d->grid_cap));
  pgb::k_cp_update<<<(unsigned)grid, 32 * pgb::kCpWarps, pgb::cp_update_smem(), s>>>(a);
  CK(cudaGetLastError());
  if (d_dgam)  // slip increments dt*gamma_dot_a: rows 91..102 of the work record, contiguous
    CK(cudaMemcpyAsync(d_dgam, a.out + 91 * nqp, sizeof(double) * 12 * nqp, cudaMemcpyDeviceToDevice, s));
  if (st) {
    unsigned long long w[4];
    CK(cudaMemcpyAsync(w, d->scratch + 1, sizeof(w), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    st->inverted = (long)w[0];
    st->nonconverged = (long)w[1];
    st->bad_diagonal = (long)w[2];
    st->other = (long)w[3];
  }
  return PGFEM_GPU_OK;
}

}  // extern "C"
