// setup_host.cpp -- host-side setup of the assembly path: synthetic box
// meshes, DOF numbering and the CSR pattern of the operator.
//
// DOF numbering keeps the reference's rule (src/generate_dof_ids.cc:306-412):
// free DOFs are numbered 1.. in first-visit order over elements, then nodes
// of the element, then components; code 1 (fixed) becomes id 0; negative
// codes (prescribed) are kept; a periodic node takes its master's ids.
// The CSR pattern is the one Psparse_ApAi produces on one rank
// (src/Psparse_ApAi.cc:161-213, 327-366, 639-658): each free DOF row holds
// the sorted, unique free DOF ids of every element touching it.  It is built
// here per node group instead of per DOF (all free DOFs of a node share one
// column set), which gives the identical arrays in a fraction of the time.
#include "pgfem_gpu.h"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// Kuhn split of the unit cube into 6 tets along the (0,0,0)-(1,1,1)
// diagonal; one tet per axis permutation, oriented to a positive volume.
const int kPerm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
const int kPermSign[6] = {+1, -1, -1, +1, +1, -1};
// Quadratic-tet edge nodes in FEMLIB's QTETRAHEDRON order
// (FEMLIB/src/femlib.cc:163-176): 4:(0,1) 5:(1,2) 6:(0,2) 7:(0,3) 8:(1,3) 9:(2,3).
const int kEdge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};

int num_threads() {
  unsigned h = std::thread::hardware_concurrency();
  return h ? (int)std::min(h, 32u) : 4;
}

template <class F>
void parallel_for(long n, F f) {
  const int nt = num_threads();
  if (n < 4096 || nt <= 1) {
    f(0, n);
    return;
  }
  std::vector<std::thread> th;
  const long chunk = (n + nt - 1) / nt;
  for (int t = 0; t < nt; t++) {
    const long b = t * chunk, e = std::min(n, b + chunk);
    if (b < e) th.emplace_back(f, b, e);
  }
  for (auto &x : th) x.join();
}

}  // namespace

extern "C" int pgfem_mesh_box_tet(int n, int nne, int periodic, long *nn_out, long *ne_out,
                                  double *X, int *conn, long *Pr) {
  if (n < 1 || (nne != 4 && nne != 10) || !nn_out || !ne_out) return PGFEM_GPU_EINVAL;
  const long N = (nne == 4) ? n : 2L * n;  // lattice intervals per axis
  const long L = N + 1;
  const long nn = L * L * L, ne = 6L * n * n * n;
  *nn_out = nn;
  *ne_out = ne;
  if (!X) return PGFEM_GPU_OK;
  const int s = (nne == 4) ? 1 : 2;  // lattice steps per cell edge
  for (long k = 0; k < L; k++)
    for (long j = 0; j < L; j++)
      for (long i = 0; i < L; i++) {
        const long id = i + L * (j + L * k);
        X[id * 3 + 0] = (double)i / (double)N;
        X[id * 3 + 1] = (double)j / (double)N;
        X[id * 3 + 2] = (double)k / (double)N;
        if (Pr) {
          long mi = i, mj = j, mk = k;
          if (periodic) {
            if (mi == N) mi = 0;
            if (mj == N) mj = 0;
            if (mk == N) mk = 0;
          }
          const long m = mi + L * (mj + L * mk);
          Pr[id] = (m == id) ? -1 : m;
        }
      }
  if (!conn) return PGFEM_GPU_OK;
  long e = 0;
  for (long ck = 0; ck < n; ck++)
    for (long cj = 0; cj < n; cj++)
      for (long ci = 0; ci < n; ci++)
        for (int t = 0; t < 6; t++) {
          int v[4][3];  // vertex offsets in cells
          v[0][0] = v[0][1] = v[0][2] = 0;
          for (int d = 0; d < 3; d++) v[1][d] = (kPerm[t][0] == d);
          for (int d = 0; d < 3; d++) v[2][d] = v[1][d] + (kPerm[t][1] == d);
          v[3][0] = v[3][1] = v[3][2] = 1;
          if (kPermSign[t] < 0)
            for (int d = 0; d < 3; d++) std::swap(v[1][d], v[2][d]);
          long lat[10][3];
          for (int a = 0; a < 4; a++) {
            lat[a][0] = s * (ci + v[a][0]);
            lat[a][1] = s * (cj + v[a][1]);
            lat[a][2] = s * (ck + v[a][2]);
          }
          if (nne == 10)
            for (int m = 0; m < 6; m++)
              for (int d = 0; d < 3; d++)
                lat[4 + m][d] = (lat[kEdge[m][0]][d] + lat[kEdge[m][1]][d]) / 2;
          for (int a = 0; a < nne; a++)
            conn[e * nne + a] = (int)(lat[a][0] + L * (lat[a][1] + L * lat[a][2]));
          e++;
        }
  return PGFEM_GPU_OK;
}

extern "C" long pgfem_generate_dof_ids(long nn, long ne, int nne, const int *conn, const long *Pr,
                                       long *id) {
  if (nn < 0 || ne < 0 || !conn || !id) return PGFEM_GPU_EINVAL;
  std::vector<uint8_t> seen(nn * 3, 0);
  long next = 1;
  for (long e = 0; e < ne; e++) {
    for (int a = 0; a < nne; a++) {
      const long nd = conn[e * nne + a];
      for (int j = 0; j < 3; j++) {
        const long k = nd * 3 + j;
        if (seen[k]) continue;
        seen[k] = 1;
        if (id[k] < 0) continue;          // prescribed: keep its code
        if (id[k] == 1) { id[k] = 0; continue; }  // fixed
        const long m = (Pr && Pr[nd] >= 0) ? Pr[nd] : -1;
        if (m >= 0) {
          const long km = m * 3 + j;
          if (!seen[km]) { seen[km] = 1; id[km] = next++; }
          id[k] = id[km];
        } else {
          id[k] = next++;
        }
      }
    }
  }
  for (long nd = 0; nd < nn; nd++)  // periodic nodes outside every element
    for (int j = 0; j < 3; j++)
      if (!seen[nd * 3 + j] && Pr && Pr[nd] >= 0) {
        id[nd * 3 + j] = id[Pr[nd] * 3 + j];
        seen[nd * 3 + j] = 1;
      }
  return next - 1;
}

extern "C" long pgfem_psparse_apai(long ne, int nne, const int *conn, const long *id, long ndof,
                                   int *Ap, int *Ai) {
  if (ne < 0 || !conn || !id || !Ap || ndof < 0) return PGFEM_GPU_EINVAL;
  // Node groups: a node's free DOFs share one row set when every free
  // component id of the node is consecutive and every node with a given
  // first free id carries the same ids (periodic images do).
  long nn = 0;
  for (long k = 0; k < ne * nne; k++) nn = std::max<long>(nn, conn[k] + 1);
  std::vector<long> first(nn, -1);  // first free dof (0-based) of each node
  std::vector<int> nfree(nn, 0);
  for (long n = 0; n < nn; n++) {
    long prev = -1;
    for (int j = 0; j < 3; j++) {
      const long g = id[n * 3 + j];
      if (g > 0) {
        if (first[n] < 0) first[n] = g - 1;
        else if (g - 1 != prev + 1) return PGFEM_GPU_EINVAL;  // non-consecutive ids
        prev = g - 1;
        nfree[n]++;
      }
    }
  }
  // group key = first free dof; rows of the group: first .. first+nfree-1
  std::vector<int> gsize(ndof, -1);
  for (long n = 0; n < nn; n++)
    if (first[n] >= 0) {
      if (first[n] >= ndof) return PGFEM_GPU_EINVAL;
      if (gsize[first[n]] >= 0 && gsize[first[n]] != nfree[n]) return PGFEM_GPU_EINVAL;
      gsize[first[n]] = nfree[n];
    }
  // neighbour lists per group (CSR over group keys)
  std::vector<long> cnt(ndof + 1, 0);
  for (long e = 0; e < ne; e++) {
    int nf = 0;
    for (int a = 0; a < nne; a++) nf += first[conn[e * nne + a]] >= 0;
    for (int a = 0; a < nne; a++) {
      const long g = first[conn[e * nne + a]];
      if (g >= 0) cnt[g + 1] += nf;
    }
  }
  for (long g = 0; g < ndof; g++) cnt[g + 1] += cnt[g];
  std::vector<long> nb(cnt[ndof]);
  {
    std::vector<long> fill(cnt.begin(), cnt.end() - 1);
    for (long e = 0; e < ne; e++)
      for (int a = 0; a < nne; a++) {
        const long g = first[conn[e * nne + a]];
        if (g < 0) continue;
        for (int b = 0; b < nne; b++) {
          const long h = first[conn[e * nne + b]];
          if (h >= 0) nb[fill[g]++] = h;
        }
      }
  }
  // sort + unique per group; column count of a group = sum of neighbour sizes
  std::vector<long> ncol(ndof, 0);
  std::vector<long> ulen(ndof, 0);
  parallel_for(ndof, [&](long b, long e) {
    for (long g = b; g < e; g++) {
      if (gsize[g] < 0) continue;
      long *beg = nb.data() + cnt[g], *end = nb.data() + cnt[g + 1];
      std::sort(beg, end);
      long *u = std::unique(beg, end);
      ulen[g] = u - beg;
      long c = 0;
      for (long *p = beg; p < u; p++) c += gsize[*p];
      ncol[g] = c;
    }
  });
  // row lengths in DOF order, prefix
  long nnz = 0;
  Ap[0] = 0;
  for (long r = 0; r < ndof; r++) {
    long g = r;
    while (g >= 0 && gsize[g] < 0) g--;  // owner group of row r
    if (g < 0 || r - g >= gsize[g]) return PGFEM_GPU_EINVAL;
    nnz += ncol[g];
    if (nnz > 0x7fffffffL) return PGFEM_GPU_ELIMIT;  // Ai_t is int (include/datatype.hpp:4)
    Ap[r + 1] = (int)nnz;
  }
  if (!Ai) return nnz;
  parallel_for(ndof, [&](long b, long e) {
    for (long g = b; g < e; g++) {
      if (gsize[g] < 0) continue;
      const long *beg = nb.data() + cnt[g];
      int *row = Ai + Ap[g];
      long c = 0;
      for (long k = 0; k < ulen[g]; k++)
        for (int j = 0; j < gsize[beg[k]]; j++) row[c++] = (int)(beg[k] + j);
      for (int s = 1; s < gsize[g]; s++) std::memcpy(Ai + Ap[g + s], row, sizeof(int) * c);
    }
  });
  return nnz;
}
