// tile_plan.hpp -- host-side plan of the tiled assembly kernel.
//
// Elements are cut into tiles of TE consecutive elements (a Kuhn cell of 6
// tets, or 4 cells for linear tets).  For every tile the plan holds
//  - its local node set (first-appearance order) and each element node's
//    local index,
//  - its local node-pair blocks ("slots"): every (A, B) node pair of its
//    elements with free rows and columns, sorted by (A, column position of B
//    inside the rows of A), with the position inside the caller's CSR rows,
//  - the K range of the CSR rows first touched by the tile, and the earlier
//    tiles that first touched the other rows it writes (its dependencies).
// First-touch ranges are contiguous because the reference numbers DOFs in
// first-visit order over elements (src/generate_dof_ids.cc:306-412) and the
// CSR rows are stored in DOF order (src/Psparse_ApAi.cc:639-658): each tile
// zeroes its own rows just before they receive contributions, which keeps the
// lines in L2 instead of streaming a 4.4 GB memset through HBM.  When the
// caller's numbering breaks that property the plan falls back to a memset.
#pragma once
#include <algorithm>
#include <cstdint>
#include <thread>
#include <vector>

namespace pgb {

constexpr int kDepMax = 16;

struct TilePlan {
  int TE = 0, NNE = 0, NLMAX = 0;
  long ntiles = 0;
  int nslots_max = 0;
  bool first_touch = false;
  std::vector<int> tile_nodes;       // ntiles * NLMAX, -1 padded
  std::vector<uint8_t> tile_nl;      // ntiles
  std::vector<uint8_t> elem_lnode;   // ne * NNE
  std::vector<uint16_t> elem_slot;   // ne * NNE * NNE, 0xFFFF = no block
  std::vector<long long> slot_off;   // ntiles + 1
  std::vector<uint32_t> slot_info;   // (A_l << 24) | (B_l << 16) | pos
  std::vector<uint16_t> aoff;        // ntiles * (NLMAX + 1): slot prefix per local node
  std::vector<long long> zlo, zhi;   // ntiles: K range zeroed by the tile
  std::vector<int> deps;             // ntiles * kDepMax, -1 padded
  std::vector<uint8_t> allfree;      // ntiles: every tile node has all three DOFs free
};

// Builds the plan; returns false when the caller's pattern misses a block.
inline bool build_tile_plan(TilePlan &P, int TE, int NNE, long ne, const std::vector<int> &conn_em,
                            const std::vector<int> &first_dof, const std::vector<uint8_t> &mask,
                            const int *Ap, const int *Ai, long ndof) {
  P.TE = TE;
  P.NNE = NNE;
  P.NLMAX = TE * NNE;
  P.ntiles = (ne + TE - 1) / TE;
  const long nt = P.ntiles;
  P.tile_nodes.assign(nt * P.NLMAX, -1);
  P.tile_nl.assign(nt, 0);
  P.elem_lnode.assign(ne * NNE, 0);
  P.elem_slot.assign(ne * NNE * NNE, 0xFFFF);
  P.aoff.assign(nt * (P.NLMAX + 1), 0);
  std::vector<std::vector<uint32_t>> tslots(nt);
  bool ok = true;

  auto work = [&](long t0, long t1) {
    std::vector<int> loc;
    std::vector<std::pair<uint32_t, uint32_t>> pairs;  // (A_l<<16|pos, B_l)
    for (long t = t0; t < t1; t++) {
      const long e0 = t * TE, e1 = std::min(ne, e0 + TE);
      loc.clear();
      for (long e = e0; e < e1; e++)
        for (int a = 0; a < NNE; a++) {
          const int n = conn_em[e * NNE + a];
          int l = (int)(std::find(loc.begin(), loc.end(), n) - loc.begin());
          if (l == (int)loc.size()) loc.push_back(n);
          P.elem_lnode[e * NNE + a] = (uint8_t)l;
        }
      P.tile_nl[t] = (uint8_t)loc.size();
      for (size_t l = 0; l < loc.size(); l++) P.tile_nodes[t * P.NLMAX + l] = loc[l];
      // distinct free pairs with their CSR column positions
      pairs.clear();
      const int nl = (int)loc.size();
      std::vector<int> pos_of(nl * nl, -1);
      for (long e = e0; e < e1; e++)
        for (int a = 0; a < NNE; a++)
          for (int b = 0; b < NNE; b++) {
            const int la = P.elem_lnode[e * NNE + a], lb = P.elem_lnode[e * NNE + b];
            const int A = loc[la], B = loc[lb];
            if (!mask[A] || !mask[B]) continue;
            int &ps = pos_of[la * nl + lb];
            if (ps < 0) {
              const int *row = Ai + Ap[first_dof[A]];
              const int len = Ap[first_dof[A] + 1] - Ap[first_dof[A]];
              const int *it = std::lower_bound(row, row + len, first_dof[B]);
              const int p = (int)(it - row);
              const int nb = __builtin_popcount(mask[B]);
              bool good = p + nb <= len && p < 0xFFFF;
              for (int k = 0; good && k < nb; k++) good = row[p + k] == first_dof[B] + k;
              if (!good) {
                ok = false;
                ps = 0;
                continue;
              }
              ps = p;
              pairs.emplace_back(((uint32_t)la << 16) | (uint32_t)p, (uint32_t)lb);
            }
          }
      std::sort(pairs.begin(), pairs.end());
      std::vector<int> slot_of(nl * nl, -1);
      auto &sl = tslots[t];
      sl.resize(pairs.size());
      uint16_t *ao = &P.aoff[t * (P.NLMAX + 1)];
      for (size_t s = 0; s < pairs.size(); s++) {
        const uint32_t la = pairs[s].first >> 16, pos = pairs[s].first & 0xFFFF, lb = pairs[s].second;
        sl[s] = (la << 24) | (lb << 16) | pos;
        slot_of[la * nl + lb] = (int)s;
        ao[la + 1]++;
      }
      for (int l = 0; l < P.NLMAX; l++) ao[l + 1] += ao[l];
      for (long e = e0; e < e1; e++)
        for (int a = 0; a < NNE; a++)
          for (int b = 0; b < NNE; b++) {
            const int la = P.elem_lnode[e * NNE + a], lb = P.elem_lnode[e * NNE + b];
            const int s = slot_of[la * nl + lb];
            if (s >= 0) P.elem_slot[(e * NNE + a) * NNE + b] = (uint16_t)s;
          }
    }
  };
  {
    unsigned h = std::thread::hardware_concurrency();
    const int nth = (int)std::max(1u, std::min(h ? h : 4u, 32u));
    std::vector<std::thread> th;
    const long chunk = (nt + nth - 1) / nth;
    for (int i = 0; i < nth; i++) {
      const long b = i * chunk, e = std::min(nt, b + chunk);
      if (b < e) th.emplace_back(work, b, e);
    }
    for (auto &x : th) x.join();
  }
  if (!ok) return false;
  P.slot_off.assign(nt + 1, 0);
  for (long t = 0; t < nt; t++) {
    P.slot_off[t + 1] = P.slot_off[t] + (long long)tslots[t].size();
    P.nslots_max = std::max(P.nslots_max, (int)tslots[t].size());
  }
  P.slot_info.resize(P.slot_off[nt]);
  for (long t = 0; t < nt; t++)
    std::copy(tslots[t].begin(), tslots[t].end(), P.slot_info.begin() + P.slot_off[t]);

  // first-touch analysis (rows = free DOFs)
  std::vector<int> ftile(ndof, -1);
  for (long t = 0; t < nt; t++)
    for (int l = 0; l < P.tile_nl[t]; l++) {
      const int n = P.tile_nodes[t * P.NLMAX + l];
      if (!mask[n]) continue;
      const int nf = __builtin_popcount(mask[n]);
      for (int k = 0; k < nf; k++)
        if (ftile[first_dof[n] + k] < 0) ftile[first_dof[n] + k] = (int)t;
    }
  bool mono = true;
  for (long d = 0; d < ndof && mono; d++) mono = ftile[d] >= 0 && (d == 0 || ftile[d] >= ftile[d - 1]);
  P.zlo.assign(nt, 0);
  P.zhi.assign(nt, 0);
  P.deps.assign(nt * kDepMax, -1);
  if (mono) {
    long d = 0;
    for (long t = 0; t < nt; t++) {
      const long d0 = d;
      while (d < ndof && ftile[d] == t) d++;
      P.zlo[t] = Ap[d0];
      P.zhi[t] = Ap[d];
    }
    for (long t = 0; t < nt && mono; t++) {
      int nd = 0;
      for (int l = 0; l < P.tile_nl[t] && mono; l++) {
        const int n = P.tile_nodes[t * P.NLMAX + l];
        if (!mask[n]) continue;
        const int f = ftile[first_dof[n]];
        if (f == t) continue;
        bool seen = false;
        for (int k = 0; k < nd; k++) seen |= P.deps[t * kDepMax + k] == f;
        if (seen) continue;
        if (nd == kDepMax) mono = false;
        else P.deps[t * kDepMax + nd++] = f;
      }
    }
  }
  P.allfree.assign(nt, 1);
  for (long t = 0; t < nt; t++)
    for (int l = 0; l < P.tile_nl[t]; l++)
      if (mask[P.tile_nodes[t * P.NLMAX + l]] != 7) P.allfree[t] = 0;
  P.first_touch = mono;
  if (!mono) {
    std::fill(P.zlo.begin(), P.zlo.end(), 0);
    std::fill(P.zhi.begin(), P.zhi.end(), 0);
    std::fill(P.deps.begin(), P.deps.end(), -1);
  }
  return true;
}

}  // namespace pgb
