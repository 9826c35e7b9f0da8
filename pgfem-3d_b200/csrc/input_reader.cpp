// input_reader.cpp -- readers of PGFem3D's input files for the assembly path.
//
// Mesh files <base><r>.in (read_input_file, src/read_input_file.cc:268-415,
// non-legacy formats: nodes src/node.cc:78-160, supports and prescribed
// values src/in.cc:29-191, elements src/element.cc:168-199 and 256-330,
// materials src/in.cc:195-223, material geometry and loads
// src/in.cc:225-290), merged over partitions r = 0..P-1 into one mesh;
// solver files <base><r>.in.st (read_solver_file / read_time_steps /
// compute_times_load, src/read_input_file.cc:517-700, src/load.cc:29-60);
// model_params.in (read_model_parameters_list, src/constitutive_model.cc:
// 1171-1309, with the CP / J2 / HE parameter blocks of src/plasticity_model.cc:
// 945-1040, src/cm_j2_plasticity.cc:865-900, src/plasticity_model_none.cc:293);
// crystal orientation files <base>_<r>.in (plasticity_model_read_orientations,
// src/plasticity_model.cc:1260-1337).
//
// Tokens are whitespace separated; a token that starts with '#' begins a
// comment that runs to the end of its line (the effect of the reference's
// scan_for_valid_line between fscanf calls); '{' and '}' are tokens of their
// own.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "pgfem_gpu.h"

namespace {

thread_local std::string g_err;

int fail(const std::string &msg) {
  g_err = msg;
  return PGFEM_GPU_EFORMAT;
}

struct Tokens {
  std::string s, path;
  size_t i = 0;

  bool load(const std::string &p) {
    path = p;
    FILE *f = fopen(p.c_str(), "rb");
    if (!f) return false;
    char buf[65536];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, f)) > 0) s.append(buf, n);
    fclose(f);
    return true;
  }
  void skip() {
    for (;;) {
      while (i < s.size() && isspace((unsigned char)s[i])) i++;
      if (i < s.size() && s[i] == '#') {
        while (i < s.size() && s[i] != '\n') i++;
        continue;
      }
      return;
    }
  }
  bool eof() {
    skip();
    return i >= s.size();
  }
  bool next(std::string &t) {
    skip();
    if (i >= s.size()) return false;
    if (s[i] == '{' || s[i] == '}') {
      t.assign(1, s[i++]);
      return true;
    }
    const size_t b = i;
    while (i < s.size() && !isspace((unsigned char)s[i]) && s[i] != '{' && s[i] != '}') i++;
    t = s.substr(b, i - b);
    return true;
  }
  bool num(double &v) {
    std::string t;
    if (!next(t)) return false;
    char *end = nullptr;
    v = strtod(t.c_str(), &end);
    return end && *end == 0 && !t.empty();
  }
  bool num(long &v) {
    std::string t;
    if (!next(t)) return false;
    char *end = nullptr;
    v = strtol(t.c_str(), &end, 10);
    return end && *end == 0 && !t.empty();
  }
  bool num(int &v) {
    long l;
    if (!num(l)) return false;
    v = (int)l;
    return true;
  }
  // peek whether the next token is an integer (without consuming it)
  bool peek_int() {
    const size_t keep = i;
    long v;
    const bool ok = num(v);
    i = keep;
    return ok;
  }
  std::string where() const {
    const long line = 1 + (long)std::count(s.begin(), s.begin() + (long)std::min(i, s.size()), '\n');
    return path + ":" + std::to_string(line);
  }
};

}  // namespace

struct pgfem_input {
  pgfem_input_info info{};
  std::vector<double> X;
  std::vector<int> conn;
  std::vector<long> codes, elem_mat, elem_hom, elem_local;
  std::vector<int> elem_part;
  std::vector<double> defl, mat_vals, cf, ee;
  std::vector<int> dev_pot, vol_pot;
  std::vector<int> bnd_id, bnd_type;  // 4 per element: the faces' boundary features
  int nparts = 0;
  std::vector<long> part_elem_off;  // merged element index of each partition's first element
  std::vector<std::vector<long>> node_map;  // per partition: merged id of each local node
  std::vector<long> Pr;                      // periodic master of each merged node, -1 if none
};

namespace {

struct Part {
  long nn = 0, ndofn = 0, ne = 0, lin_maxit = 0, nmat = 0, nconc = 0, norient = 0;
  double lin_err = 0, lim_zero = 0;
  std::vector<long> toe, gnn, dom;
  std::vector<double> X;
  std::vector<long> codes;
  std::vector<double> defl;
  std::vector<long> conn, emat, ehom;
  std::vector<int> bid, btype;  // per element and face: boundary feature id and type
  std::vector<double> mats, cf, ee;
  std::vector<int> devp, volp;
  long nln = 0, nel_s = 0, nel_v = 0;
};

// Physics layout of a mesh file: one supports section per physics, in the
// order of multiphysics.in, each with ndim codes per node; the mechanical
// section (ndim 3) is the one kept.
struct PhysLayout {
  int nphys = 1;
  std::vector<int> ndim{3};
  int mech = 0;
  bool multiphysics = false;  // the header's ndofn then counts every physics
};

int read_part(const std::string &path, Part &p, const PhysLayout &L) {
  Tokens t;
  if (!t.load(path)) return fail("cannot open " + path);
  auto bad = [&](const char *what) { return fail(std::string("bad ") + what + " at " + t.where()); };
  if (!t.num(p.nn) || !t.num(p.ndofn) || !t.num(p.ne)) return bad("header (nn ndofn ne)");
  if (!t.num(p.lin_maxit) || !t.num(p.lin_err) || !t.num(p.lim_zero)) return bad("solver header");
  if (!t.num(p.nmat) || !t.num(p.nconc) || !t.num(p.norient)) return bad("material header");
  if (p.nn <= 0 || p.ne < 0 || p.nmat < 0 || p.nconc < 0 || p.norient < 0) return bad("header sizes");
  if (!L.multiphysics && p.ndofn != 3)
    return fail(path + ": ndofn " + std::to_string(p.ndofn) + " (the mechanical path has 3)");
  p.toe.resize(p.ne);
  for (long e = 0; e < p.ne; e++)
    if (!t.num(p.toe[e])) return bad("element type line");
  // nodes: Gnn Dom id x y z model_type model_id pr
  p.gnn.assign(p.nn, -2);
  p.dom.assign(p.nn, 0);
  p.X.assign(3 * p.nn, 0.0);
  for (long k = 0; k < p.nn; k++) {
    long g, d, id, mt, mid, pr;
    double x[3];
    if (!t.num(g) || !t.num(d) || !t.num(id) || !t.num(x[0]) || !t.num(x[1]) || !t.num(x[2]) || !t.num(mt) ||
        !t.num(mid) || !t.num(pr))
      return bad("node line");
    if (id < 0 || id >= p.nn || p.gnn[id] != -2) return bad("node id");
    p.gnn[id] = g;
    p.dom[id] = d;
    for (int j = 0; j < 3; j++) p.X[3 * id + j] = x[j];
  }
  // supports and prescribed values, one section per physics (read_supports,
  // src/read_input_file.cc:362-370); the mechanical section is kept
  long npd = 0;
  p.codes.assign(3 * p.nn, 0);
  for (int ph = 0; ph < L.nphys; ph++) {
    const bool keep = ph == L.mech;
    const int nd = L.ndim[ph];
    long nsup;
    if (!t.num(nsup) || nsup < 0) return bad("support count");
    for (long k = 0; k < nsup; k++) {
      long n;
      if (!t.num(n) || n < 0 || n >= p.nn) return bad("support node");
      for (int j = 0; j < nd; j++) {
        long c;
        if (!t.num(c)) return bad("support code");
        if (keep) p.codes[3 * n + j] = c;
      }
    }
    long np_;
    if (!t.num(np_) || np_ < 0) return bad("prescribed count");
    if (keep) {
      npd = np_;
      p.defl.resize(npd);
    }
    for (long k = 0; k < np_; k++) {
      double v;
      if (!t.num(v)) return bad("prescribed value");
      if (keep) p.defl[k] = v;
    }
  }
  for (long n = 0; n < p.nn; n++)
    for (int j = 0; j < 3; j++) {
      const long c = p.codes[3 * n + j];
      if (c < -npd || c > 1) return bad("support code range");
    }
  // elements: id nodes[toe] ftype fid pr bnd_id[4] bnd_type[4]
  long nne = p.ne ? p.toe[0] : 0;
  for (long e = 0; e < p.ne; e++)
    if (p.toe[e] != nne) return fail(path + ": mixed element types (one type per mesh on this path)");
  if (p.ne && nne != 4 && nne != 10)
    return fail(path + ": element type " + std::to_string(nne) + " (linear or quadratic tets on this path)");
  p.conn.assign(p.ne * nne, -1);
  p.bid.assign(4 * p.ne, 0);
  p.btype.assign(4 * p.ne, 0);
  std::vector<char> seen(p.ne, 0);
  for (long k = 0; k < p.ne; k++) {
    long id;
    if (!t.num(id) || id < 0 || id >= p.ne || seen[id]) return bad("element id");
    seen[id] = 1;
    for (long a = 0; a < nne; a++) {
      long n;
      if (!t.num(n) || n < 0 || n >= p.nn) return bad("element node");
      p.conn[id * nne + a] = n;
    }
    for (int k2 = 0; k2 < 3; k2++) {  // ftype fid pr
      long v;
      if (!t.num(v)) return bad("element face data");
    }
    for (int f = 0; f < 4; f++)
      if (!t.num(p.bid[4 * id + f])) return bad("element face feature id");
    for (int f = 0; f < 4; f++)
      if (!t.num(p.btype[4 * id + f])) return bad("element face feature type");
  }
  // element materials: id mat[2] hom[2]
  p.emat.assign(2 * p.ne, 0);
  p.ehom.assign(2 * p.ne, 0);
  for (long k = 0; k < p.ne; k++) {
    long id;
    if (!t.num(id) || id < 0 || id >= p.ne) return bad("element material id");
    if (!t.num(p.emat[2 * id]) || !t.num(p.emat[2 * id + 1]) || !t.num(p.ehom[2 * id]) ||
        !t.num(p.ehom[2 * id + 1]))
      return bad("element material");
    if (p.emat[2 * id] < 0 || p.emat[2 * id] >= std::max(1L, p.nmat)) return bad("element material index");
  }
  // materials: Ex Ey Ez Gyz Gxz Gxy nyz nxz nxy ax ay az sig devPotFlag volPotFlag
  p.mats.assign(13 * p.nmat, 0.0);
  p.devp.assign(p.nmat, 0);
  p.volp.assign(p.nmat, 0);
  for (long m = 0; m < p.nmat; m++) {
    for (int j = 0; j < 13; j++)
      if (!t.num(p.mats[13 * m + j])) return bad("material line");
    if (!t.num(p.devp[m]) || !t.num(p.volp[m])) return bad("material potential flags");
  }
  // material geometry
  p.cf.assign(p.nconc, 0.0);
  for (long k = 0; k < p.nconc; k++)
    if (!t.num(p.cf[k])) return bad("concentration");
  p.ee.assign(9 * p.norient, 0.0);
  for (long k = 0; k < 9 * p.norient; k++)
    if (!t.num(p.ee[k])) return bad("orientation");
  {
    long SH;
    double a1, a2;
    if (!t.num(SH) || !t.num(a1) || !t.num(a2)) return bad("material geometry (SH a1 a2)");
  }
  // loads: counted and stepped over (nodal and element loads are not on this path)
  if (!t.num(p.nln) || p.nln < 0) return bad("nodal load count");
  for (long k = 0; k < p.nln; k++) {
    double v;
    for (int j = 0; j < 4; j++)
      if (!t.num(v)) return bad("nodal load");
  }
  if (!t.num(p.nel_s) || p.nel_s < 0) return bad("surface load count");
  const int nsur = nne == 10 ? 6 : 3;
  for (long k = 0; k < p.nel_s; k++) {
    double v;
    for (int j = 0; j < 1 + nsur + 3; j++)
      if (!t.num(v)) return bad("surface load");
  }
  if (!t.num(p.nel_v) || p.nel_v < 0) return bad("volume load count");
  return PGFEM_GPU_OK;
}

// Supports from <bc_base>_<r>.bc (count, then "node c0 c1 c2" lines) and the
// prescribed values from <bc_base>.bcv (count, values): the BC-directory
// variant of read_input_file (src/read_input_file.cc:320-360, read_Dirichlet_BCs /
// read_Dirichlet_BCs_values, src/in.cc:29-168), which replaces the mesh file's
// own supports section.
int read_bc_files(const std::string &bc_base, int r, Part &p) {
  Tokens v;
  const std::string fv = bc_base + ".bcv";
  if (!v.load(fv)) return fail("cannot open " + fv);
  long npd;
  if (!v.num(npd) || npd < 0) return fail("bad prescribed count at " + v.where());
  p.defl.assign(npd, 0.0);
  for (long k = 0; k < npd; k++)
    if (!v.num(p.defl[k])) return fail("bad prescribed value at " + v.where());
  Tokens t;
  const std::string fb = bc_base + "_" + std::to_string(r) + ".bc";
  if (!t.load(fb)) return fail("cannot open " + fb);
  long nsup;
  if (!t.num(nsup) || nsup < 0) return fail("bad support count at " + t.where());
  p.codes.assign(3 * p.nn, 0);
  for (long k = 0; k < nsup; k++) {
    long n;
    if (!t.num(n) || n < 0 || n >= p.nn) return fail("bad support node at " + t.where());
    for (int j = 0; j < 3; j++) {
      long c;
      if (!t.num(c) || c < -npd || c > 1) return fail("bad support code at " + t.where());
      p.codes[3 * n + j] = c;
    }
  }
  return PGFEM_GPU_OK;
}

bool close(double a, double b) { return std::fabs(a - b) <= 1e-12 * std::max(1.0, std::max(std::fabs(a), std::fabs(b))); }

}  // namespace

extern "C" {

const char *pgfem_input_last_error(void) { return g_err.c_str(); }

int pgfem_input_read_mesh(const char *base, int nparts, pgfem_input **out) {
  return pgfem_input_read_mesh_bc(base, nparts, nullptr, out);
}

int pgfem_input_read_mesh_bc(const char *base, int nparts, const char *bc_base, pgfem_input **out) {
  const int ndim = 3;
  return pgfem_input_read_mesh_mp(base, nparts, bc_base, 1, &ndim, 0, out);
}

int pgfem_input_read_mesh_mp(const char *base, int nparts, const char *bc_base, int nphys, const int *ndim,
                             int mech, pgfem_input **out) {
  if (!base || nparts < 1 || !out || nphys < 1 || !ndim || mech < 0 || mech >= nphys || ndim[mech] != 3)
    return PGFEM_GPU_EINVAL;
  for (int k = 0; k < nphys; k++)
    if (ndim[k] < 1 || ndim[k] > 3) return PGFEM_GPU_EINVAL;
  PhysLayout L;
  if (!bc_base) {
    L.nphys = nphys;
    L.ndim.assign(ndim, ndim + nphys);
    L.mech = mech;
  }  // with a BC directory the mesh file holds one supports section, read and replaced
  L.multiphysics = nphys > 1;
  *out = nullptr;
  std::vector<Part> parts(nparts);
  for (int r = 0; r < nparts; r++) {
    int e = read_part(std::string(base) + std::to_string(r) + ".in", parts[r], L);
    if (!e && bc_base) e = read_bc_files(bc_base, r, parts[r]);
    if (e) return e;
  }
  auto *in = new pgfem_input();
  in->nparts = nparts;
  const Part &p0 = parts[0];
  pgfem_input_info &I = in->info;
  I.nne = 0;
  for (const Part &p : parts)
    if (p.ne) {
      I.nne = (int)p.toe[0];
      break;
    }
  I.npres = (long)p0.defl.size();
  I.nmat = (int)p0.nmat;
  I.nconc = p0.nconc;
  I.norient = p0.norient;
  I.lin_maxit = p0.lin_maxit;
  I.lin_err = p0.lin_err;
  I.lim_zero = p0.lim_zero;
  auto reject = [&](const std::string &m) {
    delete in;
    return fail(m);
  };
  // merged node numbering: partition-boundary nodes (Gnn >= 0) by Gnn and
  // position, interior nodes (Gnn = -1) per partition; first appearance
  // order.  Nodes that share a global number at different positions are
  // periodic images: each becomes a node of its own, linked to the first
  // image as its periodic master -- the reference's rule (a node's periodic
  // master is the first node with the same global number,
  // generate_local_dof_ids, src/generate_dof_ids.cc:81-96).
  std::map<long, std::vector<long>> gmap;
  std::vector<std::vector<long>> lmap(nparts);
  for (int r = 0; r < nparts; r++) {
    const Part &p = parts[r];
    if (p.ne && p.toe[0] != I.nne) return reject("partitions with different element types");
    if ((long)p.defl.size() != I.npres) return reject("partitions with different prescribed value counts");
    for (long k = 0; k < I.npres; k++)
      if (!close(p.defl[k], p0.defl[k])) return reject("partitions with different prescribed values");
    if (p.nmat != p0.nmat) return reject("partitions with different material counts");
    for (size_t k = 0; k < p.mats.size(); k++)
      if (!close(p.mats[k], p0.mats[k])) return reject("partitions with different materials");
    for (long m = 0; m < p.nmat; m++)
      if (p.devp[m] != p0.devp[m] || p.volp[m] != p0.volp[m]) return reject("partitions with different materials");
    lmap[r].assign(p.nn, -1);
    for (long n = 0; n < p.nn; n++) {
      long id = (long)in->X.size() / 3, master = -1;
      bool fresh = true;
      if (p.gnn[n] >= 0) {
        std::vector<long> &images = gmap[p.gnn[n]];
        for (long cand : images) {
          bool same = true;
          for (int j = 0; j < 3 && same; j++) same = close(in->X[3 * cand + j], p.X[3 * n + j]);
          if (same) {
            id = cand;
            fresh = false;
            break;
          }
        }
        if (fresh) {
          if (!images.empty()) master = images[0];
          images.push_back(id);
        }
      }
      lmap[r][n] = id;
      if (fresh) {
        for (int j = 0; j < 3; j++) {
          in->X.push_back(p.X[3 * n + j]);
          in->codes.push_back(p.codes[3 * n + j]);
        }
        in->Pr.push_back(master);
        if (master >= 0) I.nperiodic++;
      } else {
        for (int j = 0; j < 3; j++) {
          long &c = in->codes[3 * id + j];
          if (c == 0) c = p.codes[3 * n + j];
          else if (p.codes[3 * n + j] != 0 && p.codes[3 * n + j] != c)
            return reject("partition-boundary node " + std::to_string(p.gnn[n]) + " with different supports");
        }
      }
    }
  }
  I.nn = (long)in->X.size() / 3;
  in->part_elem_off.assign(nparts + 1, 0);
  for (int r = 0; r < nparts; r++) {
    const Part &p = parts[r];
    in->part_elem_off[r + 1] = in->part_elem_off[r] + p.ne;
    for (long e = 0; e < p.ne; e++) {
      for (int a = 0; a < I.nne; a++) in->conn.push_back((int)lmap[r][p.conn[e * I.nne + a]]);
      in->elem_mat.push_back(p.emat[2 * e]);
      in->elem_mat.push_back(p.emat[2 * e + 1]);
      in->elem_hom.push_back(p.ehom[2 * e]);
      in->elem_hom.push_back(p.ehom[2 * e + 1]);
      in->elem_part.push_back(r);
      in->elem_local.push_back(e);
      for (int f = 0; f < 4; f++) {
        in->bnd_id.push_back(p.bid[4 * e + f]);
        in->bnd_type.push_back(p.btype[4 * e + f]);
      }
    }
    I.nln += p.nln;
    I.nel_s += p.nel_s;
    I.nel_v += p.nel_v;
  }
  I.ne = in->part_elem_off[nparts];
  in->node_map = std::move(lmap);
  in->defl = p0.defl;
  in->mat_vals = p0.mats;
  in->dev_pot = p0.devp;
  in->vol_pot = p0.volp;
  in->cf = p0.cf;
  in->ee = p0.ee;
  *out = in;
  return PGFEM_GPU_OK;
}

int pgfem_input_get_info(const pgfem_input *in, pgfem_input_info *info) {
  if (!in || !info) return PGFEM_GPU_EINVAL;
  *info = in->info;
  return PGFEM_GPU_OK;
}

int pgfem_input_get_mesh(const pgfem_input *in, double *X, int *conn, long *codes, double *defl) {
  if (!in || !X || !conn || !codes || (in->info.npres && !defl)) return PGFEM_GPU_EINVAL;
  memcpy(X, in->X.data(), sizeof(double) * in->X.size());
  memcpy(conn, in->conn.data(), sizeof(int) * in->conn.size());
  memcpy(codes, in->codes.data(), sizeof(long) * in->codes.size());
  if (in->info.npres) memcpy(defl, in->defl.data(), sizeof(double) * in->defl.size());
  return PGFEM_GPU_OK;
}

int pgfem_input_get_elements(const pgfem_input *in, long *mat, long *hom, int *part, long *local_id) {
  if (!in) return PGFEM_GPU_EINVAL;
  const size_t ne = (size_t)in->info.ne;
  if (mat) memcpy(mat, in->elem_mat.data(), sizeof(long) * 2 * ne);
  if (hom) memcpy(hom, in->elem_hom.data(), sizeof(long) * 2 * ne);
  if (part) memcpy(part, in->elem_part.data(), sizeof(int) * ne);
  if (local_id) memcpy(local_id, in->elem_local.data(), sizeof(long) * ne);
  return PGFEM_GPU_OK;
}

int pgfem_input_get_materials(const pgfem_input *in, double *vals, int *dev_pot, int *vol_pot) {
  if (!in || (in->info.nmat && (!vals || !dev_pot || !vol_pot))) return PGFEM_GPU_EINVAL;
  if (!in->info.nmat) return PGFEM_GPU_OK;
  memcpy(vals, in->mat_vals.data(), sizeof(double) * in->mat_vals.size());
  memcpy(dev_pot, in->dev_pot.data(), sizeof(int) * in->dev_pot.size());
  memcpy(vol_pot, in->vol_pot.data(), sizeof(int) * in->vol_pot.size());
  return PGFEM_GPU_OK;
}

int pgfem_input_read_orientations(const pgfem_input *in, const char *base, double *angles, int *euler_type) {
  if (!in || !base || !angles) return PGFEM_GPU_EINVAL;
  const long ne = in->info.ne;
  for (long k = 0; k < 3 * ne; k++) angles[k] = NAN;
  int etype = 0;
  for (int r = 0; r < in->nparts; r++) {
    const std::string path = std::string(base) + "_" + std::to_string(r) + ".in";
    FILE *f = fopen(path.c_str(), "r");
    if (!f) return fail("cannot open " + path);
    const long e0 = in->part_elem_off[r], npe = in->part_elem_off[r + 1] - e0;
    char line[1024];
    long lineno = 0;
    while (fgets(line, sizeof line, f)) {
      lineno++;
      if (line[0] == '#') {  // "# EulerAngleType: k"
        const char *key = strstr(line, "EulerAngleType:");
        if (key) etype = atoi(key + strlen("EulerAngleType:"));
        continue;
      }
      long e, ip;
      double a[3];
      const int got = sscanf(line, "%ld %ld %lf %lf %lf", &e, &ip, a, a + 1, a + 2);
      if (got <= 0) continue;  // blank line
      if (got != 5) {
        fclose(f);
        return fail(path + ":" + std::to_string(lineno) + ": bad orientation line");
      }
      if (e < 0) {  // every element of material `ip` of this partition
        for (long k = 0; k < npe; k++)
          if (in->elem_mat[2 * (e0 + k)] == ip)
            for (int j = 0; j < 3; j++) angles[3 * (e0 + k) + j] = a[j];
      } else {
        if (e >= npe || ip != 0) {  // one integration point per linear tet
          fclose(f);
          return fail(path + ":" + std::to_string(lineno) + ": element or point out of range");
        }
        for (int j = 0; j < 3; j++) angles[3 * (e0 + e) + j] = a[j];
      }
    }
    fclose(f);
  }
  if (euler_type) *euler_type = etype;
  return PGFEM_GPU_OK;
}

int pgfem_input_get_periodic(const pgfem_input *in, long *Pr) {
  if (!in || !Pr) return PGFEM_GPU_EINVAL;
  memcpy(Pr, in->Pr.data(), sizeof(long) * in->Pr.size());
  return PGFEM_GPU_OK;
}

int pgfem_input_get_partition(const pgfem_input *in, int part, long *nn, long *ne, long *node_map) {
  if (!in || part < 0 || part >= in->nparts) return PGFEM_GPU_EINVAL;
  const std::vector<long> &m = in->node_map[part];
  if (nn) *nn = (long)m.size();
  if (ne) *ne = in->part_elem_off[part + 1] - in->part_elem_off[part];
  if (node_map) memcpy(node_map, m.data(), sizeof(long) * m.size());
  return PGFEM_GPU_OK;
}

void pgfem_input_destroy(pgfem_input *in) { delete in; }

int pgfem_euler_rotation(long n, const double *angles, double *R) {
  if (n < 0 || (n && (!angles || !R))) return PGFEM_GPU_EINVAL;
  for (long k = 0; k < n; k++) {
    const double ph = angles[3 * k], th = angles[3 * k + 1], ps = angles[3 * k + 2];
    const double cx = cos(ph), sx = sin(ph), cy = cos(th), sy = sin(th), cz = cos(ps), sz = sin(ps);
    const double Ax[9] = {1, 0, 0, 0, cx, -sx, 0, sx, cx};
    const double Ay[9] = {cy, 0, sy, 0, 1, 0, -sy, 0, cy};
    const double Az[9] = {cz, -sz, 0, sz, cz, 0, 0, 0, 1};
    double T[9];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        T[i * 3 + j] = Ay[i * 3] * Ax[j] + Ay[i * 3 + 1] * Ax[3 + j] + Ay[i * 3 + 2] * Ax[6 + j];
    double *Rk = R + 9 * k;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        Rk[i * 3 + j] = Az[i * 3] * T[j] + Az[i * 3 + 1] * T[3 + j] + Az[i * 3 + 2] * T[6 + j];
  }
  return PGFEM_GPU_OK;
}

int pgfem_input_read_multiphysics(const char *path, int max_phys, int *ids, int *ndim, int *n) {
  if (!path || !n || max_phys < 0 || (max_phys && (!ids || !ndim))) return PGFEM_GPU_EINVAL;
  Tokens t;
  if (!t.load(path)) return fail(std::string("cannot open ") + path);
  auto bad = [&](const char *what) { return fail(std::string("bad ") + what + " at " + t.where()); };
  int np;
  if (!t.num(np) || np < 1) return bad("physics count");
  for (int k = 0; k < np; k++) {
    int id, nd, nc, nv;
    std::string name;
    if (!t.num(id) || !t.next(name) || !t.num(nd)) return bad("physics line (id name ndim)");
    if (!t.num(nc) || nc < 0) return bad("coupling count");
    for (int j = 0; j < nc; j++) {
      int c;
      if (!t.num(c)) return bad("coupled physics id");
    }
    if (!t.num(nv) || nv < 0) return bad("output variable count");
    for (int j = 0; j < nv; j++) {
      int v;
      if (!t.num(v)) return bad("output variable id");
    }
    if (k < max_phys) {
      ids[k] = id;
      ndim[k] = nd;
    }
  }
  *n = np;
  return PGFEM_GPU_OK;
}

int pgfem_input_read_solver_file(const char *path, long npd, pgfem_solver_file *sf, double *times,
                                 long *print_steps, long *load_steps, double *load_incr) {
  if (!path || !sf) return PGFEM_GPU_EINVAL;
  Tokens t;
  if (!t.load(path)) return fail(std::string("cannot open ") + path);
  auto bad = [&](const char *what) { return fail(std::string("bad ") + what + " at " + t.where()); };
  pgfem_solver_file s{};
  if (!t.num(s.nor_min) || !t.num(s.iter_max) || !t.num(s.npres) || !t.num(s.FNR)) return bad("solver line");
  if (s.FNR == 2 || s.FNR == 3)
    if (!t.num(s.dAL0) || !t.num(s.dALMAX)) return bad("arc-length line");
  if (s.FNR == 4) {
    if (!t.num(s.physicsno) || !t.num(s.max_NR_staggering) || s.physicsno < 1) return bad("multiphysics line");
    for (int k = 0; k < s.physicsno; k++) {
      int sub, setr;
      if (!t.num(sub) || !t.num(setr)) return bad("per-physics solver line");
      if (k == 0) s.max_subdivision = sub;
      if (setr) {
        double du;
        if (!t.num(du)) return bad("initial residual scale");
      }
    }
  }
  if (!t.num(s.nt) || s.nt < 0) return bad("time step count");
  for (long k = 0; k <= s.nt; k++) {
    double v;
    if (!t.num(v)) return bad("time");
    if (times) times[k] = v;
  }
  if (!t.num(s.n_print) || s.n_print < 0) return bad("output step count");
  for (long k = 0; k < s.n_print; k++) {
    long v;
    if (!t.num(v)) return bad("output step");
    if (print_steps) print_steps[k] = v;
  }
  // no load section: the history is in a load directory (<input>/load/<physics>.load,
  // src/read_input_file.cc:646-673), not read here
  if (t.eof()) {
    s.n_load = 0;
    s.n_incr = npd >= 0 ? npd : s.npres;
    *sf = s;
    return PGFEM_GPU_OK;
  }
  if (!t.num(s.n_load) || s.n_load < 0) return bad("load step count");
  for (long k = 0; k < s.n_load; k++) {
    long v;
    if (!t.num(v)) return bad("load step");
    if (load_steps) load_steps[k] = v;
  }
  // prescribed-value increments, one per prescribed value of the mesh per
  // load step (the reference reads them while stepping; all of them here)
  s.n_incr = npd >= 0 ? npd : s.npres;
  for (long k = 0; k < s.n_load * s.n_incr; k++) {
    double v;
    if (!t.num(v)) return bad("load increment");
    if (load_incr) load_incr[k] = v;
  }
  *sf = s;
  return PGFEM_GPU_OK;
}

int pgfem_input_read_model_params(const char *path, int max_entries, pgfem_model_params *out, int *n) {
  if (!path || !n || max_entries < 0 || (max_entries && !out)) return PGFEM_GPU_EINVAL;
  Tokens t;
  if (!t.load(path)) return fail(std::string("cannot open ") + path);
  auto bad = [&](const char *what) { return fail(std::string("bad ") + what + " at " + t.where()); };
  int count;
  if (!t.num(count) || count < 0) return bad("entry count");
  int k = 0;
  for (; k < count; k++) {
    pgfem_model_params m{};
    std::string tok;
    if (!t.num(m.mat_id) || !t.num(m.model_type)) return bad("entry header (mat_id model_type)");
    if (!t.next(tok) || tok != "{") return bad("opening brace");
    if (m.model_type == PGFEM_CM_UQCM) {
      if (!t.num(m.model_type)) return bad("UQ model type");
      m.uq = 1;
    }
    if (m.mat_id >= 0 && m.model_type == PGFEM_CM_CRYSTAL_PLASTICITY) {
      // gamma_dot_0 m G0 g0 gs_0 gamma_dot_s w; unit cell; orientation option (+ its data)
      for (int j = 0; j < 7; j++)
        if (!t.num(m.p[j])) return bad("crystal plasticity parameters");
      m.np = 7;
      if (!t.num(m.unit_cell) || !t.num(m.ort_option[0])) return bad("slip system / orientation option");
      if (m.ort_option[0] == 0 && !t.num(m.ort_option[1])) return bad("orientation option");
      if (m.ort_option[0] == 2) {
        std::string f;
        if (!t.next(f) || f == "}" || f.size() >= sizeof(m.ort_file)) return bad("orientation file");
        strcpy(m.ort_file, f.c_str());
      }
      if (m.ort_option[0] == 3)
        for (int j = 0; j < 3; j++)
          if (!t.num(m.ort_angles[j])) return bad("orientation angles");
      if (t.peek_int()) {
        int set;
        t.num(set);
        if (set) {
          m.solver_set = 1;
          if (!t.num(m.max_itr_stag) || !t.num(m.max_itr_hardening) || !t.num(m.max_itr_M) ||
              !t.num(m.max_subdivision) || !t.num(m.tol_hardening) || !t.num(m.tol_M) || !t.num(m.computer_zero))
            return bad("crystal plasticity solver parameters");
        }
      }
    } else if (m.mat_id >= 0 && m.model_type == PGFEM_CM_J2_PLASTICITY_DAMAGE) {
      // beta hp k0; damage mu w_max P1 P2 Yin; da db_p db_m va vb_p vb_m
      for (int j = 0; j < 14; j++)
        if (!t.num(m.p[j])) return bad("J2 plasticity parameters");
      m.np = 14;
    }
    // the rest of the block (other models, or data this path does not use)
    while (t.next(tok) && tok != "}") {
    }
    if (tok != "}") return bad("closing brace");
    if (k < max_entries) out[k] = m;
  }
  *n = k;
  return PGFEM_GPU_OK;
}

// The material of a J2 entry (CM_J2P_PARAM::read_param,
// src/cm_j2_plasticity.cc:865-932: G and nu from the mesh file's material line,
// then beta hp k0 and the damage block).  Elasticity is the spatial
// neo-Hookean form with the material line's volumetric potential; the return
// map is J2 with yield function ||dev tau|| - sqrt(2/3) (k0 + hp ep) and linear
// isotropic hardening: sigma_y = k0, H = hp.  beta = 0 (the reference's own
// driver value, tests/constitutive_model/cm_j2_plasticity_driver.cc:64-83) is
// the only hardening mix carried; damage must be off (mu = 0: the damage
// variable never evolves).  Other values return PGFEM_GPU_EINVAL.
int pgfem_input_j2_material(const pgfem_model_params *mp, double E, double nu, int vol_pot,
                            pgfem_material_desc *out) {
  if (!mp || !out || mp->model_type != PGFEM_CM_J2_PLASTICITY_DAMAGE || mp->np != 14) return PGFEM_GPU_EINVAL;
  const double beta = mp->p[0], hp = mp->p[1], k0 = mp->p[2], mu = mp->p[3];
  if (beta != 0.0 || mu != 0.0 || !(k0 > 0.0) || !(hp >= 0.0) || !(E > 0.0) || !(nu > -1.0 && nu < 0.5))
    return PGFEM_GPU_EINVAL;
  if (!(vol_pot <= 0 || vol_pot == 2 || vol_pot == 3 || vol_pot == 99)) return PGFEM_GPU_EINVAL;
  pgfem_material_desc m{};
  m.model = PGFEM_MODEL_J2;
  m.E = E;
  m.nu = nu;
  m.sigma_y = k0;
  m.H = hp;
  m.dev_pot = 1;
  m.vol_pot = vol_pot <= 0 ? 99 : vol_pot;
  *out = m;
  return PGFEM_GPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Restart files of one rank (write_restart_constitutive_model /
// read_restart_constitutive_model, src/restart.cc:187-300): per node the pairs
// "u_nm1 u_n" of x, y, z on one line; then per element its point count and per
// point the model's block of write_restart -- HE (HE_PARAM::write_restart,
// src/plasticity_model_none.cc:298-311): Fn, Fnm1; CP (CP_PARAM::write_restart,
// src/plasticity_model.cc:883-911): Fn, Fnm1, pFn, pFnm1 (cm_write_tensor_restart,
// src/constitutive_model.cc:4005-4013, one tensor of 9 per line), tau_n[12],
// gamma_dot_n[12], then g_n g_nm1 L_n L_nm1; J2 (CM_J2P_PARAM::write_restart,
// src/cm_j2_plasticity.cc:784-808): Fn, pSn, Fnm1, pSnm1, then w_n w_nm1 X_n
// X_nm1 H_n H_nm1 ep_n ep_nm1 gam_n gam_nm1 on one line and the damage flag
// (an integer) on the next.  Numbers in %.17e.
// ---------------------------------------------------------------------------
extern "C" {

int pgfem_restart_block_size(int model) {
  switch (model) {
    case PGFEM_MODEL_HE: return 18;
    case PGFEM_MODEL_CP: return 4 * 9 + 12 + 12 + 4;
    case PGFEM_MODEL_J2: return 4 * 9 + 10 + 1;
    default: return -1;
  }
}

int pgfem_restart_format(const char *path, long nn, long ne, int n_ip, int model, const double *u_nm1,
                         const double *u_n, const double *blocks) {
  const int bs = pgfem_restart_block_size(model);
  if (!path || nn < 0 || ne < 0 || n_ip < 1 || bs < 0 || (nn && (!u_nm1 || !u_n)) || (ne && !blocks))
    return PGFEM_GPU_EINVAL;
  FILE *f = fopen(path, "w");
  if (!f) return fail(std::string("cannot create ") + path);
  for (long a = 0; a < nn; a++) {
    for (int b = 0; b < 3; b++) fprintf(f, "%.17e %.17e ", u_nm1[3 * a + b], u_n[3 * a + b]);
    fprintf(f, "\n");
  }
  auto tensor = [&](const double *t) {
    fprintf(f, "%.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e %.17e\n", t[0], t[1], t[2], t[3], t[4], t[5], t[6],
            t[7], t[8]);
  };
  for (long e = 0; e < ne; e++) {
    fprintf(f, "%d\n", n_ip);
    for (int q = 0; q < n_ip; q++) {
      const double *b = blocks + ((size_t)e * n_ip + q) * bs;
      tensor(b);
      tensor(b + 9);
      if (model == PGFEM_MODEL_J2) {
        tensor(b + 18);
        tensor(b + 27);
        for (int k = 0; k < 10; k++) fprintf(f, k < 9 ? "%.17e " : "%.17e\n", b[36 + k]);
        fprintf(f, "%d\n", (int)b[46]);
      }
      if (model == PGFEM_MODEL_CP) {
        tensor(b + 18);
        tensor(b + 27);
        for (int k = 0; k < 12; k++) fprintf(f, "%.17e ", b[36 + k]);
        fprintf(f, "\n");
        for (int k = 0; k < 12; k++) fprintf(f, "%.17e ", b[48 + k]);
        fprintf(f, "\n");
        fprintf(f, "%.17e %.17e %.17e %.17e\n", b[60], b[61], b[62], b[63]);
      }
    }
  }
  const bool ok = !ferror(f);
  fclose(f);
  return ok ? PGFEM_GPU_OK : fail(std::string("write error on ") + path);
}

int pgfem_restart_parse(const char *path, long nn, long ne, int n_ip, int model, double *u_nm1, double *u_n,
                        double *blocks) {
  const int bs = pgfem_restart_block_size(model);
  if (!path || nn < 0 || ne < 0 || n_ip < 1 || bs < 0 || (nn && (!u_nm1 || !u_n)) || (ne && !blocks))
    return PGFEM_GPU_EINVAL;
  Tokens t;
  if (!t.load(path)) return fail(std::string("cannot open ") + path);
  auto bad = [&](const char *what) { return fail(std::string("bad ") + what + " at " + t.where()); };
  for (long a = 0; a < nn; a++)
    for (int b = 0; b < 3; b++)
      if (!t.num(u_nm1[3 * a + b]) || !t.num(u_n[3 * a + b])) return bad("nodal displacement");
  for (long e = 0; e < ne; e++) {
    long nip;
    if (!t.num(nip)) return bad("point count");
    if (nip != n_ip) return bad("point count (element type)");
    for (int q = 0; q < n_ip; q++) {
      double *b = blocks + ((size_t)e * n_ip + q) * bs;
      for (int k = 0; k < bs; k++)
        if (!t.num(b[k]))
          return bad(model == PGFEM_MODEL_CP   ? "crystal plasticity block"
                     : model == PGFEM_MODEL_J2 ? "J2 plasticity block"
                                               : "hyperelastic block");
    }
  }
  if (!t.eof()) return bad("trailing data (mesh or model does not match the file)");
  return PGFEM_GPU_OK;
}

}  // extern "C"

extern "C" {

int pgfem_restart_write_partitions(const pgfem_input *in, const char *name, int step, int model, int n_ip,
                                   const double *u_nm1, const double *u_n, const double *blocks) {
  const int bs = pgfem_restart_block_size(model);
  if (!in || !name || step < 0 || n_ip < 1 || bs < 0 || !u_nm1 || !u_n || !blocks) return PGFEM_GPU_EINVAL;
  for (int r = 0; r < in->nparts; r++) {
    const std::vector<long> &nm = in->node_map[r];
    const long e0 = in->part_elem_off[r], ne = in->part_elem_off[r + 1] - e0;
    std::vector<double> a(3 * nm.size()), b(3 * nm.size());
    for (size_t i = 0; i < nm.size(); i++)
      for (int j = 0; j < 3; j++) {
        a[3 * i + j] = u_nm1[3 * nm[i] + j];
        b[3 * i + j] = u_n[3 * nm[i] + j];
      }
    const std::string path = std::string(name) + "_" + std::to_string(r) + "_" + std::to_string(step) + ".res";
    const int e = pgfem_restart_format(path.c_str(), (long)nm.size(), ne, n_ip, model, a.data(), b.data(),
                                       blocks + (size_t)e0 * n_ip * bs);
    if (e) return e;
  }
  return PGFEM_GPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Surface loads: NBC/<physics>.nbc (read_Neumann_boundary_conditions,
// src/read_input_file.cc:168-214; NeumannBoundaryElement::read_loads,
// src/PGFem3D_data_structure.cc:934-948), the element faces they load
// (construct_list_of_boundary_elements, :825-895, from the elements' face
// features, src/element.cc:168-199) and their load values at a time
// (compute_load_values, :956-972).  The reference evaluates each load file's
// first line with the exprtk library as a function of t with exprtk's
// constants (string_function_of_time, src/utils.cc:3423-3440); this reader
// evaluates the arithmetic subset written below (comments, numbers, t, pi, epsilon, inf,
// + - * / % ^, comparisons, and / or, "c ? a : b", if(c, a, b), min, max,
// clamp, abs, sgn, sqrt, exp, log, log10, log2, pow, hypot, floor, ceil,
// round, trunc, frac, sin, cos, tan, asin, acos, atan, atan2, sinh, cosh,
// tanh), and rejects anything else with EFORMAT rather than guessing.
// ---------------------------------------------------------------------------
struct pgfem_nbc {
  std::vector<int> ftype, fid, ltype;
  std::vector<std::string> expr;  // 3 per feature, load_type of them set
};

namespace {

struct Expr {
  const std::string &s;
  double t;
  size_t i = 0;
  std::string err;

  Expr(const std::string &src, double tv) : s(src), t(tv) {}
  // white space and comments (# or // to the end of the line, /* ... */)
  void ws() {
    for (;;) {
      while (i < s.size() && isspace((unsigned char)s[i])) i++;
      if (i < s.size() && (s[i] == '#' || s.compare(i, 2, "//") == 0)) {
        while (i < s.size() && s[i] != '\n') i++;
      } else if (s.compare(i, 2, "/*") == 0) {
        const size_t e = s.find("*/", i + 2);
        i = e == std::string::npos ? s.size() : e + 2;
      } else {
        return;
      }
    }
  }
  bool eat(const char *tok) {
    ws();
    const size_t n = strlen(tok);
    if (s.compare(i, n, tok) != 0) return false;
    // a word operator must not run into an identifier
    if (isalpha((unsigned char)tok[0]) && i + n < s.size() && (isalnum((unsigned char)s[i + n]) || s[i + n] == '_'))
      return false;
    i += n;
    return true;
  }
  bool fail_at(const std::string &m) {
    if (err.empty()) err = m + " at column " + std::to_string(i + 1);
    return false;
  }
  bool ternary(double &v) {
    if (!logic_or(v)) return false;
    if (eat("?")) {
      double a, b;
      if (!ternary(a)) return false;
      if (!eat(":")) return fail_at("expected ':'");
      if (!ternary(b)) return false;
      v = v != 0.0 ? a : b;
    }
    return true;
  }
  bool logic_or(double &v) {
    if (!logic_and(v)) return false;
    for (;;) {
      if (eat("||") || eat("or") || eat("|")) {
        double w;
        if (!logic_and(w)) return false;
        v = (v != 0.0 || w != 0.0) ? 1.0 : 0.0;
      } else {
        return true;
      }
    }
  }
  bool logic_and(double &v) {
    if (!compare(v)) return false;
    for (;;) {
      if (eat("&&") || eat("and") || eat("&")) {
        double w;
        if (!compare(w)) return false;
        v = (v != 0.0 && w != 0.0) ? 1.0 : 0.0;
      } else {
        return true;
      }
    }
  }
  bool compare(double &v) {
    if (!additive(v)) return false;
    for (;;) {
      int op;
      if (eat("<=")) op = 0;
      else if (eat(">=")) op = 1;
      else if (eat("==")) op = 2;
      else if (eat("!=") || eat("<>")) op = 3;
      else if (eat("<")) op = 4;
      else if (eat(">")) op = 5;
      else if (eat("=")) op = 2;
      else return true;
      double w;
      if (!additive(w)) return false;
      const bool r[6] = {v <= w, v >= w, v == w, v != w, v < w, v > w};
      v = r[op] ? 1.0 : 0.0;
    }
  }
  bool additive(double &v) {
    if (!multiplicative(v)) return false;
    for (;;) {
      if (eat("+")) {
        double w;
        if (!multiplicative(w)) return false;
        v += w;
      } else if (eat("-")) {
        double w;
        if (!multiplicative(w)) return false;
        v -= w;
      } else {
        return true;
      }
    }
  }
  bool multiplicative(double &v) {
    if (!unary(v)) return false;
    for (;;) {
      if (eat("*")) {
        double w;
        if (!unary(w)) return false;
        v *= w;
      } else if (eat("/")) {
        double w;
        if (!unary(w)) return false;
        v /= w;
      } else if (eat("%")) {
        double w;
        if (!unary(w)) return false;
        v = std::fmod(v, w);
      } else {
        return true;
      }
    }
  }
  bool unary(double &v) {
    if (eat("-")) {
      if (!unary(v)) return false;
      v = -v;
      return true;
    }
    if (eat("+")) return unary(v);
    if (eat("not")) {
      if (!unary(v)) return false;
      v = v == 0.0 ? 1.0 : 0.0;
      return true;
    }
    return power(v);
  }
  bool power(double &v) {
    if (!primary(v)) return false;
    if (eat("^")) {
      double w;
      if (!unary(w)) return false;  // right associative
      v = std::pow(v, w);
    }
    return true;
  }
  bool args(std::vector<double> &a) {
    if (!eat("(")) return fail_at("expected '('");
    if (eat(")")) return true;
    for (;;) {
      double v;
      if (!ternary(v)) return false;
      a.push_back(v);
      if (eat(")")) return true;
      if (!eat(",")) return fail_at("expected ',' or ')'");
    }
  }
  bool primary(double &v) {
    ws();
    if (i >= s.size()) return fail_at("unexpected end");
    if (eat("(")) {
      if (!ternary(v)) return false;
      if (!eat(")")) return fail_at("expected ')'");
      return true;
    }
    const char c = s[i];
    if (isdigit((unsigned char)c) || c == '.') {
      const char *b = s.c_str() + i;
      char *end = nullptr;
      v = strtod(b, &end);
      if (end == b) return fail_at("bad number");
      i += (size_t)(end - b);
      return true;
    }
    if (!isalpha((unsigned char)c) && c != '_') return fail_at(std::string("unexpected '") + c + "'");
    const size_t b = i;
    while (i < s.size() && (isalnum((unsigned char)s[i]) || s[i] == '_')) i++;
    std::string w = s.substr(b, i - b);
    for (char &ch : w) ch = (char)tolower((unsigned char)ch);
    if (w == "t") return v = t, true;
    if (w == "pi") return v = 3.14159265358979323846, true;
    if (w == "epsilon") return v = 2.220446049250313e-16, true;
    if (w == "inf") return v = HUGE_VAL, true;
    if (w == "true") return v = 1.0, true;
    if (w == "false") return v = 0.0, true;
    std::vector<double> a;
    const size_t at = b;
    if (!args(a)) return false;
    auto need = [&](size_t n) {
      if (a.size() == n) return true;
      i = at;
      return fail_at(w + " takes " + std::to_string(n) + " argument(s)");
    };
    if (w == "min" || w == "max") {
      if (a.empty()) return need(1);
      v = a[0];
      for (double x : a) v = w == "min" ? std::min(v, x) : std::max(v, x);
      return true;
    }
    if (w == "if") return need(3) && (v = a[0] != 0.0 ? a[1] : a[2], true);
    if (w == "clamp") return need(3) && (v = std::min(std::max(a[1], a[0]), a[2]), true);
    if (w == "pow") return need(2) && (v = std::pow(a[0], a[1]), true);
    if (w == "atan2") return need(2) && (v = std::atan2(a[0], a[1]), true);
    if (w == "hypot") return need(2) && (v = std::hypot(a[0], a[1]), true);
    if (w == "mod") return need(2) && (v = std::fmod(a[0], a[1]), true);
    if (!need(1)) return false;
    const double x = a[0];
    if (w == "abs") v = std::fabs(x);
    else if (w == "sgn") v = x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0);
    else if (w == "sqrt") v = std::sqrt(x);
    else if (w == "exp") v = std::exp(x);
    else if (w == "log") v = std::log(x);
    else if (w == "log10") v = std::log10(x);
    else if (w == "log2") v = std::log2(x);
    else if (w == "floor") v = std::floor(x);
    else if (w == "ceil") v = std::ceil(x);
    else if (w == "round") v = std::round(x);
    else if (w == "trunc") v = std::trunc(x);
    else if (w == "frac") v = x - std::trunc(x);
    else if (w == "sin") v = std::sin(x);
    else if (w == "cos") v = std::cos(x);
    else if (w == "tan") v = std::tan(x);
    else if (w == "asin") v = std::asin(x);
    else if (w == "acos") v = std::acos(x);
    else if (w == "atan") v = std::atan(x);
    else if (w == "sinh") v = std::sinh(x);
    else if (w == "cosh") v = std::cosh(x);
    else if (w == "tanh") v = std::tanh(x);
    else {
      i = at;
      return fail_at("unknown function or name '" + w + "'");
    }
    return true;
  }
  // a whole expression, optionally ended by ';'
  bool run(double &v) {
    if (!ternary(v)) return false;
    eat(";");
    ws();
    if (i != s.size()) return fail_at("trailing text");
    return true;
  }
};

}  // namespace

extern "C" {

int pgfem_input_get_element_faces(const pgfem_input *in, int *bnd_type, int *bnd_id) {
  if (!in) return PGFEM_GPU_EINVAL;
  if (bnd_type) std::copy(in->bnd_type.begin(), in->bnd_type.end(), bnd_type);
  if (bnd_id) std::copy(in->bnd_id.begin(), in->bnd_id.end(), bnd_id);
  return PGFEM_GPU_OK;
}

int pgfem_load_expression(const char *expr, double t, double *value) {
  if (!expr || !value) return PGFEM_GPU_EINVAL;
  const std::string s(expr);
  Expr x(s, t);
  double v = 0.0;
  if (!x.run(v)) return fail("load expression \"" + s + "\": " + x.err);
  *value = v;
  return PGFEM_GPU_OK;
}

int pgfem_input_read_nbc(const char *ipath, const char *physics, pgfem_nbc **out) {
  if (!ipath || !physics || !out) return PGFEM_GPU_EINVAL;
  *out = nullptr;
  auto *nb = new pgfem_nbc();
  const std::string dir = std::string(ipath) + "/NBC";
  Tokens t;
  if (!t.load(dir + "/" + physics + ".nbc")) {  // no NBC directory or file: no surface loads
    *out = nb;
    return PGFEM_GPU_OK;
  }
  auto reject = [&](const std::string &m) {
    delete nb;
    return fail(m);
  };
  long nf;
  if (!t.num(nf) || nf < 0) return reject("bad feature count at " + t.where());
  for (long f = 0; f < nf; f++) {
    int ft, fi, lt;
    if (!t.num(ft) || !t.num(fi) || !t.num(lt)) return reject("bad feature line at " + t.where());
    if (lt < 1 || lt > 3) return reject("load type " + std::to_string(lt) + " at " + t.where() + " (1 to 3 values)");
    for (long g = 0; g < f; g++)
      if (nb->ftype[g] == ft && nb->fid[g] == fi)
        return reject("feature (" + std::to_string(ft) + ", " + std::to_string(fi) + ") listed twice at " + t.where());
    nb->ftype.push_back(ft);
    nb->fid.push_back(fi);
    nb->ltype.push_back(lt);
    for (int k = 0; k < 3; k++) {
      std::string line;
      if (k < lt) {
        std::string fn;
        if (!t.next(fn)) return reject("missing load file name at " + t.where());
        FILE *fp = fopen((dir + "/" + fn).c_str(), "rb");
        if (!fp) return reject("cannot open " + dir + "/" + fn);
        int ch;
        while ((ch = fgetc(fp)) != EOF && ch != '\n') line.push_back((char)ch);
        fclose(fp);
        double v;
        Expr x(line, 0.0);
        if (!x.run(v)) return reject(dir + "/" + fn + ": " + x.err);
      }
      nb->expr.push_back(line);
    }
  }
  *out = nb;
  return PGFEM_GPU_OK;
}

int pgfem_nbc_get_features(const pgfem_nbc *nb, int *nfeature, int *ftype, int *fid, int *load_type) {
  if (!nb) return PGFEM_GPU_EINVAL;
  const size_t n = nb->ftype.size();
  if (nfeature) *nfeature = (int)n;
  if (ftype) std::copy(nb->ftype.begin(), nb->ftype.end(), ftype);
  if (fid) std::copy(nb->fid.begin(), nb->fid.end(), fid);
  if (load_type) std::copy(nb->ltype.begin(), nb->ltype.end(), load_type);
  return PGFEM_GPU_OK;
}

int pgfem_nbc_faces(const pgfem_nbc *nb, const pgfem_input *in, long *nface, long *elem, int *face, int *feature) {
  if (!nb || !in || !nface) return PGFEM_GPU_EINVAL;
  long k = 0;
  for (long e = 0; e < in->info.ne; e++)
    for (int f = 0; f < 4; f++) {
      int hit = -1;
      for (size_t g = 0; g < nb->ftype.size(); g++)
        if (nb->ftype[g] == in->bnd_type[4 * e + f] && nb->fid[g] == in->bnd_id[4 * e + f]) hit = (int)g;
      if (hit < 0) continue;
      if (elem) elem[k] = e;
      if (face) face[k] = f;
      if (feature) feature[k] = hit;
      k++;
    }
  *nface = k;
  return PGFEM_GPU_OK;
}

int pgfem_nbc_load_values(const pgfem_nbc *nb, double t, double *load) {
  if (!nb || !load) return PGFEM_GPU_EINVAL;
  for (size_t f = 0; f < nb->ftype.size(); f++)
    for (int k = 0; k < 3; k++) {
      double v = 0.0;
      if (k < nb->ltype[f]) {
        Expr x(nb->expr[3 * f + k], t);
        if (!x.run(v)) return fail("load expression \"" + nb->expr[3 * f + k] + "\": " + x.err);
      }
      load[3 * f + k] = v;
    }
  return PGFEM_GPU_OK;
}

void pgfem_nbc_destroy(pgfem_nbc *nb) { delete nb; }

}  // extern "C"
