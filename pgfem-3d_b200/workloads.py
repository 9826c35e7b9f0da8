"""Synthetic workloads of the assembly path (structured unit-cube tet meshes).

No public benchmark or dataset exists for this path; every input is
generated from a seed with splitmix64 (keyed by seed and array index), so the
GPU path, the CPU oracle and any rerun see bit-identical inputs.

Workloads (units: MPa, mm-free unit cube):
  he_p1     n^3 cells x 6 linear tets, compressible neo-Hookean E=200 GPa,
            nu=0.3; u = 0.01 x e_x + U(-a,a)^3, a = 1e-3 h; x=0 face fixed.
  j2_p2     n^3 cells x 6 quadratic tets (4-point rule), J2 E=200 GPa,
            nu=0.3, sigma_y=250 MPa, H=2 GPa; state Cp^-1 = I, eqps = 0;
            u = (Fbar - I) X + U(-a,a)^3, a = 1e-4 h, all DOFs free.  The
            stretch of Fbar sits at the onset of yield (eps = sigma_y/2mu) so
            that about half of the points yield; a 2 % stretch would yield
            every point (trial stress ~ 4 GPa vs 250 MPa).
"""
import numpy as np

import pgfem_gpu as pg

MASK64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed, n, stream=0):
    """n uniform doubles in [0,1) from splitmix64(seed, stream, index)."""
    with np.errstate(over="ignore"):
        idx = np.arange(n, dtype=np.uint64)
        z = (np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15) + np.uint64(stream) * np.uint64(0xD1B54A32D192ED03)
             + (idx + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


class Problem:
    """Mesh + DOFs + CSR pattern + material + one displacement iterate."""

    def __init__(self, name, X, conn, ids, ndof, Ap, Ai, mat, u, u_presc=None, state=None, F0=None,
                 R_cp=None, dt=0.0, Pr=None, meta=None):
        self.name, self.X, self.conn, self.ids, self.ndof = name, X, conn, ids, ndof
        self.Ap, self.Ai, self.mat, self.u, self.u_presc = Ap, Ai, mat, u, u_presc
        self.state, self.F0, self.R_cp, self.dt, self.Pr = state, F0, R_cp, dt, Pr
        self.meta = meta or {}

    @property
    def nne(self):
        return self.conn.shape[1]

    @property
    def ne(self):
        return self.conn.shape[0]

    @property
    def nint(self):
        return 4 if self.nne == 10 else 1

    @property
    def nqp(self):
        return self.ne * self.nint

    @property
    def nnz(self):
        return int(self.Ap[-1])

    def context(self):
        ctx = pg.Context(self.X, self.conn, self.ids, self.ndof, self.Ap, self.Ai, self.mat,
                         npres=0 if self.u_presc is None else len(self.u_presc), F0=self.F0, R_cp=self.R_cp)
        if self.state is not None:
            ctx.set_state(self.state)
        return ctx


def nodal_to_free(ids, disp):
    """Free-DOF vector from a nodal displacement field (nn,3)."""
    ndof = int(ids.max())
    u = np.zeros(max(ndof, 0))
    m = ids > 0
    u[ids[m] - 1] = disp[m]
    return u


# local faces of a tet by their vertex nodes (FEMLIB's Tet2Tri numbering)
TET_FACES = np.array([[0, 2, 1], [0, 1, 3], [1, 2, 3], [0, 3, 2]])


def box_faces(X, conn, axis, value, tol=1e-12):
    """The element faces lying on the plane X[axis] = value: (elem, face)
    arrays, face the local face 0..3 whose three vertex nodes are on it (the
    synthetic meshes' stand-in for the reference's boundary features)."""
    on = np.abs(X[:, axis] - value) <= tol
    hit = on[conn[:, TET_FACES]].all(axis=2)  # (ne, 4)
    e, f = np.nonzero(hit)
    return e.astype(np.int64), f.astype(np.int32)


def he_p1(n=10, seed=0):
    X, conn, Pr = pg.mesh_box_tet(n, 4)
    nn = X.shape[0]
    h = 1.0 / n
    codes = np.zeros((nn, 3), dtype=np.int64)
    codes[X[:, 0] == 0.0] = 1
    ids, ndof = pg.generate_dof_ids(conn, nn, codes)
    Ap, Ai = pg.psparse_apai(conn, ids, ndof)
    a = 1e-3 * h
    r = splitmix64(seed, nn * 3).reshape(nn, 3)
    disp = (2.0 * r - 1.0) * a
    disp[:, 0] += 0.01 * X[:, 0]
    u = nodal_to_free(ids, disp)
    mat = pg.material(pg.MODEL_HE, E=200e3, nu=0.3)
    return Problem("he_p1_n%d" % n, X, conn, ids, ndof, Ap, Ai, mat, u, meta=dict(n=n, seed=seed))


def tension(n=4, nne=4, model="he", stretch=0.01, predictor=False):
    """Uniaxial tension of the unit cube for a Newton-Raphson load step: the
    x = 0 face fixed, the x-displacement of the x = 1 face prescribed
    (one prescribed value, u_presc[0] = stretch), every other DOF free,
    starting from zero or, with predictor, from the linear field
    u_x = stretch * x.  model "he" (neo-Hookean) or "j2" (state at identity)."""
    X, conn, _ = pg.mesh_box_tet(n, nne)
    nn = X.shape[0]
    codes = np.zeros((nn, 3), dtype=np.int64)
    codes[X[:, 0] == 0.0] = 1
    codes[X[:, 0] == 1.0, 0] = -1
    ids, ndof = pg.generate_dof_ids(conn, nn, codes)
    Ap, Ai = pg.psparse_apai(conn, ids, ndof)
    if model == "he":
        mat = pg.material(pg.MODEL_HE, E=200e3, nu=0.3)
        state = None
    else:
        mat = pg.material(pg.MODEL_J2, E=200e3, nu=0.3, sigma_y=250.0, H=2000.0)
        nqp = conn.shape[0] * (4 if nne == 10 else 1)
        state = np.zeros((nqp, 10))
        state[:, [0, 4, 8]] = 1.0
    disp = np.zeros((nn, 3))
    if predictor:
        disp[:, 0] = stretch * X[:, 0]
    u = nodal_to_free(ids, disp) if ndof else np.zeros(0)
    return Problem("tension_%s_p%d_n%d" % (model, 1 if nne == 4 else 2, n), X, conn, ids, ndof, Ap, Ai, mat,
                   u, u_presc=np.array([stretch]), state=state,
                   meta=dict(n=n, stretch=stretch, model=model))


def j2_yield_strain(E=200e3, nu=0.3, sigma_y=250.0):
    mu = E / (2.0 * (1.0 + nu))
    return sigma_y / (2.0 * mu)


def _first_layers(X, conn, layers, n):
    """The first `layers` z-layers of cells (the leading elements in element
    order) with their nodes, renumbered compactly in the original order."""
    ne_sub = 6 * n * n * layers
    conn = conn[:ne_sub]
    used = np.unique(conn)
    remap = np.full(X.shape[0], -1, dtype=np.int64)
    remap[used] = np.arange(len(used))
    return used, X[used], remap[conn].astype(np.int32)


def j2_p2(n=64, seed=1, stretch=None, perturb=1e-4, max_cells_z=None):
    X, conn, Pr = pg.mesh_box_tet(n, 10)
    nn_full = X.shape[0]
    h = 1.0 / n
    eps = j2_yield_strain() if stretch is None else stretch
    a = perturb * h
    r = splitmix64(seed, nn_full * 3).reshape(nn_full, 3)
    if max_cells_z is not None and max_cells_z < n:
        used, X, conn = _first_layers(X, conn, max_cells_z, n)
        r = r[used]
    nn = X.shape[0]
    codes = np.zeros((nn, 3), dtype=np.int64)
    ids, ndof = pg.generate_dof_ids(conn, nn, codes)
    Ap, Ai = pg.psparse_apai(conn, ids, ndof)
    disp = (2.0 * r - 1.0) * a
    disp[:, 0] += eps * X[:, 0]
    u = nodal_to_free(ids, disp)
    mat = pg.material(pg.MODEL_J2, E=200e3, nu=0.3, sigma_y=250.0, H=2000.0)
    nqp = conn.shape[0] * 4
    state = np.zeros((nqp, 10))
    state[:, [0, 4, 8]] = 1.0
    return Problem("j2_p2_n%d" % n, X, conn, ids, ndof, Ap, Ai, mat, u, state=state,
                   meta=dict(n=n, seed=seed, stretch=eps))


# ----------------------------------------------------------------------------
# crystal plasticity
# ----------------------------------------------------------------------------
CP_STEPS = 20  # load steps of the 1 % tension ramp
CP_DT = 0.1


def quat_to_rot(q):
    """Rotation matrices (n,3,3) from unit quaternions (n,4) = (x, y, z, w)."""
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = np.empty((len(q), 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def shoemake_quaternions(seed, n):
    """Uniform random rotations (Shoemake 1992) as unit quaternions."""
    u = splitmix64(seed, 3 * n, stream=7).reshape(n, 3)
    a, b = np.sqrt(1 - u[:, 0]), np.sqrt(u[:, 0])
    t1, t2 = 2 * np.pi * u[:, 1], 2 * np.pi * u[:, 2]
    return np.stack([a * np.sin(t1), a * np.cos(t1), b * np.sin(t2), b * np.cos(t2)], axis=1)


def voronoi_grains(centroids, seed, ngrains):
    """Grain id of each point: nearest of ngrains seeded uniform centres."""
    c = splitmix64(seed, 3 * ngrains, stream=5).reshape(ngrains, 3)
    gid = np.empty(len(centroids), dtype=np.int64)
    cc = (c * c).sum(1)
    for s in range(0, len(centroids), 65536):
        # |x - c|^2 - |x|^2 = |c|^2 - 2 x.c ranks the centres like the distance
        d = cc[None, :] - 2.0 * (centroids[s:s + 65536] @ c.T)
        gid[s:s + 65536] = d.argmin(1)
    return gid


def cp_material(max_iter=25, tol=1e-10):
    return pg.material(pg.MODEL_CP, E=200e3, nu=0.3, gamma_dot_0=1e-3, m=0.05, G0=200.0, g0=60.0, gs_0=250.0,
                       gamma_dot_s=1.0, w=0.0, cp_tol=tol, cp_max_iter=max_iter)


class CpProblem(Problem):
    """Config-3 style problem: the load ramp u(s) = s/CP_STEPS * u_final."""

    def displacement(self, step):
        return self.u_final * (step / CP_STEPS)


def cp_p1(n=48, seed=2, ngrains=512, perturb=1e-4):
    X, conn, Pr = pg.mesh_box_tet(n, 4)
    nn = X.shape[0]
    h = 1.0 / n
    codes = np.zeros((nn, 3), dtype=np.int64)
    ids, ndof = pg.generate_dof_ids(conn, nn, codes)
    Ap, Ai = pg.psparse_apai(conn, ids, ndof)
    cen = X[conn].mean(axis=1)
    gid = voronoi_grains(cen, seed, ngrains)
    Rg = quat_to_rot(shoemake_quaternions(seed, ngrains))
    R_cp = np.ascontiguousarray(Rg[gid].reshape(-1, 9))
    r = splitmix64(seed, nn * 3).reshape(nn, 3)
    disp = (2.0 * r - 1.0) * perturb * h
    disp[:, 0] += 0.01 * X[:, 0]
    u_final = nodal_to_free(ids, disp)
    state = np.zeros((conn.shape[0], 10))
    state[:, [0, 4, 8]] = 1.0
    state[:, 9] = 60.0
    p = CpProblem("cp_p1_n%d" % n, X, conn, ids, ndof, Ap, Ai, cp_material(), u_final.copy(), state=state,
                  R_cp=R_cp, dt=CP_DT, meta=dict(n=n, seed=seed, ngrains=ngrains))
    p.u_final = u_final
    p.grain = gid
    p.quat = shoemake_quaternions(seed, ngrains)[gid]
    return p


def fcc_slip_systems():
    """FCC {111}<110> slip directions s and normals n (unit, crystal frame), 12 x 3 each."""
    N = np.array([[1, 1, 1], [-1, 1, 1], [1, -1, 1], [1, 1, -1]], dtype=float) / np.sqrt(3.0)
    D = np.array([[[0, 1, -1], [1, 0, -1], [1, -1, 0]], [[0, 1, -1], [1, 0, 1], [1, 1, 0]],
                  [[0, 1, 1], [1, 0, -1], [1, 1, 0]], [[0, 1, 1], [1, 0, 1], [1, -1, 0]]], dtype=float) / np.sqrt(2.0)
    s = D.reshape(12, 3)
    n = np.repeat(N, 3, axis=0)
    return s, n


# ------------------------------------------------------------ FE2 RVE batch --
RVE_SEED = 3


class RveBatch(Problem):
    """Independent periodic unit cells (FE2 micro-structures) held as one mesh:
    nodes, elements and DOFs of RVE r occupy the ranges node_off[r]..,
    elem_off[r].., dof_off[r]..; the CSR pattern is block diagonal; RVE r sees
    the macro deformation F0s[r] (F = I + grad u + F0s[r])."""

    def rve(self, r):
        """RVE r on its own (local numbering), for per-RVE reference checks."""
        n0, n1 = self.node_off[r], self.node_off[r + 1]
        e0, e1 = self.elem_off[r], self.elem_off[r + 1]
        d0, d1 = self.dof_off[r], self.dof_off[r + 1]
        conn = (self.conn[e0:e1] - n0).astype(np.int32)
        ids = self.ids[n0:n1].copy()
        ids[ids > 0] -= d0
        Ap = (self.Ap[d0:d1 + 1] - self.Ap[d0]).astype(np.int32)
        Ai = (self.Ai[self.Ap[d0]:self.Ap[d1]] - d0).astype(np.int32)
        ni = self.nint
        state = None if self.state is None else self.state[e0 * ni:e1 * ni]
        return Problem("%s_rve%d" % (self.name, r), self.X[n0:n1], conn, ids, d1 - d0, Ap, Ai, self.mat,
                       self.u[d0:d1].copy(), state=state, F0=self.F0s[r].copy(), meta=dict(n=int(self.n_r[r])))

    def context(self):
        ctx = super().context()
        ctx.set_mesh_groups(self.elem_off, self.F0s)
        return ctx


def rve_batch(nrve=256, seed=RVE_SEED, nmin=8, nmax=24, fluct=1e-3, subset=None, nne=4):
    """Config 5: nrve periodic unit cubes, n_r^3 cells x 6 linear tets with n_r
    uniform in nmin..nmax, macro F0 = sym(U(-0.02, 0.02)^{3x3}) per RVE, a
    seeded periodic fluctuation field of amplitude fluct * h_r, J2 material
    (E 200 GPa, nu 0.3, yield 250 MPa, H 2 GPa), state at identity.
    subset: indices of the RVEs to build (a rank's shard); sizes, macro
    deformations and fluctuations are those of the full batch.  nne 10 builds
    quadratic tets (4 points per element) instead."""
    ns_all = nmin + np.minimum((splitmix64(seed, nrve, stream=7) * (nmax - nmin + 1)).astype(np.int64),
                               nmax - nmin)
    A_all = (2.0 * splitmix64(seed, 9 * nrve, stream=8) - 1.0).reshape(nrve, 3, 3) * 0.02
    sel = np.arange(nrve) if subset is None else np.asarray(subset, dtype=np.int64)
    ns = ns_all[sel]
    Xs, conns, idss, node_off, elem_off, dof_off = [], [], [], [0], [0], [0]
    us = []
    for r, n in zip(sel, ns):
        X, conn, Pr = pg.mesh_box_tet(int(n), nne, periodic=True)
        nn = X.shape[0]
        ids, ndof = pg.generate_dof_ids(conn, nn, np.zeros((nn, 3), dtype=np.int64), Pr=Pr)
        Xs.append(X)
        conns.append(conn.astype(np.int64) + node_off[-1])
        ids = ids.copy()
        ids[ids > 0] += dof_off[-1]
        idss.append(ids)
        node_off.append(node_off[-1] + nn)
        elem_off.append(elem_off[-1] + conn.shape[0])
        dof_off.append(dof_off[-1] + ndof)
        # periodic fluctuation: one value per free DOF, scaled by the cell size,
        # from a stream keyed by the RVE's index in the full batch
        us.append((2.0 * splitmix64(seed * 1000003 + int(r), ndof, stream=9) - 1.0) * fluct / float(n))
    X = np.concatenate(Xs)
    conn = np.concatenate(conns).astype(np.int32)
    ids = np.concatenate(idss)
    ndof = dof_off[-1]
    Ap, Ai = pg.psparse_apai(conn, ids, ndof)
    A = A_all[sel]
    F0s = (0.5 * (A + np.transpose(A, (0, 2, 1)))).reshape(len(sel), 9)
    u = np.concatenate(us)
    mat = pg.material(pg.MODEL_J2, E=200e3, nu=0.3, sigma_y=250.0, H=2000.0)
    state = np.zeros((conn.shape[0] * (4 if nne == 10 else 1), 10))
    state[:, [0, 4, 8]] = 1.0
    p = RveBatch("rve_batch_%d" % nrve, X, conn, ids, ndof, Ap, Ai, mat, u, state=state,
                 meta=dict(nrve=nrve, seed=seed, nmin=nmin, nmax=nmax, subset=sel.tolist()))
    p.n_r = ns
    p.node_off = np.array(node_off, dtype=np.int64)
    p.elem_off = np.array(elem_off, dtype=np.int64)
    p.dof_off = np.array(dof_off, dtype=np.int64)
    p.F0s = F0s
    return p
