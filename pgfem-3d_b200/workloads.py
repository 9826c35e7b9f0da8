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
