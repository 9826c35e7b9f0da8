"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product path never uses it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

HE, J2, CP = 0, 1, 2


class OrcMaterial(C.Structure):
    _fields_ = [("model", C.c_int), ("E", C.c_double), ("nu", C.c_double),
                ("sigma_y", C.c_double), ("H", C.c_double),
                ("gamma_dot_0", C.c_double), ("m", C.c_double), ("G0", C.c_double),
                ("g0", C.c_double), ("gs_0", C.c_double), ("gamma_dot_s", C.c_double),
                ("w", C.c_double), ("cp_tol", C.c_double), ("cp_max_iter", C.c_int),
                ("dev_pot", C.c_int), ("vol_pot", C.c_int)]


class OrcProblem(C.Structure):
    _fields_ = [("nn", C.c_long), ("ne", C.c_long), ("nne", C.c_int),
                ("X", C.c_void_p), ("conn", C.c_void_p), ("id", C.c_void_p), ("ndof", C.c_long),
                ("Ap", C.c_void_p), ("Ai", C.c_void_p), ("F0", C.c_void_p), ("R_cp", C.c_void_p),
                ("nbc_off", C.c_void_p), ("nbc_face", C.c_void_p), ("nbc_type", C.c_void_p),
                ("nbc_load", C.c_void_p), ("nbc_load_n", C.c_void_p), ("nbc_load_nm1", C.c_void_p)]


_lib = None
_P = C.c_void_p


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        sig = {
            "orc_state_size": (C.c_int, [C.c_int]),
            "orc_nint": (C.c_int, [C.c_int]),
            "orc_generate_dof_ids": (C.c_long, [C.c_long, C.c_long, C.c_int, _P, _P, _P]),
            "orc_psparse_apai": (C.c_long, [C.c_long, C.c_int, _P, _P, C.c_long, _P, _P]),
            "orc_cm_update": (C.c_int, [_P, _P, C.c_double, _P, _P, _P, _P, _P, _P]),
            "orc_element": (C.c_int, [_P, _P, C.c_long, _P, C.c_double, _P, _P, _P, _P]),
            "orc_assemble": (C.c_int, [_P, _P, _P, _P, C.c_double, _P, _P, _P, _P, C.c_long, C.c_long,
                                       C.c_int, _P]),
            "orc_assemble_bform": (C.c_int, [_P, _P, _P, _P, C.c_double, _P, _P, _P, _P, C.c_long,
                                             C.c_long, C.c_int]),
            "orc_cp_update_batch": (C.c_long, [_P, C.c_long, _P, C.c_double, _P, _P, _P, _P, _P, _P, _P,
                                               _P, C.c_int, _P]),
            "orc_assemble_transient": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, C.c_double, C.c_double,
                                                 C.c_double, C.c_double, _P, _P]),
            "orc_assemble_transient_state": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, C.c_double, C.c_double,
                                                       C.c_double, C.c_double, _P, _P, _P, _P, _P]),
            "orc_cp_tangent_pair": (C.c_int, [_P, _P, _P, C.c_double, _P, _P, _P, _P]),
            "orc_element_3f": (C.c_int, [_P, _P, C.c_long, _P, C.c_double, C.c_double, _P, _P, _P, _P, _P]),
            "orc_assemble_3f": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
            "orc_update_3f": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
            "orc_assemble_3f_transient": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, C.c_double,
                                                    C.c_double, C.c_double, C.c_double, _P, _P]),
            "orc_update_3f_transient": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, C.c_double,
                                                  C.c_double, C.c_double, _P, _P]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def material(model, E=200e3, nu=0.3, sigma_y=0.0, H=0.0, gamma_dot_0=0.0, m=1.0, G0=0.0, g0=0.0,
             gs_0=0.0, gamma_dot_s=1.0, w=0.0, cp_tol=1e-10, cp_max_iter=25, dev_pot=1, vol_pot=99):
    return OrcMaterial(model, E, nu, sigma_y, H, gamma_dot_0, m, G0, g0, gs_0, gamma_dot_s, w, cp_tol,
                       cp_max_iter, dev_pot, vol_pot)


def from_pg_material(m, dev_pot=None):
    """Oracle material from a pgfem_gpu.MaterialDesc (same field meanings; the
    deviatoric potential flag is taken from the record unless given)."""
    if dev_pot is None:
        dev_pot = 2 if getattr(m, "dev_pot", 1) == 2 else 1
    return material(m.model, m.E, m.nu, m.sigma_y, m.H, m.gamma_dot_0, m.m, m.G0, m.g0, m.gs_0,
                    m.gamma_dot_s, m.w, m.cp_tol, m.cp_max_iter, dev_pot, getattr(m, "vol_pot", 99))


def state_size(model):
    return lib().orc_state_size(model)


def generate_dof_ids(conn, nn, codes, Pr=None):
    ids = np.ascontiguousarray(codes, dtype=np.int64).copy()
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    Pr = None if Pr is None else np.ascontiguousarray(Pr, dtype=np.int64)
    ndof = lib().orc_generate_dof_ids(nn, conn.shape[0], conn.shape[1], _p(conn), _p(Pr), _p(ids))
    return ids, ndof


def psparse_apai(conn, ids, ndof):
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    ids = np.ascontiguousarray(ids, dtype=np.int64)
    Ap = np.zeros(ndof + 1, dtype=np.int32)
    nnz = lib().orc_psparse_apai(conn.shape[0], conn.shape[1], _p(conn), _p(ids), ndof, _p(Ap), None)
    Ai = np.zeros(max(nnz, 1), dtype=np.int32)
    lib().orc_psparse_apai(conn.shape[0], conn.shape[1], _p(conn), _p(ids), ndof, _p(Ap), _p(Ai))
    return Ap, Ai[:nnz]


def cm_update(mat, F, state_n=None, dt=0.0, Rcp=None):
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(9)
    S = np.zeros(9)
    L = np.zeros(81)
    ns = state_size(mat.model)
    snp1 = np.zeros(max(ns, 1))
    sn = None if state_n is None else np.ascontiguousarray(state_n, dtype=np.float64)
    Rcp = None if Rcp is None else np.ascontiguousarray(Rcp, dtype=np.float64)
    it = C.c_int()
    err = lib().orc_cm_update(C.byref(mat), _p(F), dt, _p(Rcp), _p(sn), _p(snp1), _p(S), _p(L), C.byref(it))
    return err, S.reshape(3, 3), L.reshape(3, 3, 3, 3), snp1, it.value


def cp_update_batch(mat, F, state_n, dt, Rcp, M0=None, g_guess=None, warm_k=0, want_fallback=False):
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(-1, 9)
    nq = F.shape[0]
    state_n = np.ascontiguousarray(state_n, dtype=np.float64).reshape(nq, 10)
    Rcp = np.ascontiguousarray(Rcp, dtype=np.float64).reshape(nq, 9)
    M0 = None if M0 is None else np.ascontiguousarray(M0, dtype=np.float64).reshape(nq, 9)
    gg = None if g_guess is None else np.ascontiguousarray(g_guess, dtype=np.float64).reshape(nq)
    snp1 = np.zeros((nq, 10))
    it = np.zeros(nq, dtype=np.int32)
    dg = np.zeros((nq, 12))
    cv = np.zeros(nq, dtype=np.int32)
    fb = np.zeros(nq, dtype=np.int32)
    bad = lib().orc_cp_update_batch(C.byref(mat), nq, _p(F), dt, _p(Rcp), _p(state_n), _p(M0), _p(gg), _p(snp1),
                                    _p(it), _p(dg), _p(cv), int(warm_k), _p(fb))
    if want_fallback:
        return bad, snp1, it, dg, cv, fb
    return bad, snp1, it, dg, cv


class Problem:
    """Oracle view of a mesh problem (keeps the arrays alive)."""

    def __init__(self, X, conn, ids, ndof, Ap, Ai, F0=None, R_cp=None):
        self.X = np.ascontiguousarray(X, dtype=np.float64)
        self.conn = np.ascontiguousarray(conn, dtype=np.int32)
        self.ids = np.ascontiguousarray(ids, dtype=np.int64)
        self.Ap = np.ascontiguousarray(Ap, dtype=np.int32)
        self.Ai = np.ascontiguousarray(Ai, dtype=np.int32)
        self.F0 = None if F0 is None else np.ascontiguousarray(F0, dtype=np.float64).reshape(9)
        self.R_cp = None if R_cp is None else np.ascontiguousarray(R_cp, dtype=np.float64)
        self.ndof = ndof
        self.s = OrcProblem(self.X.shape[0], self.conn.shape[0], self.conn.shape[1], _p(self.X),
                            _p(self.conn), _p(self.ids), ndof, _p(self.Ap), _p(self.Ai), _p(self.F0),
                            _p(self.R_cp))

    def set_neumann(self, elem, face, load_type, load, load_n=None, load_nm1=None):
        """Surface loads on element faces (the reference's NeumannBoundaryElement
        list, src/PGFem3D_data_structure.cc:825-895, flattened to one entry per
        face): elem (0-based), local face 0..3, number of load values (1 pressure,
        2..3 traction) and the values at t_{n+1} (nface x 3); for the transient
        element also at t_n and t_{n-1}.  Empty lists clear."""
        elem = np.asarray(elem, dtype=np.int64).ravel()
        if elem.size == 0:
            self.nbc = None
            self.s.nbc_off = self.s.nbc_face = self.s.nbc_type = self.s.nbc_load = None
            self.s.nbc_load_n = self.s.nbc_load_nm1 = None
            return
        order = np.argsort(elem, kind="stable")
        ne = self.conn.shape[0]
        off = np.zeros(ne + 1, dtype=np.int64)
        np.add.at(off, elem + 1, 1)
        off = np.cumsum(off)
        face = np.ascontiguousarray(np.asarray(face, dtype=np.int32).ravel()[order])
        ltype = np.ascontiguousarray(np.asarray(load_type, dtype=np.int32).ravel()[order])
        load = np.ascontiguousarray(np.asarray(load, dtype=np.float64).reshape(-1, 3)[order])
        hist = [None if x is None else np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1, 3)[order])
                for x in (load_n, load_nm1)]
        self.nbc = (off, face, ltype, load, hist)
        self.s.nbc_off, self.s.nbc_face, self.s.nbc_type, self.s.nbc_load = (_p(off), _p(face), _p(ltype),
                                                                             _p(load))
        self.s.nbc_load_n, self.s.nbc_load_nm1 = _p(hist[0]), _p(hist[1])

    @property
    def nnz(self):
        return int(self.Ap[-1])

    def element(self, mat, e, u_e, state_n=None, dt=0.0, want_K=True):
        nd = self.conn.shape[1] * 3
        fe = np.zeros(nd)
        lk = np.zeros((nd, nd)) if want_K else None
        nint = lib().orc_nint(self.conn.shape[1])
        ns = state_size(mat.model)
        snp1 = np.zeros(max(nint * ns, 1))
        sn = None if state_n is None else np.ascontiguousarray(state_n, dtype=np.float64)
        u_e = np.ascontiguousarray(u_e, dtype=np.float64)
        err = lib().orc_element(C.byref(self.s), C.byref(mat), e, _p(u_e), dt, _p(sn), _p(snp1), _p(fe), _p(lk))
        return err, fe, lk, snp1

    def element_3f(self, mat, e, u_e, P, theta, want_K=True, state_n=None):
        """Three-field (CM3F) element of the hyperelastic or J2 model: (err, fe,
        lk, blocks) with blocks = (fp, ft, Ktp, Ktt, Kup[3 nne])."""
        nd = self.conn.shape[1] * 3
        fe = np.zeros(nd)
        lk = np.zeros((nd, nd)) if want_K else None
        blk = np.zeros(4 + nd)
        u_e = np.ascontiguousarray(u_e, dtype=np.float64)
        sn = None if state_n is None else np.ascontiguousarray(state_n, dtype=np.float64)
        err = lib().orc_element_3f(C.byref(self.s), C.byref(mat), e, _p(u_e), float(P), float(theta), _p(sn), None,
                                   _p(fe), _p(lk), _p(blk))
        return err, fe, lk, (blk[0], blk[1], blk[2], blk[3], blk[4:].copy())

    def assemble_3f(self, mat, u, P, theta, u_presc=None, want_K=True, state_n=None):
        """Global R, K of the three-field element (P, theta per element); with a
        J2 state at t_n also the state at t_{n+1}: (err, R, K[, state_np1])."""
        R = np.zeros(self.ndof)
        K = np.zeros(self.nnz) if want_K else None
        ns = state_size(mat.model)
        nint = lib().orc_nint(self.conn.shape[1])
        snp1 = np.zeros((self.conn.shape[0] * nint, ns)) if ns else None
        a = [np.ascontiguousarray(x, dtype=np.float64) if x is not None else None
             for x in (u, u_presc, P, theta, state_n)]
        err = lib().orc_assemble_3f(C.byref(self.s), C.byref(mat), *[_p(x) for x in a], _p(snp1), _p(R), _p(K))
        return (err, R, K) if state_n is None else (err, R, K, snp1)

    def assemble_3f_transient(self, mat, us, Ps, thetas, alpha, dt_np1, dt_n, rho, presc=(None, None, None),
                              want_K=True):
        """Transient three-field R, K (hyperelastic): us, presc, Ps, thetas are
        the values at t_{n+1}, t_n, t_{n-1}.  Returns (err, R, K)."""
        R = np.zeros(self.ndof)
        K = np.zeros(self.nnz) if want_K else None
        a = [np.ascontiguousarray(x, dtype=np.float64) if x is not None else None for x in (*us, *presc)]
        P3 = np.ascontiguousarray(np.stack(Ps, axis=1), dtype=np.float64)
        T3 = np.ascontiguousarray(np.stack(thetas, axis=1), dtype=np.float64)
        err = lib().orc_assemble_3f_transient(C.byref(self.s), C.byref(mat), *[_p(x) for x in a], _p(P3), _p(T3),
                                              alpha, dt_np1, dt_n, rho, _p(R), _p(K))
        return err, R, K

    def update_3f_transient(self, mat, us, du, Ps, thetas, alpha, dt_np1, dt_n, presc=(None, None, None)):
        """Element pressure / volume increments of the transient three-field
        element after the displacement increment du.  Returns (err, dP, dtheta)."""
        ne = self.conn.shape[0]
        dP, dth = np.zeros(ne), np.zeros(ne)
        a = [np.ascontiguousarray(x, dtype=np.float64) if x is not None else None for x in (*us, *presc, du)]
        P3 = np.ascontiguousarray(np.stack(Ps, axis=1), dtype=np.float64)
        T3 = np.ascontiguousarray(np.stack(thetas, axis=1), dtype=np.float64)
        err = lib().orc_update_3f_transient(C.byref(self.s), C.byref(mat), *[_p(x) for x in a], _p(P3), _p(T3),
                                            alpha, dt_np1, dt_n, _p(dP), _p(dth))
        return err, dP, dth

    def update_3f(self, mat, u, du, P, theta, u_presc=None, state_n=None):
        """Element pressure / volume increments after the displacement increment du."""
        ne = self.conn.shape[0]
        dP, dth = np.zeros(ne), np.zeros(ne)
        a = [np.ascontiguousarray(x, dtype=np.float64) if x is not None else None
             for x in (u, u_presc, du, P, theta, state_n)]
        err = lib().orc_update_3f(C.byref(self.s), C.byref(mat), *[_p(x) for x in a], _p(dP), _p(dth))
        return err, dP, dth

    def assemble(self, mat, u, u_presc=None, state_n=None, dt=0.0, want_K=True, e0=0, e1=None,
                 nthreads=1, bform=False):
        ne = self.conn.shape[0]
        e1 = ne if e1 is None else e1
        nint = lib().orc_nint(self.conn.shape[1])
        ns = state_size(mat.model)
        R = np.zeros(self.ndof)
        K = np.zeros(self.nnz) if want_K else None
        snp1 = np.zeros((ne * nint, max(ns, 1))) if ns else None
        sn = None if state_n is None else np.ascontiguousarray(state_n, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        up = None if u_presc is None else np.ascontiguousarray(u_presc, dtype=np.float64)
        if bform:
            err = lib().orc_assemble_bform(C.byref(self.s), C.byref(mat), _p(u), _p(up), dt, _p(sn), _p(snp1),
                                           _p(R), _p(K), e0, e1, nthreads)
        else:
            err = lib().orc_assemble(C.byref(self.s), C.byref(mat), _p(u), _p(up), dt, _p(sn), _p(snp1), _p(R),
                                     _p(K), e0, e1, nthreads, None)
        return err, R, K, snp1


def assemble_transient(P, mat, u_np1, u_n, u_nm1, alpha, dt_np1, dt_n, rho, p_np1=None, p_n=None, p_nm1=None,
                       want_K=True):
    """Transient (mid-point rule) R, K of the hyperelastic element: the oracle's
    orc_assemble_transient.  Returns (err, R, K)."""
    R = np.zeros(P.ndof)
    K = np.zeros(P.nnz) if want_K else None
    arr = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None
           for a in (u_np1, u_n, u_nm1, p_np1, p_n, p_nm1)]
    err = lib().orc_assemble_transient(C.byref(P.s), C.byref(mat), *[_p(a) for a in arr], alpha, dt_np1, dt_n, rho,
                                       _p(R), _p(K))
    return err, R, K


def assemble_transient_cp(P, mat, u_np1, u_n, u_nm1, alpha, dt_np1, dt_n, rho, state_nm1, state_n,
                          p_np1=None, p_n=None, p_nm1=None, want_K=True):
    """Transient (mid-point rule) R, K of the crystal-plasticity element with the
    state at t_{n-1} and t_n (AoS ne*nint*10): orc_assemble_transient_state.
    Returns (err, R, K, state_np1)."""
    R = np.zeros(P.ndof)
    K = np.zeros(P.nnz) if want_K else None
    arr = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None
           for a in (u_np1, u_n, u_nm1, p_np1, p_n, p_nm1)]
    s0 = np.ascontiguousarray(state_nm1, dtype=np.float64)
    s1 = np.ascontiguousarray(state_n, dtype=np.float64)
    s2 = np.zeros_like(s1)
    err = lib().orc_assemble_transient_state(C.byref(P.s), C.byref(mat), *[_p(a) for a in arr], alpha, dt_np1,
                                             dt_n, rho, _p(s0), _p(s1), _p(s2), _p(R), _p(K))
    return err, R, K, s2


def newton_step(P, mat, u0, u_presc=None, state_n=None, dt=0.0, iter_max=10, nor_min=1e-10,
                computer_zero=1e-15, nthreads=8):
    """One load step of full Newton-Raphson on the CPU, the checker of
    pgfem_gpu_newton_step: the reference's loop (src/Newton_Raphson.cc:931-1330
    with FNR = 1, no line search) -- assemble R and K, nor = ||R|| / ||R_0||
    (:1203-1217), stop when nor <= nor_min or ||R|| <= computer_zero (:1323),
    else solve K du = -R (here a sparse direct solve) and u += du.
    Returns (u, [nor per iteration], converged, state_np1)."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.linalg import spsolve
    u = np.array(u0, dtype=np.float64, copy=True)
    hist, NORM = [], 1.0
    for it in range(iter_max + 1):
        err, R, K, snp1 = P.assemble(mat, u, u_presc, state_n=state_n, dt=dt, nthreads=nthreads)
        if err:
            return u, hist, False, snp1
        nor2 = float(np.linalg.norm(R))
        if it == 0:
            NORM = nor2 if nor2 > computer_zero else (computer_zero if computer_zero > 0 else 1.0)
        nor = nor2 / NORM
        hist.append(nor)
        if nor <= nor_min or nor2 <= computer_zero:
            return u, hist, True, snp1
        if it >= iter_max:
            return u, hist, False, snp1
        Km = csr_matrix((K, P.Ai, P.Ap), shape=(P.ndof, P.ndof))
        u = u + spsolve(Km.tocsc(), -R)
    return u, hist, False, snp1


# ---------------------------------------------------------------------------
# Synthetic workload built without the product library (the CPU arm of the
# benchmark times the oracle on it, so that no product code is loaded there).
# ---------------------------------------------------------------------------
# Kuhn split of the unit cube into 6 tets along the (0,0,0)-(1,1,1) diagonal
# (one tet per axis permutation, oriented to a positive volume) and the
# quadratic-tet edge nodes in FEMLIB's order (FEMLIB/src/femlib.cc:163-176).
_KUHN_PERM = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]
_KUHN_SIGN = [1, -1, -1, 1, 1, -1]
_EDGES = [(0, 1), (1, 2), (0, 2), (0, 3), (1, 3), (2, 3)]


def mesh_box_tet(n, nne):
    """Structured n^3 unit-cube mesh, 6 Kuhn tets per cell, node-lexicographic
    numbering on the lattice (n or 2n intervals), cell-major element order."""
    N = n if nne == 4 else 2 * n
    L = N + 1
    s = 1 if nne == 4 else 2
    k, j, i = np.meshgrid(np.arange(L), np.arange(L), np.arange(L), indexing="ij")
    X = np.stack([i.ravel() / N, j.ravel() / N, k.ravel() / N], axis=1)
    cells = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), axis=-1).reshape(-1, 3)
    cells = cells[:, ::-1]  # (ci, cj, ck) with ci fastest
    conn = np.zeros((6 * n ** 3, nne), dtype=np.int64)
    for t in range(6):
        v = np.zeros((4, 3), dtype=np.int64)
        v[1, _KUHN_PERM[t][0]] = 1
        v[2] = v[1]
        v[2, _KUHN_PERM[t][1]] += 1
        v[3] = 1
        if _KUHN_SIGN[t] < 0:
            v[[1, 2]] = v[[2, 1]]
        lat = [s * (cells + v[a]) for a in range(4)]
        if nne == 10:
            lat += [(lat[a] + lat[b]) // 2 for a, b in _EDGES]
        for a in range(nne):
            conn[t::6, a] = lat[a][:, 0] + L * (lat[a][:, 1] + L * lat[a][:, 2])
    return X, conn.astype(np.int32)


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


def j2_p2_problem(n, seed=1, perturb=1e-4, max_cells_z=None, E=200e3, nu=0.3, sigma_y=250.0, H=2000.0):
    """The J2 quadratic-tet workload (n^3 cells, stretch at the yield onset
    sigma_y / 2 mu along x plus a seeded perturbation of perturb * h), or its
    first max_cells_z layers of cells, built with the oracle's own mesher, DOF
    numbering and CSR pattern.  Returns (Problem, material, u, state_n)."""
    X, conn = mesh_box_tet(n, 10)
    r = splitmix64(seed, X.shape[0] * 3).reshape(-1, 3)
    if max_cells_z is not None and max_cells_z < n:
        conn = conn[:6 * n * n * max_cells_z]
        used = np.unique(conn)
        remap = np.full(X.shape[0], -1, dtype=np.int64)
        remap[used] = np.arange(len(used))
        X, r, conn = X[used], r[used], remap[conn].astype(np.int32)
    ids, ndof = generate_dof_ids(conn, X.shape[0], np.zeros((X.shape[0], 3), dtype=np.int64))
    Ap, Ai = psparse_apai(conn, ids, ndof)
    a = perturb * (1.0 / n)
    mu = E / (2.0 * (1.0 + nu))
    disp = (2.0 * r - 1.0) * a
    disp[:, 0] += sigma_y / (2.0 * mu) * X[:, 0]
    u = np.zeros(ndof)
    m = ids > 0
    u[ids[m] - 1] = disp[m]
    state = np.zeros((conn.shape[0] * 4, 10))
    state[:, [0, 4, 8]] = 1.0
    mat = material(J2, E=E, nu=nu, sigma_y=sigma_y, H=H)
    return Problem(X, conn, ids, ndof, Ap, Ai), mat, u, state


def from_workload(p):
    """Oracle Problem + material for a pgfem-3d_b200 workloads.Problem."""
    return Problem(p.X, p.conn, p.ids, p.ndof, p.Ap, p.Ai, F0=p.F0, R_cp=p.R_cp), from_pg_material(p.mat)


def cp_tangent_pair(mat, Fn, Fnp1, dt, Rcp, state_n):
    """(err, dM/dF from the oracle's Newton, dM/dF from the reference's formula), 9 x 9 each."""
    a = [np.ascontiguousarray(x, dtype=np.float64) for x in (Fn, Fnp1, Rcp, state_n)]
    d1, d2 = np.zeros(81), np.zeros(81)
    err = lib().orc_cp_tangent_pair(C.byref(mat), _p(a[0]), _p(a[1]), dt, _p(a[2]), _p(a[3]), _p(d1), _p(d2))
    return err, d1.reshape(9, 9), d2.reshape(9, 9)
