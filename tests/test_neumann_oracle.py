"""Surface loads (Neumann terms) in the oracle, on the CPU.

The oracle's face terms (oracle/pgfem_oracle.cpp, neumann_faces) are checked
against a second, literal restatement written here in numpy from the
reference's own tensor expressions -- compute_Neumann_boundary_conditions
(src/fd_residuals.cc:123-273) and compute_Neumann_boundary_conditions_stiffnes_mat
(src/stiffmat_fd.cc:359-500) with the 4-index dFIdF and the shape tensor of
compute_shape_tensor (FEMLIB/src/femlib.cc:47-69) -- and against known
answers on undeformed elements: a traction t on faces 0..2 sums to -t A over
the face's nodes, a pressure p to -p n A with n the outward normal; face 3,
whose points the reference's table puts on the plane zet = 0, gives -(2/3) t A
on a linear tet.
"""
import numpy as np
import pytest

import oracle

TET2TRI = [[0, 2, 1], [0, 1, 3], [1, 2, 3], [0, 3, 2]]
QTET2QTRI = [[0, 2, 1, 6, 5, 4], [0, 1, 3, 4, 8, 7], [1, 2, 3, 5, 9, 8], [0, 3, 2, 7, 9, 6]]
KEZMAP = [[1, 0, 2], [0, 2, 1], [0, 1, 2], [0, 1, 2]]
# reference tet node coordinates (xi, eta, zeta), quadratic: mid-edge nodes 01 12 02 03 13 23
XI4 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)
XI10 = np.vstack([XI4, 0.5 * (XI4[[0, 1, 0, 0, 1, 2]] + XI4[[1, 2, 2, 3, 3, 3]])])


def shape(nne, k, e, z):
    l0 = 1.0 - k - e - z
    if nne == 4:
        return (np.array([l0, k, e, z]),
                np.array([[-1, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float))
    N = np.array([(2 * l0 - 1) * l0, (2 * k - 1) * k, (2 * e - 1) * e, (2 * z - 1) * z, 4 * l0 * k, 4 * k * e,
                  4 * l0 * e, 4 * l0 * z, 4 * k * z, 4 * e * z])
    s = 4 * (k + e + z) - 3
    dN = np.array([[s, s, s], [4 * k - 1, 0, 0], [0, 4 * e - 1, 0], [0, 0, 4 * z - 1],
                   [4 * (1 - 2 * k - e - z), -4 * k, -4 * k], [4 * e, 4 * k, 0],
                   [-4 * e, 4 * (1 - k - 2 * e - z), -4 * e], [-4 * z, -4 * z, 4 * (1 - k - e - 2 * z)],
                   [4 * z, 0, 4 * k], [0, 4 * z, 4 * e]])
    return N, dN


def face_dN(nb, k, e):
    if nb == 3:
        return np.array([[-1, -1], [1, 0], [0, 1]], dtype=float)
    return np.array([[4 * e + 4 * k - 3, 4 * e + 4 * k - 3], [4 * k - 1, 0], [0, 4 * e - 1],
                     [4 - 8 * k - 4 * e, -4 * k], [4 * e, 4 * k], [-4 * e, 4 - 4 * k - 8 * e]])


def ref_face_terms(Xe, ue, f, ltype, load):
    """The reference's face loop, line by line (quasi-static branch)."""
    nne = len(Xe)
    quad = nne == 10
    v2b = QTET2QTRI[f] if quad else TET2TRI[f]
    nb = len(v2b)
    km = KEZMAP[f]
    pts = [(2 / 3, 1 / 6), (1 / 6, 1 / 6), (1 / 6, 2 / 3)] if quad else [(1 / 3, 1 / 3)]
    wts = [1 / 6] * 3 if quad else [0.5]
    Pnp1 = np.zeros(3)
    Pnp1[:ltype] = load[:ltype]
    if ltype == 1:
        Pnp1[2:] = Pnp1[0]
    be = np.zeros(nne * 3)
    lk = np.zeros((nne * 3, nne * 3))
    for (gk, ge), wt in zip(pts, wts):
        kez = [0.0, 0.0, 0.0]
        kez[km[0]] = gk
        kez[km[1]] = ge
        if f == 2:
            kez[km[2]] = 1.0 - gk - ge
        N, dNk = shape(nne, *kez)
        dXv = np.einsum("ai,aj->ij", Xe, dNk)
        dNdX = dNk @ np.linalg.inv(dXv)
        dNb = face_dN(nb, kez[km[0]], kez[km[1]])
        dX = np.zeros((3, 2))
        for ib in range(3):
            for ic in range(2):
                for ia in range(nb):
                    dX[ib, ic] += dNb[ia, ic] * Xe[v2b[ia], ib]
        v = np.cross(dX[:, 0], dX[:, 1])
        J = np.linalg.norm(v)
        normal = v / J
        detJxW = J * wt
        F = np.eye(3) + np.einsum("ai,aj->ij", ue, dNdX)
        Jn = np.linalg.det(F)
        FI = np.linalg.inv(F)
        PN = Pnp1[0] * normal if ltype == 1 else Pnp1
        FITN = np.einsum("ji,j->i", FI, PN)
        for ia in range(nb):
            nid = v2b[ia]
            be[nid * 3:nid * 3 + 3] += N[nid] * detJxW * (-1.0) * Jn * FITN
        PNs = Pnp1 * normal if ltype == 1 else Pnp1
        ST = np.zeros((nne, 3, 3, 3))
        for a in range(nne):
            for b in range(3):
                ST[a, b, b, :] = dNdX[a, :]
        dFIdF = -np.einsum("jk,li->ijkl", FI, FI)
        for ia in range(nb):
            a_nid = v2b[ia]
            for ic in range(nb):
                c_nid = v2b[ic]
                for d in range(3):
                    STcd = ST[ic, d]  # idx_4_gen(ic, id, 0, 0, ...) as in the reference
                    FIT = (np.einsum("lk,kl->", FI, STcd) * FI.T - np.einsum("ijkl,kl->ij", dFIdF, STcd)) @ PNs
                    lk[a_nid * 3 + d, c_nid * 3 + d] += N[a_nid] * detJxW * (-1.0) * Jn * FIT[d]
    return be, lk


def one_element(nne, seed, perturb=0.05):
    rng = np.random.default_rng(seed)
    base = XI10 if nne == 10 else XI4
    A = np.array([[1.1, 0.1, -0.05], [0.05, 0.9, 0.1], [0.0, -0.1, 1.2]])
    X = base @ A.T + perturb * rng.uniform(-1, 1, base.shape)
    conn = np.arange(nne, dtype=np.int32)[None, :]
    ids = np.arange(1, 3 * nne + 1, dtype=np.int64).reshape(nne, 3)
    nd = 3 * nne
    Ap = np.arange(0, nd * nd + 1, nd, dtype=np.int32)
    Ai = np.tile(np.arange(nd, dtype=np.int32), nd)
    return oracle.Problem(X, conn, ids, nd, Ap, Ai), X


def face_terms_oracle(P, mat, u_e, faces):
    """The oracle's face terms of element 0: with faces minus without."""
    P.set_neumann([], [], [], [])
    _, f0, k0, _ = P.element(mat, 0, u_e)
    e = np.zeros(len(faces), dtype=np.int64)
    P.set_neumann(e, [f for f, _, _ in faces], [t for _, t, _ in faces], [ld for _, _, ld in faces])
    err, f1, k1, _ = P.element(mat, 0, u_e)
    assert err == 0
    return f1 - f0, k1 - k0


@pytest.mark.parametrize("nne", [4, 10])
@pytest.mark.parametrize("ltype", [1, 2, 3])
def test_face_terms_equal_literal_restatement(nne, ltype):
    P, X = one_element(nne, seed=nne + ltype)
    mat = oracle.material(oracle.HE, E=1e-9)  # volume terms far below the face terms
    rng = np.random.default_rng(7 * ltype + nne)
    u_e = 0.03 * rng.uniform(-1, 1, (nne, 3))
    for f in range(4):
        load = np.array([0.7, -1.3, 2.1])
        fo, ko = face_terms_oracle(P, mat, u_e.ravel(), [(f, ltype, load)])
        fr, kr = ref_face_terms(X, u_e, f, ltype, load)
        assert np.abs(fo - fr).max() <= 1e-12 * np.abs(fr).max(), (f, np.abs(fo - fr).max())
        assert np.abs(ko - kr).max() <= 1e-12 * np.abs(kr).max(), (f, np.abs(ko - kr).max())
        # only component-diagonal entries of the face's node pairs
        nz = np.argwhere(np.abs(ko) > 0)
        assert np.all(nz[:, 0] % 3 == nz[:, 1] % 3)


@pytest.mark.parametrize("nne", [4, 10])
def test_several_faces_add(nne):
    P, X = one_element(nne, seed=3)
    mat = oracle.material(oracle.HE, E=1e-9)  # volume terms far below the face terms
    u_e = 0.02 * np.random.default_rng(5).uniform(-1, 1, (nne, 3))
    faces = [(0, 3, np.array([1.0, 2.0, 3.0])), (2, 1, np.array([-4.0, 0.0, 0.0])), (1, 2, np.array([0.5, 0.25, 9.0]))]
    fo, ko = face_terms_oracle(P, mat, u_e.ravel(), faces)
    fr = sum(ref_face_terms(X, u_e, f, t, ld)[0] for f, t, ld in faces)
    kr = sum(ref_face_terms(X, u_e, f, t, ld)[1] for f, t, ld in faces)
    assert np.abs(fo - fr).max() <= 1e-12 * np.abs(fr).max()
    assert np.abs(ko - kr).max() <= 1e-12 * np.abs(kr).max()


def _area_normal(X, f):
    a, b, c = X[TET2TRI[f]]
    v = np.cross(b - a, c - a)
    return 0.5 * np.linalg.norm(v), v / np.linalg.norm(v)


@pytest.mark.parametrize("nne", [4, 10])
def test_known_answers_undeformed(nne):
    # straight-edged element (no perturbation), u = 0: F = I
    P, X = one_element(nne, seed=1, perturb=0.0)
    mat = oracle.material(oracle.HE, E=1e-9)  # volume terms far below the face terms
    u0 = np.zeros(3 * nne)
    t = np.array([3.0, -2.0, 5.0])
    centroid = X[:4].mean(axis=0)
    for f in range(4):
        A, n = _area_normal(X, f)
        assert np.dot(X[TET2TRI[f][0]] - centroid, n) > 0  # Tet2Tri faces point outward
        fo, _ = face_terms_oracle(P, mat, u0, [(f, 3, t)])
        total = fo.reshape(nne, 3).sum(axis=0)
        if f < 3:
            assert np.allclose(total, -t * A, rtol=1e-13, atol=1e-13), (f, total, -t * A)
            fp, _ = face_terms_oracle(P, mat, u0, [(f, 1, np.array([2.5, 0, 0]))])
            assert np.allclose(fp.reshape(nne, 3).sum(axis=0), -2.5 * n * A, rtol=1e-13, atol=1e-13)
        elif nne == 4:
            # points on zet = 0 while the nodes are {0, 3, 2}: N_3 = 0 there
            assert np.allclose(total, -(2.0 / 3.0) * t * A, rtol=1e-13, atol=1e-13)
        # only the face's own nodes are loaded
        loaded = np.nonzero(np.abs(fo.reshape(nne, 3)).sum(axis=1))[0]
        face_nodes = QTET2QTRI[f] if nne == 10 else TET2TRI[f]
        assert set(loaded.tolist()) <= set(face_nodes)


def test_assembled_faces_equal_element_sums():
    """orc_assemble adds each face through its element (box mesh, two features)."""
    import workloads as wl
    p = wl.he_p1(n=3, seed=4)
    P, mat = oracle.from_workload(p)
    e1, f1 = wl.box_faces(p.X, p.conn, 0, 1.0)
    e2, f2 = wl.box_faces(p.X, p.conn, 2, 1.0)
    assert len(e1) == 2 * 9 and len(e2) == 2 * 9  # two triangles per cell face
    err, R0, K0, _ = P.assemble(mat, p.u)
    elem = np.concatenate([e1, e2])
    face = np.concatenate([f1, f2])
    lt = np.array([3] * len(e1) + [1] * len(e2))
    ld = np.array([[10.0, -5.0, 2.0]] * len(e1) + [[7.0, 0, 0]] * len(e2))
    P.set_neumann(elem, face, lt, ld)
    err, R1, K1, _ = P.assemble(mat, p.u)
    assert err == 0
    # total applied load on the undeformed-ish box: sum of R change ~ -(t A1 + p n A2) (u small)
    dR = R1 - R0
    assert np.abs(dR).max() > 0 and np.abs(K1 - K0).max() > 0
    # per element: the element's own face terms
    err, Rb, Kb, _ = P.assemble(mat, p.u, bform=True)
    assert np.abs(Rb - R1).max() <= 1e-10 * np.abs(R1).max()
    assert np.abs(Kb - K1).max() <= 1e-10 * np.abs(K1).max()
