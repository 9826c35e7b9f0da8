"""Known-answer and consistency checks of the CPU oracle itself.

- central differences of the element residual reproduce the consistent
  tangent (HE; J2 elastic and plastic points)
- the spatial B-form ("best CPU") assembly equals the reference-form
  4-nested compute_stiffness_matrix assembly
- patch test: an affine displacement gives zero residual on interior DOFs
- rigid rotation leaves S unchanged; HE and J2 elastic K are symmetric
- the threaded assembly equals the serial one, periodic cells included
"""
import numpy as np
import pytest

import oracle
import workloads as wl


def rot(a, b, c):
    def Rx(t):
        return np.array([[1, 0, 0], [0, np.cos(t), -np.sin(t)], [0, np.sin(t), np.cos(t)]])

    def Rz(t):
        return np.array([[np.cos(t), -np.sin(t), 0], [np.sin(t), np.cos(t), 0], [0, 0, 1]])
    return Rz(a) @ Rx(b) @ Rz(c)


def small_problem(kind, n=2, stretch=None, vol_pot=99):
    if kind == "he":
        p = wl.he_p1(n=n, seed=7)
    else:
        p = wl.j2_p2(n=n, seed=3, stretch=stretch, perturb=2e-2)
    p.mat.vol_pot = vol_pot
    P, mat = oracle.from_workload(p)
    return p, P, mat


def elem_u(p, e, u):
    ue = np.zeros(p.nne * 3)
    for a in range(p.nne):
        for j in range(3):
            i = p.ids[p.conn[e, a], j]
            ue[a * 3 + j] = u[i - 1] if i > 0 else 0.0
    return ue


@pytest.mark.parametrize("kind,stretch,vol_pot", [("he", None, 99), ("j2", 1e-4, 99), ("j2", 6e-3, 99),
                                                   ("he", None, 2), ("he", None, 3), ("j2", 6e-3, 2),
                                                   ("j2", 6e-3, 3)])
def test_tangent_matches_central_differences(kind, stretch, vol_pot):
    """Also for the Doll-Schweizerhof volumetric potentials (volPotFlag 2, 3)."""
    p, P, mat = small_problem(kind, stretch=stretch, vol_pot=vol_pot)
    rng = np.random.default_rng(0)
    for e in rng.choice(p.ne, 4, replace=False):
        ue = elem_u(p, e, p.u)
        sn = None if p.state is None else p.state[e * p.nint:(e + 1) * p.nint].ravel()
        err, fe, lk, _ = P.element(mat, e, ue, sn)
        assert err == 0
        h = 1e-7 * max(1.0, np.abs(ue).max())
        fd = np.zeros_like(lk)
        for k in range(len(ue)):
            up, um = ue.copy(), ue.copy()
            up[k] += h
            um[k] -= h
            _, fp, _, _ = P.element(mat, e, up, sn, want_K=False)
            _, fm, _, _ = P.element(mat, e, um, sn, want_K=False)
            fd[:, k] = (fp - fm) / (2 * h)
        assert np.linalg.norm(fd - lk) <= 1e-6 * np.linalg.norm(lk), (e, np.linalg.norm(fd - lk) / np.linalg.norm(lk))


def test_j2_plastic_points_exist_in_plastic_case():
    p, P, mat = small_problem("j2", stretch=6e-3)
    err, R, K, snp1 = P.assemble(mat, p.u, state_n=p.state)
    assert err == 0
    assert (snp1[:, 9] > 0).mean() > 0.5


@pytest.mark.parametrize("kind,stretch,vol_pot", [("he", None, 99), ("j2", None, 99), ("j2", 6e-3, 99),
                                                   ("he", None, 2), ("j2", 6e-3, 3)])
def test_bform_equals_reference_form(kind, stretch, vol_pot):
    p, P, mat = small_problem(kind, n=3, stretch=stretch, vol_pot=vol_pot)
    err, R, K, s1 = P.assemble(mat, p.u, state_n=p.state)
    err2, R2, K2, s2 = P.assemble(mat, p.u, state_n=p.state, bform=True)
    assert err == 0 and err2 == 0
    assert np.linalg.norm(R2 - R) <= 1e-12 * np.linalg.norm(R)
    assert np.linalg.norm(K2 - K) <= 1e-12 * np.linalg.norm(K)
    if s1 is not None:
        assert np.abs(s2 - s1).max() <= 1e-12 * max(1.0, np.abs(s1).max())


def test_multithreaded_assembly_equals_serial():
    p, P, mat = small_problem("j2", n=3)
    _, R1, K1, _ = P.assemble(mat, p.u, state_n=p.state, nthreads=1)
    _, R4, K4, _ = P.assemble(mat, p.u, state_n=p.state, nthreads=4)
    assert np.linalg.norm(R4 - R1) <= 1e-13 * np.linalg.norm(R1)
    assert np.linalg.norm(K4 - K1) <= 1e-13 * np.linalg.norm(K1)


def test_multithreaded_assembly_on_periodic_cell_equals_serial():
    """Periodic cells map distinct slave and master nodes to one DOF: the
    threaded assembly's element colours must keep elements that share a DOF
    apart, not only elements that share a node (repeated, since a race shows
    only on some runs)."""
    b = wl.rve_batch(nrve=9, nmin=3, nmax=7, seed=5)
    for r in range(len(b.n_r)):
        q = b.rve(r)
        P, mat = oracle.from_workload(q)
        _, R1, K1, _ = P.assemble(mat, q.u, state_n=q.state, nthreads=1)
        for _ in range(6):
            _, R8, K8, _ = P.assemble(mat, q.u, state_n=q.state, nthreads=8)
            assert np.abs(R8 - R1).max() <= 1e-13 * np.abs(R1).max()
            assert np.abs(K8 - K1).max() <= 1e-13 * np.abs(K1).max()


@pytest.mark.parametrize("nne", [4, 10])
def test_patch_affine_displacement_interior_residual_zero(nne):
    import pgfem_gpu as pg
    X, conn, Pr = pg.mesh_box_tet(3, nne)
    nn = X.shape[0]
    codes = np.zeros((nn, 3), dtype=np.int64)
    ids, ndof = oracle.generate_dof_ids(conn, nn, codes)
    Ap, Ai = oracle.psparse_apai(conn, ids, ndof)
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai)
    G = np.array([[2e-3, 1e-3, -5e-4], [4e-4, -1e-3, 2e-4], [1e-4, 3e-4, 1.5e-3]])
    disp = X @ G.T
    u = wl.nodal_to_free(ids, disp)
    mat = oracle.material(oracle.HE)
    err, R, K, _ = P.assemble(mat, u)
    assert err == 0
    interior = np.all((X > 1e-12) & (X < 1 - 1e-12), axis=1)
    rows = ids[interior].ravel() - 1
    assert np.abs(R[rows]).max() <= 1e-10 * np.abs(R).max()
    # all-free: internal forces sum to zero per component
    for c in range(3):
        assert abs(R[ids[:, c] - 1].sum()) <= 1e-11 * np.abs(R).max()


@pytest.mark.parametrize("model", [oracle.HE, oracle.J2])
def test_rigid_rotation_invariance(model):
    mat = oracle.material(model, sigma_y=250.0, H=2000.0)
    F = np.eye(3) + np.array([[3e-3, 1e-3, 0], [0, -1e-3, 2e-3], [5e-4, 0, 2e-3]])
    st = np.zeros(10)
    st[[0, 4, 8]] = 1.0
    e1, S1, _, _, _ = oracle.cm_update(mat, F, st)
    Q = rot(0.3, -1.1, 2.0)
    e2, S2, _, _, _ = oracle.cm_update(mat, Q @ F, st)
    assert e1 == 0 and e2 == 0
    assert np.abs(S1 - S2).max() <= 1e-10 * np.abs(S1).max()


def test_he_stiffness_symmetric():
    p, P, mat = small_problem("he", n=2)
    err, fe, lk, _ = P.element(mat, 5, elem_u(p, 5, p.u))
    assert err == 0
    assert np.abs(lk - lk.T).max() <= 1e-10 * np.abs(lk).max()


@pytest.mark.parametrize("w", [0.0, 0.005])
def test_cp_tangent_matches_central_differences(w):
    """w > 0: the saturation stress depends on the slip rate, and its
    derivative enters the local Jacobian and the tangent."""
    p = wl.cp_p1(n=3, seed=2, ngrains=4)
    if w:
        p.mat.w = w
        p.mat.gamma_dot_s = 5e10
    P, mat = oracle.from_workload(p)
    st = p.state.copy()
    for s in range(1, 5):  # load to a plastic state
        err, R, K, st = P.assemble(mat, p.displacement(s), state_n=st, dt=p.dt)
        assert err == 0
    u = p.displacement(5)
    for e in (1, 40, 100):
        ue = elem_u(p, e, u)
        err, fe, lk, _ = P.element(mat, e, ue, st[e], dt=p.dt)
        assert err == 0
        h = 1e-8
        fd = np.zeros_like(lk)
        for k in range(12):
            up, um = ue.copy(), ue.copy()
            up[k] += h
            um[k] -= h
            _, fp, _, _ = P.element(mat, e, up, st[e], dt=p.dt, want_K=False)
            _, fm, _, _ = P.element(mat, e, um, st[e], dt=p.dt, want_K=False)
            fd[:, k] = (fp - fm) / (2 * h)
        assert np.linalg.norm(fd - lk) <= 1e-6 * np.linalg.norm(lk)


def test_cp_local_newton_converges_with_uneven_iterations():
    p = wl.cp_p1(n=3, seed=2, ngrains=4)
    mat = oracle.from_pg_material(p.mat)
    st = p.state.copy()
    seen = set()
    for s in range(1, 6):
        F = p1_deformation_gradients(p, p.displacement(s))
        bad, st, it, dg, cv = oracle.cp_update_batch(mat, F, st, p.dt, p.R_cp)
        assert bad == 0 and cv.all()
        seen |= set(np.unique(it).tolist())
    assert max(seen) - min(seen) >= 5


def test_cp_warm_start_from_converged_increment_needs_no_iterations():
    p = wl.cp_p1(n=3, seed=2, ngrains=4)
    mat = oracle.from_pg_material(p.mat)
    st = p.state.copy()
    F = p1_deformation_gradients(p, p.displacement(1))
    _, st, _, _, _ = oracle.cp_update_batch(mat, F, st, p.dt, p.R_cp)
    F = p1_deformation_gradients(p, p.displacement(2))
    _, s_cold, it_cold, dg, _ = oracle.cp_update_batch(mat, F, st, p.dt, p.R_cp)
    M0 = cp_guess_from_slip(p, dg)
    _, s_warm, it_warm, _, cv = oracle.cp_update_batch(mat, F, st, p.dt, p.R_cp, M0=M0[:, :9], g_guess=M0[:, 9] * 0 + s_cold[:, 9])
    assert cv.all()
    assert it_warm.max() <= 2 and it_cold.mean() > it_warm.mean()
    assert np.abs(s_warm - s_cold).max() <= 1e-9 * np.abs(s_cold).max()


def p1_deformation_gradients(p, u):
    """F per linear tet from a free-DOF displacement vector (numpy)."""
    X = p.X[p.conn]
    ue = np.zeros((p.ne, 4, 3))
    for a in range(4):
        for j in range(3):
            i = p.ids[p.conn[:, a], j]
            ue[:, a, j] = np.where(i > 0, u[i - 1], 0.0)
    D = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=2)
    dU = np.stack([ue[:, 1] - ue[:, 0], ue[:, 2] - ue[:, 0], ue[:, 3] - ue[:, 0]], axis=2)
    F = np.eye(3)[None] + dU @ np.linalg.inv(D)
    return F.reshape(-1, 9)


def cp_guess_from_slip(p, dgam):
    """Initial guess M0 = I - sum dgam_a P_a (and a g column placeholder) from slip increments."""
    s, n = wl.fcc_slip_systems()
    R = p.R_cp.reshape(-1, 3, 3)
    rs = np.einsum("eij,aj->eai", R, s)
    rn = np.einsum("eij,aj->eai", R, n)
    P = np.einsum("eai,eaj->eaij", rs, rn)
    M0 = np.eye(3)[None] - np.einsum("ea,eaij->eij", dgam, P)
    return np.concatenate([M0.reshape(-1, 9), np.zeros((len(M0), 1))], axis=1)


@pytest.mark.parametrize("vol_pot", [2, 3])
def test_volumetric_potentials_change_the_answer(vol_pot):
    """The Doll-Schweizerhof potentials are really used (R differs from the
    U_Common answer at finite volume change)."""
    p, P, mat = small_problem("j2", stretch=6e-3, vol_pot=99)
    _, R0, _, _ = P.assemble(mat, p.u, state_n=p.state)
    p2, P2, mat2 = small_problem("j2", stretch=6e-3, vol_pot=vol_pot)
    _, R1, _, _ = P2.assemble(mat2, p2.u, state_n=p2.state)
    assert np.linalg.norm(R1 - R0) > 1e-6 * np.linalg.norm(R0)
