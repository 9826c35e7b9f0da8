"""The transient (inertia, mid-point rule) element of the oracle on the CPU
(oracle/pgfem_oracle.cpp, orc_assemble_transient; the reference's
residual_with_inertia / stiffness_with_inertia, src/dynamics.cc:183-432, for
the hyperelastic model), checked by known answers on a mesh with every DOF
free: at rest the residual vanishes and the mass part of K sums to
-rho V / dt_np1 per component; a rigid motion of constant acceleration a
(u_k = a t_k^2 / 2) leaves only the inertia force, which sums to
-rho V a (dt_n + dt_np1) / 2; the K of the element is
-M / dt_np1 - alpha (1 - alpha) dt_np1 K(u_{n+alpha})."""
import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
import workloads as wl


def free_box(n, nne):
    X, conn, _ = pg.mesh_box_tet(n, nne)
    codes = np.zeros((X.shape[0], 3), dtype=np.int64)
    ids, ndof = pg.generate_dof_ids(conn, X.shape[0], codes)
    Ap, Ai = pg.psparse_apai(conn, ids, ndof)
    return X, conn, ids, ndof, Ap, Ai


@pytest.mark.parametrize("nne", [4, 10])
def test_rest_and_mass(nne):
    X, conn, ids, ndof, Ap, Ai = free_box(2, nne)
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai)
    mat = oracle.material(oracle.HE)
    z = np.zeros(ndof)
    rho, dt1, dt0, al = 3.0, 0.2, 0.1, 0.4
    err, R, K = oracle.assemble_transient(P, mat, z, z, z, al, dt1, dt0, rho)
    assert err == 0 and np.abs(R).max() == 0.0
    _, _, K0, _ = P.assemble(mat, z)  # quasi-static K at rest
    Mpart = -(K + al * (1 - al) * dt1 * K0) * dt1  # = M
    rows = np.repeat(np.arange(ndof), np.diff(Ap))
    cx = (ids[:, 0] - 1)  # x-component rows / columns
    mx = np.isin(rows, cx) & np.isin(Ai, cx)
    assert np.isclose(Mpart[mx].sum(), rho * 1.0, rtol=1e-12)  # unit cube
    # the mass couples equal components only
    comp = np.zeros(ndof, dtype=int)
    for c in range(3):
        comp[ids[:, c] - 1] = c
    off = comp[rows] != comp[Ai]
    assert np.abs(Mpart[off]).max() <= 1e-14 * np.abs(K).max() * dt1  # roundoff of the subtraction only


@pytest.mark.parametrize("nne", [4, 10])
def test_constant_acceleration_rigid_motion(nne):
    X, conn, ids, ndof, Ap, Ai = free_box(2, nne)
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai)
    mat = oracle.material(oracle.HE)
    a = np.array([2.0, -1.0, 0.5])
    dt0, dt1, al, rho = 0.1, 0.15, 0.6, 5.0
    t = np.array([0.3, 0.3 + dt0, 0.3 + dt0 + dt1])
    us = []
    for tk in t:
        disp = np.tile(0.5 * a * tk ** 2, (X.shape[0], 1))
        us.append(wl.nodal_to_free(ids, disp))
    err, R, K = oracle.assemble_transient(P, mat, us[2], us[1], us[0], al, dt1, dt0, rho)
    assert err == 0
    for c in range(3):
        tot = R[ids[:, c] - 1].sum()
        assert np.isclose(tot, -rho * 1.0 * a[c] * (dt0 + dt1) / 2, rtol=1e-10)


def test_linear_in_the_static_parts():
    """With rho -> 0 the residual is the mid-point blend of quasi-static residuals."""
    p = wl.he_p1(n=2, seed=3)
    P, mat = oracle.from_workload(p)
    rng = np.random.default_rng(1)
    u2, u1, u0 = (p.u + 1e-3 * rng.uniform(-1, 1, p.ndof) for _ in range(3))
    al, dt1, dt0 = 0.3, 0.2, 0.1
    err, R, K = oracle.assemble_transient(P, mat, u2, u1, u0, al, dt1, dt0, 0.0)
    _, Ra, Ka, _ = P.assemble(mat, (1 - al) * u1 + al * u2)
    _, Rb, _, _ = P.assemble(mat, (1 - al) * u0 + al * u1, want_K=False)
    assert np.allclose(R, -dt1 * (1 - al) * Ra - dt0 * al * Rb, rtol=1e-12, atol=1e-12 * np.abs(Ra).max())
    assert np.allclose(K, -al * (1 - al) * dt1 * Ka, rtol=1e-12, atol=1e-12 * np.abs(Ka).max())


def _surface_part(P, mat, us, al, dt1, dt0, faces, loads3):
    """Transient R, K with the faces loaded minus without (the surface part)."""
    el, fc, lt = faces
    P.set_neumann(el, fc, lt, loads3[0], load_n=loads3[1], load_nm1=loads3[2])
    err, R1, K1 = oracle.assemble_transient(P, mat, us[2], us[1], us[0], al, dt1, dt0, 2.0)
    assert err == 0
    P.set_neumann([], [], [], np.zeros((0, 3)))
    err, R0, K0 = oracle.assemble_transient(P, mat, us[2], us[1], us[0], al, dt1, dt0, 2.0)
    assert err == 0
    return R1 - R0, K1 - K0


@pytest.mark.parametrize("nne", [4, 10])
def test_surface_loads_constant_in_time(nne):
    """With u and the loads the same at the three times the transient surface
    terms are the quasi-static ones scaled: traction -(dt_np1 (1 - a) + dt_n a)
    on R and -dt_np1 a (1 - a) on K; a pressure at a = 0 (only the older value,
    projected on the normal, enters) -dt_np1 on R and nothing on K."""
    X, conn, ids, ndof, Ap, Ai = free_box(2, nne)
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai)
    mat = oracle.material(oracle.HE)
    u = 1e-3 * np.random.default_rng(5).uniform(-1, 1, ndof)
    el, fc = wl.box_faces(X, conn, 0, 1.0)
    dt1, dt0 = 0.2, 0.1
    for lt, val, al in ((3, [3.0, -1.0, 2.0], 0.35), (1, [5.0, 0.0, 0.0], 0.0)):
        loads = np.tile(val, (len(el), 1))
        Rs, Ks = _surface_part(P, mat, (u, u, u), al, dt1, dt0, (el, fc, np.full(len(el), lt)), (loads,) * 3)
        P.set_neumann(el, fc, np.full(len(el), lt), loads)
        _, Rq1, Kq1, _ = P.assemble(mat, u)
        P.set_neumann([], [], [], np.zeros((0, 3)))
        _, Rq0, Kq0, _ = P.assemble(mat, u)
        cR = -(dt1 * (1 - al) + dt0 * al) if lt != 1 else -dt1
        cK = -dt1 * al * (1 - al)
        np.testing.assert_allclose(Rs, cR * (Rq1 - Rq0), rtol=0, atol=1e-12 * np.abs(Rs).max())
        np.testing.assert_allclose(Ks, cK * (Kq1 - Kq0), rtol=0, atol=1e-10 * np.abs(Kq1 - Kq0).max())


# ---- crystal plasticity: the mid-point plastic state ---------------------------
def _cp_history(n=2, ngrains=4):
    """A CP problem marched through two quasi-static steps of its ramp (slip
    active): the states at t_{n-1} (step 1) and t_n (step 2) and the
    displacements of steps 1, 2, 3 as u_{n-1}, u_n, u_{n+1}."""
    p = wl.cp_p1(n=n, seed=2, ngrains=ngrains)
    P, mat = oracle.from_workload(p)
    us = [p.displacement(s) for s in (1, 2, 3)]
    err, _, _, s_nm1 = P.assemble(mat, us[0], state_n=p.state, dt=p.dt, want_K=False)
    assert err == 0
    err, _, _, s_n = P.assemble(mat, us[1], state_n=s_nm1, dt=p.dt, want_K=False)
    assert err == 0
    return p, P, mat, us, s_nm1, s_n


def test_cp_transient_end_points_are_the_quasi_static_residual():
    """alpha = 1 keeps only the older mid point at (F_n, pF_n): R = -dt_n r_n;
    alpha = 0 only the newer one at the same point: R = -dt_np1 r_n; r_n is the
    quasi-static residual of the step that produced the state at t_n, K = 0
    (rho = 0).  This pins which state each mid point reads."""
    p, P, mat, us, s_nm1, s_n = _cp_history()
    err, r_n, _, s_chk = P.assemble(mat, us[1], state_n=s_nm1, dt=p.dt, want_K=False)
    assert err == 0 and np.abs(s_chk - s_n).max() <= 1e-13
    dt1, dt0 = p.dt, 0.7 * p.dt
    for al, coef in ((1.0, -dt0), (0.0, -dt1)):
        err, R, K, _ = oracle.assemble_transient_cp(P, mat, us[2], us[1], us[0], al, dt1, dt0, 0.0, s_nm1, s_n)
        assert err == 0
        np.testing.assert_allclose(R, coef * r_n, rtol=0, atol=1e-12 * np.abs(r_n).max())
        assert np.abs(K).max() == 0.0


def test_cp_transient_without_slip_is_the_hyperelastic_one():
    """A slip resistance far above the stress stops every slip system
    (gamma_dot = 0, pF = I, dM/du = 0): the CP transient is the hyperelastic
    one with the same elasticity, inertia included."""
    p, P, mat, us, _, _ = _cp_history()
    ne = p.conn.shape[0]
    st = np.zeros((ne, 10))
    st[:, [0, 4, 8]] = 1.0
    st[:, 9] = 1e30
    mhe = oracle.from_pg_material(p.mat)
    mhe.model = oracle.HE
    al, dt1, dt0, rho = 0.35, p.dt, 0.8 * p.dt, 7.5e-3
    err, R, K, s2 = oracle.assemble_transient_cp(P, mat, us[2], us[1], us[0], al, dt1, dt0, rho, st, st)
    assert err == 0
    np.testing.assert_array_equal(s2, st)
    err, Rh, Kh = oracle.assemble_transient(P, mhe, us[2], us[1], us[0], al, dt1, dt0, rho)
    assert err == 0
    np.testing.assert_allclose(R, Rh, rtol=0, atol=1e-13 * np.abs(Rh).max())
    np.testing.assert_allclose(K, Kh, rtol=0, atol=1e-13 * np.abs(Kh).max())


def test_cp_transient_stiffness_is_the_derivative():
    """K of the CP transient (mid-point plastic part through pF_{n+1}, the
    consistent derivative of the local update) against central differences
    of R in u_{n+1}, with slip active and inertia on."""
    p, P, mat, us, s_nm1, s_n = _cp_history()
    rng = np.random.default_rng(11)
    u2 = us[2] + 2e-4 * rng.uniform(-1, 1, p.ndof) / p.meta["n"]
    al, dt1, dt0, rho = 0.4, p.dt, 0.6 * p.dt, 3e-3
    err, R, K, s2 = oracle.assemble_transient_cp(P, mat, u2, us[1], us[0], al, dt1, dt0, rho, s_nm1, s_n)
    assert err == 0
    assert np.abs(s2[:, :9] - s_n[:, :9]).max() > 1e-6  # the plastic part moved in this step
    cols = rng.choice(p.ndof, 8, replace=False)
    h = 1e-7
    for j in cols:
        up, um = u2.copy(), u2.copy()
        up[j] += h
        um[j] -= h
        _, Rp, _, _ = oracle.assemble_transient_cp(P, mat, up, us[1], us[0], al, dt1, dt0, rho, s_nm1, s_n,
                                                   want_K=False)
        _, Rm, _, _ = oracle.assemble_transient_cp(P, mat, um, us[1], us[0], al, dt1, dt0, rho, s_nm1, s_n,
                                                   want_K=False)
        fd = (Rp - Rm) / (2 * h)
        col = np.zeros(p.ndof)
        for i in range(p.ndof):  # column j of the CSR K
            row = slice(p.Ap[i], p.Ap[i + 1])
            hit = np.nonzero(p.Ai[row] == j)[0]
            if hit.size:
                col[i] = K[p.Ap[i] + hit[0]]
        assert np.abs(col - fd).max() <= 1e-6 * np.abs(col).max(), (j, np.abs(col - fd).max(), np.abs(col).max())
