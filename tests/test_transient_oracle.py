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
