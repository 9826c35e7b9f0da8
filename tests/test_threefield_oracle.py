"""The three-field (CM3F) element of the oracle on the CPU (hyperelastic model;
the J2 model of this library with its isochoric return map)
(oracle/pgfem_oracle.cpp, orc_element_3f / orc_assemble_3f / orc_update_3f:
the reference's constitutive-model element with one pressure and one volume
per element, src/constitutive_model.cc:695-881, src/constitutive_model_3f.cc,
src/condense.cc:300-385), checked by identities of the mixed formulation:

* with theta and P at their local solution theta* = sum w J / sum w,
  P* = kappa U'(theta*) (fp = ft = 0), the condensed residual is
  g(u) = fu(u, P*(u), theta*(u)) and the condensed stiffness is its exact
  derivative -- checked against central differences of g;
* the condensed residual does not depend on P (the pressure terms cancel);
* Kup is the derivative of fp with respect to u (central differences);
* under a homogeneous deformation (J the same at every point) with
  theta = J and P = kappa U'(J), the three-field R equals the one-field R;
* one Newton correction of the local unknowns (compute_d_theta_dP) from a
  displacement increment du lands on theta*(u + du), P*(u + du) to second
  order in du."""
import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
import workloads as wl


def _problem(n, nne, fix=False):
    X, conn, _ = pg.mesh_box_tet(n, nne)
    codes = np.zeros((X.shape[0], 3), dtype=np.int64)
    if fix:
        codes[X[:, 0] == 0.0] = 1
    ids, ndof = pg.generate_dof_ids(conn, X.shape[0], codes)
    Ap, Ai = pg.psparse_apai(conn, ids, ndof)
    return X, conn, ids, ndof, Ap, Ai


def _mat(vol_pot=99):
    return oracle.material(oracle.HE, E=200.0, nu=0.45, vol_pot=vol_pot)


def _local(P, mat, e, ue, sn=None):
    """theta* and P* of element e at ue (from the blocks at theta = 0)."""
    _, _, _, (fp0, ft, Ktp, Ktt, Kup) = P.element_3f(mat, e, ue, 0.0, 0.0, want_K=False, state_n=sn)
    W = -Ktp
    th = fp0 / W  # fp(theta = 0) = sum w J
    kap = mat.E / (3.0 * (1.0 - 2.0 * mat.nu))
    dU = th - 1.0 if mat.vol_pot not in (2, 3) else (
        0.5 * (np.exp(th - 1.0) - 1.0 / th) if mat.vol_pot == 2 else (th - 1.0) / (2 * th) + 0.5 * np.log(th))
    return th, kap * dU


@pytest.mark.parametrize("nne,vol_pot", [(10, 99), (10, 2), (10, 3), (4, 99)])
def test_condensed_stiffness_is_derivative_of_condensed_residual(nne, vol_pot):
    X, conn, ids, ndof, Ap, Ai = _problem(1, nne)
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai)
    mat = _mat(vol_pot)
    rng = np.random.default_rng(7)
    e = 2
    nd = 3 * nne
    ue = 0.03 * rng.uniform(-1, 1, nd)

    def g(u):
        th, pr = _local(P, mat, e, u)
        err, fe, _, _ = P.element_3f(mat, e, u, pr, th, want_K=False)
        assert err == 0
        return fe

    th, pr = _local(P, mat, e, ue)
    err, fe, lk, _ = P.element_3f(mat, e, ue, pr, th)
    assert err == 0
    np.testing.assert_allclose(fe, g(ue), rtol=0, atol=1e-14 * np.abs(fe).max())
    h = 1e-6
    Kfd = np.zeros((nd, nd))
    for c in range(nd):
        d = np.zeros(nd)
        d[c] = h
        Kfd[:, c] = (g(ue + d) - g(ue - d)) / (2 * h)
    assert np.abs(lk - Kfd).max() <= 1e-6 * np.abs(lk).max()


def test_residual_independent_of_pressure_and_Kup():
    X, conn, ids, ndof, Ap, Ai = _problem(1, 10)
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai)
    mat = _mat()
    rng = np.random.default_rng(3)
    ue = 0.02 * rng.uniform(-1, 1, 30)
    _, fa, _, _ = P.element_3f(mat, 1, ue, 5.0, 1.01, want_K=False)
    _, fb, _, (_, _, _, _, Kup) = P.element_3f(mat, 1, ue, -40.0, 1.01, want_K=False)
    np.testing.assert_allclose(fa, fb, rtol=0, atol=1e-12 * np.abs(fa).max())
    h = 1e-6
    for c in range(30):
        d = np.zeros(30)
        d[c] = h
        fp_p = P.element_3f(mat, 1, ue + d, 0.0, 1.0, want_K=False)[3][0]
        fp_m = P.element_3f(mat, 1, ue - d, 0.0, 1.0, want_K=False)[3][0]
        assert abs((fp_p - fp_m) / (2 * h) - Kup[c]) <= 1e-7 * np.abs(Kup).max()


@pytest.mark.parametrize("nne", [4, 10])
def test_homogeneous_deformation_equals_one_field(nne):
    X, conn, ids, ndof, Ap, Ai = _problem(2, nne)
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai)
    mat = _mat()
    Fbar = np.array([[1.02, 0.01, 0.0], [0.0, 0.99, 0.005], [0.003, 0.0, 1.01]])
    u = wl.nodal_to_free(ids, X @ (Fbar - np.eye(3)).T)
    J = np.linalg.det(Fbar)
    kap = mat.E / (3.0 * (1.0 - 2.0 * mat.nu))
    ne = conn.shape[0]
    err, R3, K3 = P.assemble_3f(mat, u, np.full(ne, kap * (J - 1.0)), np.full(ne, J))
    assert err == 0
    err, R1, K1, _ = P.assemble(mat, u)
    assert err == 0
    np.testing.assert_allclose(R3, R1, rtol=0, atol=1e-12 * np.abs(R1).max())
    assert np.abs(K3).max() > 0


def test_local_update_is_second_order():
    X, conn, ids, ndof, Ap, Ai = _problem(2, 10, fix=True)
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai)
    mat = _mat()
    rng = np.random.default_rng(11)
    ne = conn.shape[0]
    u = 0.01 * rng.uniform(-1, 1, ndof)
    du = rng.uniform(-1, 1, ndof)
    pr0, th0 = 3.0 * rng.uniform(-1, 1, ne), 1.0 + 0.01 * rng.uniform(-1, 1, ne)
    errs = []
    for s in (1e-3, 5e-4):
        err, dP, dth = P.update_3f(mat, u, s * du, pr0, th0)
        assert err == 0
        # the linearised local solution at u + s du
        th1, pr1 = th0 + dth, pr0 + dP
        ue = np.zeros(30)
        e_err = []
        for e in range(ne):
            for a in range(10):
                for j in range(3):
                    i = ids[conn[e, a], j]
                    ue[a * 3 + j] = (u + s * du)[i - 1] if i > 0 else 0.0
            ths, prs = _local(P, mat, e, ue)
            e_err.append(max(abs(th1[e] - ths), abs(pr1[e] - prs) / mat.E))
        errs.append(max(e_err))
    # from arbitrary (P, theta) the correction jumps to the local solution up
    # to the second-order remainder: halving du quarters the error
    assert errs[1] < 0.3 * errs[0]


def test_j2_condensed_stiffness_is_derivative_of_condensed_residual():
    """The J2 model (state at t_n fixed, points yielding): the same identity."""
    X, conn, ids, ndof, Ap, Ai = _problem(1, 10)
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai)
    mat = oracle.material(oracle.J2, E=200.0, nu=0.45, sigma_y=0.2, H=5.0)
    rng = np.random.default_rng(17)
    e = 3
    ue = 0.03 * rng.uniform(-1, 1, 30)
    sn = np.zeros((4, 10))
    sn[:, [0, 4, 8]] = 1.0

    def g(u):
        th, pr = _local(P, mat, e, u, sn)
        err, fe, _, _ = P.element_3f(mat, e, u, pr, th, want_K=False, state_n=sn)
        assert err == 0
        return fe

    th, pr = _local(P, mat, e, ue, sn)
    err, fe, lk, _ = P.element_3f(mat, e, ue, pr, th, state_n=sn)
    assert err == 0
    h = 1e-7
    Kfd = np.zeros((30, 30))
    for c in range(30):
        d = np.zeros(30)
        d[c] = h
        Kfd[:, c] = (g(ue + d) - g(ue - d)) / (2 * h)
    assert np.abs(lk - Kfd).max() <= 1e-5 * np.abs(lk).max()
    # the points yield, and the plastic element differs from the hyperelastic one
    mat_he = oracle.material(oracle.HE, E=200.0, nu=0.45)
    _, fe_he, _, _ = P.element_3f(mat_he, e, ue, pr, th, want_K=False)
    assert np.linalg.norm(fe - fe_he) > 1e-2 * np.linalg.norm(fe)


# ---- transient (inertia) three-field element --------------------------------
def _tr_setup(n=2, nne=10, fix=True, seed=3):
    X, conn, ids, ndof, Ap, Ai = _problem(n, nne, fix=fix)
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai)
    rng = np.random.default_rng(seed)
    ne = conn.shape[0]
    us = [0.01 * k * rng.uniform(-1, 1, ndof) for k in (3, 2, 1)]  # t_{n+1}, t_n, t_{n-1}
    Ps = [2.0 * k * rng.uniform(-1, 1, ne) for k in (3, 2, 1)]
    ths = [1.0 + 0.004 * k * rng.uniform(-1, 1, ne) for k in (3, 2, 1)]
    return P, us, Ps, ths


def test_transient_3f_constant_in_time_is_the_scaled_quasi_static_element():
    """u, P, theta the same at the three times, rho = 0: both mid points are
    the quasi-static point, so R = -(dt_np1 (1 - a) + dt_n a) R_qs and
    K = -dt_np1 a (1 - a) K_qs (the blocks' common factor drops out of the
    condensation ratios)."""
    P, us, Ps, ths = _tr_setup()
    mat = _mat()
    al, dt1, dt0 = 0.35, 0.2, 0.15
    err, R, K = P.assemble_3f_transient(mat, [us[0]] * 3, [Ps[0]] * 3, [ths[0]] * 3, al, dt1, dt0, 0.0)
    assert err == 0
    err, Rq, Kq = P.assemble_3f(mat, us[0], Ps[0], ths[0])
    assert err == 0
    np.testing.assert_allclose(R, -(dt1 * (1 - al) + dt0 * al) * Rq, rtol=0, atol=1e-12 * np.abs(Rq).max())
    np.testing.assert_allclose(K, -dt1 * al * (1 - al) * Kq, rtol=0, atol=1e-12 * np.abs(Kq).max())


def test_transient_3f_inertia_part_is_the_one_field_one():
    P, us, Ps, ths = _tr_setup()
    mat = _mat()
    al, dt1, dt0, rho = 0.6, 0.2, 0.15, 40.0
    _, R1, K1 = P.assemble_3f_transient(mat, us, Ps, ths, al, dt1, dt0, rho)
    _, R0, K0 = P.assemble_3f_transient(mat, us, Ps, ths, al, dt1, dt0, 0.0)
    _, r1, k1 = oracle.assemble_transient(P, mat, *us, al, dt1, dt0, rho)
    _, r0, k0 = oracle.assemble_transient(P, mat, *us, al, dt1, dt0, 0.0)
    np.testing.assert_allclose(R1 - R0, r1 - r0, rtol=0, atol=1e-12 * np.abs(r1 - r0).max())
    np.testing.assert_allclose(K1 - K0, k1 - k0, rtol=0, atol=1e-12 * np.abs(k1 - k0).max())


def test_transient_3f_newton_converges_quadratically():
    """Newton on (u_{n+1}, P_{n+1}, theta_{n+1}) with the condensed transient K
    and the transient local update (compute_d_theta_dP with the combined
    blocks): the condensed residual falls quadratically, so K and the update
    are the exact linearisation of the mid-point three-field system."""
    P, us, Ps, ths = _tr_setup(seed=5)
    mat = _mat()
    al, dt1, dt0, rho = 0.5, 0.05, 0.04, 20.0
    from scipy.sparse import csr_matrix
    from scipy.sparse.linalg import spsolve
    u2, P2, t2 = us[0].copy(), Ps[0].copy(), ths[0].copy()
    hist = []
    for it in range(8):
        err, R, K = P.assemble_3f_transient(mat, [u2, us[1], us[2]], [P2, Ps[1], Ps[2]], [t2, ths[1], ths[2]],
                                            al, dt1, dt0, rho)
        assert err == 0
        hist.append(np.linalg.norm(R))
        if hist[-1] <= 1e-11 * hist[0]:
            break
        du = spsolve(csr_matrix((K, P.Ai, P.Ap), shape=(P.ndof, P.ndof)).tocsc(), -R)
        err, dP, dth = P.update_3f_transient(mat, [u2, us[1], us[2]], du, [P2, Ps[1], Ps[2]],
                                             [t2, ths[1], ths[2]], al, dt1, dt0)
        assert err == 0
        u2, P2, t2 = u2 + du, P2 + dP, t2 + dth
    assert hist[-1] <= 1e-11 * hist[0] and len(hist) <= 6, hist
    rates = [hist[k + 1] / hist[k] ** 2 for k in range(1, len(hist) - 1) if hist[k] > 1e-8 * hist[0]]
    assert rates and max(rates) * hist[0] < 10.0, (hist, rates)
