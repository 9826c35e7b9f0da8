"""The three-field (CM3F) element on the GPU against the oracle, through the C
ABI (pgfem_gpu_set_three_field and the R+K, residual, local-update and Newton
entry points; the reference's element with one pressure and one volume per
element, src/constitutive_model.cc:695-881, src/constitutive_model_3f.cc,
src/condense.cc:300-385).

Quadratic-tet tension boxes of the hyperelastic model (and of this library's
J2 model, state at t_n given, yielding), perturbed nodes, element
pressures and volumes away from their local solution: R and K of the condensed
element equal the oracle's at 1e-10 (with surface loads too), the residual
call equals the R of the R+K call, the local update (compute_d_theta_dP)
equals the oracle's, and the device Newton step -- local update after each
solve -- follows the oracle's Newton loop to the same displacements,
pressures and volumes.  The calls the three-field element does not cover are
rejected.  The transient form (inertia, mid-point rule; P and theta at t_n and
t_{n-1} kept by the context): R, K and the local update equal the oracle's
(orc_assemble_3f_transient / orc_update_3f_transient) at 1e-10, with surface
loads too, and a commit moves the current P, theta to t_n and t_n to t_{n-1}."""
import numpy as np
import pytest
from scipy.sparse import csr_matrix
from scipy.sparse.linalg import spsolve

import oracle
import pgfem_gpu as pg
import workloads as wl
from test_gpu_parity import check_K, check_R

pytestmark = pytest.mark.gpu


def _case(n=3, seed=5, vol_pot=99, curve=True):
    p = wl.tension(n=n, nne=10, model="he", stretch=0.01, predictor=True)
    p.mat = pg.material(pg.MODEL_HE, E=200e3, nu=0.45, vol_pot=vol_pot)
    rng = np.random.default_rng(seed)
    if curve:
        p.X = p.X + 0.02 / n * rng.uniform(-1, 1, p.X.shape)
    ne = p.conn.shape[0]
    P = 50.0 * rng.uniform(-1, 1, ne)
    th = 1.0 + 0.01 * rng.uniform(-1, 1, ne)
    return p, P, th


@pytest.mark.parametrize("vol_pot", [99, 2, 3])
def test_R_K_match_oracle(gpu, vol_pot):
    p, P, th = _case(vol_pot=vol_pot)
    ctx = p.context()
    ctx.set_three_field(P, th)
    assert ctx.three_field_enabled()
    R, K, st = ctx.assemble_RK(p.u, p.u_presc)
    assert st.ok(), st.as_dict()
    Po, mat = oracle.from_workload(p)
    err, Ro, Ko = Po.assemble_3f(mat, p.u, P, th, u_presc=p.u_presc)
    assert err == 0
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    # the condensation carries weight: the one-field element differs
    _, R1, K1, _ = Po.assemble(mat, p.u, p.u_presc)
    assert np.linalg.norm(R1 - Ro) > 1e-3 * np.linalg.norm(Ro)
    # the residual call
    Rr, st = ctx.assemble_R(p.u, p.u_presc)
    assert st.ok()
    check_R(Rr, Ro)
    # P and theta read back; switching back gives the one-field element
    Pg, thg = ctx.get_three_field()
    assert np.array_equal(Pg, P) and np.array_equal(thg, th)
    ctx.set_three_field(None, None)
    R1g, _ = ctx.assemble_R(p.u, p.u_presc)
    check_R(R1g, R1)
    ctx.close()


def test_with_surface_loads(gpu):
    p, P, th = _case(seed=9)
    el, fc = wl.box_faces(p.X, p.conn, 2, 1.0)
    p.X = p.X  # faces picked before any further change
    ft = np.zeros(len(el), dtype=np.int32)
    ctx = p.context()
    ctx.set_neumann(el, fc, ft, np.array([1]), np.array([[30.0, 0.0, 0.0]]))
    ctx.set_three_field(P, th)
    R, K, st = ctx.assemble_RK(p.u, p.u_presc)
    assert st.ok()
    Po, mat = oracle.from_workload(p)
    Po.set_neumann(el, fc, np.ones(len(el), dtype=np.int64), np.tile([30.0, 0.0, 0.0], (len(el), 1)))
    err, Ro, Ko = Po.assemble_3f(mat, p.u, P, th, u_presc=p.u_presc)
    assert err == 0
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    ctx.close()


def test_local_update_matches_oracle(gpu):
    p, P, th = _case(seed=2)
    ctx = p.context()
    ctx.set_three_field(P, th)
    du = 1e-3 * np.random.default_rng(4).uniform(-1, 1, p.ndof)
    dP, dth, st = ctx.three_field_increments(p.u, du, p.u_presc)
    assert st.ok()
    Po, mat = oracle.from_workload(p)
    err, dPo, dtho = Po.update_3f(mat, p.u, du, P, th, u_presc=p.u_presc)
    assert err == 0
    assert np.abs(dP - dPo).max() <= 1e-10 * np.abs(dPo).max()
    assert np.abs(dth - dtho).max() <= 1e-10 * np.abs(dtho).max()
    ctx.close()


def _oracle_newton(Po, mat, u, u_presc, P, th, iter_max=15, nor_min=1e-10, state_n=None):
    u, P, th = u.copy(), P.copy(), th.copy()
    hist, NORM = [], 1.0
    for it in range(iter_max + 1):
        res = Po.assemble_3f(mat, u, P, th, u_presc=u_presc, state_n=state_n)
        err, R, K = res[:3]
        assert err == 0
        nor2 = float(np.linalg.norm(R))
        NORM = nor2 if it == 0 else NORM
        hist.append(nor2 / NORM)
        if hist[-1] <= nor_min:
            return u, P, th, hist, True
        du = spsolve(csr_matrix((K, Po.Ai, Po.Ap), shape=(Po.ndof, Po.ndof)).tocsc(), -R)
        err, dP, dth = Po.update_3f(mat, u, du, P, th, u_presc=u_presc, state_n=state_n)
        assert err == 0
        P, th, u = P + dP, th + dth, u + du
    return u, P, th, hist, False


def test_device_newton_matches_oracle(gpu):
    import torch
    p, _, _ = _case(n=3, seed=3, curve=False)
    ne = p.conn.shape[0]
    P0, th0 = np.zeros(ne), np.ones(ne)
    Po, mat = oracle.from_workload(p)
    uo, Pio, tho, ho, ok = _oracle_newton(Po, mat, p.u, p.u_presc, P0, th0)
    assert ok and len(ho) >= 3
    ctx = p.context()
    ctx.set_three_field(P0, th0)
    s = pg.Solver(p.Ap, p.Ai, p.ndof, maxit=20000, kdim=100, tol=1e-12)
    du = torch.from_numpy(p.u.copy()).cuda()
    dp = torch.from_numpy(p.u_presc.copy()).cuda()
    info = s.newton_step(ctx, du.data_ptr(), dp.data_ptr(), iter_max=15, nor_min=1e-10)
    assert info.converged and not info.lin_failed and info.elem_failures == 0
    h = info.history()
    assert len(h) == len(ho), (h, ho)
    u = du.cpu().numpy()
    assert np.linalg.norm(u - uo) <= 1e-8 * np.linalg.norm(uo)
    Pg, thg = ctx.get_three_field()
    # theta follows u (1e-8 relative); P = kappa U'(theta) amplifies theta's
    # difference by kappa
    kap = 200e3 / (3 * (1 - 2 * 0.45))
    assert np.abs(thg - tho).max() <= 1e-8
    assert np.abs(Pg - Pio).max() <= 1e-8 * kap
    # at the solution the local constraints hold: theta = mean J, P = kappa U'(theta)
    assert np.abs(Pg - kap * (thg - 1.0)).max() <= 1e-6 * np.abs(Pg).max()
    ctx.close()


def test_rejections(gpu):
    p1 = wl.he_p1(n=2, seed=1)
    c1 = p1.context()
    with pytest.raises(pg.PgfemError):
        c1.set_three_field(np.zeros(p1.ne), np.ones(p1.ne))
    c1.close()
    p, P, th = _case(n=2)
    ctx = p.context()
    with pytest.raises(pg.PgfemError):
        ctx.set_three_field(P, -th)  # a volume must be positive
    ctx.set_three_field(P, th)
    with pytest.raises(pg.PgfemError):
        ctx.stiffmatel_fd([0], p.u, p.u_presc)
    ctx.close()


def test_j2_R_K_state_match_oracle(gpu):
    p = wl.j2_p2(n=3, seed=11, stretch=4e-3, perturb=5e-3)
    rng = np.random.default_rng(21)
    P = 300.0 * rng.uniform(-1, 1, p.ne)
    th = 1.0 + 0.002 * rng.uniform(-1, 1, p.ne)
    ctx = p.context()
    ctx.set_three_field(P, th)
    R, K, st = ctx.assemble_RK(p.u)
    assert st.ok(), st.as_dict()
    Po, mat = oracle.from_workload(p)
    err, Ro, Ko, so = Po.assemble_3f(mat, p.u, P, th, state_n=p.state)
    assert err == 0
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    sg = ctx.get_state(1)
    assert np.abs(sg - so).max() <= 1e-10 * np.abs(so).max()
    assert (so[:, 9] > 0).mean() > 0.3  # points yield
    ctx.close()


def test_j2_device_newton_matches_oracle(gpu):
    import torch
    p = wl.tension(n=2, nne=10, model="j2", stretch=0.003, predictor=True)
    ne = p.conn.shape[0]
    P0, th0 = np.zeros(ne), np.ones(ne)
    Po, mat = oracle.from_workload(p)
    uo, Pio, tho, ho, ok = _oracle_newton(Po, mat, p.u, p.u_presc, P0, th0, state_n=p.state)
    assert ok
    ctx = p.context()
    ctx.set_three_field(P0, th0)
    s = pg.Solver(p.Ap, p.Ai, p.ndof, maxit=20000, kdim=100, tol=1e-12)
    du = torch.from_numpy(p.u.copy()).cuda()
    dp = torch.from_numpy(p.u_presc.copy()).cuda()
    info = s.newton_step(ctx, du.data_ptr(), dp.data_ptr(), iter_max=15, nor_min=1e-10)
    assert info.converged and not info.lin_failed and info.elem_failures == 0
    assert len(info.history()) == len(ho)
    u = du.cpu().numpy()
    assert np.linalg.norm(u - uo) <= 1e-8 * np.linalg.norm(uo)
    Pg, thg = ctx.get_three_field()
    kap = 200e3 / (3 * (1 - 2 * 0.3))
    assert np.abs(thg - tho).max() <= 1e-8
    assert np.abs(Pg - Pio).max() <= 1e-8 * kap
    ctx.close()


def test_larger_mesh_free_body_and_translations(gpu):
    """24^3 cells (the config-2 mesh at a smaller n, every DOF free, K values
    above L2): the condensed internal forces of a free body sum to zero per
    component, and K maps a rigid translation to zero."""
    p = wl.j2_p2(n=24, seed=1)
    p.mat = pg.material(pg.MODEL_HE, E=200e3, nu=0.45)
    p.state = None
    rng = np.random.default_rng(8)
    ctx = p.context()
    ctx.set_three_field(300.0 * rng.uniform(-1, 1, p.ne), 1.0 + 0.002 * rng.uniform(-1, 1, p.ne))
    R, K, st = ctx.assemble_RK(p.u)
    assert st.ok()
    Km = csr_matrix((K, p.Ai, p.Ap), shape=(p.ndof, p.ndof))
    for c in range(3):
        rows = p.ids[:, c] - 1
        assert abs(R[rows].sum()) <= 1e-10 * np.abs(R[rows]).sum()
        t = np.zeros(p.ndof)
        t[rows] = 1.0
        assert np.abs(Km @ t).max() <= 1e-10 * np.abs(Km).sum(axis=1).max()
    ctx.close()


def _tr_case(seed=9, curve=True):
    """Displacements, prescribed values, element pressures and volumes at
    t_{n+1}, t_n, t_{n-1} of a curved quadratic-tet tension box."""
    p, P, th = _case(seed=seed, vol_pot=3, curve=curve)  # a potential whose U'' varies: theta's history weighs in R
    rng = np.random.default_rng(seed + 1)
    h = 1.0 / p.meta["n"]
    us = [p.u * f + 1e-3 * h * rng.uniform(-1, 1, p.ndof) for f in (1.0, 0.7, 0.4)]
    ps = [p.u_presc * f for f in (1.0, 0.7, 0.4)]
    Ps = [P, 0.8 * P + 3.0, 0.5 * P - 4.0]
    ths = [th, 1.0 + 0.7 * (th - 1.0) + 1e-3, 1.0 + 0.4 * (th - 1.0) - 1e-3]
    return p, us, ps, Ps, ths


def _tr_context(p, Ps, ths):
    ctx = p.context()
    ctx.set_three_field(Ps[0], ths[0])
    ctx.set_three_field_history(Ps[1], ths[1], Ps[2], ths[2])
    return ctx


@pytest.mark.parametrize("alpha", [0.5, 0.3])
def test_transient_R_K_update_match_oracle(gpu, alpha):
    p, us, ps, Ps, ths = _tr_case()
    ctx = _tr_context(p, Ps, ths)
    dt1, dt0, rho = 0.02, 0.015, 2.0e4
    R, K, st = ctx.assemble_RK_transient(us[0], us[1], us[2], alpha, dt1, dt0, rho, presc=tuple(ps))
    assert st.ok(), st.as_dict()
    Po, mat = oracle.from_workload(p)
    err, Ro, Ko = Po.assemble_3f_transient(mat, us, Ps, ths, alpha, dt1, dt0, rho, presc=tuple(ps))
    assert err == 0
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    # the three-field history and the inertia both carry weight
    _, Rh, _ = Po.assemble_3f_transient(mat, us, [Ps[0]] * 3, [ths[0]] * 3, alpha, dt1, dt0, rho,
                                        presc=tuple(ps))
    assert np.linalg.norm(Ro - Rh) > 1e-3 * np.linalg.norm(Ro)
    _, R0, _ = Po.assemble_3f_transient(mat, us, Ps, ths, alpha, dt1, dt0, 0.0, presc=tuple(ps))
    assert np.linalg.norm(Ro - R0) > 1e-2 * np.linalg.norm(Ro)
    # residual only
    R2, K2, st = ctx.assemble_RK_transient(us[0], us[1], us[2], alpha, dt1, dt0, rho, presc=tuple(ps),
                                           want_K=False)
    assert K2 is None and st.ok()
    check_R(R2, Ro)
    # the local update
    du = 1e-3 / p.meta["n"] * np.random.default_rng(3).uniform(-1, 1, p.ndof)
    dP, dth, st = ctx.three_field_increments_transient(us[0], us[1], us[2], du, alpha, dt1, dt0,
                                                       presc=tuple(ps))
    assert st.ok()
    err, dPo, dtho = Po.update_3f_transient(mat, us, du, Ps, ths, alpha, dt1, dt0, presc=tuple(ps))
    assert err == 0
    assert np.abs(dth - dtho).max() <= 1e-10 * np.abs(dtho).max()
    assert np.abs(dP - dPo).max() <= 1e-10 * np.abs(dPo).max()
    # commit: the current P, theta become t_n, t_n becomes t_{n-1}
    ctx.commit_state()
    Pn = [Ps[0] + 1.0, Ps[0], Ps[1]]
    tn = [ths[0] * 1.001, ths[0], ths[1]]
    ctx.set_three_field(Pn[0], tn[0])
    un = [us[0] * 1.2, us[0], us[1]]
    pn = [ps[0] * 1.2, ps[0], ps[1]]
    R, K, st = ctx.assemble_RK_transient(un[0], un[1], un[2], alpha, dt1, dt0, rho, presc=tuple(pn))
    assert st.ok()
    err, Ro, Ko = Po.assemble_3f_transient(mat, un, Pn, tn, alpha, dt1, dt0, rho, presc=tuple(pn))
    assert err == 0
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    ctx.close()


def test_transient_with_surface_loads(gpu):
    p, us, ps, Ps, ths = _tr_case(seed=4, curve=False)  # faces on the plane z = 1
    ctx = _tr_context(p, Ps, ths)
    el, fc = wl.box_faces(p.X, p.conn, 2, 1.0)
    assert len(el) > 0
    ft = np.zeros(len(el), dtype=np.int32)
    types = np.array([3])
    L2 = np.array([[300.0, -100.0, 50.0]])
    L1, L0 = 0.7 * L2 + 20.0, 0.4 * L2 - 30.0
    ctx.set_neumann(el, fc, ft, types, L2)
    ctx.set_neumann_load_history(L1, L0)
    alpha, dt1, dt0, rho = 0.4, 0.02, 0.015, 2.0e4
    R, K, st = ctx.assemble_RK_transient(us[0], us[1], us[2], alpha, dt1, dt0, rho, presc=tuple(ps))
    assert st.ok(), st.as_dict()
    Po, mat = oracle.from_workload(p)
    Po.set_neumann(el, fc, types[ft], L2[ft], load_n=L1[ft], load_nm1=L0[ft])
    err, Ro, Ko = Po.assemble_3f_transient(mat, us, Ps, ths, alpha, dt1, dt0, rho, presc=tuple(ps))
    assert err == 0
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    P0, _ = oracle.from_workload(p)
    _, R0, _ = P0.assemble_3f_transient(mat, us, Ps, ths, alpha, dt1, dt0, rho, presc=tuple(ps))
    assert np.linalg.norm(Ro - R0) > 1e-3 * np.linalg.norm(Ro)
    ctx.close()


def test_transient_rejections(gpu):
    p, us, ps, Ps, ths = _tr_case()
    ctx = _tr_context(p, Ps, ths)
    for a in (0.0, 1.0):  # the local update divides by alpha (1 - alpha)
        with pytest.raises(pg.PgfemError):
            ctx.assemble_RK_transient(us[0], us[1], us[2], a, 0.02, 0.015, 1.0, presc=tuple(ps))
        with pytest.raises(pg.PgfemError):
            ctx.three_field_increments_transient(us[0], us[1], us[2], us[0], a, 0.02, 0.015, presc=tuple(ps))
    ctx.close()
    c2 = p.context()
    with pytest.raises(pg.PgfemError):  # not three-field
        c2.three_field_increments_transient(us[0], us[1], us[2], us[0], 0.5, 0.02, 0.015, presc=tuple(ps))
    with pytest.raises(pg.PgfemError):
        c2.set_three_field_history(Ps[1], ths[1], Ps[2], ths[2])
    c2.close()
