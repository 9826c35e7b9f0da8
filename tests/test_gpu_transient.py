"""The transient (inertia, mid-point rule) element on the GPU against the
oracle, through the C ABI (pgfem_gpu_assemble_RK_transient; the reference's
residual_with_inertia / stiffness_with_inertia, src/dynamics.cc:183-432, for
the hyperelastic model): linear tets with a fixed face, quadratic tets with
prescribed displacements (values at three times), two alphas and unequal
steps, R and K at the parity tolerance (1e-10); below the density threshold
the call is the quasi-static assembly at t_{n+1}; with surface loads (tractions
and pressures, values at the three times) the mid-point surface terms equal the
oracle's; J2 contexts, surface loads without their earlier values and bad time
parameters are rejected.  Crystal plasticity (linear tets): with the states at
t_{n-1} and t_n from two committed load steps, R, K and the state at t_{n+1}
equal the oracle's mid-point element (orc_assemble_transient_state), with and
without surface loads; the commit moves the state at t_n to t_{n-1}."""
import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
import workloads as wl
from test_gpu_parity import check_K, check_R

pytestmark = pytest.mark.gpu


def _three_states(p, seed, amp=2e-3):
    rng = np.random.default_rng(seed)
    h = 1.0 / p.meta["n"]
    us = [p.u * (k + 1) / 3 + amp * h * rng.uniform(-1, 1, p.ndof) for k in range(3)]
    ps = None
    if p.u_presc is not None:
        ps = [p.u_presc * (k + 1) / 3 for k in range(3)]
    return us, ps


@pytest.mark.parametrize("maker,alpha", [("p1", 0.5), ("p1", 0.8), ("p2", 0.5), ("p2", 0.3)])
def test_transient_matches_oracle(gpu, maker, alpha):
    if maker == "p1":
        p = wl.he_p1(n=4, seed=2)
    else:
        p = wl.tension(n=3, nne=10, model="he", stretch=0.004, predictor=True)
    us, ps = _three_states(p, seed=7)
    dt1, dt0 = 0.02, 0.015
    rho = 2.0e4  # inertia and stiffness terms of one order (E 200e3, h ~ 0.3, dt ~ 0.02)
    ctx = p.context()
    R, K, st = ctx.assemble_RK_transient(us[2], us[1], us[0], alpha, dt1, dt0, rho,
                                         presc=(ps[2], ps[1], ps[0]) if ps else (None, None, None))
    assert st.ok(), st.as_dict()
    P, mat = oracle.from_workload(p)
    args = dict(p_np1=ps[2], p_n=ps[1], p_nm1=ps[0]) if ps else {}
    err, Ro, Ko = oracle.assemble_transient(P, mat, us[2], us[1], us[0], alpha, dt1, dt0, rho, **args)
    assert err == 0
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    # both the inertia and the quasi-static parts carry weight
    _, R0, K0 = oracle.assemble_transient(P, mat, us[2], us[1], us[0], alpha, dt1, dt0, 0.0, **args)
    assert np.linalg.norm(Ro - R0) > 0.05 * np.linalg.norm(Ro)
    assert np.linalg.norm(R0) > 0.05 * np.linalg.norm(Ro)
    # residual only
    R1, K1, st1 = ctx.assemble_RK_transient(us[2], us[1], us[0], alpha, dt1, dt0, rho,
                                            presc=(ps[2], ps[1], ps[0]) if ps else (None, None, None),
                                            want_K=False)
    assert K1 is None and st1.ok()
    check_R(R1, Ro)
    ctx.close()


def test_below_density_threshold_is_quasi_static(gpu):
    p = wl.he_p1(n=3, seed=4)
    us, _ = _three_states(p, seed=2)
    ctx = p.context()
    R, K, st = ctx.assemble_RK_transient(us[2], us[1], us[0], 0.5, 0.1, 0.1, 1e-17)
    Rs, Ks, _ = ctx.assemble_RK(us[2])
    check_R(R, Rs, 1e-13)  # two atomic-scatter assemblies: the summation order differs
    check_K(K, Ks, p.Ap, 1e-13)
    ctx.close()


def test_transient_rejections(gpu):
    p = wl.he_p1(n=2, seed=1)
    us, _ = _three_states(p, seed=1)
    ctx = p.context()
    for a, d1, d0 in [(-0.1, 0.1, 0.1), (1.5, 0.1, 0.1), (0.5, 0.0, 0.1), (0.5, 0.1, -1.0)]:
        with pytest.raises(pg.PgfemError):
            ctx.assemble_RK_transient(us[2], us[1], us[0], a, d1, d0, 1.0)
    e, f = wl.box_faces(p.X, p.conn, 0, 1.0)
    ctx.set_neumann(e, f, np.zeros(len(e), dtype=np.int32), [1], [[1.0, 0, 0]])
    with pytest.raises(pg.PgfemError):
        ctx.assemble_RK_transient(us[2], us[1], us[0], 0.5, 0.1, 0.1, 1.0)
    ctx.close()
    q = wl.j2_p2(n=2, seed=1)
    cq = q.context()
    with pytest.raises(pg.PgfemError):
        cq.assemble_RK_transient(q.u, q.u, q.u, 0.5, 0.1, 0.1, 1.0)
    cq.close()



@pytest.mark.parametrize("maker,alpha", [("p1", 0.6), ("p2", 0.4)])
def test_transient_with_surface_loads(gpu, maker, alpha):
    if maker == "p1":
        p = wl.he_p1(n=4, seed=3)
    else:
        p = wl.tension(n=3, nne=10, model="he", stretch=0.004, predictor=True)
    us, ps = _three_states(p, seed=9)
    planes = [(0, 1.0), (2, 1.0), (1, 0.0)]
    types = np.array([3, 1, 2])
    el, fc, ft = [], [], []
    for k, (axis, v) in enumerate(planes):
        e, f = wl.box_faces(p.X, p.conn, axis, v)
        el.append(e)
        fc.append(f)
        ft.append(np.full(len(e), k, dtype=np.int32))
    el, fc, ft = np.concatenate(el), np.concatenate(fc), np.concatenate(ft)
    L2 = np.array([[12.0, -7.0, 3.0], [25.0, 0.0, 0.0], [-4.0, 6.0, 0.0]])
    L1, L0 = 0.7 * L2 + 1.0, 0.4 * L2 - 2.0
    dt1, dt0, rho = 0.02, 0.015, 2.0e4
    ctx = p.context()
    ctx.set_neumann(el, fc, ft, types, L2)
    ctx.set_neumann_load_history(L1, L0)
    pr = (ps[2], ps[1], ps[0]) if ps else (None, None, None)
    R, K, st = ctx.assemble_RK_transient(us[2], us[1], us[0], alpha, dt1, dt0, rho, presc=pr)
    assert st.ok(), st.as_dict()
    P, mat = oracle.from_workload(p)
    P.set_neumann(el, fc, types[ft], L2[ft], load_n=L1[ft], load_nm1=L0[ft])
    args = dict(p_np1=ps[2], p_n=ps[1], p_nm1=ps[0]) if ps else {}
    err, Ro, Ko = oracle.assemble_transient(P, mat, us[2], us[1], us[0], alpha, dt1, dt0, rho, **args)
    assert err == 0
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    # the surface terms carry weight
    P0, _ = oracle.from_workload(p)
    _, R0, _ = oracle.assemble_transient(P0, mat, us[2], us[1], us[0], alpha, dt1, dt0, rho, **args)
    assert np.linalg.norm(Ro - R0) > 1e-3 * np.linalg.norm(Ro)
    # the quasi-static calls still use the values at t_{n+1}
    Rq, Kq, st = ctx.assemble_RK(us[2], ps[2] if ps else None)
    P.set_neumann(el, fc, types[ft], L2[ft])
    _, Rqo, Kqo, _ = P.assemble(mat, us[2], ps[2] if ps else None)
    check_R(Rq, Rqo)
    check_K(Kq, Kqo, p.Ap)
    ctx.close()


def _cp_marched(n=3, ngrains=8):
    """A CP context and the oracle after two committed quasi-static load steps:
    the states at t_{n-1} and t_n, the displacements of steps 1, 2 and a
    perturbed step 3 as u_{n-1}, u_n, u_{n+1}."""
    p = wl.cp_p1(n=n, seed=2, ngrains=ngrains)
    ctx = p.context()
    P, mat = oracle.from_workload(p)
    st = p.state.copy()
    hist = []
    for s in (1, 2):
        u = p.displacement(s)
        _, _, status = ctx.assemble_RK(u, dt=p.dt)
        assert status.ok(), status.as_dict()
        ctx.commit_state()
        err, _, _, st = P.assemble(mat, u, state_n=st, dt=p.dt, want_K=False, nthreads=8)
        assert err == 0
        hist.append(st)
    s_nm1, s_n = hist
    assert np.abs(ctx.get_state(2) - s_nm1).max() <= 1e-10 * np.abs(s_nm1).max()
    assert np.abs(ctx.get_state(0) - s_n).max() <= 1e-10 * np.abs(s_n).max()
    rng = np.random.default_rng(5)
    u2 = p.displacement(3) + 2e-4 * rng.uniform(-1, 1, p.ndof) / n
    return p, ctx, P, mat, (p.displacement(1), p.displacement(2), u2), s_nm1, s_n


@pytest.mark.parametrize("alpha", [0.5, 0.3])
def test_cp_transient_matches_oracle(gpu, alpha):
    p, ctx, P, mat, us, s_nm1, s_n = _cp_marched()
    dt1, dt0, rho = p.dt, 0.8 * p.dt, 5.0e4
    R, K, st = ctx.assemble_RK_transient(us[2], us[1], us[0], alpha, dt1, dt0, rho)
    assert st.ok(), st.as_dict()
    err, Ro, Ko, so = oracle.assemble_transient_cp(P, mat, us[2], us[1], us[0], alpha, dt1, dt0, rho, s_nm1, s_n)
    assert err == 0
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    sg = ctx.get_state(1)
    assert np.abs(sg - so).max() <= 1e-10 * np.abs(so).max()
    assert np.abs(so[:, :9] - s_n[:, :9]).max() > 1e-6  # the plastic part moves in this step
    # inertia and the plastic mid points both carry weight
    _, R0, _, _ = oracle.assemble_transient_cp(P, mat, us[2], us[1], us[0], alpha, dt1, dt0, 0.0, s_nm1, s_n)
    assert np.linalg.norm(Ro - R0) > 1e-2 * np.linalg.norm(Ro)
    _, Rf, _, _ = oracle.assemble_transient_cp(P, mat, us[2], us[1], us[0], alpha, dt1, dt0, rho, s_n, s_n)
    assert np.linalg.norm(Ro - Rf) > 1e-3 * np.linalg.norm(Ro)  # the state at t_{n-1} matters
    # residual only: the same R
    R2, K2, st = ctx.assemble_RK_transient(us[2], us[1], us[0], alpha, dt1, dt0, rho, want_K=False)
    assert K2 is None and st.ok()
    check_R(R2, R, 1e-13)
    # the device-buffer entry point: the same R and K
    import torch
    d_us = [torch.from_numpy(np.ascontiguousarray(u)).cuda() for u in (us[2], us[1], us[0])]
    d_R = torch.empty(p.ndof, dtype=torch.float64, device="cuda")
    d_K = torch.empty(p.nnz, dtype=torch.float64, device="cuda")
    ctx.assemble_RK_transient_device([d.data_ptr() for d in d_us], [0, 0, 0], alpha, dt1, dt0, rho, d_R.data_ptr(),
                                     d_K.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    check_R(d_R.cpu().numpy(), R, 1e-13)
    check_K(d_K.cpu().numpy(), K, p.Ap, 1e-13)
    # commit: t_n -> t_{n-1}, t_{n+1} -> t_n
    ctx.commit_state()
    assert np.abs(ctx.get_state(2) - s_n).max() <= 1e-10 * np.abs(s_n).max()
    assert np.abs(ctx.get_state(0) - so).max() <= 1e-10 * np.abs(so).max()
    ctx.close()


def test_cp_transient_with_surface_loads(gpu):
    p, ctx, P, mat, us, s_nm1, s_n = _cp_marched()
    el, fc, ft = [], [], []
    for k, (axis, v) in enumerate([(0, 1.0), (2, 1.0)]):
        e, f = wl.box_faces(p.X, p.conn, axis, v)
        el.append(e)
        fc.append(f)
        ft.append(np.full(len(e), k, dtype=np.int32))
    el, fc, ft = np.concatenate(el), np.concatenate(fc), np.concatenate(ft)
    types = np.array([3, 1])
    L2 = np.array([[40.0, -15.0, 9.0], [60.0, 0.0, 0.0]])
    L1, L0 = 0.7 * L2 + 3.0, 0.4 * L2 - 5.0
    ctx.set_neumann(el, fc, ft, types, L2)
    ctx.set_neumann_load_history(L1, L0)
    alpha, dt1, dt0, rho = 0.4, p.dt, 0.6 * p.dt, 5.0e4
    R, K, st = ctx.assemble_RK_transient(us[2], us[1], us[0], alpha, dt1, dt0, rho)
    assert st.ok(), st.as_dict()
    P.set_neumann(el, fc, types[ft], L2[ft], load_n=L1[ft], load_nm1=L0[ft])
    err, Ro, Ko, so = oracle.assemble_transient_cp(P, mat, us[2], us[1], us[0], alpha, dt1, dt0, rho, s_nm1, s_n)
    assert err == 0
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    P0, _ = oracle.from_workload(p)
    _, R0, _, _ = oracle.assemble_transient_cp(P0, mat, us[2], us[1], us[0], alpha, dt1, dt0, rho, s_nm1, s_n)
    assert np.linalg.norm(Ro - R0) > 1e-3 * np.linalg.norm(Ro)
    ctx.close()
