"""GPU crystal plasticity (config 3 family) against the CPU oracle, through the C ABI:
R, K and the state over several load steps of the tension ramp, the local
Newton iteration counts, and the warm-started solve (same answer, fewer
iterations).  Tolerance: 1e-10 relative (norm-wise; K per entry row-scaled)."""
import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
import workloads as wl
from test_gpu_parity import check_K, check_R
from test_oracle_selfcheck import cp_guess_from_slip, p1_deformation_gradients

pytestmark = pytest.mark.gpu
TOL = 1e-10


def test_cp_load_steps_match_oracle(gpu):
    p = wl.cp_p1(n=4, seed=2, ngrains=8)
    ctx = p.context()
    P, mat = oracle.from_workload(p)
    st = p.state.copy()
    for s in range(1, 6):
        u = p.displacement(s)
        R, K, status = ctx.assemble_RK(u, dt=p.dt)
        assert status.ok(), status.as_dict()
        err, Ro, Ko, so = P.assemble(mat, u, state_n=st, dt=p.dt, nthreads=8)
        assert err == 0
        check_R(R, Ro)
        check_K(K, Ko, p.Ap)
        sg = ctx.get_state(1)
        assert np.abs(sg - so).max() <= TOL * np.abs(so).max()
        ctx.commit_state()
        st = so


def test_cp_iterations_match_oracle_and_are_uneven(gpu):
    p = wl.cp_p1(n=4, seed=2, ngrains=8)
    ctx = p.context()
    mat = oracle.from_pg_material(p.mat)
    st = p.state.copy()
    for s in range(1, 4):
        u = p.displacement(s)
        ctx.assemble_RK(u, dt=p.dt)
        it, dg = ctx.cp_iterations(want_slip=True)
        _, so, ito, dgo, cv = oracle.cp_update_batch(mat, p1_deformation_gradients(p, u), st, p.dt, p.R_cp)
        assert cv.all()
        assert np.mean(np.abs(it - ito) <= 1) > 0.99
        assert np.abs(dg - dgo).max() <= 1e-9 * max(np.abs(dgo).max(), 1e-30)
        ctx.commit_state()
        st = so
    assert it.max() - it.min() >= 3


def test_cp_warm_start_same_answer_fewer_iterations(gpu):
    p = wl.cp_p1(n=4, seed=2, ngrains=8)
    ctx = p.context()
    mat = oracle.from_pg_material(p.mat)
    ctx.assemble_RK(p.displacement(1), dt=p.dt)
    ctx.commit_state()
    st_n = ctx.get_state(0)
    u = p.displacement(2)
    R0, K0, _ = ctx.assemble_RK(u, dt=p.dt)
    it0, dg = ctx.cp_iterations(want_slip=True)
    s0 = ctx.get_state(1)
    guess = cp_guess_from_slip(p, dg)
    guess[:, 9] = s0[:, 9]
    ctx.set_cp_guess(guess)
    R1, K1, st = ctx.assemble_RK(u, dt=p.dt)
    it1 = ctx.cp_iterations()
    s1 = ctx.get_state(1)
    assert st.ok()
    assert it1.max() <= 2 and it1.mean() < it0.mean()
    # both solves meet the 1e-10 local residual; they agree to what that implies
    check_R(R1, R0, 1e-7)
    assert np.abs(s1 - s0).max() <= 1e-9 * np.abs(s0).max()
    # the warm-started GPU solve equals the oracle's solve from the same guess
    _, so, ito, _, cv = oracle.cp_update_batch(mat, p1_deformation_gradients(p, u), st_n, p.dt, p.R_cp,
                                               M0=guess[:, :9], g_guess=guess[:, 9])
    assert cv.all()
    assert np.abs(s1 - so).max() <= TOL * np.abs(so).max()
    ctx.set_cp_guess(None)


def test_cp_element_level_entry_points(gpu):
    """stiffmatel_fd / resid_on_elem for crystal plasticity (the reference's
    stiffness_el_constitutive_model_1f with compute_dMdu,
    src/constitutive_model.cc:2545-2676, src/plasticity_model.cc:867-881): the
    dense element blocks of listed elements (every element DOF, idx_K order)
    equal the oracle's element at the same state and load step (1e-10), and
    assemble into the CSR K of the assembly call."""
    p = wl.cp_p1(n=4, seed=2, ngrains=8)
    ctx = p.context()
    P, mat = oracle.from_workload(p)
    ctx.assemble_RK(p.displacement(1), dt=p.dt)
    ctx.commit_state()
    st_n = ctx.get_state(0)
    u = p.displacement(2)
    elems = np.array([0, 5, 77, 200, p.ne - 1])
    lk, fe, st = ctx.stiffmatel_fd(elems, u, dt=p.dt)
    fe2, st2 = ctx.resid_on_elem(elems, u, dt=p.dt)
    assert st.ok() and st2.ok()
    for k, e in enumerate(elems):
        ue = np.zeros(12)
        for a in range(4):
            for j in range(3):
                i = p.ids[p.conn[e, a], j]
                ue[a * 3 + j] = u[i - 1] if i > 0 else 0.0
        err, feo, lko, _ = P.element(mat, e, ue, st_n[e], dt=p.dt)
        assert err == 0
        assert np.linalg.norm(fe[k] - feo) <= TOL * np.linalg.norm(feo)
        assert np.linalg.norm(fe2[k] - feo) <= TOL * np.linalg.norm(feo)
        assert np.linalg.norm(lk[k].ravel() - lko.ravel()) <= TOL * np.linalg.norm(lko)
    # the blocks of all elements assemble into the assembly's K
    allel = np.arange(p.ne)
    lka, _, _ = ctx.stiffmatel_fd(allel, u, dt=p.dt)
    R, K, _ = ctx.assemble_RK(u, dt=p.dt)
    Kd = np.zeros((p.ndof, p.ndof))
    for e in allel:
        idx = np.array([p.ids[p.conn[e, a], j] for a in range(4) for j in range(3)])
        m = idx > 0
        Kd[np.ix_(idx[m] - 1, idx[m] - 1)] += lka[e].reshape(12, 12)[np.ix_(m, m)]
    rows = np.repeat(np.arange(p.ndof), np.diff(p.Ap))
    assert np.abs(Kd[rows, p.Ai] - K).max() <= 1e-10 * np.abs(K).max()
