"""The benchmark configurations at their stated sizes on the GPU, checked
against the oracle (the whole-mesh oracle would take too long, so samples).

- Crystal plasticity, 48^3 cells x 6 linear tets (663,552 elements), 512
  grains: GPU load steps 1..9 committed, then step 10: the assembled R rows and
  K rows of 100 seeded nodes (every element touching them, >= 2,000 elements,
  run by the oracle from the GPU's state at step 9) and the state of those
  elements equal the oracle (1e-10).
- The learned warm start on the same mesh and step: the warm-started solve
  and the plain solve reach the same state within the local tolerance, and on
  2,000 seeded points the GPU's warm-then-cold Newton equals the oracle's from
  the same network guesses (1e-10).
- The FE2 batch of 256 periodic RVEs of 8^3..24^3 cells (8.9 M elements) in
  one assembly: the smallest, the largest and 6 seeded RVEs each equal the
  oracle run on that RVE alone (R, K block, state; 1e-10).
"""
import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
import surrogate as sg
import workloads as wl
from test_gpu_parity import TOL, check_K, check_R
from test_oracle_selfcheck import p1_deformation_gradients

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cp48():
    p = wl.cp_p1(n=48, seed=2, ngrains=512)
    ctx = p.context()
    for s in range(1, 10):
        _, st = ctx.assemble_R(p.displacement(s), dt=p.dt)
        assert st.ok(), (s, st.as_dict())
        ctx.commit_state()
    return p, ctx, ctx.get_state(0)


def _sample(p, nodes_n=100, seed=10):
    rng = np.random.default_rng(seed)
    nodes = np.sort(rng.choice(p.X.shape[0], nodes_n, replace=False))
    elems = np.nonzero(np.isin(p.conn, nodes).any(axis=1))[0]
    return nodes, elems


def test_config3_crystal_plasticity_full_size_sampled_rows(gpu, cp48):
    p, ctx, st9 = cp48
    u = p.displacement(10)
    R, K, st = ctx.assemble_RK(u, dt=p.dt)
    assert st.ok(), st.as_dict()
    s10 = ctx.get_state(1)
    nodes, elems = _sample(p)
    assert len(elems) >= 2000
    P, mat = oracle.from_workload(p)
    rows = np.sort(p.ids[nodes].ravel() - 1)
    pos = {r: i for i, r in enumerate(rows)}
    Ro = np.zeros(len(rows))
    Krows = {r: {} for r in rows}
    for e in elems:
        idx = p.ids[p.conn[e]].ravel() - 1
        err, fe, lk, snp1 = P.element(mat, e, u[idx], st9[e], dt=p.dt)
        assert err == 0
        assert np.abs(s10[e] - snp1).max() <= TOL * np.abs(snp1).max()
        for a, r in enumerate(idx):
            if r in pos:
                Ro[pos[r]] += fe[a]
                kr = Krows[r]
                for b, c in enumerate(idx):
                    kr[c] = kr.get(c, 0.0) + lk[a, b]
    check_R(R[rows], Ro)
    for r in rows:
        cols = p.Ai[p.Ap[r]:p.Ap[r + 1]]
        assert sorted(Krows[r]) == cols.tolist()  # every element of the row was run
        ko = np.array([Krows[r][c] for c in cols])
        kg = K[p.Ap[r]:p.Ap[r + 1]]
        assert np.abs(kg - ko).max() <= TOL * np.abs(ko).max()


def test_config4_warm_start_full_size(gpu, cp48):
    import torch
    p, ctx, st9 = cp48
    u = p.displacement(10)
    ctx.reset_state()
    ctx.set_cp_surrogate(None)
    R0, st0 = ctx.assemble_R(u, dt=p.dt)
    it0 = ctx.cp_iterations()
    s0 = ctx.get_state(1)
    # a network trained on the GPU from plain-Newton pairs of smaller meshes
    x, t, _ = sg.generate_pairs(n=12, ngrains=64)
    net, hist, _ = sg.train(x, t, seed=1, epochs=15, batch=4096, lr=3e-3, lr_min=3e-5)
    del x, t
    ctx.reset_state()
    ctx.set_cp_warm_limit(8)
    ctx.set_cp_surrogate(net)
    R1, st1 = ctx.assemble_R(u, dt=p.dt)
    it1 = ctx.cp_iterations()
    s1 = ctx.get_state(1)
    assert st0.ok() and st1.ok()
    assert it1.mean() < it0.mean(), (it0.mean(), it1.mean())
    # same converged answer (both meet the 1e-10 local residual)
    assert np.abs(s1 - s0).max() <= 1e-9 * np.abs(s0).max()
    check_R(R1, R0, 1e-7)
    # the GPU's warm-then-cold Newton equals the oracle's from the same guesses
    xg = torch.empty((p.ne, 34), dtype=torch.float32, device="cuda")
    tg = torch.empty((p.ne, 12), dtype=torch.float32, device="cuda")
    ctx.cp_training_pairs(xg.data_ptr(), tg.data_ptr())
    rng = np.random.default_rng(4)
    pts = np.sort(rng.choice(p.ne, 2000, replace=False))
    y = net.predict(xg.cpu().numpy()[pts])
    guess = sg.guess_from_prediction(p, y, st9, points=pts)
    mat = oracle.from_pg_material(p.mat)
    F = p1_deformation_gradients(p, u)[pts]
    bad, so, ito, _, cv, fbo = oracle.cp_update_batch(mat, F, st9[pts], p.dt, p.R_cp[pts], M0=guess[:, :9],
                                                      g_guess=guess[:, 9], warm_k=8, want_fallback=True)
    assert bad == 0 and cv.all()
    assert np.abs(s1[pts] - so).max() <= TOL * np.abs(so).max()
    assert np.mean(np.abs(it1[pts] - ito) <= 1) > 0.99
    ctx.set_cp_surrogate(None)


def test_config5_rve_batch_full_size(gpu):
    p = wl.rve_batch()  # 256 RVEs, 8..24 cells per side
    assert len(p.n_r) == 256 and p.n_r.min() == 8 and p.n_r.max() == 24
    ctx = p.context()
    R, K, st = ctx.assemble_RK(p.u)
    assert st.ok(), st.as_dict()
    S = ctx.get_state(1)
    rng = np.random.default_rng(6)
    pick = {int(np.argmin(p.n_r)), int(np.argmax(p.n_r))} | set(rng.choice(256, 6, replace=False).tolist())
    assert len(pick) >= 7
    for r in sorted(pick):
        q = p.rve(r)
        Po, mat = oracle.from_workload(q)
        err, Ro, Ko, so = Po.assemble(mat, q.u, state_n=q.state, nthreads=8)
        assert err == 0
        d0, d1 = p.dof_off[r], p.dof_off[r + 1]
        check_R(R[d0:d1], Ro)
        check_K(K[p.Ap[d0]:p.Ap[d1]], Ko, q.Ap)
        e0, e1 = p.elem_off[r], p.elem_off[r + 1]
        assert np.abs(S[e0:e1] - so).max() <= TOL * np.abs(so).max()
