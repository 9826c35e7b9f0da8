"""Learned warm start of the CP local Newton, through the C ABI:

- the device features equal a numpy restatement (F F_n^-1 - I and pF_n - I in
  the lattice frame, slip resistances, lattice quaternion) and the targets
  equal the converged slip;
- with a network attached, every point still meets the 1e-10 local residual
  and the result equals the CPU oracle started from the same guess, including
  the cold-start fallback after warm_k iterations (a deliberately poor,
  untrained network exercises the fallback);
- a network trained on the GPU from plain-Newton pairs of other seeds needs
  fewer Newton iterations than the cold start on an unseen mesh and load step,
  for the same converged answer.
"""
import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
import surrogate as sg
import workloads as wl
from test_gpu_parity import check_R
from test_oracle_selfcheck import p1_deformation_gradients

pytestmark = pytest.mark.gpu


def quat_np(R):
    """Shepperd's rotation-matrix -> quaternion (w >= 0), rows of R (n x 9)."""
    out = np.zeros((R.shape[0], 4))
    for k, r in enumerate(R.reshape(-1, 3, 3)):
        tr = np.trace(r)
        if tr > 0:
            s = 2 * np.sqrt(tr + 1)
            q = [0.25 * s, (r[2, 1] - r[1, 2]) / s, (r[0, 2] - r[2, 0]) / s, (r[1, 0] - r[0, 1]) / s]
        elif r[0, 0] > r[1, 1] and r[0, 0] > r[2, 2]:
            s = 2 * np.sqrt(1 + r[0, 0] - r[1, 1] - r[2, 2])
            q = [(r[2, 1] - r[1, 2]) / s, 0.25 * s, (r[0, 1] + r[1, 0]) / s, (r[0, 2] + r[2, 0]) / s]
        elif r[1, 1] > r[2, 2]:
            s = 2 * np.sqrt(1 + r[1, 1] - r[0, 0] - r[2, 2])
            q = [(r[0, 2] - r[2, 0]) / s, (r[0, 1] + r[1, 0]) / s, 0.25 * s, (r[1, 2] + r[2, 1]) / s]
        else:
            s = 2 * np.sqrt(1 + r[2, 2] - r[0, 0] - r[1, 1])
            q = [(r[1, 0] - r[0, 1]) / s, (r[0, 2] + r[2, 0]) / s, (r[1, 2] + r[2, 1]) / s, 0.25 * s]
        q = np.array(q)
        out[k] = -q if q[0] < 0 else q
    return out


def features_np(p, u, u_prev, state_n):
    F = p1_deformation_gradients(p, u).reshape(-1, 3, 3)
    Fn = p1_deformation_gradients(p, u_prev).reshape(-1, 3, 3)
    R = p.R_cp.reshape(-1, 3, 3)
    Rt = np.transpose(R, (0, 2, 1))
    dF = (Rt @ F @ np.linalg.inv(Fn) @ R).reshape(-1, 9) - np.eye(3).ravel()
    pF = (Rt @ state_n[:, :9].reshape(-1, 3, 3) @ R).reshape(-1, 9) - np.eye(3).ravel()
    g = np.repeat(state_n[:, 9:10], 12, axis=1)
    return np.concatenate([dF, pF, g, quat_np(p.R_cp)], axis=1)


def test_features_and_targets_match_numpy(gpu):
    import torch
    p = wl.cp_p1(n=4, seed=2, ngrains=8)
    ctx = p.context()
    ctx.assemble_R(p.displacement(1), dt=p.dt)
    ctx.commit_state()
    st_n = ctx.get_state(0)
    ctx.assemble_R(p.displacement(2), dt=p.dt)
    x = torch.empty((p.ne, 34), dtype=torch.float32, device="cuda")
    t = torch.empty((p.ne, 12), dtype=torch.float32, device="cuda")
    ctx.cp_training_pairs(x.data_ptr(), t.data_ptr())
    xo = features_np(p, p.displacement(2), p.displacement(1), st_n)
    xg = x.cpu().numpy()
    for lo, hi in ((0, 9), (9, 18), (18, 30), (30, 34)):
        scale = max(np.abs(xo[:, lo:hi]).max(), 1e-30)
        assert np.abs(xg[:, lo:hi] - xo[:, lo:hi]).max() <= 1e-6 * scale, (lo, hi)
    _, dg = ctx.cp_iterations(want_slip=True)
    assert np.array_equal(t.cpu().numpy(), dg.astype(np.float32))


def _ramp_state(p, ctx, steps):
    for s in range(1, steps + 1):
        ctx.assemble_R(p.displacement(s), dt=p.dt)
        ctx.commit_state()


def test_attached_network_matches_oracle_with_fallback(gpu):
    """An untrained network with a deliberately large output scale: poor guesses,
    many cold restarts after warm_k = 3 iterations; GPU and oracle agree."""
    import torch
    p = wl.cp_p1(n=6, seed=5, ngrains=16)
    ctx = p.context()
    _ramp_state(p, ctx, 4)
    st_n = ctx.get_state(0)
    u = p.displacement(5)
    net = pg.Mlp(seed=9)
    x0 = features_np(p, u, p.displacement(4), st_n).astype(np.float32)
    net.set_scaling(x0.mean(0), x0.std(0) + 1e-3, np.full(12, 4e-4, np.float32))
    ctx.set_cp_warm_limit(3)
    ctx.set_cp_surrogate(net)
    R, st = ctx.assemble_R(u, dt=p.dt)
    assert st.ok(), st.as_dict()
    it, dg = ctx.cp_iterations(want_slip=True)
    fb = ctx.cp_fallbacks()
    s_gpu = ctx.get_state(1)
    # the same guess on the host: device features -> network -> numpy guess
    x = torch.empty((p.ne, 34), dtype=torch.float32, device="cuda")
    t = torch.empty((p.ne, 12), dtype=torch.float32, device="cuda")
    ctx.cp_training_pairs(x.data_ptr(), t.data_ptr())
    y = net.predict(x.cpu().numpy())
    guess = sg.guess_from_prediction(p, y, st_n)
    mat = oracle.from_pg_material(p.mat)
    bad, so, ito, dgo, cv, fbo = oracle.cp_update_batch(mat, p1_deformation_gradients(p, u), st_n, p.dt, p.R_cp,
                                                        M0=guess[:, :9], g_guess=guess[:, 9], warm_k=3,
                                                        want_fallback=True)
    assert bad == 0 and cv.all()
    assert fb >= 0.05 * p.ne and abs(fb - int(fbo.sum())) <= 0.01 * p.ne + 1, (fb, fbo.sum())
    assert np.abs(s_gpu - so).max() <= 1e-10 * np.abs(so).max()
    assert np.abs(dg - dgo).max() <= 1e-9 * np.abs(dgo).max()
    assert np.mean(np.abs(it - ito) <= 1) > 0.99
    # same converged answer as the plain solve
    ctx.set_cp_surrogate(None)
    ctx.reset_state()
    R0, st0 = ctx.assemble_R(u, dt=p.dt)
    s0 = ctx.get_state(1)
    check_R(R, R0, 1e-7)
    assert np.abs(s_gpu - s0).max() <= 1e-9 * np.abs(s0).max()


def test_trained_network_saves_newton_iterations(gpu):
    x, t, info = sg.generate_pairs(n=8, ngrains=32)
    assert info["pairs"] >= 0.99 * 20 * 6 * 8 ** 3
    net, hist, _ = sg.train(x, t, seed=1, epochs=40, batch=1024, lr=3e-3, lr_min=3e-5)
    assert hist[-1] < 0.2 * hist[0], hist
    # unseen mesh (seed 2) and load step 10, cold versus warm
    p = wl.cp_p1(n=8, seed=2, ngrains=32)
    ctx = p.context()
    _ramp_state(p, ctx, 9)
    u = p.displacement(10)
    R0, st0 = ctx.assemble_R(u, dt=p.dt)
    it0 = ctx.cp_iterations()
    s0 = ctx.get_state(1)
    ctx.reset_state()
    ctx.set_cp_warm_limit(8)
    ctx.set_cp_surrogate(net)
    R1, st1 = ctx.assemble_R(u, dt=p.dt)
    it1 = ctx.cp_iterations()
    s1 = ctx.get_state(1)
    assert st0.ok() and st1.ok()
    assert it1.mean() < 0.6 * it0.mean(), (it0.mean(), it1.mean(), ctx.cp_fallbacks())
    check_R(R1, R0, 1e-7)
    assert np.abs(s1 - s0).max() <= 1e-9 * np.abs(s0).max()
