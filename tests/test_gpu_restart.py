"""Restart files from and into a device context (pgfem_gpu_write_restart /
pgfem_gpu_read_restart) in the reference's per-rank layout.

- crystal plasticity box (the reference's own inputs): after three device load
  steps the written file holds the total nodal displacements of t_{n-1} and
  t_n, F from them, pF and g at t_n (committed state) and t_{n-1} (the state
  before the last commit), tau_n and gamma_dot_n of the state at t_n in the
  reference's system order (pgfem_cp_resolved_shear, pinned to the
  reference's own restart output on the CPU), zero L_n, L_nm1;
  a fresh context that reads it returns the same displacements and state,
  and its next load step equals the original context's (to the rounding of
  the atomic scatter's summation order, 1e-12)
- hyperelastic box patch test: the converged affine stretch writes
  Fn = diag(2, 1, 1) at every point and Fnm1 = I
- J2 quadratic tets past yield: the written file holds the reference's J2
  block (pS = G (I - Cp^-1), ep, gam); a fresh context that reads it holds the
  same state (1e-14) and assembles the same R and K (1e-12)
"""
import numpy as np
import pytest

import pgfem_gpu as pg
from test_oracle_golden import cp_box, cp_box_steps

pytestmark = pytest.mark.gpu

DN4 = np.array([[-1.0, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1]])


def nodal(ids, u, presc):
    out = np.zeros(ids.shape)
    free = ids > 0
    out[free] = u[ids[free] - 1]
    pres = ids < 0
    out[pres] = presc[-ids[pres] - 1]
    return out


def F_linear_tets(X, conn, un):
    dX = np.einsum("eai,ac->eic", X[conn], DN4)
    dU = np.einsum("eai,ac->eic", un[conn], DN4)
    return np.eye(3) + dU @ np.linalg.inv(dX)


def test_crystal_plasticity_restart_round_trip(gpu, tmp_path):
    import torch
    d, X, conn, ids, ndof, Ap, Ai, R_cp, mat = cp_box()
    npres = len(d["defl"])

    def context():
        return pg.Context(X, conn, ids, ndof, Ap, Ai, mat, npres=npres, R_cp=R_cp)

    ctx = context()
    s = pg.Solver(Ap, Ai, ndof, maxit=5000, kdim=100, tol=1e-13)
    du = torch.zeros(ndof, dtype=torch.float64, device="cuda")
    steps = list(cp_box_steps(d))
    hist = []
    for dt, presc in steps[:3]:
        prev_state = ctx.get_state(0)
        info = s.newton_step(ctx, du.data_ptr(), torch.from_numpy(presc).cuda().data_ptr(), dt=dt, iter_max=20,
                             nor_min=1e-10)
        assert info.converged
        ctx.commit_state()
        hist.append((du.cpu().numpy(), presc))
    (u1, p1), (u2, p2) = hist[-2], hist[-1]
    assert np.array_equal(ctx.get_state(2), prev_state)  # the context's state at t_{n-1}
    path = str(tmp_path / "box_0_3.res")
    pg.write_restart(ctx, path, u1, u2, p1, p2, state_nm1=prev_state)
    a, b, blocks = pg.restart_parse(path, pg.MODEL_CP, X.shape[0], conn.shape[0], 1)
    assert np.array_equal(a, nodal(ids, u1, p1)) and np.array_equal(b, nodal(ids, u2, p2))
    st = ctx.get_state(0)
    blk = blocks[:, 0]
    assert np.abs(blk[:, 0:9] - F_linear_tets(X, conn, b).reshape(-1, 9)).max() <= 1e-14
    assert np.abs(blk[:, 9:18] - F_linear_tets(X, conn, a).reshape(-1, 9)).max() <= 1e-14
    assert np.array_equal(blk[:, 18:27], st[:, :9]) and np.array_equal(blk[:, 60], st[:, 9])
    assert np.array_equal(blk[:, 27:36], prev_state[:, :9]) and np.array_equal(blk[:, 61], prev_state[:, 9])
    tau, gdot = pg.cp_resolved_shear(mat, blk[:, 0:9], st[:, :9], st[:, 9], R_cp)
    assert np.array_equal(blk[:, 36:48], tau) and np.array_equal(blk[:, 48:60], gdot)
    assert np.abs(tau).max() > 1.0 and not blk[:, 62:64].any()
    # a fresh context resumes from the file
    ctx2 = context()
    r1, r2 = pg.read_restart(ctx2, path)
    assert np.array_equal(r1, u1) and np.array_equal(r2, u2)
    assert np.array_equal(ctx2.get_state(0), st)
    assert np.array_equal(ctx2.get_state(2), prev_state)  # pF_{n-1}, g_{n-1} from the file
    dt, presc = steps[3]
    dp = torch.from_numpy(presc).cuda()
    du2 = torch.from_numpy(r2.copy()).cuda()
    i1 = s.newton_step(ctx, du.data_ptr(), dp.data_ptr(), dt=dt, iter_max=20, nor_min=1e-10)
    i2 = s.newton_step(ctx2, du2.data_ptr(), dp.data_ptr(), dt=dt, iter_max=20, nor_min=1e-10)
    assert i1.converged and i2.converged and len(i1.history()) == len(i2.history())
    for h1, h2 in zip(i1.history(), i2.history()):  # rounding-level norms at convergence differ
        assert abs(h1 - h2) <= 1e-6 * h2 if h2 > 1e-8 else h1 <= 1e-10
    assert torch.allclose(du, du2, rtol=0, atol=1e-12 * float(du.abs().max()))
    s1, s2 = ctx.get_state(1), ctx2.get_state(1)
    assert np.abs(s1 - s2).max() <= 1e-12 * np.abs(s1).max()


def test_hyperelastic_restart_holds_the_deformation(gpu, tmp_path):
    import torch
    from test_gpu_box_fixture import box
    d, X, conn, ids, ndof, Ap, Ai, mat, defl = box(tmp_path, "LT")
    ctx = pg.Context(X, conn, ids, ndof, Ap, Ai, mat, npres=len(defl))
    s = pg.Solver(Ap, Ai, ndof, maxit=2000, kdim=100, tol=1e-13)
    du = torch.zeros(ndof, dtype=torch.float64, device="cuda")
    info = s.newton_step(ctx, du.data_ptr(), torch.from_numpy(defl.copy()).cuda().data_ptr(), iter_max=30,
                         nor_min=1e-13)
    assert info.converged
    u = du.cpu().numpy()
    path = str(tmp_path / "box_LT_0_1.res")
    pg.write_restart(ctx, path, np.zeros(ndof), u, np.zeros_like(defl), defl)
    _, b, blocks = pg.restart_parse(path, pg.MODEL_HE, X.shape[0], conn.shape[0], 1)
    assert np.abs(blocks[:, 0, 0:9] - np.diag([1.0 + defl[0], 1.0, 1.0]).ravel()).max() <= 1e-10
    assert np.abs(blocks[:, 0, 9:18] - np.eye(3).ravel()).max() == 0.0
    r1, r2 = pg.read_restart(ctx, path)
    assert not r1.any() and np.array_equal(r2, u)


def test_j2_restart_round_trip(gpu, tmp_path):
    import workloads as wl
    p = wl.j2_p2(n=2, seed=1, stretch=6e-3, perturb=2e-2)
    ctx = p.context()
    s0 = ctx.get_state(0)
    R, K, st = ctx.assemble_RK(p.u)
    assert st.ok()
    ctx.commit_state()
    s1 = ctx.get_state(0)
    assert (s1[:, 9] > 0).any()
    path = str(tmp_path / "j2_0_1.res")
    zero = np.zeros(p.ndof)
    pg.write_restart(ctx, path, zero, p.u, state_nm1=s0)
    nn, ne = p.X.shape[0], p.conn.shape[0]
    a, b, blocks = pg.restart_parse(path, pg.MODEL_J2, nn, ne, 4)
    G = 200e3 / (2 * 1.3)
    blk = blocks.reshape(-1, 47)
    assert np.allclose(blk[:, 9:18], G * (np.eye(3).ravel() - s1[:, :9]), rtol=0, atol=1e-9 * G)
    assert np.array_equal(blk[:, 42], s1[:, 9]) and not blk[:, 43].any()
    assert np.allclose(blk[:, 44], np.sqrt(1.5) * s1[:, 9], rtol=1e-14, atol=0)
    assert not blk[:, [36, 37, 38, 39, 40, 41, 45, 46]].any()
    ctx2 = p.context()
    r1, r2 = pg.read_restart(ctx2, path)
    assert not r1.any() and np.allclose(r2, p.u, rtol=0, atol=0)
    assert np.abs(ctx2.get_state(0) - s1).max() <= 1e-14 * max(1.0, np.abs(s1).max())
    u3 = p.u * 1.1
    Ra, Ka, _ = ctx.assemble_RK(u3)
    Rb, Kb, _ = ctx2.assemble_RK(u3)
    assert np.linalg.norm(Rb - Ra) <= 1e-12 * np.linalg.norm(Ra)
    assert np.linalg.norm(Kb - Ka) <= 1e-12 * np.linalg.norm(Ka)
