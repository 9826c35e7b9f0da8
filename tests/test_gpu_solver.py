"""Device linear solve and Newton-Raphson load step (the consumer of K),
through the C ABI:

- pgfem_gpu_spmv equals scipy's CSR product on the same values (summation
  order differs: 1e-13 relative per entry of the largest |y|);
- pgfem_gpu_solve (GMRES with a short restart length, so that it restarts,
  and BiCGSTAB; diagonal scaling or none) on an assembled stiffness reaches
  its relative residual tolerance 1e-12 and equals scipy's sparse direct
  solve to 1e-8 relative; a second call on the same solver object gives the
  bit-identical answer; an exact initial guess takes no iteration;
- pgfem_gpu_newton_step on tension problems (neo-Hookean linear tets from
  rest, J2 quadratic tets past yield from the linear predictor) takes the same number of Newton iterations as the
  CPU oracle's Newton (oracle.newton_step: oracle assembly + sparse direct
  solve, src/Newton_Raphson.cc loop), with the same residual history where
  it is above 1e-8, and converges to the same displacement and state (1e-8);
  the J2 quadratic-tet case on 6^3 cells is one where BiCGSTAB with diagonal
  scaling breaks down, and GMRES (the reference's default solver) does not."""
import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
import workloads as wl

pytestmark = pytest.mark.gpu


def csr(p, K):
    from scipy.sparse import csr_matrix
    return csr_matrix((K, p.Ai, p.Ap), shape=(p.ndof, p.ndof))


def assembled_K(p):
    ctx = p.context()
    _, K, st = ctx.assemble_RK(p.u, u_presc=p.u_presc)
    assert st.ok()
    return ctx, K


def test_spmv_matches_scipy(gpu):
    import torch
    p = wl.tension(n=6, nne=4, model="he")
    rng = np.random.default_rng(1)
    K = rng.normal(size=p.nnz)
    x = rng.normal(size=p.ndof)
    s = pg.Solver(p.Ap, p.Ai, p.ndof)
    dK, dx = torch.from_numpy(K).cuda(), torch.from_numpy(x).cuda()
    dy = torch.empty(p.ndof, dtype=torch.float64, device="cuda")
    s.spmv(dK.data_ptr(), dx.data_ptr(), dy.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    y = dy.cpu().numpy()
    yo = csr(p, K) @ x
    assert np.abs(y - yo).max() <= 1e-13 * np.abs(yo).max()


@pytest.mark.parametrize("method", [pg.SOLVER_GMRES, pg.SOLVER_BCG_STAB])
@pytest.mark.parametrize("precond", [pg.PRECOND_DIAG_SCALE, pg.PRECOND_NONE])
def test_krylov_matches_direct_solve(gpu, method, precond):
    import torch
    from scipy.sparse.linalg import spsolve
    p = wl.tension(n=6, nne=4, model="he", stretch=0.01)
    ctx, K = assembled_K(p)
    rng = np.random.default_rng(2)
    b = rng.normal(size=p.ndof)
    xo = spsolve(csr(p, K).tocsc(), b)
    s = pg.Solver(p.Ap, p.Ai, p.ndof, solver=method, precond=precond, maxit=20000, kdim=40, tol=1e-12)
    dK, db = torch.from_numpy(K).cuda(), torch.from_numpy(b).cuda()
    for call in range(2):  # the second call reuses the work vectors
        dx = torch.zeros(p.ndof, dtype=torch.float64, device="cuda")
        info = s.solve(dK.data_ptr(), db.data_ptr(), dx.data_ptr(), torch.cuda.current_stream().cuda_stream)
        assert info.converged and not info.breakdown and info.iters > 0, (call, info.iters, info.res_norm)
        assert info.res_norm <= (1e-11 if method == pg.SOLVER_GMRES else 1e-12)
        x = dx.cpu().numpy()
        assert np.linalg.norm(b - csr(p, K) @ x) <= 1e-11 * np.linalg.norm(b)
        assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo), call
        if method == pg.SOLVER_GMRES:
            assert info.iters > 40  # at least one restart
        if call == 0:
            it0, x0 = info.iters, x
        else:
            assert info.iters == it0 and np.array_equal(x, x0)  # fixed-order reductions
    # exact initial guess: converged before the first iteration
    dx = torch.from_numpy(xo.copy()).cuda()
    info = s.solve(dK.data_ptr(), db.data_ptr(), dx.data_ptr())
    assert info.converged and info.iters == 0


@pytest.mark.parametrize("case", [("he", 4, 4, 0.02), ("j2", 10, 2, 0.003), ("j2", 10, 6, 0.003)])
def test_newton_step_matches_oracle(gpu, case):
    import torch
    model, nne, n, stretch = case
    p = wl.tension(n=n, nne=nne, model=model, stretch=stretch, predictor=(model == "j2"))
    P, mat = oracle.from_workload(p)
    uo, ho, ok, so = oracle.newton_step(P, mat, p.u, p.u_presc, state_n=p.state, iter_max=15, nor_min=1e-10)
    assert ok
    ctx = p.context()
    s = pg.Solver(p.Ap, p.Ai, p.ndof, maxit=20000, kdim=100, tol=1e-12)
    du = torch.from_numpy(p.u.copy()).cuda()
    dp = torch.from_numpy(p.u_presc.copy()).cuda()
    info = s.newton_step(ctx, du.data_ptr(), dp.data_ptr(), iter_max=15, nor_min=1e-10)
    assert info.converged and not info.lin_failed and info.elem_failures == 0
    h = info.history()
    assert len(h) == len(ho), (h, ho)
    for a, b in zip(h, ho):
        if b > 1e-8:
            assert abs(a - b) <= 1e-6 * b, (h, ho)
    u = du.cpu().numpy()
    assert np.linalg.norm(u - uo) <= 1e-8 * np.linalg.norm(uo)
    if so is not None:
        sg = ctx.get_state(1)
        assert np.abs(sg - so).max() <= 1e-8 * np.abs(so).max()
        assert (so[:, 9] > 0).mean() > 0.5  # the step yields
    assert info.lin_iters > info.iters
