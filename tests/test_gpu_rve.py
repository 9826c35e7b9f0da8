"""FE2 RVE batch on the GPU, through the C ABI: every RVE of a batch of uneven
periodic cells, assembled in one launch with its own macro deformation,
equals the oracle run on that RVE alone (R, K block, state; 1e-10); every
launch schedule (elements per block x work-stealing size) gives the same
result; the captured CUDA graph replays it; the autotuner picks a valid
schedule."""
import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
import workloads as wl
from test_gpu_parity import TOL, check_K, check_R

pytestmark = pytest.mark.gpu


def _oracle_rve(q):
    P, mat = oracle.from_workload(q)
    err, R, K, s = P.assemble(mat, q.u, state_n=q.state, nthreads=8)
    assert err == 0
    return R, K, s


@pytest.fixture(scope="module")
def batch():
    return wl.rve_batch(nrve=9, nmin=3, nmax=7, seed=5)


def test_every_rve_matches_its_own_oracle(gpu, batch):
    p = batch
    ctx = p.context()
    R, K, st = ctx.assemble_RK(p.u)
    assert st.ok(), st.as_dict()
    S = ctx.get_state(1)
    for r in range(len(p.n_r)):
        q = p.rve(r)
        Ro, Ko, so = _oracle_rve(q)
        d0, d1 = p.dof_off[r], p.dof_off[r + 1]
        check_R(R[d0:d1], Ro)
        check_K(K[p.Ap[d0]:p.Ap[d1]], Ko, q.Ap)
        e0, e1 = p.elem_off[r], p.elem_off[r + 1]
        assert np.abs(S[e0:e1] - so).max() <= TOL * np.abs(so).max()
        assert (so[:, 9] > 0).mean() > 0.5  # macro strains of a few percent yield


def test_schedules_and_graph_replay_agree(gpu, batch):
    import torch
    p = batch
    ctx = p.context()
    R0, K0, _ = ctx.assemble_RK(p.u)
    for epb in (16, 32, 64):
        for grab in (0, 1, 4):
            ctx.set_schedule(epb, grab)
            assert ctx.schedule() == (epb, grab)
            R, K, st = ctx.assemble_RK(p.u)
            assert st.ok()
            check_R(R, R0, 1e-13)
            check_K(K, K0, p.Ap, 1e-13)
    d_u = torch.from_numpy(p.u).cuda()
    d_R = torch.empty(p.ndof, dtype=torch.float64, device="cuda")
    d_K = torch.empty(p.nnz, dtype=torch.float64, device="cuda")
    epb, grab, ms = ctx.autotune(d_u.data_ptr(), None, d_R.data_ptr(), d_K.data_ptr(), reps=2)
    assert epb in (16, 32, 64) and grab in (1, 2, 4, 8, 16) and ms > 0
    assert ctx.schedule() == (epb, grab)
    g = ctx.graph_create(d_u.data_ptr(), None, d_R.data_ptr(), d_K.data_ptr())
    d_R.fill_(np.nan)
    d_K.fill_(np.nan)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        g.launch(stream)
    torch.cuda.synchronize()
    check_R(d_R.cpu().numpy(), R0, 1e-13)
    check_K(d_K.cpu().numpy(), K0, p.Ap, 1e-13)
    # the graph reads d_u at replay time
    d_u.mul_(0.5)
    g.launch(stream)
    torch.cuda.synchronize()
    R5, K5, _ = ctx.assemble_RK(p.u * 0.5)
    check_R(d_R.cpu().numpy(), R5, 1e-13)
    g.destroy()
    with pytest.raises(pg.PgfemError):
        ctx.set_schedule(24, 1)


def test_quadratic_tet_groups_use_their_own_macro_deformation(gpu):
    """Mesh groups on a quadratic-tet context: each RVE of the batch sees its
    own macro F through the default two-kernel path (the point kernel applies
    the group's F0); every RVE equals the oracle run on it alone."""
    p = wl.rve_batch(nrve=3, nmin=2, nmax=3, seed=11, nne=10)
    assert len(set(map(tuple, np.round(p.F0s, 12)))) == 3
    ctx = p.context()
    R, K, st = ctx.assemble_RK(p.u)
    assert st.ok(), st.as_dict()
    S = ctx.get_state(1)
    for r in range(len(p.n_r)):
        q = p.rve(r)
        Ro, Ko, so = _oracle_rve(q)
        d0, d1 = p.dof_off[r], p.dof_off[r + 1]
        check_R(R[d0:d1], Ro)
        check_K(K[p.Ap[d0]:p.Ap[d1]], Ko, q.Ap)
        e0, e1 = p.elem_off[r] * 4, p.elem_off[r + 1] * 4
        assert np.abs(S[e0:e1] - so).max() <= TOL * np.abs(so).max()
