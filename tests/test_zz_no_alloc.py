"""pgfem_gpu_cp_integrate_noalloc: the crystal plasticity point update for callers
that must not allocate device memory (code under another framework's memory
pool, latency-critical callbacks that cannot afford cudaMalloc's implicit
synchronisation, hosts that forbid allocation after start-up).  Its working
memory is a fixed array inside the library, so it is limited to 4096 points per
call and calls must not overlap on the GPU.

The GPU test drives two consecutive load steps through the C ABI with
caller-owned device buffers and checks each result against the CP assembly
entry point (pgfem_gpu_assemble_RK) on the same steps: the state at t_{n+1}
within the 1e-10 relative tolerance of the other CP tests, the slip increments
within 1e-9, the Newton iteration counts equal up to one for floating-point
ties.  The second call would see a stale ticket counter or stale failure counts
if the shared array were not cleared between calls.  This file is collected
last so that a failure here stops a -x run only after every other test ran."""
import numpy as np
import pytest

import pgfem_gpu as pg
import workloads as wl
from test_oracle_selfcheck import p1_deformation_gradients

TOL = 1e-10


def test_noalloc_rejects_batches_beyond_the_limit():
    """The size check comes before any device work, so it also runs without a GPU."""
    p = wl.cp_p1(n=2, seed=2, ngrains=2)
    n = pg.CP_NOALLOC_MAX_POINTS + 1
    bufs = [np.zeros((10, n)) for _ in range(4)]
    with pytest.raises(pg.PgfemError) as e:
        pg.cp_integrate_noalloc(p.mat, n, *[b.ctypes.data for b in bufs[:3]], 0.1, bufs[3].ctypes.data)
    assert pg.ERRORS[e.value.code] == "ELIMIT"


@pytest.mark.gpu
def test_noalloc_matches_cp_assembly_on_two_calls_in_a_row(gpu):
    import torch
    p = wl.cp_p1(n=8, seed=2, ngrains=16)  # 3072 points: several persistent CTAs
    nq = p.ne
    assert nq <= pg.CP_NOALLOC_MAX_POINTS
    ctx = p.context()
    dev = torch.device("cuda:0")

    def soa(a):
        return torch.from_numpy(np.ascontiguousarray(np.asarray(a).reshape(nq, -1).T)).to(dev)

    d_R = soa(p.R_cp)
    d_sn = soa(p.state)
    d_snp1 = torch.empty((10, nq), dtype=torch.float64, device=dev)
    d_dg = torch.empty((12, nq), dtype=torch.float64, device=dev)
    d_it = torch.empty(nq, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    for step in (1, 2):
        u = p.displacement(step)
        # existing entry point: the CP assembly of this step
        _, _, st_ref = ctx.assemble_RK(u, dt=p.dt)
        assert st_ref.ok(), st_ref.as_dict()
        s_ref = ctx.get_state(1)
        it_ref, dg_ref = ctx.cp_iterations(want_slip=True)
        ctx.commit_state()
        # no-allocation entry point on device buffers
        d_F = soa(p1_deformation_gradients(p, u))
        d_snp1.fill_(np.nan)
        d_it.fill_(-1)
        torch.cuda.synchronize()
        if step == 1:
            st = pg.cp_integrate_noalloc(p.mat, nq, d_F.data_ptr(), d_R.data_ptr(), d_sn.data_ptr(), p.dt,
                                         d_snp1.data_ptr(), d_dg.data_ptr(), d_it.data_ptr(), stream=stream)
            assert st.ok(), st.as_dict()
        else:  # asynchronous form, then wait on the stream
            assert pg.cp_integrate_noalloc(p.mat, nq, d_F.data_ptr(), d_R.data_ptr(), d_sn.data_ptr(), p.dt,
                                           d_snp1.data_ptr(), d_dg.data_ptr(), d_it.data_ptr(), stream=stream,
                                           want_status=False) is None
            torch.cuda.synchronize()
        s = d_snp1.cpu().numpy().T
        it = d_it.cpu().numpy()
        dg = d_dg.cpu().numpy().T
        assert np.isfinite(s).all()
        assert np.abs(s - s_ref).max() <= TOL * np.abs(s_ref).max(), step
        assert np.abs(dg - dg_ref).max() <= 1e-9 * np.abs(dg_ref).max(), step
        assert (np.abs(it - it_ref) <= 1).all() and np.mean(it == it_ref) > 0.99, step
        if step == 2:
            assert it.max() > 0 and np.abs(dg).max() > 0  # the second step does plastic work
        d_sn = d_snp1.clone()  # t_{n+1} becomes t_n for the next call
