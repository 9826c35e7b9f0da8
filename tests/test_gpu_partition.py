"""Domain-decomposed assembly with the device backend: two ranks (gloo,
spawned processes sharing one GPU -- their kernels never wait on each other),
each assembling its boundary and interior pieces on device contexts of this
library and exchanging the partial rows of rows it does not own; the owned rows
of R and K equal the single-context GPU assembly of the whole mesh (1e-12 of
the norm: only the summation order differs).  Linear tets with a fixed face
(HE), quadratic tets (J2, the tensor-core path, state per point), crystal
plasticity (rotations and state per element) and prescribed displacements."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _make(kind):
    import workloads as wl
    if kind == "he_p1":
        return wl.he_p1(n=4, seed=3), 0.0
    if kind == "j2_p2":
        return wl.j2_p2(n=4, seed=2, stretch=4e-3, perturb=5e-3), 0.0
    if kind == "tension_p2":
        return wl.tension(n=3, nne=10, model="he", stretch=0.004, predictor=True), 0.0
    p = wl.cp_p1(n=4, seed=2, ngrains=8)
    p.u = p.displacement(2)
    return p, p.dt


def _worker(rank, ws, port, kind, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "pgfem-3d_b200")]
    import datetime

    import torch
    import torch.distributed as dist

    import partition
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=120))
    try:
        p, dt = _make(kind)
        nint = 4 if p.nne == 10 else 1
        be = partition.DeviceBackend(p.mat, state=p.state, nint=nint, npres=0 if p.u_presc is None else len(p.u_presc),
                                     dt=dt, R_cp=p.R_cp)
        da = partition.DistributedAssembly(p.X, p.conn, p.ids, p.ndof, p.Ap, p.Ai, be)
        r0, r1 = da.owned_rows
        R, K, st = da.assemble_RK(da.gather_ghosts(p.u[r0:r1]), p.u_presc)
        ctx = p.context()
        Rg, Kg, stg = ctx.assemble_RK(p.u, p.u_presc, dt=dt)
        k0, k1 = int(p.Ap[r0]), int(p.Ap[r1])
        rR = np.linalg.norm(R - Rg[r0:r1]) / np.linalg.norm(Rg[r0:r1])
        rK = np.linalg.norm(K - Kg[k0:k1]) / np.linalg.norm(Kg[k0:k1])
        npieces = len(da.plan.pieces)
        be.close()
        ctx.close()
        q.put((rank, rR, rK, st.tolist(), stg.ok(), npieces, r1 - r0))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["he_p1", "j2_p2", "tension_p2", "cp_p1"])
def test_two_ranks_on_device_contexts(gpu, kind):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, kind, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = sorted([q.get(timeout=300) for _ in range(2)])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for rank, rR, rK, st, okg, npieces, nrows in res:
        assert okg and st == [0, 0, 0, 0]
        assert nrows > 0
        assert rR <= 1e-12 and rK <= 1e-12, (kind, rank, rR, rK)
    assert res[1][5] == 2  # the upper slab has a boundary and an interior piece
