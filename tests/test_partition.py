"""Domain-decomposed assembly (partition.py) on CPU over gloo: each rank
assembles its slab's boundary and interior pieces with the oracle, sends the
partial rows of rows it does not own to their owners (the reference's
Lk[proc] exchange, src/PLoc_Sparse.cc:143-170,
src/communication/ISIR_SparseComm.cc:119-200), and then holds exactly the
single-rank answer on its owned rows: the owned block of the pattern equals
the global Psparse_ApAi rows bit for bit, R and K to 1e-12 of the norm
(only the summation order differs).  The ghost displacements come from the
owners (reverse exchange); the status word is reduced with MAX (one rank
reports an inverted element, every rank sees it)."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "pgfem-3d_b200"), os.path.join(ROOT, "oracle")]
    import datetime

    import torch.distributed as dist

    import oracle
    import partition
    import workloads as wl
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        p = wl.j2_p2(n=4, seed=2, stretch=4e-3, perturb=5e-3)
        P, mat = oracle.from_workload(p)

        def backend(pc, u_local, u_presc):
            Pl = oracle.Problem(pc.X, pc.conn, pc.ids, pc.ndof, pc.Ap, pc.Ai)
            sn = p.state[(pc.elems[:, None] * 4 + np.arange(4)).ravel()]
            err, R, K, _ = Pl.assemble(mat, u_local, state_n=sn)
            st = np.zeros(4, dtype=np.int64)
            st[0] = err  # the oracle counts inverted elements in err
            if rank == ws - 1 and backend.flag:
                st[0] = 1  # a failure on one rank only
            return R, K, st
        backend.flag = False

        da = partition.DistributedAssembly(p.X, p.conn, p.ids, p.ndof, p.Ap, p.Ai, backend)
        r0, r1 = da.owned_rows
        u_owned = p.u[r0:r1].copy()
        u_pieces = da.gather_ghosts(u_owned)
        ghosts_ok = all(np.array_equal(u, pc.local_u(p.u)) for u, pc in zip(u_pieces, da.plan.pieces))
        R, K, st = da.assemble_RK(u_pieces)
        err, Rg, Kg, _ = P.assemble(mat, p.u, state_n=p.state)
        k0, k1 = int(p.Ap[r0]), int(p.Ap[r1])
        pattern_ok = bool(np.array_equal(da.plan.Ap_owned, p.Ap[r0:r1 + 1] - k0) and
                          np.array_equal(da.plan.Ai_owned, p.Ai[k0:k1]))
        rR = np.linalg.norm(R - Rg[r0:r1]) / np.linalg.norm(Rg[r0:r1])
        rK = np.linalg.norm(K - Kg[k0:k1]) / np.linalg.norm(Kg[k0:k1])
        backend.flag = True
        _, _, st2 = da.assemble_RK(u_pieces)
        npieces = len(da.plan.pieces)
        q.put((rank, r0, r1, pattern_ok, ghosts_ok, rR, rK, st.tolist(), st2.tolist(), npieces,
               sorted(da.plan.send), sorted(da.recv)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws", [2, 3])
def test_partitioned_assembly_equals_single_rank(ws):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q)) for r in range(ws)]
    for pr in procs:
        pr.start()
    res = sorted([q.get(timeout=240) for _ in range(ws)])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    bounds = [(r0, r1) for _, r0, r1, *_ in res]
    assert bounds[0][0] == 0 and all(bounds[i][1] == bounds[i + 1][0] for i in range(ws - 1))
    for rank, r0, r1, pattern_ok, ghosts_ok, rR, rK, st, st2, npieces, sends, recvs in res:
        assert r1 > r0
        assert pattern_ok and ghosts_ok
        assert rR <= 1e-12 and rK <= 1e-12, (rank, rR, rK)
        assert st == [0, 0, 0, 0] and st2[0] == 1
        # first-visit numbering: a slab's foreign rows belong to lower ranks
        assert all(q < rank for q in sends) and all(q > rank for q in recvs)
        if rank > 0:
            assert sends  # partial rows go down
        if ws == 2:
            assert npieces == 2 - (rank == 0)  # rank 0 touches only its own rows: no boundary piece


def test_row_ownership_is_blocked_and_first_visit():
    sys.path[:0] = [os.path.join(ROOT, "pgfem-3d_b200")]
    import partition
    import workloads as wl
    p = wl.j2_p2(n=4, seed=2)
    eb = partition.slab_bounds(p.ne, 4)
    rb = partition.row_bounds(p.conn, p.ids, p.ndof, eb)
    assert rb[0] == 0 and rb[-1] == p.ndof and np.all(np.diff(rb) > 0)
    rev = p.ids.copy()
    m = rev > 0
    rev[m] = p.ndof + 1 - rev[m]  # not first-visit: rejected
    with pytest.raises(ValueError):
        partition.row_bounds(p.conn, rev, p.ndof, eb)
