"""The N>1 host path of bench.py on CPU: world_size 2 over gloo, each rank a
separate process.  The RVE shards of the ranks are disjoint and cover the
batch (no data-path collective needed), a rank's shard has the sizes, macro
deformations and fluctuations of the same RVEs in the full batch, and the
reported time is the maximum over ranks."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "pgfem-3d_b200")]
    import torch.distributed as dist

    import bench
    import workloads as wl
    ws_, rank_, _ = bench.dist_setup(ws, backend="gloo")
    shard = bench.rve_shard(10, ws_, rank_)
    shards = [None] * ws_
    dist.all_gather_object(shards, shard)
    t = bench.allreduce_max(float(rank_ + 1) * 1.5, ws_)
    tot = bench.allreduce_sum(rank_ + 1, ws_)
    bench.barrier(ws_)
    full = wl.rve_batch(nrve=10, nmin=2, nmax=4)
    part = wl.rve_batch(nrve=10, nmin=2, nmax=4, subset=shard)
    same = bool(np.array_equal(part.n_r, full.n_r[shard]) and np.allclose(part.F0s, full.F0s[shard]))
    uok = all(np.array_equal(part.rve(i).u, full.rve(r).u) for i, r in enumerate(shard))
    q.put((rank_, shards, t, tot, same, uok))
    dist.destroy_process_group()


def test_two_rank_gloo_shards_and_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, shards, t, tot, same, uok in res:
        assert sorted(sum(shards, [])) == list(range(10))
        assert not set(shards[0]) & set(shards[1])
        assert t == 3.0 and tot == 3.0
        assert same and uok
