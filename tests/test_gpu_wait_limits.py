"""Failure path of the bounded device-side waits, made on the host.

The producer/consumer hand-off of the linear-tet R+K kernel and the
tensor-core completion waits of the warm-start network are bounded.  A test
switch withholds one hand-off (the producer's first arrive; the network's
first MMA chain of each CTA, so that no MMA is in flight): with the bound cut
to a millisecond the waits run out, the kernels return early without a trap,
the host sees the failure (status.other > 0 for the assembly,
PGFEM_GPU_ETIMEOUT for the network), and the next call on the same context
or network equals the oracle.  No GPU fault is provoked: every access stays
in bounds and every wait ends by its time bound.
"""
import numpy as np
import pytest

import mlp_oracle as MO
import oracle
import pgfem_gpu as pg
import workloads as wl

pytestmark = pytest.mark.gpu


def test_assembly_handoff_wait_runs_out_and_context_recovers(gpu):
    p = wl.he_p1(5, seed=4)
    ctx = p.context()
    P, mat = oracle.from_workload(p)
    err, Ro, Ko, _ = P.assemble(mat, p.u)
    assert err == 0
    ctx.set_wait_test(1e-3, stall_next=True)
    R, K, st = ctx.assemble_RK(p.u)
    assert st.other > 0 and st.inverted == 0 and st.nonconverged == 0
    ctx.read_status(clear=True)
    R, K, st = ctx.assemble_RK(p.u)  # the switch is one-shot
    assert st.ok(), st.as_dict()
    assert np.linalg.norm(R - Ro) <= 1e-10 * np.linalg.norm(Ro)
    assert np.linalg.norm(K - Ko) <= 1e-10 * np.linalg.norm(Ko)


def test_network_completion_wait_runs_out_and_network_recovers(gpu):
    rng = np.random.default_rng(1)
    m = pg.Mlp(seed=5)
    params = MO.init_params(3)
    m.set_params(params)
    xm = np.zeros(34, np.float32)
    xs = np.ones(34, np.float32)
    ys = np.full(12, 1e-3, np.float32)
    m.set_scaling(xm, xs, ys)
    x = rng.normal(size=(300, 34)).astype(np.float32)
    m.set_wait_test(1e-3, stall_next=True)
    with pytest.raises(pg.PgfemError, match="ETIMEOUT"):
        m.predict(x)
    y = m.predict(x)
    yo = MO.forward(params, x, xm, xs, ys)
    assert np.linalg.norm(y - yo) <= 1e-3 * np.linalg.norm(yo)


def test_wait_limits_are_validated(gpu):
    ctx = wl.he_p1(2).context()
    for bad in (0.0, -1.0, 100.0):
        with pytest.raises(pg.PgfemError, match="EINVAL"):
            ctx.set_wait_test(bad)
        with pytest.raises(pg.PgfemError, match="EINVAL"):
            pg.Mlp(seed=1).set_wait_test(bad)
