"""Layout of the FE2 RVE batch workload (CPU): the union mesh's CSR pattern
is block diagonal and each block equals the RVE's own Psparse_ApAi pattern;
DOF, node and element ranges are consistent; macro deformations are symmetric
and within the stated amplitude."""
import numpy as np

import oracle
import workloads as wl


def test_batch_pattern_is_block_diagonal_per_rve():
    p = wl.rve_batch(nrve=7, nmin=3, nmax=6)
    assert len(p.n_r) == 7 and p.n_r.min() >= 3 and p.n_r.max() <= 6
    assert p.elem_off[-1] == p.ne and p.node_off[-1] == p.X.shape[0] and p.dof_off[-1] == p.ndof
    for r in range(7):
        q = p.rve(r)
        assert q.ne == 6 * int(p.n_r[r]) ** 3
        # periodic: one node's DOFs per lattice point
        assert q.ndof == 3 * int(p.n_r[r]) ** 3
        Ap, Ai = oracle.psparse_apai(q.conn, q.ids, q.ndof)
        assert np.array_equal(Ap, q.Ap) and np.array_equal(Ai, q.Ai)
        d0, d1 = p.dof_off[r], p.dof_off[r + 1]
        cols = p.Ai[p.Ap[d0]:p.Ap[d1]]
        assert cols.min() >= d0 and cols.max() < d1


def test_macro_deformations_symmetric_and_bounded():
    p = wl.rve_batch(nrve=16, nmin=3, nmax=4)
    F = p.F0s.reshape(-1, 3, 3)
    assert np.allclose(F, np.transpose(F, (0, 2, 1)))
    assert np.abs(F).max() <= 0.02 and np.abs(F).max() > 0.005
