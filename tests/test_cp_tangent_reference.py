"""The crystal-plasticity tangent dM/dF (M = pF_n pF_{n+1}^-1) on the CPU: the
oracle's implicit derivative of its Newton system -- the tangent the GPU path
and the oracle's K use -- against central differences of the converged update,
and the reference's own formula (plasticity_compute_dMdu,
src/plasticity_model.cc:578-699, restated literally in
oracle/orc_cp_ref_tangent.inc) fed with the same converged state.

Finding recorded here: the implicit derivative equals the finite differences
(5e-7), the reference's formula does not (its U is built as sum aC_a (x) P_a,
the transpose of the Jacobian's structure, and (L:C) P_a in place of the
derivative of Ce S) -- so the reference's crystal-plasticity K is not the
derivative of its own update, and this library's CP K, the consistent
tangent, differs from it.  The converged state does not depend on K: the
state pin to the reference's restart output stands."""
import numpy as np

import oracle
import workloads as wl


def _march(steps=4):
    m = oracle.from_pg_material(wl.cp_material())
    q = np.array([[0.3, -0.5, 0.7, 0.4]])
    R = wl.quat_to_rot(q / np.linalg.norm(q)).reshape(9)
    D = np.array([[5e-4, 1e-4, 0], [0, -1.5e-4, 5e-5], [3e-5, 0, -1.5e-4]])
    I = np.eye(3)
    Fn, st = I.copy(), np.concatenate([I.reshape(9), [m.g0]])
    for k in range(1, steps):
        Fk = I + k * D
        bad, snp1, it, dg, cv = oracle.cp_update_batch(m, Fk.reshape(1, 9), st.reshape(1, 10), 0.1, R.reshape(1, 9))
        assert bad == 0
        Fn, st = Fk, snp1[0].copy()
    return m, R, Fn, Fn + D, st


def test_implicit_tangent_is_the_derivative_reference_formula_is_not():
    m, R, Fn, Fk, st = _march()
    dt = 0.1

    def Mof(F):
        bad, snp1, it, dg, cv = oracle.cp_update_batch(m, F.reshape(1, 9), st.reshape(1, 10), dt, R.reshape(1, 9))
        assert bad == 0 and it[0] > 2  # the step slips
        return (st[:9].reshape(3, 3) @ np.linalg.inv(snp1[0, :9].reshape(3, 3))).reshape(9)

    h = 1e-8
    Dfd = np.zeros((9, 9))
    for kl in range(9):
        e = np.zeros(9)
        e[kl] = h
        Dfd[:, kl] = (Mof(Fk.reshape(9) + e) - Mof(Fk.reshape(9) - e)) / (2 * h)
    err, dN, dR = oracle.cp_tangent_pair(m, Fn.reshape(9), Fk.reshape(9), dt, R, st)
    assert err == 0
    scale = np.abs(Dfd).max()
    assert np.abs(dN - Dfd).max() <= 5e-7 * scale
    assert np.abs(dR - Dfd).max() > 0.5 * scale
