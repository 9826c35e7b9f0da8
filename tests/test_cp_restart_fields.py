"""The crystal plasticity restart fields tau_n and gamma_dot_n
(pgfem_cp_resolved_shear, host) against the reference's own restart output
of its tension case (ref_out_tension/box_<r>_49.res, in the committed
fixture): from the file's F_n, pF_n and g_n and the grains' rotations, the
resolved shear of every slip system of every element equals the file's tau_n
to 2e-6 of the element's largest (the file's own state reproduces its stress
to that precision) and the slip rates its gamma_dot_n to 5e-5 (the flow rule
raises tau to the power 1/m = 20).  The flow rule applied to the file's own
tau_n and g_n gives its gamma_dot_n to 1e-12: the rate law, the exponent and
the use of g_n are the reference's."""
import numpy as np

import pgfem_gpu as pg
from test_oracle_golden import cp_box


def test_resolved_shear_and_slip_rates_equal_reference_restart():
    d, X, conn, ids, ndof, Ap, Ai, R_cp, mat = cp_box()
    F = np.array(d["ref_F"])
    pF = np.array(d["ref_pF"])
    g = np.array(d["ref_g"])
    tau_ref = np.array(d["ref_tau"])
    gd_ref = np.array(d["ref_gdot"])
    assert tau_ref.shape == (conn.shape[0], 12) and np.abs(tau_ref).max() > 1.0
    tau, gd = pg.cp_resolved_shear(mat, F, pF, g, R_cp)
    scale = np.abs(tau_ref).max(axis=1, keepdims=True)
    assert np.all(np.abs(tau - tau_ref) <= 2e-6 * scale)
    gscale = np.abs(gd_ref).max(axis=1, keepdims=True)
    assert np.all(np.abs(gd - gd_ref) <= 5e-5 * gscale)
    # the rate law itself, on the file's own tau and g
    p = d["cp_params"]
    r = tau_ref / g[:, None]
    law = p[0] * r * np.abs(r) ** (1.0 / p[1] - 1.0)
    assert np.all(np.abs(law - gd_ref) <= 1e-12 * gscale)
