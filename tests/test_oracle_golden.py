"""Pins the CPU oracle to the reference's own known answers.

The reference's box patch test (tests/box/tension_disp, run by
tests/box/common.sh.in) stretches the unit box to twice its length with the
lateral DOFs held (verification_tests/box_patch_{LT,QT}/tension_disp inputs)
using the linear deviatoric potential + U_Common volumetric potential, and
checks the homogenised stress S_xx against
verification_tests/output/stress_tension_disp.out (4.600000e+00) at 1e-14.
Here the oracle's residual and consistent tangent drive a Newton solve on the
reference's own meshes (24 linear and 24 quadratic tets) from u = 0; the
converged state must reproduce that number.
"""
import json
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load_box(lq):
    d = json.load(open(os.path.join(GOLDEN, "box_%s_tension_disp.json" % lq)))
    X = np.array(d["X"])
    conn = np.array(d["conn"], dtype=np.int32)
    codes = np.array(d["codes"], dtype=np.int64)
    return d, X, conn, codes


@pytest.mark.parametrize("lq", ["LT", "QT"])
def test_box_tension_disp_matches_reference_output(lq):
    d, X, conn, codes = load_box(lq)
    nn = X.shape[0]
    ids, ndof = oracle.generate_dof_ids(conn, nn, codes)
    Ap, Ai = oracle.psparse_apai(conn, ids, ndof)
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai)
    m = d["material"]
    mat = oracle.material(oracle.HE, E=m["Ex"], nu=m["nyz"], dev_pot=m["devPotFlag"])
    assert m["volPotFlag"] == 99
    u_presc = np.array(d["defl"])
    u = np.zeros(ndof)
    rows = np.repeat(np.arange(ndof), np.diff(Ap))
    hist = []
    for it in range(30):
        err, R, K, _ = P.assemble(mat, u, u_presc)
        assert err == 0
        nr = np.linalg.norm(R)
        hist.append(nr)
        if nr < 1e-12:
            break
        Kd = np.zeros((ndof, ndof))
        np.add.at(Kd, (rows, Ai), K)
        u -= np.linalg.solve(Kd, R)
    assert hist[-1] < 1e-12, hist
    # quadratic convergence of the consistent tangent: the last steps shrink fast
    assert len(hist) <= 12, hist
    # homogenised PK2 stress: the equilibrium state is homogeneous (affine u_x = x)
    free_nodes_x = {}
    for n in range(nn):
        if ids[n, 0] > 0:
            free_nodes_x[n] = u[ids[n, 0] - 1]
    for n, ux in free_nodes_x.items():
        assert abs(ux - X[n, 0] * u_presc[0]) < 1e-10
    F = np.diag([1.0 + u_presc[0], 1.0, 1.0])
    err, S, _, _, _ = oracle.cm_update(mat, F)
    assert err == 0
    assert abs(S[0, 0] - d["expected_S_xx"]) <= 1e-14 * abs(d["expected_S_xx"]) + 1e-14
