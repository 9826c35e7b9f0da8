"""The reference's own box patch test run through the GPU path.

verification_tests/box_patch_{LT,QT}/tension_disp stretches the unit box to
twice its length with the lateral DOFs held (24 linear / 24 quadratic tets,
the linear deviatoric + U_Common potentials, devPotFlag 2) and the reference
checks the homogenised stress against verification_tests/output/
stress_tension_disp.out = 4.6 (tests/box/common.sh.in).  Here the product
does every step on the device: DOF ids and the CSR pattern from the host
setup, then one Newton-Raphson load step of device assembly + device GMRES
(pgfem_gpu_newton_step) from u = 0, and the constitutive-level entry point
for the stress of the converged deformation.  The inputs are the committed
fixtures extracted from the reference's mesh files
(tests/golden/make_box_fixtures.py)."""
import json
import os

import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
from test_gpu_parity import check_K, check_R

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def box(lq):
    d = json.load(open(os.path.join(GOLDEN, "box_%s_tension_disp.json" % lq)))
    X = np.array(d["X"])
    conn = np.array(d["conn"], dtype=np.int32)
    codes = np.array(d["codes"], dtype=np.int64)
    ids, ndof = pg.generate_dof_ids(conn, X.shape[0], codes)
    Ap, Ai = pg.psparse_apai(conn, ids, ndof)
    m = d["material"]
    assert m["devPotFlag"] == 2 and m["volPotFlag"] == 99
    mat = pg.material(pg.MODEL_HE, E=m["Ex"], nu=m["nyz"], dev_pot=m["devPotFlag"])
    return d, X, conn, ids, ndof, Ap, Ai, mat, np.array(d["defl"])


@pytest.mark.parametrize("lq", ["LT", "QT"])
def test_box_tension_disp_on_the_gpu_matches_reference_output(gpu, lq):
    import torch
    d, X, conn, ids, ndof, Ap, Ai, mat, defl = box(lq)
    ctx = pg.Context(X, conn, ids, ndof, Ap, Ai, mat, npres=len(defl))
    # the first iterate's R and K equal the oracle's on the reference mesh
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai)
    om = oracle.from_pg_material(mat)
    u0 = np.zeros(ndof)
    err, Ro, Ko, _ = P.assemble(om, u0, defl)
    assert err == 0
    R, K, st = ctx.assemble_RK(u0, defl)
    assert st.ok()
    check_R(R, Ro)
    check_K(K, Ko, Ap)
    # one load step on the device
    s = pg.Solver(Ap, Ai, ndof, maxit=2000, kdim=100, tol=1e-13)
    du = torch.zeros(ndof, dtype=torch.float64, device="cuda")
    dp = torch.from_numpy(defl.copy()).cuda()
    info = s.newton_step(ctx, du.data_ptr(), dp.data_ptr(), iter_max=30, nor_min=1e-13)
    assert info.converged and not info.lin_failed and info.elem_failures == 0, info.history()
    assert info.iters <= 12, info.history()
    u = du.cpu().numpy()
    # the equilibrium field is the affine stretch u_x = defl * x
    for n in range(X.shape[0]):
        if ids[n, 0] > 0:
            assert abs(u[ids[n, 0] - 1] - defl[0] * X[n, 0]) < 1e-10
    Rf, _ = ctx.assemble_R(u, defl)
    assert np.linalg.norm(Rf) <= 1e-10 * np.linalg.norm(Ro)
    # homogenised PK2 stress of the converged deformation, on the device
    F = np.diag([1.0 + defl[0], 1.0, 1.0]).reshape(1, 9)
    S, _, _, q = pg.cm_integrate(mat, F, want_L=False)
    assert q[0] == 0
    assert abs(S[0, 0] - d["expected_S_xx"]) <= 1e-14 * abs(d["expected_S_xx"]) + 1e-14
