"""The reference's own input cases run through the GPU path.

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
(tests/golden/make_box_fixtures.py), written back in the mesh-file format and
read by the library's reader (pgfem_input_read_mesh).

The reference's crystal plasticity box (verification_tests/crystal_plasticity,
8 partitions merged, 257 linear tets, its grain orientations, CP parameters,
time steps and prescribed-value increments; tests/golden/
make_cp_box_fixture.py) runs its 50 load steps of device Newton with state
commits; every step equals the oracle's Newton on the same inputs, and the
final state reproduces the reference's own step-49 restart output (slip
resistance within 2e-4 relative, plastic deformation gradient within 5e-5)."""
import json
import os

import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
from input_files import write_box_fixture
from test_gpu_parity import check_K, check_R

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def box(tmp_path, lq):
    base = str(tmp_path / "box_")
    d = write_box_fixture(base, lq)
    m = pg.InputMesh(base, 1)
    assert m.dev_pot[0] == 2 and m.vol_pot[0] == 99
    ids, ndof, Ap, Ai = m.dof_setup()
    return d, m.X, m.conn, ids, ndof, Ap, Ai, m.material(), m.defl


@pytest.mark.parametrize("lq", ["LT", "QT"])
def test_box_tension_disp_on_the_gpu_matches_reference_output(gpu, tmp_path, lq):
    import torch
    d, X, conn, ids, ndof, Ap, Ai, mat, defl = box(tmp_path, lq)
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


def test_crystal_plasticity_box_load_steps_match_oracle_and_reference(gpu):
    import torch
    from test_oracle_golden import CP_REF_G_RTOL, CP_REF_PF_ATOL, CP_REF_U_ATOL, cp_box, cp_box_steps, nodal_total
    d, X, conn, ids, ndof, Ap, Ai, R_cp, mat = cp_box()
    ctx = pg.Context(X, conn, ids, ndof, Ap, Ai, mat, npres=len(d["defl"]), R_cp=R_cp)
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai, R_cp=R_cp)
    om = oracle.from_pg_material(mat)
    s = pg.Solver(Ap, Ai, ndof, maxit=5000, kdim=100, tol=1e-13)
    st = np.zeros((conn.shape[0], 10))
    st[:, [0, 4, 8]] = 1.0
    st[:, 9] = d["cp_params"][3]
    uo = np.zeros(ndof)
    du = torch.zeros(ndof, dtype=torch.float64, device="cuda")
    for dt, presc in cp_box_steps(d):
        uo, ho, ok, so = oracle.newton_step(P, om, uo, presc, state_n=st, dt=dt, iter_max=20, nor_min=1e-10)
        assert ok
        dp = torch.from_numpy(presc).cuda()
        info = s.newton_step(ctx, du.data_ptr(), dp.data_ptr(), dt=dt, iter_max=20, nor_min=1e-10)
        assert info.converged and not info.lin_failed and info.elem_failures == 0, info.history()
        assert len(info.history()) == len(ho)
        u = du.cpu().numpy()
        assert np.linalg.norm(u - uo) <= 1e-8 * np.linalg.norm(uo)
        sg = ctx.get_state(1)
        assert np.abs(sg - so).max() <= 1e-8 * np.abs(so).max()
        ctx.commit_state()
        st = so
    # the device run reproduces the reference's own step-49 restart output
    g_ref, pF_ref = np.array(d["ref_g"]), np.array(d["ref_pF"])
    sg = ctx.get_state(0)
    assert np.abs(sg[:, 9] - g_ref).max() <= CP_REF_G_RTOL * g_ref.max()
    assert np.abs(sg[:, :9] - pF_ref).max() <= CP_REF_PF_ATOL
    assert np.abs(nodal_total(ids, du.cpu().numpy(), presc) - np.array(d["ref_u"])).max() <= CP_REF_U_ATOL
