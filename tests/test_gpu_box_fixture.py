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
make_cp_box_fixture.py) runs three load steps of device Newton with state
commits; every step equals the oracle's Newton on the same inputs."""
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


def test_crystal_plasticity_box_load_steps_match_oracle(gpu):
    import torch
    d = json.load(open(os.path.join(GOLDEN, "cp_box_tension.json")))
    X = np.array(d["X"])
    conn = np.array(d["conn"], dtype=np.int32)
    ids, ndof = pg.generate_dof_ids(conn, X.shape[0], np.array(d["codes"]))
    Ap, Ai = pg.psparse_apai(conn, ids, ndof)
    R_cp = pg.euler_rotation(np.array(d["angles"])).reshape(-1, 9)
    p = d["cp_params"]
    mat = pg.material(pg.MODEL_CP, E=d["Ex"], nu=d["nyz"], gamma_dot_0=p[0], m=p[1], G0=p[2], g0=p[3], gs_0=p[4],
                      gamma_dot_s=p[5], w=p[6])
    ctx = pg.Context(X, conn, ids, ndof, Ap, Ai, mat, npres=len(d["defl"]), R_cp=R_cp)
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai, R_cp=R_cp)
    om = oracle.from_pg_material(mat)
    s = pg.Solver(Ap, Ai, ndof, maxit=5000, kdim=100, tol=1e-13)
    st = np.zeros((conn.shape[0], 10))
    st[:, [0, 4, 8]] = 1.0
    st[:, 9] = p[3]
    uo = np.zeros(ndof)
    du = torch.zeros(ndof, dtype=torch.float64, device="cuda")
    presc = np.array(d["defl"])
    for k in range(len(d["load_incr"])):
        dt = d["times"][k + 1] - d["times"][k]
        uo, ho, ok, so = oracle.newton_step(P, om, uo, presc, state_n=st, dt=dt, iter_max=15, nor_min=1e-10)
        assert ok
        dp = torch.from_numpy(presc.copy()).cuda()
        info = s.newton_step(ctx, du.data_ptr(), dp.data_ptr(), dt=dt, iter_max=15, nor_min=1e-10)
        assert info.converged and not info.lin_failed and info.elem_failures == 0, info.history()
        assert len(info.history()) == len(ho)
        u = du.cpu().numpy()
        assert np.linalg.norm(u - uo) <= 1e-8 * np.linalg.norm(uo)
        sg = ctx.get_state(1)
        assert np.abs(sg - so).max() <= 1e-8 * np.abs(so).max()
        ctx.commit_state()
        st = so
        presc = presc + np.array(d["load_incr"][k])
    assert np.abs(st[:, 9] - p[3]).max() > 0  # the grains harden by the third step
