"""Pins the CPU oracle to the reference's own known answers.

(1) box patch test (below); (2) the crystal plasticity tension case of
verification_tests/crystal_plasticity: its 8-partition mesh, grain
orientations, parameters and 50 load steps, against the state the reference
wrote in its step-49 restart files (nodal displacements, deformation gradient,
slip resistance and plastic deformation gradient of every element), including
the reference's own numdiff criterion (1e-5) on u_n, F_n and pF_n.

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


# The reference's crystal plasticity tension case writes its state after 50
# load steps (tests/golden/make_cp_box_fixture.py); its local solver stops at
# 1e-5 and its elasticity lives in an absent library, so agreement is judged
# at the size of those tolerances (measured: g 6.5e-5 relative, pF 1.7e-5,
# nodal displacements 1.3e-6 of at most 1.0e-2).
CP_REF_G_RTOL = 2e-4
CP_REF_PF_ATOL = 5e-5
CP_REF_U_ATOL = 5e-6


def nodal_total(ids, u, presc):
    """Nodal displacements (nn, 3): free DOFs from u, prescribed ones from presc."""
    out = np.zeros(ids.shape)
    out[ids > 0] = u[ids[ids > 0] - 1]
    out[ids < 0] = presc[-ids[ids < 0] - 1]
    return out


def cp_box():
    import pgfem_gpu as pg
    d = json.load(open(os.path.join(GOLDEN, "cp_box_tension.json")))
    X = np.array(d["X"])
    conn = np.array(d["conn"], dtype=np.int32)
    ids, ndof = oracle.generate_dof_ids(conn, X.shape[0], np.array(d["codes"], dtype=np.int64))
    Ap, Ai = oracle.psparse_apai(conn, ids, ndof)
    R_cp = pg.euler_rotation(np.array(d["angles"])).reshape(-1, 9)
    p = d["cp_params"]
    mat = pg.material(pg.MODEL_CP, E=d["Ex"], nu=d["nyz"], gamma_dot_0=p[0], m=p[1], G0=p[2], g0=p[3], gs_0=p[4],
                      gamma_dot_s=p[5], w=p[6])
    return d, X, conn, ids, ndof, Ap, Ai, R_cp, mat


def cp_box_steps(d):
    """(dt, prescribed values) of each solve: the mesh's values first, then one
    increment per load step (times has one more entry than the solves)."""
    presc = np.array(d["defl"])
    for k in range(len(d["times"]) - 1):
        yield d["times"][k + 1] - d["times"][k], presc.copy()
        if k < len(d["load_incr"]):
            presc = presc + np.array(d["load_incr"][k])


def test_crystal_plasticity_box_matches_reference_restart():
    d, X, conn, ids, ndof, Ap, Ai, R_cp, mat = cp_box()
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai, R_cp=R_cp)
    om = oracle.from_pg_material(mat)
    st = np.zeros((conn.shape[0], 10))
    st[:, [0, 4, 8]] = 1.0
    st[:, 9] = d["cp_params"][3]
    u = np.zeros(ndof)
    nsolve = 0
    presc = None
    for dt, presc in cp_box_steps(d):
        u, h, ok, st = oracle.newton_step(P, om, u, presc, state_n=st, dt=dt, iter_max=20, nor_min=1e-10)
        assert ok, h
        nsolve += 1
    assert nsolve == d["ref_step"] + 1 == 50
    g_ref, pF_ref = np.array(d["ref_g"]), np.array(d["ref_pF"])
    assert np.abs(st[:, 9] - g_ref).max() <= CP_REF_G_RTOL * g_ref.max()
    assert np.abs(st[:, :9] - pF_ref).max() <= CP_REF_PF_ATOL
    un = nodal_total(ids, u, presc)
    assert np.abs(un - np.array(d["ref_u"])).max() <= CP_REF_U_ATOL
    # the reference's own test criterion on its restart files (numdiff, absolute
    # or relative 1e-5): every u_n and F_n entry, and 99 % of the pF_n entries
    def numdiff_pass(a, b):
        ad = np.abs(a - b)
        return (ad <= 1e-5) | (ad <= 1e-5 * np.abs(b))
    dN = np.array([[-1.0, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    dX = np.einsum("eai,ac->eic", X[conn], dN)
    dU = np.einsum("eai,ac->eic", un[conn], dN)
    F = (np.eye(3) + dU @ np.linalg.inv(dX)).reshape(-1, 9)
    assert numdiff_pass(un, np.array(d["ref_u"])).all()
    assert numdiff_pass(F, np.array(d["ref_F"])).all()
    assert numdiff_pass(st[:, :9], pF_ref).mean() >= 0.99
    # the comparison is sharp: the plastic part of pF is 200x the tolerance
    assert np.abs(pF_ref - np.eye(3).ravel()).max() > 200 * CP_REF_PF_ATOL


@pytest.mark.parametrize("nne", [4, 10])
def test_oracle_mesher_equals_product_mesher(nne):
    """The oracle's restated box mesher (used by the CPU arm of the benchmark
    so that it loads no product code) gives the product mesher's nodes and
    connectivity."""
    import pgfem_gpu as pg
    Xp, cp, _ = pg.mesh_box_tet(3, nne)
    Xo, co = oracle.mesh_box_tet(3, nne)
    assert np.array_equal(cp, co)
    assert np.array_equal(Xp, Xo)


@pytest.mark.parametrize("layers", [None, 2])
def test_oracle_j2_workload_equals_product_workload(layers):
    import workloads as wl
    p = wl.j2_p2(n=3, seed=1, max_cells_z=layers)
    P, mat, u, state = oracle.j2_p2_problem(3, seed=1, max_cells_z=layers)
    assert np.array_equal(P.ids, p.ids) and P.ndof == p.ndof
    assert np.array_equal(P.Ap, p.Ap) and np.array_equal(P.Ai, p.Ai)
    assert np.array_equal(u, p.u) and np.array_equal(state, p.state)
    assert np.array_equal(P.X, p.X) and np.array_equal(P.conn, p.conn)
