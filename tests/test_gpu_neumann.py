"""Surface loads (Neumann terms) on the GPU against the oracle, through the C ABI.

Box meshes with loaded boundary planes -- a traction (3 values) on x = 1, a
pressure (1 value) on z = 1, a 2-value traction on y = 0 and, where x = 0 is
fixed, a traction whose rows are all dropped -- and node coordinates perturbed
after the faces are picked (curved quadratic faces, the face Jacobian varies
over the face).  R and K of the R+K and residual calls (every kernel path:
linear-tet column split, quadratic-tet tensor-core, colour scatter, linear
deviatoric potential, crystal plasticity) and the element-level blocks equal
the oracle with the same faces (1e-10, the parity tolerance); new load values
and clearing the faces take effect; bad faces are rejected.
"""
import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
import workloads as wl
from test_gpu_parity import TOL, check_K, check_R

pytestmark = pytest.mark.gpu

LOADS = np.array([[12.0, -7.0, 3.0], [25.0, 0.0, 0.0], [-4.0, 6.0, 0.0], [9.0, 9.0, 9.0]])
TYPES = np.array([3, 1, 2, 3])


def _faces(p):
    planes = [(0, 1.0), (2, 1.0), (1, 0.0), (0, 0.0)]
    el, fc, ft = [], [], []
    for k, (axis, v) in enumerate(planes):
        e, f = wl.box_faces(p.X, p.conn, axis, v)
        el.append(e)
        fc.append(f)
        ft.append(np.full(len(e), k, dtype=np.int32))
    return np.concatenate(el), np.concatenate(fc), np.concatenate(ft)


def _curve(p, seed=3, amp=0.04):
    n = p.meta.get("n", 4)
    r = np.random.default_rng(seed).uniform(-1, 1, p.X.shape)
    p.X = p.X + amp / n * r


def _oracle_with_faces(p, el, fc, ft, loads=LOADS):
    P, mat = oracle.from_workload(p)
    P.set_neumann(el, fc, TYPES[ft], loads[ft])
    return P, mat


def _check_problem(p, dt=0.0, mode=None):
    el, fc, ft = _faces(p)
    assert len(el) > 0
    _curve(p)
    ctx = p.context()
    if mode is not None:
        ctx.set_scatter_mode(mode)
    ctx.set_neumann(el, fc, ft, TYPES, LOADS)
    R, K, st = ctx.assemble_RK(p.u, p.u_presc, dt=dt)
    assert st.ok(), st.as_dict()
    P, mat = _oracle_with_faces(p, el, fc, ft)
    err, Ro, Ko, _ = P.assemble(mat, p.u, p.u_presc, state_n=p.state, dt=dt, nthreads=8)
    assert err == 0
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    # the faces carry weight in the comparison
    P0, _ = oracle.from_workload(p)
    _, R0, K0, _ = P0.assemble(mat, p.u, p.u_presc, state_n=p.state, dt=dt, nthreads=8)
    assert np.linalg.norm(Ro - R0) > 1e-3 * np.linalg.norm(Ro)
    assert np.abs(Ko - K0).max() > 0
    R1, st1 = ctx.assemble_R(p.u, p.u_presc, dt=dt)
    assert st1.ok()
    check_R(R1, Ro)
    return ctx, el, fc, ft, R0


def test_linear_tets_he(gpu):
    p = wl.he_p1(n=4, seed=2)
    ctx, el, fc, ft, R0 = _check_problem(p)
    # new values: only the loads change
    loads2 = LOADS * np.array([[2.0], [-1.0], [0.5], [3.0]])
    ctx.set_neumann_loads(loads2)
    R, K, st = ctx.assemble_RK(p.u)
    P, mat = _oracle_with_faces(p, el, fc, ft, loads2)
    err, Ro, Ko, _ = P.assemble(mat, p.u, nthreads=8)
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    # cleared: the plain assembly
    ctx.set_neumann([], [], [], [], np.zeros((0, 3)))
    R, st = ctx.assemble_R(p.u)
    check_R(R, R0)
    ctx.close()


def test_linear_tets_colour_scatter(gpu):
    p = wl.he_p1(n=4, seed=5)
    _check_problem(p, mode=pg.SCATTER_COLOUR)[0].close()


def test_quadratic_tets_j2_tensor_core_path(gpu):
    p = wl.j2_p2(n=3, seed=11, stretch=4e-3, perturb=5e-3)
    ctx = _check_problem(p)[0]
    assert ctx.launches_per_assembly() == 4  # u expansion, points, tensor-core R+K, faces
    ctx.close()


def test_quadratic_tets_prescribed_and_fixed(gpu):
    p = wl.tension(n=3, nne=10, model="he", stretch=0.004, predictor=True)
    _check_problem(p)[0].close()


def test_linear_deviatoric_potential(gpu):
    p = wl.he_p1(n=3, seed=8)
    p.mat = pg.material(pg.MODEL_HE, E=200e3, nu=0.3, dev_pot=2)
    _check_problem(p)[0].close()


def test_crystal_plasticity(gpu):
    p = wl.cp_p1(n=4, seed=2, ngrains=8)
    el, fc, ft = _faces(p)
    ctx = p.context()
    ctx.set_neumann(el, fc, ft, TYPES, LOADS)
    P, mat = _oracle_with_faces(p, el, fc, ft)
    u = p.displacement(1)
    R, K, st = ctx.assemble_RK(u, dt=p.dt)
    assert st.ok(), st.as_dict()
    err, Ro, Ko, _ = P.assemble(mat, u, state_n=p.state, dt=p.dt, nthreads=8)
    assert err == 0
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    ctx.close()


@pytest.mark.parametrize("maker", ["p1", "p2", "cp"])
def test_element_level_blocks(gpu, maker):
    if maker == "p1":
        p = wl.he_p1(n=3, seed=4)
    elif maker == "p2":
        p = wl.j2_p2(n=2, seed=11, stretch=4e-3, perturb=5e-3)
    else:
        p = wl.cp_p1(n=3, seed=2, ngrains=8)
    el, fc, ft = _faces(p)
    if maker != "cp":
        _curve(p)
    ctx = p.context()
    ctx.set_neumann(el, fc, ft, TYPES, LOADS)
    P, mat = _oracle_with_faces(p, el, fc, ft)
    u = p.displacement(1) if maker == "cp" else p.u
    dt = p.dt
    counts = np.bincount(el, minlength=p.ne)
    elems = np.unique(np.concatenate([np.nonzero(counts >= 2)[0][:3], el[:4], [0, p.ne - 1]]))
    lk, fe, st = ctx.stiffmatel_fd(elems, u, dt=dt)
    fe2, st2 = ctx.resid_on_elem(elems, u, dt=dt)
    assert st.ok() and st2.ok()
    st_n = ctx.get_state(0).reshape(p.ne, -1) if p.state is not None else None
    nd = 3 * p.nne
    for k, e in enumerate(elems):
        ue = np.zeros(nd)
        for a in range(p.nne):
            for j in range(3):
                i = p.ids[p.conn[e, a], j]
                ue[a * 3 + j] = u[i - 1] if i > 0 else 0.0
        sn = None if st_n is None else st_n[e]
        err, feo, lko, _ = P.element(mat, e, ue, sn, dt=dt)
        assert err == 0
        assert np.linalg.norm(fe[k] - feo) <= TOL * np.linalg.norm(feo)
        assert np.linalg.norm(fe2[k] - feo) <= TOL * np.linalg.norm(feo)
        assert np.linalg.norm(lk[k].ravel() - lko.ravel()) <= TOL * np.linalg.norm(lko)
    ctx.close()


def test_bad_faces_rejected(gpu):
    p = wl.he_p1(n=2, seed=1)
    ctx = p.context()
    good = dict(elem=[0], face=[1], feature=[0], load_type=[3], load_np1=[[1.0, 2.0, 3.0]])
    ctx.set_neumann(**good)
    for key, bad in [("elem", [p.ne]), ("elem", [-1]), ("face", [4]), ("feature", [1]), ("load_type", [0]),
                     ("load_type", [4])]:
        args = dict(good)
        args[key] = bad
        with pytest.raises(pg.PgfemError):
            ctx.set_neumann(**args)
    with pytest.raises(pg.PgfemError):  # wrong number of features
        ctx.set_neumann_loads(np.zeros((2, 3)))
    ctx.close()


def test_input_files_drive_surface_loads(gpu, tmp_path):
    """A mesh with face features and NBC files read through the input API,
    the loaded faces and their load values at t handed to the context."""
    from test_nbc_reader import _box_input, _write_nbc
    tmp = str(tmp_path)
    base, X, conn, _, _ = _box_input(tmp, nne=10, n=2)
    _write_nbc(tmp, ["2", "2 5 3 tx ty tz", "2 7 1 p"], {"tx": "100*t", "ty": "20", "tz": "-50*t",
                                                        "p": "if(t < 1, 30*t, 30)"})
    mesh = pg.InputMesh(base)
    nb = pg.NbcFile(tmp)
    ids, ndof, Ap, Ai = mesh.dof_setup()
    mat = mesh.material(0)
    ctx = pg.Context(mesh.X, mesh.conn, ids, ndof, Ap, Ai, mat)
    el, fc, ft = nb.faces(mesh)
    ctx.set_neumann(el, fc, ft, nb.load_type, nb.load_values(0.0))
    u = 1e-3 * np.random.default_rng(2).uniform(-1, 1, ndof)
    P = oracle.Problem(mesh.X, mesh.conn, ids, ndof, Ap, Ai)
    om = oracle.from_pg_material(mat)
    for t in (0.5, 2.0):
        loads = nb.load_values(t)
        ctx.set_neumann_loads(loads)
        R, K, st = ctx.assemble_RK(u)
        assert st.ok()
        P.set_neumann(el, fc, nb.load_type[ft], loads[ft])
        err, Ro, Ko, _ = P.assemble(om, u)
        assert err == 0
        check_R(R, Ro)
        check_K(K, Ko, Ap)
    ctx.close()
