"""Readers of PGFem3D's input files (host code of the library, CPU).

- the reference's box patch-test mesh, written in the mesh-file format, reads
  back to the same nodes, elements, supports, prescribed values and material
  line, and its DOF setup equals the oracle's
- a mesh split into partitions (shared nodes by global number, interior nodes
  per file, shuffled local ids) merges back to the original topology
- solver files (plain, arc-length and multiphysics headers; times, output
  steps, load steps and increments), model_params.in (crystal plasticity with
  orientation files and local solver block, J2, hyperelastic, comments),
  orientation files (per element and per material lines)
- malformed or missing files fail with EFORMAT and say where
"""
import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
from input_files import material_line, write_box_fixture, write_mesh, write_partitions


@pytest.mark.parametrize("lq", ["LT", "QT"])
def test_box_fixture_reads_back(tmp_path, lq):
    base = str(tmp_path / "box_")
    d = write_box_fixture(base, lq)
    m = pg.InputMesh(base, 1)
    assert m.info.nn == len(d["X"]) and m.info.ne == len(d["conn"]) and m.info.nne == (4 if lq == "LT" else 10)
    assert np.array_equal(m.X, np.array(d["X"]))
    assert np.array_equal(m.conn, np.array(d["conn"]))
    assert np.array_equal(m.codes, np.array(d["codes"]))
    assert np.array_equal(m.defl, np.array(d["defl"]))
    assert m.info.nmat == 1 and m.dev_pot[0] == 2 and m.vol_pot[0] == 99
    assert m.materials[0, 0] == d["material"]["Ex"] and m.materials[0, 6] == d["material"]["nyz"]
    assert (m.info.nln, m.info.nel_s, m.info.nel_v) == (0, 0, 0)
    mat = m.material()
    assert mat.model == pg.MODEL_HE and mat.dev_pot == 2 and mat.E == d["material"]["Ex"]
    ids, ndof, Ap, Ai = m.dof_setup()
    ido, ndofo = oracle.generate_dof_ids(m.conn, m.info.nn, m.codes)
    Apo, Aio = oracle.psparse_apai(m.conn, ido, ndofo)
    assert ndof == ndofo and np.array_equal(ids, ido)
    assert np.array_equal(Ap, Apo) and np.array_equal(Ai[:Ap[-1]], Aio[:Apo[-1]])


@pytest.mark.parametrize("nne", [4, 10])
def test_partitions_merge_to_the_original_mesh(tmp_path, nne):
    X, conn, _ = pg.mesh_box_tet(3, nne)
    nn = X.shape[0]
    codes = np.zeros((nn, 3), dtype=np.int64)
    codes[X[:, 0] == 0.0] = 1
    codes[X[:, 0] == 1.0, 0] = -1
    ne = conn.shape[0]
    rng = np.random.default_rng(1)
    split = np.sort(rng.choice(np.arange(1, ne), 2, replace=False))
    parts = np.split(np.arange(ne), split)
    base = str(tmp_path / "cube_")
    maps = write_partitions(base, X, conn, codes, [0.1], [material_line(2e5, 0.3, 1, 99)], parts)
    m = pg.InputMesh(base, len(parts))
    assert m.info.nn == nn and m.info.ne == ne
    # merged node -> original node, by the partition maps
    orig = -np.ones(nn, dtype=int)
    for e in range(ne):
        r, le = m.elem_part[e], m.elem_local[e]
        assert parts[r][le] == np.concatenate(parts)[e]
    for r, els in enumerate(parts):
        loc = {int(n): i for i, n in enumerate(maps[r])}
        e0 = sum(len(p) for p in parts[:r])
        for k, e in enumerate(els):
            for a in range(nne):
                g = m.conn[e0 + k, a]
                o = conn[e, a]
                assert orig[g] in (-1, o)
                orig[g] = o
                assert loc[int(o)] >= 0
    assert (orig >= 0).all() and len(set(orig)) == nn
    for r in range(len(parts)):  # the partition maps: local node -> merged node
        nm, e0, ne_r = m.partition(r)
        assert ne_r == len(parts[r]) and e0 == sum(len(p) for p in parts[:r])
        assert np.array_equal(orig[nm], maps[r])
    assert np.array_equal(m.X, X[orig])
    assert np.array_equal(m.codes, codes[orig])
    assert np.array_equal(orig[m.conn], conn[np.concatenate(parts)])


def test_shared_number_at_two_positions_is_a_periodic_image(tmp_path):
    X, conn, _ = pg.mesh_box_tet(2, 4)
    codes = np.zeros((X.shape[0], 3), dtype=np.int64)
    parts = np.split(np.arange(conn.shape[0]), [20])
    base = str(tmp_path / "bad_")
    maps = write_partitions(base, X, conn, codes, [], [material_line(2e5, 0.3, 1, 99)], parts)
    # move a shared node in partition 1's file: the same global number at
    # another position is a periodic image of the first (its DOFs are shared)
    shared = set(np.unique(conn[parts[0]])) & set(np.unique(conn[parts[1]]))
    n = sorted(shared)[0]
    X2 = X.copy()
    X2[n, 0] += 0.5
    loc = {int(v): i for i, v in enumerate(maps[1])}
    Xl = X2[maps[1]]
    lconn = np.vectorize(loc.get)(conn[parts[1]])
    gnn = np.array([v if v in shared else -1 for v in maps[1]])
    write_mesh(base + "1.in", Xl, lconn, codes[maps[1]], [], [material_line(2e5, 0.3, 1, 99)], gnn=gnn,
               dom=np.zeros(len(maps[1]), dtype=int))
    m = pg.InputMesh(base, 2)
    assert m.info.nn == X.shape[0] + 1 and m.info.nperiodic == 1
    img = int(np.where(m.Pr >= 0)[0][0])
    assert np.allclose(m.X[img], X2[n]) and np.allclose(m.X[m.Pr[img]], X[n])
    ids, ndof, _, _ = m.dof_setup()
    assert np.array_equal(ids[img], ids[m.Pr[img]]) and ndof == 3 * X.shape[0]
    # one node with different supports in the two files is an error
    maps = write_partitions(base, X, conn, codes, [0.5], [material_line(2e5, 0.3, 1, 99)], parts)
    c1 = codes[maps[1]].copy()
    c1[list(maps[1]).index(n)] = [-1, 0, 0]
    write_mesh(base + "1.in", X[maps[1]], np.vectorize(loc.get)(conn[parts[1]]), c1, [0.5],
               [material_line(2e5, 0.3, 1, 99)], gnn=gnn, dom=np.zeros(len(maps[1]), dtype=int))
    c0 = codes[maps[0]].copy()
    c0[list(maps[0]).index(n)] = [1, 1, 1]
    loc0 = {int(v): i for i, v in enumerate(maps[0])}
    gnn0 = np.array([v if v in shared else -1 for v in maps[0]])
    write_mesh(base + "0.in", X[maps[0]], np.vectorize(loc0.get)(conn[parts[0]]), c0, [0.5],
               [material_line(2e5, 0.3, 1, 99)], gnn=gnn0, dom=np.zeros(len(maps[0]), dtype=int))
    with pytest.raises(pg.PgfemError, match="EFORMAT.*different supports"):
        pg.InputMesh(base, 2)


def test_missing_and_malformed_files_say_where(tmp_path):
    with pytest.raises(pg.PgfemError, match="EFORMAT.*cannot open"):
        pg.InputMesh(str(tmp_path / "none_"), 1)
    base = str(tmp_path / "box_")
    write_box_fixture(base, "LT")
    lines = open(base + "0.in").read().split("\n")
    open(base + "0.in", "w").write("\n".join(lines[:30]))  # cut inside the support list
    with pytest.raises(pg.PgfemError, match=r"EFORMAT.*box_0\.in:\d+"):
        pg.InputMesh(base, 1)


def test_solver_files(tmp_path):
    p = tmp_path / "a.in.st"
    nt = 50
    times = np.arange(nt + 1) * 2e-4
    inc = np.column_stack([2e-4 * (1 + 1e-3 * np.arange(49)), -1e-4 * (1 - 1e-3 * np.arange(49))])
    # the header's npres (3) is not the increments' count (the mesh's 2 prescribed values)
    p.write_text("1.0e-5 5 3 1\n\n%d\n%s \n\n1\n49 \n\n49\n%s \n\n%s\n" % (
        nt, " ".join("%.6e" % t for t in times), " ".join(str(i) for i in range(1, 50)),
        " ".join("%.17g" % v for v in inc.ravel())))
    sf, t, ps, ls, li = pg.read_solver_file(str(p), npd=2)
    assert (sf.nor_min, sf.iter_max, sf.npres, sf.FNR, sf.nt, sf.n_incr) == (1e-5, 5, 3, 1, nt, 2)
    assert np.allclose(t, times, rtol=1e-6, atol=0) and list(ps) == [49] and list(ls) == list(range(1, 50))
    assert np.array_equal(li, inc)
    # arc length and multiphysics headers, comments, no loads
    q = tmp_path / "b.in.st"
    q.write_text("# solver\n1e-7 5 4 2\n0.1 0.5\n\n1\n0 1\n\n2\n0 1\n\n0\n")
    sf, t, ps, ls, li = pg.read_solver_file(str(q))
    assert (sf.FNR, sf.dAL0, sf.dALMAX, sf.nt, sf.n_print, sf.n_load) == (2, 0.1, 0.5, 1, 2, 0)
    r = tmp_path / "c.in.st"
    r.write_text("1e-6 8 0 4\n1 3\n\n6 1 0.25\n\n2\n0 1 2\n\n1\n2\n\n0\n")
    sf, t, ps, ls, li = pg.read_solver_file(str(r))
    assert (sf.FNR, sf.physicsno, sf.max_NR_staggering, sf.max_subdivision, sf.nt) == (4, 1, 3, 6, 2)
    r.write_text("1e-5 10 4 1 \n\n3\n0 1 2 3 \n\n3\n0 1 2 \n")  # load history in a load directory
    sf, t, ps, ls, li = pg.read_solver_file(str(r), 0)
    assert (sf.nt, sf.n_print, sf.n_load) == (3, 3, 0) and list(ps) == [0, 1, 2]
    r.write_text("1e-6 8 0 1\n\n3\n0 1\n")
    with pytest.raises(pg.PgfemError, match="EFORMAT.*time"):
        pg.read_solver_file(str(r))


def test_model_params(tmp_path):
    p = tmp_path / "model_params.in"
    p.write_text("""3 # number of materials

0 1
{
# gamma_dot_0 m    G0     g0      gs_0    gamma_dot_s     w
          1.0 0.05 58.41  27.17   61.8    50.0e+9         0.005
# 0 0 0
 0 2 CO/co
# read_OnOff max_itr_stag  max_itr_hardening  max_itr_M  max_subdivision tol_hardening  tol_M   computer_zero
  1          10             1                  20        -1               1.0e-5      1.0e-5  1.0e-15
}
1 4
{
0.5 2000.0 250.0
1.0 0.9 1.0 2.0 0.1
0 0 0 0 0 0
}

2 0
{
}
""")
    cp, j2, he = pg.read_model_params(str(p))
    assert (cp.mat_id, cp.model_type, cp.np) == (0, pg.CM_CRYSTAL_PLASTICITY, 7)
    assert list(cp.p)[:7] == [1.0, 0.05, 58.41, 27.17, 61.8, 50.0e9, 0.005]
    assert (cp.unit_cell, cp.ort_option[0], cp.ort_file) == (0, 2, b"CO/co")
    assert (cp.solver_set, cp.max_itr_stag, cp.max_itr_hardening, cp.max_itr_M, cp.max_subdivision) == (1, 10, 1, 20, -1)
    assert (cp.tol_hardening, cp.tol_M, cp.computer_zero) == (1e-5, 1e-5, 1e-15)
    m = pg.cp_material(cp, E=67868.76, nu=0.34128)
    assert (m.model, m.gamma_dot_0, m.m, m.G0, m.g0, m.gs_0, m.w) == (pg.MODEL_CP, 1.0, 0.05, 58.41, 27.17, 61.8, 0.005)
    assert (j2.mat_id, j2.model_type, j2.np) == (1, pg.CM_J2_PLASTICITY_DAMAGE, 14)
    assert list(j2.p)[:3] == [0.5, 2000.0, 250.0]
    assert (he.mat_id, he.model_type, he.np) == (2, pg.CM_HYPER_ELASTICITY, 0)
    p.write_text("1\n0 1\n{\n1.0 0.05\n")
    with pytest.raises(pg.PgfemError, match="EFORMAT"):
        pg.read_model_params(str(p))


def test_j2_material_from_the_reference_parameter_block(tmp_path):
    """A J2 entry (beta hp k0 / damage / split-damage lines, the reference's own
    driver values: beta 0, hp 300, k0 0.5, damage off) gives sigma_y = k0,
    H = hp, E and nu from the mesh's material line and its volumetric potential;
    beta != 0 and active damage (mu != 0) are refused."""
    p = tmp_path / "model_params.in"
    block = "1\n0 4\n{\n%s %s %s\n%s 1.0 0.0 0.0 0.0\n0 0 0 0 0 0\n}\n"
    p.write_text(block % (0.0, 300.0, 0.5, 0.0))
    (j2,) = pg.read_model_params(str(p))
    G, nu = 6.0, 0.49
    E = 2 * G * (1 + nu)
    m = pg.j2_material(j2, E, nu, vol_pot=2)
    assert (m.model, m.sigma_y, m.H, m.vol_pot, m.dev_pot) == (pg.MODEL_J2, 0.5, 300.0, 2, 1)
    assert (m.E, m.nu) == (E, nu)
    assert pg.j2_material(j2, E, nu, vol_pot=0).vol_pot == 99
    for beta, mu in ((0.5, 0.0), (0.0, 1.0)):
        p.write_text(block % (beta, 300.0, 0.5, mu))
        (j2b,) = pg.read_model_params(str(p))
        with pytest.raises(pg.PgfemError, match="EINVAL"):
            pg.j2_material(j2b, E, nu)
    with pytest.raises(pg.PgfemError, match="EINVAL"):
        pg.j2_material(j2, E, nu, vol_pot=5)


def test_orientations_and_rotations(tmp_path):
    X, conn, _ = pg.mesh_box_tet(2, 4)
    ne = conn.shape[0]
    parts = np.split(np.arange(ne), [30])
    base = str(tmp_path / "box_")
    write_partitions(base, X, conn, np.zeros((X.shape[0], 3), dtype=np.int64), [],
                     [material_line(2e5, 0.3, 1, 2)], parts)
    m = pg.InputMesh(base, 2)
    rng = np.random.default_rng(5)
    ang = rng.uniform(-3, 3, (ne, 3))
    with open(str(tmp_path / "co_0.in"), "w") as f:
        f.write("# EulerAngleType: 1\n# element_ID, Integration_point_ID, phi, theta, psi\n")
        for k in range(30):
            f.write("%d 0 %.17g %.17g %.17g\n" % (k, *ang[k]))
    with open(str(tmp_path / "co_1.in"), "w") as f:  # every element of material 0
        f.write("-1 0 %.17g %.17g %.17g\n" % tuple(ang[30]))
    a, et = m.orientations(str(tmp_path / "co"))
    assert et == 1 and np.array_equal(a[:30], ang[:30]) and np.array_equal(a[30:], np.tile(ang[30], (ne - 30, 1)))
    R = pg.euler_rotation(a)

    def rx(t):
        return np.array([[1, 0, 0], [0, np.cos(t), -np.sin(t)], [0, np.sin(t), np.cos(t)]])

    def ry(t):
        return np.array([[np.cos(t), 0, np.sin(t)], [0, 1, 0], [-np.sin(t), 0, np.cos(t)]])

    def rz(t):
        return np.array([[np.cos(t), -np.sin(t), 0], [np.sin(t), np.cos(t), 0], [0, 0, 1]])
    for k in range(ne):
        assert np.allclose(R[k], rz(a[k, 2]) @ ry(a[k, 1]) @ rx(a[k, 0]), atol=1e-15)
    assert np.allclose(np.einsum("kij,kil->kjl", R, R), np.eye(3), atol=1e-14)
    with pytest.raises(pg.PgfemError, match="EFORMAT.*co_9"):
        pg.InputMesh(base, 2).orientations(str(tmp_path / "co_9"))


def test_bc_directory_supports(tmp_path):
    """Supports and prescribed values from a BC directory (<bc>_<r>.bc,
    <bc>.bcv) replace the mesh files' own sections."""
    X, conn, _ = pg.mesh_box_tet(3, 4)
    nn = X.shape[0]
    codes = np.zeros((nn, 3), dtype=np.int64)
    codes[X[:, 0] == 0.0] = 1
    codes[X[:, 0] == 1.0, 0] = -1
    codes[X[:, 0] == 1.0, 1] = -2
    parts = np.split(np.arange(conn.shape[0]), [50, 110])
    base = str(tmp_path / "cube_")
    maps = write_partitions(base, X, conn, np.zeros_like(codes), [], [material_line(2e5, 0.3, 1, 99)], parts)
    bc = tmp_path / "BC"
    bc.mkdir()
    (bc / "Mechanical.bcv").write_text("2\n0.25\n-0.125\n")
    for r, nodes in enumerate(maps):
        sup = [i for i, n in enumerate(nodes) if codes[n].any()]
        (bc / ("Mechanical_%d.bc" % r)).write_text(
            "%d\n" % len(sup) + "".join("%4d  %d %d %d\n" % (i, *codes[nodes[i]]) for i in sup))
    plain = pg.InputMesh(base, 3)
    assert not plain.codes.any() and plain.info.npres == 0
    m = pg.InputMesh(base, 3, bc_base=str(bc / "Mechanical"))
    assert m.info.npres == 2 and list(m.defl) == [0.25, -0.125]
    orig = np.zeros(nn, dtype=int)
    for r in range(3):
        orig[m.partition(r)[0]] = maps[r]
    assert np.array_equal(m.codes, codes[orig])
    ids, ndof, Ap, Ai = m.dof_setup()
    assert ndof == 3 * nn - 3 * (X[:, 0] == 0.0).sum() - 2 * (X[:, 0] == 1.0).sum()
    (bc / "Mechanical_1.bc").write_text("1\n0  -3 0 0\n")
    with pytest.raises(pg.PgfemError, match="EFORMAT.*support code"):
        pg.InputMesh(base, 3, bc_base=str(bc / "Mechanical"))


def test_reference_fe2_micro_structure():
    """The reference's periodic FE2 micro-structure (tube-shear case, three
    partitions, BC directory; tests/golden/make_fe2_micro_fixture.py): the
    merged mesh carries the periodic links of its shared global numbers, the
    product's DOF ids and CSR pattern with those links equal the oracle's, and
    the oracle assembles it under a macro deformation."""
    import json
    import os
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "fe2_micro_pack.json")))
    X = np.array(d["X"])
    conn = np.array(d["conn"], dtype=np.int32)
    codes = np.array(d["codes"], dtype=np.int64)
    Pr = np.array(d["Pr"], dtype=np.int64)
    assert X.shape == (360, 3) and conn.shape == (1350, 4) and (Pr >= 0).sum() == 94
    # images sit one cell length apart along the axes
    off = X[Pr >= 0] - X[Pr[Pr >= 0]]
    assert np.allclose(np.abs(off), np.round(np.abs(off))) and (np.abs(off).sum(1) >= 1).all()
    ids, ndof = pg.generate_dof_ids(conn, X.shape[0], codes, Pr)
    ido, ndofo = oracle.generate_dof_ids(conn, X.shape[0], codes, Pr)
    assert ndof == ndofo == 726 and np.array_equal(ids, ido)
    sl = np.where(Pr >= 0)[0]
    assert np.array_equal(ids[sl], ids[Pr[sl]])
    Ap, Ai = pg.psparse_apai(conn, ids, ndof)
    Apo, Aio = oracle.psparse_apai(conn, ido, ndofo)
    assert np.array_equal(Ap, Apo) and np.array_equal(Ai[:Ap[-1]], Aio[:Apo[-1]])
    F0 = np.array([[0.01, 0.004, 0.0], [0.004, -0.005, 0.002], [0.0, 0.002, 0.003]])
    P = oracle.Problem(X, conn, ids, ndof, Ap, Ai, F0=F0.ravel())
    mat = oracle.material(oracle.HE, E=d["Ex"], nu=d["nyz"])
    u = np.random.default_rng(0).uniform(-1e-4, 1e-4, ndof)
    err, R, K, _ = P.assemble(mat, u, np.array(d["defl"]))
    assert err == 0 and np.isfinite(R).all() and np.isfinite(K).all() and np.abs(R).max() > 0


def test_multiphysics_mesh_keeps_the_mechanical_supports(tmp_path):
    """A heat-transfer + mechanics mesh (multiphysics.in lists heat transfer
    first): the thermal supports section (one code per node) is stepped over
    and the mechanical one kept."""
    (tmp_path / "multiphysics.in").write_text("""# physics
2
1 heat_transfer 1
0
2
0 1
# mechanics
0 solid_mechanics 3
1 1
4
0 3 6 11
""")
    ids, nd = pg.read_multiphysics(str(tmp_path / "multiphysics.in"))
    assert (ids, nd) == ([1, 0], [1, 3])
    X, conn, _ = pg.mesh_box_tet(2, 4)
    nn = X.shape[0]
    codes = np.zeros((nn, 3), dtype=np.int64)
    codes[X[:, 2] == 0.0] = 1
    codes[X[:, 2] == 1.0, 2] = -1
    tcodes = np.where(X[:, 0] == 0.0, -1, 0)
    write_mesh(str(tmp_path / "mp_0.in"), X, conn, codes, [0.05], [material_line(2e5, 0.3, 1, 99)],
               before=[(tcodes, [300.0])])
    m = pg.InputMesh(str(tmp_path / "mp_"), 1, physics=(ids, nd))
    assert np.array_equal(m.codes, codes) and list(m.defl) == [0.05]
    with pytest.raises(pg.PgfemError, match="EFORMAT"):
        pg.InputMesh(str(tmp_path / "mp_"), 1)  # read as single-physics: the layout does not fit


def test_entry_points_reject_bad_arguments(tmp_path):
    """Null handles, null outputs and out-of-range arguments return EINVAL
    (no crash) from every reader and restart entry point."""
    import ctypes as C
    L = pg.lib()
    EINVAL = -1
    h = C.c_void_p()
    assert L.pgfem_input_read_mesh(None, 1, C.byref(h)) == EINVAL
    assert L.pgfem_input_read_mesh(b"x_", 0, C.byref(h)) == EINVAL
    assert L.pgfem_input_read_mesh(b"x_", 1, None) == EINVAL
    one = np.array([3], dtype=np.int32)
    assert L.pgfem_input_read_mesh_mp(b"x_", 1, None, 1, one.ctypes.data, 1, C.byref(h)) == EINVAL  # mech out of range
    bad = np.array([2], dtype=np.int32)
    assert L.pgfem_input_read_mesh_mp(b"x_", 1, None, 1, bad.ctypes.data, 0, C.byref(h)) == EINVAL  # mechanics needs 3
    assert L.pgfem_input_get_info(None, None) == EINVAL
    assert L.pgfem_input_get_mesh(None, None, None, None, None) == EINVAL
    assert L.pgfem_input_get_elements(None, None, None, None, None) == EINVAL
    assert L.pgfem_input_get_periodic(None, None) == EINVAL
    assert L.pgfem_input_get_partition(None, 0, None, None, None) == EINVAL
    assert L.pgfem_input_read_orientations(None, b"co", None, None) == EINVAL
    assert L.pgfem_euler_rotation(-1, None, None) == EINVAL
    n = C.c_int()
    assert L.pgfem_input_read_model_params(None, 0, None, C.byref(n)) == EINVAL
    assert L.pgfem_input_read_multiphysics(None, 0, None, None, C.byref(n)) == EINVAL
    assert L.pgfem_input_read_solver_file(None, -1, None, None, None, None, None) == EINVAL
    assert L.pgfem_restart_block_size(7) < 0
    assert L.pgfem_input_j2_material(None, C.c_double(1.0), C.c_double(0.3), 99, None) == EINVAL
    assert L.pgfem_restart_format(None, 1, 1, 1, pg.MODEL_HE, None, None, None) == EINVAL
    assert L.pgfem_restart_parse(b"x.res", 1, 1, 0, pg.MODEL_HE, None, None, None) == EINVAL
    assert L.pgfem_restart_write_partitions(None, b"x", 0, pg.MODEL_CP, 1, None, None, None) == EINVAL
    # a valid handle with a partition out of range
    from input_files import write_box_fixture
    base = str(tmp_path / "box_")
    write_box_fixture(base, "LT")
    m = pg.InputMesh(base, 1)
    assert L.pgfem_input_get_partition(m._h, 1, None, None, None) == EINVAL
    assert L.pgfem_input_get_partition(m._h, -1, None, None, None) == EINVAL
