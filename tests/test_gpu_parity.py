"""GPU parity of the assembly path against the CPU oracle, through the C ABI.

Tolerance (FP64 path): R and K agree with the oracle to 1e-10 relative in
norm, R per entry to 1e-10 max|R|, K per entry to 1e-10 of the row's max
|K_ij| (row-scaled), state per entry to 1e-10 relative.
"""
import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
import workloads as wl

TOL = 1e-10
pytestmark = pytest.mark.gpu


def check_R(Rg, Ro, tol=TOL):
    assert np.linalg.norm(Rg - Ro) <= tol * np.linalg.norm(Ro), np.linalg.norm(Rg - Ro) / np.linalg.norm(Ro)
    assert np.abs(Rg - Ro).max() <= tol * np.abs(Ro).max()


def check_K(Kg, Ko, Ap, tol=TOL):
    assert np.linalg.norm(Kg - Ko) <= tol * np.linalg.norm(Ko), np.linalg.norm(Kg - Ko) / np.linalg.norm(Ko)
    rows = np.repeat(np.arange(len(Ap) - 1), np.diff(Ap))
    rmax = np.zeros(len(Ap) - 1)
    np.maximum.at(rmax, rows, np.abs(Ko))
    assert np.all(np.abs(Kg - Ko) <= tol * rmax[rows])


def oracle_assemble(p, nthreads=8):
    P, mat = oracle.from_workload(p)
    err, R, K, s = P.assemble(mat, p.u, p.u_presc, state_n=p.state, dt=p.dt, nthreads=nthreads)
    assert err == 0
    return R, K, s


def test_config1_he_p1_full_size(gpu):
    p = wl.he_p1(10)
    ctx = p.context()
    R, K, st = ctx.assemble_RK(p.u)
    assert st.ok(), st.as_dict()
    Ro, Ko, _ = oracle_assemble(p)
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)


@pytest.mark.parametrize("n,stretch,perturb", [(3, None, 1e-4), (4, None, 1e-4), (3, 4e-3, 5e-3)])
def test_j2_p2_parity(gpu, n, stretch, perturb):
    p = wl.j2_p2(n=n, seed=11, stretch=stretch, perturb=perturb)
    ctx = p.context()
    R, K, st = ctx.assemble_RK(p.u)
    assert st.ok(), st.as_dict()
    Ro, Ko, so = oracle_assemble(p)
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    sg = ctx.get_state(1)
    assert np.abs(sg - so).max() <= TOL * np.abs(so).max()
    frac = (so[:, 9] > 0).mean()
    if stretch is None:
        assert 0.05 < frac < 0.95, frac


def test_j2_p1_parity(gpu):
    p = wl.he_p1(5)
    p.mat = pg.material(pg.MODEL_J2, E=200e3, nu=0.3, sigma_y=250.0, H=2000.0)
    p.u = p.u * 0.3
    p.state = np.zeros((p.nqp, 10))
    p.state[:, [0, 4, 8]] = 1.0
    ctx = p.context()
    R, K, st = ctx.assemble_RK(p.u)
    assert st.ok()
    Ro, Ko, so = oracle_assemble(p)
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    assert (so[:, 9] > 0).any()


def test_colour_scatter_deterministic_and_equal(gpu):
    p = wl.j2_p2(n=3, seed=5, perturb=5e-3)
    ctx = p.context()
    Ra, Ka, _ = ctx.assemble_RK(p.u)
    ctx.set_scatter_mode(pg.SCATTER_COLOUR)
    R1, K1, _ = ctx.assemble_RK(p.u)
    R2, K2, _ = ctx.assemble_RK(p.u)
    assert np.array_equal(R1, R2) and np.array_equal(K1, K2)
    check_R(R1, Ra, 1e-12)
    check_K(K1, Ka, p.Ap, 1e-12)


def test_assemble_R_only_equals_RK(gpu):
    p = wl.j2_p2(n=3, seed=5, perturb=5e-3)
    ctx = p.context()
    R, K, _ = ctx.assemble_RK(p.u)
    R2, st = ctx.assemble_R(p.u)
    assert st.ok()
    check_R(R2, R, 1e-13)


def test_element_level_entry_points(gpu):
    p = wl.j2_p2(n=3, seed=9, perturb=5e-3, stretch=3e-3)
    ctx = p.context()
    P, mat = oracle.from_workload(p)
    elems = np.array([0, 7, 31, 100, 161])
    lk, fe, st = ctx.stiffmatel_fd(elems, p.u)
    fe2, st2 = ctx.resid_on_elem(elems, p.u)
    assert st.ok() and st2.ok()
    for k, e in enumerate(elems):
        ue = np.zeros(30)
        for a in range(10):
            for j in range(3):
                i = p.ids[p.conn[e, a], j]
                ue[a * 3 + j] = p.u[i - 1] if i > 0 else 0.0
        err, feo, lko, _ = P.element(mat, e, ue, p.state[e * 4:(e + 1) * 4].ravel())
        assert err == 0
        assert np.linalg.norm(fe[k] - feo) <= TOL * np.linalg.norm(feo)
        assert np.linalg.norm(fe2[k] - feo) <= TOL * np.linalg.norm(feo)
        assert np.linalg.norm(lk[k] - lko) <= TOL * np.linalg.norm(lko)


def sym_L(L):
    L = L.reshape(-1, 3, 3, 3, 3)
    L = 0.5 * (L + L.transpose(0, 2, 1, 3, 4))
    return 0.5 * (L + L.transpose(0, 1, 2, 4, 3))


@pytest.mark.parametrize("model", [pg.MODEL_HE, pg.MODEL_J2])
def test_cm_integrate_matches_oracle(gpu, model):
    rng = np.random.default_rng(2)
    nq = 64
    F = np.eye(3)[None] + rng.uniform(-4e-3, 4e-3, (nq, 3, 3))
    mat = pg.material(model, sigma_y=250.0, H=2000.0)
    st = np.zeros((nq, 10))
    st[:, [0, 4, 8]] = 1.0
    S, L, snp1, q = pg.cm_integrate(mat, F.reshape(nq, 9), st)
    assert (q == 0).all()
    om = oracle.from_pg_material(mat)
    for i in range(nq):
        err, So, Lo, so, _ = oracle.cm_update(om, F[i], st[i])
        assert err == 0
        assert np.abs(S[i] - So.ravel()).max() <= TOL * np.abs(So).max()
        Ls, Los = sym_L(L[i]), sym_L(Lo)
        assert np.abs(Ls - Los).max() <= TOL * np.abs(Los).max()
        if model == pg.MODEL_J2:
            assert np.abs(snp1[i] - so).max() <= TOL * np.abs(so).max()


def test_state_commit_and_reset(gpu):
    p = wl.j2_p2(n=2, seed=4, perturb=5e-3, stretch=3e-3)
    ctx = p.context()
    ctx.assemble_RK(p.u)
    s1 = ctx.get_state(1)
    assert (s1[:, 9] > 0).any()
    ctx.reset_state()
    assert np.array_equal(ctx.get_state(1), ctx.get_state(0))
    ctx.assemble_RK(p.u)
    ctx.commit_state()
    assert np.array_equal(ctx.get_state(0), s1)
    # a second load step from the committed state matches the oracle
    u2 = p.u * 1.5
    R, K, _ = ctx.assemble_RK(u2)
    P, mat = oracle.from_workload(p)
    _, Ro, Ko, so = P.assemble(mat, u2, state_n=s1)
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)


def test_inverted_element_is_counted_not_trapped(gpu):
    p = wl.he_p1(3)
    u = p.u.copy()
    node = p.conn[40, 3]
    for j in range(3):
        if p.ids[node, j] > 0:
            u[p.ids[node, j] - 1] -= 2.0  # push a vertex through its element
    ctx = p.context()
    R, K, st = ctx.assemble_RK(u)
    assert st.inverted > 0
    # the context stays usable
    R2, K2, st2 = ctx.assemble_RK(p.u)
    assert st2.ok()


def test_pattern_mismatch_is_rejected(gpu):
    p = wl.he_p1(2)
    Ai = p.Ai.copy()
    Ai[5] = Ai[6]  # corrupt one column id
    with pytest.raises(pg.PgfemError) as ei:
        pg.Context(p.X, p.conn, p.ids, p.ndof, p.Ap, Ai, p.mat)
    assert ei.value.code == -4


@pytest.mark.parametrize("model", ["j2", "he"])
def test_quadratic_tet_ragged_tile_and_repeat(gpu, model):
    """The quadratic-tet R+K path (point kernel, then the tensor-core element
    assembly over tiles of four elements) on 162 elements, so that the last
    tile is partly empty, against the oracle; a second call on the same
    context gives the same R and K (the record and Y buffers carry nothing
    over between calls)."""
    p = wl.j2_p2(n=3, seed=7, perturb=5e-3)
    if model == "he":
        p.mat = pg.material(pg.MODEL_HE, E=200e3, nu=0.3)
        p.state = None
    assert p.conn.shape[0] % 4 == 2
    ctx = p.context()
    assert ctx.launches_per_assembly() == 3
    Ro, Ko, so = oracle_assemble(p)
    R, K, st = ctx.assemble_RK(p.u)
    assert st.ok(), st.as_dict()
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    if so is not None:
        sg = ctx.get_state(1)
        assert np.abs(sg - so).max() <= TOL * np.abs(so).max()
    R2, K2, st2 = ctx.assemble_RK(p.u)
    assert st2.ok()
    check_R(R2, R, 1e-13)
    check_K(K2, K, p.Ap, 1e-13)


@pytest.mark.parametrize("model", ["j2", "he"])
def test_linear_tet_schedules_agree(gpu, model):
    """The linear-tet R+K path (point kernel, then the warp-specialised
    column-split assembly) with each schedule -- elements per block 16/32/64,
    static or work stealing -- on 5^3 x 6 = 750 elements, so that the last
    tile of every tile size is partly empty; each against the oracle."""
    p = wl.he_p1(5, seed=4)
    p.u = p.u * 0.3
    if model == "j2":
        p.mat = pg.material(pg.MODEL_J2, E=200e3, nu=0.3, sigma_y=250.0, H=2000.0)
        p.state = np.zeros((p.nqp, 10))
        p.state[:, [0, 4, 8]] = 1.0
    assert p.ne % 16 and p.ne % 32 and p.ne % 64
    ctx = p.context()
    Ro, Ko, so = oracle_assemble(p)
    if so is not None:
        assert (so[:, 9] > 0).any()
    for epb in (16, 32, 64):
        for grab in (0, 2):
            ctx.set_schedule(epb, grab)
            R, K, st = ctx.assemble_RK(p.u)
            assert st.ok(), (epb, grab, st.as_dict())
            check_R(R, Ro)
            check_K(K, Ko, p.Ap)
            if so is not None:
                assert np.abs(ctx.get_state(1) - so).max() <= TOL * np.abs(so).max(), (epb, grab)


@pytest.mark.parametrize("nne", [4, 10])
def test_non_first_visit_numbering_matches_oracle(gpu, nne):
    """Nodes numbered in reverse order (ids stay consecutive per node, but rows
    are no longer first touched in element order): the default R+K path
    against the oracle."""
    import pgfem_gpu as pgm
    X, conn, _ = pgm.mesh_box_tet(3, nne)
    nn = X.shape[0]
    ids = np.zeros((nn, 3), dtype=np.int64)
    order = np.arange(nn)[::-1]
    ids[order] = (np.arange(nn)[:, None] * 3 + np.arange(3)[None, :] + 1)
    ndof = 3 * nn
    Ap, Ai = pgm.psparse_apai(conn, ids, ndof)
    r = wl.splitmix64(5, nn * 3).reshape(nn, 3)
    disp = (2 * r - 1) * 1e-4 / 3 + np.outer(X[:, 0], [wl.j2_yield_strain(), 0, 0])
    u = wl.nodal_to_free(ids, disp)
    mat = pg.material(pg.MODEL_J2, sigma_y=250.0, H=2000.0)
    nqp = conn.shape[0] * (4 if nne == 10 else 1)
    state = np.zeros((nqp, 10))
    state[:, [0, 4, 8]] = 1.0
    prob = wl.Problem("rev", X, conn, ids, ndof, Ap, Ai, mat, u, state=state)
    ctx = prob.context()
    R, K, st = ctx.assemble_RK(u)
    assert st.ok()
    Ro, Ko, _ = oracle_assemble(prob)
    check_R(R, Ro)
    check_K(K, Ko, Ap)


def test_scatter_modes_other_than_atomic_and_colour_are_rejected(gpu):
    ctx = wl.he_p1(4).context()
    for mode in (2, 3, -1):
        with pytest.raises(pg.PgfemError):
            ctx.set_scatter_mode(mode)


@pytest.mark.parametrize("nne", [4, 10])
def test_linear_deviatoric_potential_matches_oracle(gpu, nne):
    """HE with the reference's linear deviatoric potential (devPotFlag 2,
    S_dev = G (C - I)) at finite strain (30 % stretch, random perturbation,
    prescribed face): R and K through the atomic and the colour scatter, the
    R-only call, the element-level entry points and the constitutive level
    equal the oracle with the same flag (1e-10)."""
    p = wl.tension(n=3, nne=nne, model="he", stretch=0.3, predictor=True)
    rng = np.random.default_rng(3)
    p.u = p.u + rng.uniform(-0.02, 0.02, p.u.shape)
    p.mat.dev_pot = 2
    Ro, Ko, _ = oracle_assemble(p)
    # the b-term is not negligible: the neo-Hookean K differs at O(1)
    P_, _ = oracle.from_workload(p)
    _, _, Kn, _ = P_.assemble(oracle.from_pg_material(p.mat, dev_pot=1), p.u, p.u_presc)
    assert np.linalg.norm(Kn - Ko) > 0.05 * np.linalg.norm(Ko)
    ctx = p.context()
    R, K, st = ctx.assemble_RK(p.u, p.u_presc)
    assert st.ok(), st.as_dict()
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    check_R(ctx.assemble_R(p.u, p.u_presc)[0], Ro)
    ctx.set_scatter_mode(pg.SCATTER_COLOUR)
    Rc, Kc, _ = ctx.assemble_RK(p.u, p.u_presc)
    check_R(Rc, Ro)
    check_K(Kc, Ko, p.Ap)
    # element level: the dense element blocks assemble to the same K
    elems = np.arange(p.conn.shape[0])
    lk, fe, _ = ctx.stiffmatel_fd(elems, p.u, p.u_presc)
    nd = nne * 3
    Kd = np.zeros((p.ndof, p.ndof))
    for e in elems:
        idx = np.array([p.ids[p.conn[e, a], j] for a in range(nne) for j in range(3)])
        m = idx > 0
        Kd[np.ix_(idx[m] - 1, idx[m] - 1)] += lk[e].reshape(nd, nd)[np.ix_(m, m)]
    rows = np.repeat(np.arange(p.ndof), np.diff(p.Ap))
    assert np.abs(Kd[rows, p.Ai] - Ko).max() <= TOL * np.abs(Ko).max()
    # constitutive level
    F = np.eye(3)[None] + rng.uniform(-0.2, 0.2, (16, 3, 3))
    S, L, _, q = pg.cm_integrate(p.mat, F.reshape(16, 9))
    assert (q == 0).all()
    om = oracle.from_pg_material(p.mat)
    for i in range(16):
        err, So, Lo, _, _ = oracle.cm_update(om, F[i])
        assert err == 0
        assert np.abs(S[i] - So.ravel()).max() <= TOL * np.abs(So).max()
        assert np.abs(sym_L(L[i]) - sym_L(Lo)).max() <= TOL * np.abs(sym_L(Lo)).max()


@pytest.mark.parametrize("nne,model,vol_pot", [(10, "j2", 2), (10, "j2", 3), (4, "j2", 3), (4, "he", 2),
                                               (10, "he", 3)])
def test_volumetric_potentials_match_oracle(gpu, nne, model, vol_pot):
    """The reference's Doll-Schweizerhof volumetric potentials (volPotFlag 2,
    3) at finite volume change, every R+K path of the element type (the
    tensor-core quadratic-tet kernel, the linear-tet column-split kernel), the
    R-only call and the constitutive level, against the oracle (1e-10)."""
    p = wl.tension(n=3, nne=nne, model=model, stretch=0.05, predictor=True)
    rng = np.random.default_rng(vol_pot)
    p.u = p.u + rng.uniform(-0.01, 0.01, p.u.shape)
    p.mat.vol_pot = vol_pot
    Ro, Ko, so = oracle_assemble(p)
    ctx = p.context()
    R, K, st = ctx.assemble_RK(p.u, p.u_presc)
    assert st.ok(), st.as_dict()
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    if so is not None:
        assert np.abs(ctx.get_state(1) - so).max() <= TOL * np.abs(so).max()
    check_R(ctx.assemble_R(p.u, p.u_presc)[0], Ro)
    F = np.eye(3)[None] + rng.uniform(-0.1, 0.1, (8, 3, 3))
    st = None
    if model == "j2":
        st = np.zeros((8, 10))
        st[:, [0, 4, 8]] = 1.0
    S, L, _, q = pg.cm_integrate(p.mat, F.reshape(8, 9), st)
    assert (q == 0).all()
    om = oracle.from_pg_material(p.mat)
    for i in range(8):
        err, So, Lo, _, _ = oracle.cm_update(om, F[i], None if st is None else st[i])
        assert err == 0
        assert np.abs(S[i] - So.ravel()).max() <= TOL * np.abs(So).max()


def test_reference_j2_parameter_block_through_the_gpu(gpu, tmp_path):
    """A model_params.in J2 entry with the reference driver's parameters (beta
    0, hp 300, k0 0.5, damage off; G 6, nu 0.49 from the material line,
    volPotFlag 2) goes reader -> material -> GPU assembly of quadratic tets
    stretched past yield, equal to the oracle with the same material (1e-10)."""
    f = tmp_path / "model_params.in"
    f.write_text("1\n0 4\n{\n0.0 300.0 0.5\n0.0 1.0 0.0 0.0 0.0\n0 0 0 0 0 0\n}\n")
    (j2,) = pg.read_model_params(str(f))
    G, nu = 6.0, 0.49
    mat = pg.j2_material(j2, 2 * G * (1 + nu), nu, vol_pot=2)
    p = wl.j2_p2(n=3, seed=5, stretch=0.08, perturb=5e-3)
    p.mat = mat
    Ro, Ko, so = oracle_assemble(p)
    assert (so[:, 9] > 0).mean() > 0.5
    ctx = p.context()
    R, K, st = ctx.assemble_RK(p.u)
    assert st.ok(), st.as_dict()
    check_R(R, Ro)
    check_K(K, Ko, p.Ap)
    assert np.abs(ctx.get_state(1) - so).max() <= TOL * np.abs(so).max()
