"""Host setup of the product library vs the oracle's restatement of the
reference: DOF numbering (src/generate_dof_ids.cc) and the CSR pattern
(src/Psparse_ApAi.cc) must be bit-exact, including fixed, prescribed and
periodic DOFs."""
import json
import os

import numpy as np
import pytest

import oracle
import pgfem_gpu as pg
import workloads as wl


def codes_for(X, kind, seed=0):
    nn = X.shape[0]
    codes = np.zeros((nn, 3), dtype=np.int64)
    if kind == "fixed_face":
        codes[X[:, 0] == 0.0] = 1
    elif kind == "mixed":
        r = wl.splitmix64(seed, nn * 3).reshape(nn, 3)
        codes[r < 0.1] = 1
        pres = r > 0.93
        codes[pres] = -(np.arange(pres.sum()) + 1)
    elif kind == "lateral":  # reference box test: only some components free
        codes[:, 1:] = 1
        codes[X[:, 0] == 1.0, 0] = -1
    return codes


@pytest.mark.parametrize("nne", [4, 10])
@pytest.mark.parametrize("kind", ["free", "fixed_face", "mixed", "lateral"])
def test_dof_ids_and_pattern_bit_exact(nne, kind):
    X, conn, Pr = pg.mesh_box_tet(3, nne)
    codes = codes_for(X, kind)
    ids_p, nd_p = pg.generate_dof_ids(conn, X.shape[0], codes)
    ids_o, nd_o = oracle.generate_dof_ids(conn, X.shape[0], codes)
    assert nd_p == nd_o
    assert np.array_equal(ids_p, ids_o)
    if kind == "mixed":
        # partially-free nodes: the node-block pattern builder refuses them only
        # when ids are not consecutive per node, which first-visit numbering never produces
        pass
    Ap_p, Ai_p = pg.psparse_apai(conn, ids_p, nd_p)
    Ap_o, Ai_o = oracle.psparse_apai(conn, ids_o, nd_o)
    assert np.array_equal(Ap_p, Ap_o)
    assert np.array_equal(Ai_p, Ai_o)


@pytest.mark.parametrize("nne", [4, 10])
def test_periodic_pattern_bit_exact(nne):
    X, conn, Pr = pg.mesh_box_tet(4, nne, periodic=True)
    nn = X.shape[0]
    assert (Pr >= 0).sum() > 0
    codes = np.zeros((nn, 3), dtype=np.int64)
    codes[0] = 1
    ids_p, nd_p = pg.generate_dof_ids(conn, nn, codes, Pr)
    ids_o, nd_o = oracle.generate_dof_ids(conn, nn, codes, Pr)
    assert nd_p == nd_o and np.array_equal(ids_p, ids_o)
    Ap_p, Ai_p = pg.psparse_apai(conn, ids_p, nd_p)
    Ap_o, Ai_o = oracle.psparse_apai(conn, ids_o, nd_o)
    assert np.array_equal(Ap_p, Ap_o) and np.array_equal(Ai_p, Ai_o)


@pytest.mark.parametrize("lq", ["LT", "QT"])
def test_reference_box_mesh_pattern(lq):
    d = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "box_%s_tension_disp.json" % lq)))
    X = np.array(d["X"])
    conn = np.array(d["conn"], dtype=np.int32)
    codes = np.array(d["codes"], dtype=np.int64)
    ids_p, nd_p = pg.generate_dof_ids(conn, X.shape[0], codes)
    ids_o, nd_o = oracle.generate_dof_ids(conn, X.shape[0], codes)
    assert np.array_equal(ids_p, ids_o)
    Ap_p, Ai_p = pg.psparse_apai(conn, ids_p, nd_p)
    Ap_o, Ai_o = oracle.psparse_apai(conn, ids_o, nd_o)
    assert np.array_equal(Ap_p, Ap_o) and np.array_equal(Ai_p, Ai_o)


def test_mesh_sizes_and_orientation():
    for n, nne in [(2, 4), (2, 10), (5, 4)]:
        X, conn, _ = pg.mesh_box_tet(n, nne)
        assert conn.shape == (6 * n ** 3, nne)
        L = (n if nne == 4 else 2 * n) + 1
        assert X.shape[0] == L ** 3
        v = X[conn[:, :4]]
        vol = np.einsum("ij,ij->i", np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), v[:, 3] - v[:, 0]) / 6
        assert np.all(vol > 0)
        assert abs(vol.sum() - 1.0) < 1e-12
        if nne == 10:  # edge nodes at the edge midpoints (FEMLIB QTETRAHEDRON order)
            for k, (a, b) in enumerate([(0, 1), (1, 2), (0, 2), (0, 3), (1, 3), (2, 3)]):
                assert np.allclose(X[conn[:, 4 + k]], 0.5 * (X[conn[:, a]] + X[conn[:, b]]))


def test_config_sizes_match_survey():
    # config 1: 6000 elements, 1331 nodes; x=0 face fixed -> 3630 free DOFs
    p = wl.he_p1(10)
    assert p.ne == 6000 and p.X.shape[0] == 1331 and p.ndof == 3630
