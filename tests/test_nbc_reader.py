"""Surface-load input files on the CPU (host code, no GPU): the element lines'
face features, NBC/<physics>.nbc with its load files, the loaded faces
(construct_list_of_boundary_elements, src/PGFem3D_data_structure.cc:825-895)
and the load expressions of time (the exprtk subset pgfem_load_expression
documents)."""
import math
import os

import numpy as np
import pytest

import pgfem_gpu as pg
import workloads as wl
from input_files import material_line, write_mesh


@pytest.mark.parametrize("expr,t,want", [
    ("1e3*t", 0.25, 250.0),
    ("2*sin(pi*t/2)", 1.0, 2.0),
    ("if(t < 1, t, 1)", 3.0, 1.0),
    ("t < 1 ? 10*t : 10", 0.5, 5.0),
    ("-2^2", 0.0, -4.0),
    ("2^3^2", 0.0, 512.0),
    ("2^-1", 0.0, 0.5),
    ("max(1, t, 3)", 7.0, 7.0),
    ("min(4, t)", 2.0, 2.0),
    ("clamp(0, t, 0.5)", 0.9, 0.5),
    ("abs(-3) + sqrt(16)", 0.0, 7.0),
    ("(1 + 2) * 3 - 4 / 8", 0.0, 8.5),
    ("5 % 3", 0.0, 2.0),
    ("not (t > 1)", 2.0, 0.0),
    ("t >= 1 and t <= 2", 1.5, 1.0),
    ("t == 1 or t = 2", 2.0, 1.0),
    ("exp(log(3)) + log10(100) + floor(2.7) + ceil(0.2)", 0.0, 8.0),
    ("atan2(1, 1) * 4", 0.0, math.pi),
    ("100*t;", 0.1, 10.0),
    ("  12.5  ", 0.0, 12.5),
    ("T * 2", 3.0, 6.0),
    ("3 * t // slope", 2.0, 6.0),
    ("/* ramp */ 4 * t", 0.5, 2.0),
])
def test_load_expressions(expr, t, want):
    assert pg.load_expression(expr, t) == pytest.approx(want, rel=1e-15, abs=1e-15)


@pytest.mark.parametrize("expr", ["t +", "foo(1)", "1 2", "x", "sin(1, 2)", "", "(1 + 2", "if(1, 2)", "t ? 1"])
def test_bad_expressions_rejected(expr):
    with pytest.raises(pg.PgfemError):
        pg.load_expression(expr, 0.0)


def _box_input(tmp, nne=4, n=2):
    X, conn, _ = pg.mesh_box_tet(n, nne)
    ne = conn.shape[0]
    bt = np.zeros((ne, 4), dtype=int)
    bi = np.zeros((ne, 4), dtype=int)
    e1, f1 = wl.box_faces(X, conn, 0, 1.0)
    e2, f2 = wl.box_faces(X, conn, 2, 1.0)
    bt[e1, f1], bi[e1, f1] = 2, 5  # T3D feature: surface 5
    bt[e2, f2], bi[e2, f2] = 2, 7  # surface 7
    codes = np.zeros((X.shape[0], 3), dtype=int)
    codes[X[:, 0] == 0.0] = 1
    base = os.path.join(tmp, "box_")
    write_mesh(base + "0.in", X, conn, codes, [], [material_line(200e3, 0.3, 1, 99)], bnd=(bt, bi))
    return base, X, conn, (e1, f1), (e2, f2)


def _write_nbc(tmp, lines, files):
    d = os.path.join(tmp, "NBC")
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "Mechanical.nbc"), "w") as f:
        f.write("\n".join(lines) + "\n")
    for name, text in files.items():
        with open(os.path.join(d, name), "w") as f:
            f.write(text + "\n")


@pytest.mark.parametrize("nne", [4, 10])
def test_nbc_files_give_faces_and_loads(tmp_path, nne):
    tmp = str(tmp_path)
    base, X, conn, (e1, f1), (e2, f2) = _box_input(tmp, nne)
    _write_nbc(tmp, ["2", "", "# feature type, id, load type, load files", "2 5 3 tx ty tz", "2 7 1 p"],
               {"tx": "100*t\nignored second line", "ty": "0", "tz": "-50*t  # an expression comment",
                "p": "25*sin(pi*t) /* pressure */"})
    nb = pg.NbcFile(tmp)
    assert nb.ftype.tolist() == [2, 2] and nb.fid.tolist() == [5, 7] and nb.load_type.tolist() == [3, 1]
    mesh = pg.InputMesh(base)
    bt, bi = mesh.element_faces()
    assert bt.shape == (conn.shape[0], 4)
    el, fc, ft = nb.faces(mesh)
    got = set(zip(el.tolist(), fc.tolist(), ft.tolist()))
    want = {(int(e), int(f), 0) for e, f in zip(e1, f1)} | {(int(e), int(f), 1) for e, f in zip(e2, f2)}
    assert got == want
    assert np.all(np.diff(el) >= 0)  # element order
    v = nb.load_values(0.5)
    assert np.allclose(v, [[50.0, 0.0, -25.0], [25.0, 0.0, 0.0]], rtol=1e-15, atol=1e-14)


def test_nbc_missing_means_no_loads(tmp_path):
    nb = pg.NbcFile(str(tmp_path))
    assert len(nb.ftype) == 0 and nb.load_values(1.0).shape == (0, 3)


@pytest.mark.parametrize("lines,files", [
    (["2", "2 5 1 p", "2 5 1 p"], {"p": "1"}),   # feature listed twice
    (["1", "2 5 4 a b c d"], {k: "1" for k in "abcd"}),  # load type out of range
    (["1", "2 5 1 missing"], {}),                # load file absent
    (["1", "2 5 1 p"], {"p": "2 * q"}),          # unknown name
    (["3", "2 5 1 p"], {"p": "1"}),              # fewer features than counted
])
def test_bad_nbc_rejected(tmp_path, lines, files):
    _write_nbc(str(tmp_path), lines, files)
    with pytest.raises(pg.PgfemError):
        pg.NbcFile(str(tmp_path))
