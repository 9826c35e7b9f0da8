"""Writers of PGFem3D-format input files for the reader tests (test helpers).

They lay out the non-legacy mesh file of read_input_file
(src/read_input_file.cc:268-415: header, element types, nodes
"Gnn Dom id x y z model_type model_id pr", supports, prescribed values,
elements "id nodes ftype fid pr bnd_id[4] bnd_type[4]", element materials
"id mat[2] hom[2]", material lines, material geometry, load counts), the
solver file of read_solver_file (:556-700) and model_params.in blocks, with
the blank lines and comments the reference's own files carry."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def material_line(Ex, nu, dev_pot, vol_pot, Ey=0.0, Ez=0.0, G=0.0):
    v = [Ex, Ey, Ez, G, 0.0, 0.0, nu, 0.0, 0.0, 1.0, 1.0, 1.0, 1700.0]
    return " ".join("%.17g" % x for x in v) + " %d %d" % (dev_pot, vol_pot)


def write_mesh(path, X, conn, codes, defl, mat_lines, gnn=None, dom=None, elem_mat=None, local_order=None,
               before=(), bnd=None):
    """One mesh file.  gnn/dom per local node (default: Gnn = id, Dom = 0);
    local_order: the order in which node lines are written (default 0..nn-1);
    before: supports sections of other physics written ahead of the
    mechanical one, each (codes (nn, ndim), values); bnd: (bnd_type, bnd_id),
    each (ne, 4), the boundary feature of every element face (default 0)."""
    nn, ne, nne = X.shape[0], conn.shape[0], conn.shape[1]
    gnn = np.arange(nn) if gnn is None else gnn
    dom = np.zeros(nn, dtype=int) if dom is None else dom
    elem_mat = np.zeros(ne, dtype=int) if elem_mat is None else elem_mat
    order = range(nn) if local_order is None else local_order
    L = ["%d 3 %d" % (nn, ne), "", "300 1.000000e-06 1.000000e-15", "", "%d 1 1" % len(mat_lines), "",
         " ".join([str(nne)] * ne), ""]
    for i in order:
        L.append("%d %d %d  %.17g %.17g %.17g 1 %d     0" % (gnn[i], dom[i], i, X[i, 0], X[i, 1], X[i, 2], i + 1))
    for c_other, v_other in before:
        c_other = np.asarray(c_other).reshape(nn, -1)
        s_other = [i for i in range(nn) if np.any(c_other[i] != 0)]
        L += ["", str(len(s_other))] + ["%d %s" % (i, " ".join(str(int(c)) for c in c_other[i])) for i in s_other]
        L += ["", str(len(v_other)), " ".join("%.17g" % v for v in v_other)]
    sup = [i for i in range(nn) if np.any(codes[i] != 0)]
    L += ["", str(len(sup))] + ["%d  %d %d %d " % (i, *codes[i]) for i in sup]
    L += ["", str(len(defl)), " ".join("%.17g" % v for v in defl), ""]
    bt, bi = (np.zeros((ne, 4), dtype=int),) * 2 if bnd is None else bnd
    for e in range(ne):
        L.append("%d  %s  4 1 0  %s  %s" % (e, " ".join(str(int(n)) for n in conn[e]),
                                           " ".join(str(int(v)) for v in bi[e]), " ".join(str(int(v)) for v in bt[e])))
    L.append("")
    L += ["%d  %d 0 %d 0 " % (e, elem_mat[e], elem_mat[e]) for e in range(ne)]
    L += [""] + list(mat_lines) + ["", "1.000000 ",
                                   "1.000000 0.000000 0.000000  0.000000 1.000000 0.000000  0.000000 0.000000 1.000000",
                                   "0 0.500000 0.500000", "", "0", "", "0", "", "0", ""]
    with open(path, "w") as f:
        f.write("\n".join(L))


def write_partitions(base, X, conn, codes, defl, mat_lines, parts, seed=0):
    """Split the mesh into len(parts) files <base><r>.in; parts[r] = element
    ids of partition r.  A node used by several partitions gets its original
    id as Gnn and the lowest such partition as Dom; other nodes Gnn = -1.
    Local node ids are a seeded shuffle.  Returns, per partition, the
    original ids of its local nodes."""
    rng = np.random.default_rng(seed)
    users = {}
    for r, els in enumerate(parts):
        for n in np.unique(conn[els]):
            users.setdefault(int(n), []).append(r)
    maps = []
    for r, els in enumerate(parts):
        nodes = np.unique(conn[els])
        nodes = nodes[rng.permutation(len(nodes))]
        loc = {int(n): i for i, n in enumerate(nodes)}
        gnn = np.array([n if len(users[int(n)]) > 1 else -1 for n in nodes])
        dom = np.array([min(users[int(n)]) for n in nodes])
        lconn = np.vectorize(loc.get)(conn[els])
        write_mesh("%s%d.in" % (base, r), X[nodes], lconn.reshape(len(els), -1), codes[nodes], defl, mat_lines,
                   gnn=gnn, dom=dom, local_order=rng.permutation(len(nodes)))
        maps.append(nodes)
    return maps


def box_fixture(lq):
    return json.load(open(os.path.join(GOLDEN, "box_%s_tension_disp.json" % lq)))


def write_box_fixture(base, lq):
    """The reference's box patch-test mesh (committed fixture) as a mesh file
    <base>0.in; returns the fixture."""
    d = box_fixture(lq)
    m = d["material"]
    write_mesh(base + "0.in", np.array(d["X"]), np.array(d["conn"]), np.array(d["codes"]), d["defl"],
               [material_line(m["Ex"], m["nyz"], m["devPotFlag"], m["volPotFlag"], Ey=m["Ey"], Ez=m["Ez"],
                              G=m["Gyz"])])
    return d
