"""Generates the box patch-test fixtures from the PGFem3D source tree.

    python tests/golden/make_box_fixtures.py /path/to/pgfem3d

Reads the reference's 1-rank tension_disp inputs
(verification_tests/box_patch_{LT,QT}/tension_disp/inputs/box_*_1CPU/box_*_0.in)
and the reference output it is checked against
(verification_tests/output/stress_tension_disp.out; the reference test
harness is tests/box/common.sh.in and tests/box/tension_disp/Makefile.am)
and writes tests/golden/box_{LT,QT}_tension_disp.json: node coordinates,
element connectivity, the support codes per DOF (0 free, 1 fixed, -k
prescribed with value defl[k-1]), the prescribed values, the material line
and the expected homogenised stress S_xx.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_input(path):
    lines = [ln.split() for ln in open(path) if ln.strip()]
    nn, ndofn, ne = map(int, lines[0])
    k = 3  # solver tolerances, "1 1 1"
    toe = list(map(int, lines[k]))
    assert len(toe) == ne
    nne = toe[0]
    k += 1
    X = []
    for i in range(nn):
        t = lines[k + i]
        X.append([float(t[3]), float(t[4]), float(t[5])])
    k += nn
    nsup = int(lines[k][0])
    k += 1
    codes = [[0, 0, 0] for _ in range(nn)]
    for i in range(nsup):
        t = list(map(int, lines[k + i]))
        codes[t[0]] = t[1:4]
    k += nsup
    npres = int(lines[k][0])
    k += 1
    defl = list(map(float, lines[k]))[:npres] if npres else []
    k += 1 if npres else 0
    conn = []
    for i in range(ne):
        t = list(map(int, lines[k + i][: 1 + nne]))
        assert t[0] == i
        conn.append(t[1:])
    k += ne
    mat = None
    for t in lines[k:]:
        if len(t) == 15:
            mat = t
            break
    assert mat is not None
    m = dict(Ex=float(mat[0]), Ey=float(mat[1]), Ez=float(mat[2]), Gyz=float(mat[3]), nyz=float(mat[6]),
             devPotFlag=int(mat[13]), volPotFlag=int(mat[14]))
    return dict(nn=nn, ne=ne, nne=nne, X=X, conn=conn, codes=codes, defl=defl, material=m)


def main(ref):
    vt = os.path.join(ref, "verification_tests")
    expected = float(open(os.path.join(vt, "output", "stress_tension_disp.out")).read().split()[0])
    for lq in ("LT", "QT"):
        src = os.path.join(vt, "box_patch_" + lq, "tension_disp", "inputs", "box_%s_1CPU" % lq, "box_%s_0.in" % lq)
        d = parse_input(src)
        d["expected_S_xx"] = expected
        d["source"] = "verification_tests/box_patch_%s/tension_disp/inputs/box_%s_1CPU/box_%s_0.in" % (lq, lq, lq)
        d["expected_source"] = "verification_tests/output/stress_tension_disp.out"
        out = os.path.join(HERE, "box_%s_tension_disp.json" % lq)
        with open(out, "w") as f:
            json.dump(d, f, indent=0)
        print(out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <path of the PGFem3D source tree>" % sys.argv[0])
    main(sys.argv[1])
