"""Generates the FE2 micro-structure fixture from the PGFem3D source tree.

    python tests/golden/make_fe2_micro_fixture.py /path/to/pgfem3d

Reads, with this library's own input readers (pgfem_input_read_mesh_bc), the
reference's periodic micro-structure of the tube-shear FE2 case,
verification_MS/tube_shear_model/in/micro/pack_3CPU: the three partition
files pack_<r>.in merged into one mesh (1350 linear tets; nodes that share a
global number at different positions become periodic images) with the
supports of its BC directory (BC/Mechanical_<r>.bc, BC/Mechanical.bcv), and
writes tests/golden/fe2_micro_pack.json (inputs only).
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "pgfem-3d_b200"))

import pgfem_gpu as pg  # noqa: E402


def main(ref):
    d = os.path.join(ref, "verification_MS", "tube_shear_model", "in", "micro", "pack_3CPU")
    m = pg.InputMesh(os.path.join(d, "pack_"), 3, bc_base=os.path.join(d, "BC", "Mechanical"))
    out = dict(X=m.X.tolist(), conn=m.conn.tolist(), codes=m.codes.tolist(), defl=m.defl.tolist(),
               Pr=m.Pr.tolist(), Ex=float(m.materials[0, 0]), nyz=float(m.materials[0, 6]),
               devPotFlag=int(m.dev_pot[0]), volPotFlag=int(m.vol_pot[0]),
               source="verification_MS/tube_shear_model/in/micro/pack_3CPU/{pack_<r>.in, BC/Mechanical_<r>.bc, "
                      "BC/Mechanical.bcv}")
    path = os.path.join(HERE, "fe2_micro_pack.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=0)
    print(path)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <path of the PGFem3D source tree>" % sys.argv[0])
    main(sys.argv[1])
