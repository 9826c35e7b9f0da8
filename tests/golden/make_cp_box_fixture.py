"""Generates the crystal-plasticity box fixture from the PGFem3D source tree.

    python tests/golden/make_cp_box_fixture.py [/path/to/pgfem3d]

Reads, with this library's own input readers (pgfem_input_*), the reference's
8-partition tension case verification_tests/crystal_plasticity:
box_8CPU_tension/box_<r>.in (257 linear tets, merged into one mesh),
model_params.in (crystal plasticity parameters), CO/co_<r>.in (grain
orientations) and box_0.in.st_tension (time steps and the prescribed-value
increments of the first load steps), and writes
tests/golden/cp_box_tension.json.  The file carries inputs only: the
reference's own results for this case come from an elastic law and a local
solver that live in an absent library, so no reference numbers are stored.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "pgfem-3d_b200"))

import pgfem_gpu as pg  # noqa: E402

NSTEPS = 3


def main(ref):
    cp = os.path.join(ref, "verification_tests", "crystal_plasticity")
    m = pg.InputMesh(os.path.join(cp, "box_8CPU_tension", "box_"), 8)
    (mp,) = [x for x in pg.read_model_params(os.path.join(cp, "model_params.in"))
             if x.model_type == pg.CM_CRYSTAL_PLASTICITY]
    angles, etype = m.orientations(os.path.join(cp, mp.ort_file.decode()))
    sf, times, _, load_steps, incr = pg.read_solver_file(os.path.join(cp, "box_0.in.st_tension"), m.info.npres)
    d = dict(X=m.X.tolist(), conn=m.conn.tolist(), codes=m.codes.tolist(), defl=m.defl.tolist(),
             Ex=float(m.materials[0, 0]), nyz=float(m.materials[0, 6]), devPotFlag=int(m.dev_pot[0]),
             volPotFlag=int(m.vol_pot[0]), cp_params=list(mp.p)[:mp.np], euler_type=etype,
             angles=angles.tolist(), nor_min=sf.nor_min, times=times[:NSTEPS + 1].tolist(),
             load_steps=load_steps[:NSTEPS].tolist(), load_incr=incr[:NSTEPS].tolist(),
             source="verification_tests/crystal_plasticity/{box_8CPU_tension/box_<r>.in, model_params.in, "
                    "CO/co_<r>.in, box_0.in.st_tension}")
    out = os.path.join(HERE, "cp_box_tension.json")
    with open(out, "w") as f:
        json.dump(d, f, indent=0)
    print(out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
