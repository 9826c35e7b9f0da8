"""Generates the crystal-plasticity box fixture from the PGFem3D source tree.

    python tests/golden/make_cp_box_fixture.py /path/to/pgfem3d

Reads, with this library's own input readers (pgfem_input_*), the reference's
8-partition tension case verification_tests/crystal_plasticity:
box_8CPU_tension/box_<r>.in (257 linear tets, merged into one mesh),
model_params.in (crystal plasticity parameters), CO/co_<r>.in (grain
orientations) and box_0.in.st_tension (time steps and the prescribed-value
increments of its 49 load steps) and the reference's own output of that run,
ref_out_tension/box_<r>_49.res (restart files of step 49: the nodal
displacements u_n and per element the deformation gradient F_n, the plastic
deformation gradient pF_n, the slip resistance g_n and the per-system resolved
shear tau_n and slip rate gamma_dot_n, read with this library's restart parser and put in merged
node / element order through the reader's partition maps), and writes
tests/golden/cp_box_tension.json.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "pgfem-3d_b200"))

import pgfem_gpu as pg  # noqa: E402

NSTEPS = 49


def main(ref):
    cp = os.path.join(ref, "verification_tests", "crystal_plasticity")
    m = pg.InputMesh(os.path.join(cp, "box_8CPU_tension", "box_"), 8)
    (mp,) = [x for x in pg.read_model_params(os.path.join(cp, "model_params.in"))
             if x.model_type == pg.CM_CRYSTAL_PLASTICITY]
    angles, etype = m.orientations(os.path.join(cp, mp.ort_file.decode()))
    sf, times, _, load_steps, incr = pg.read_solver_file(os.path.join(cp, "box_0.in.st_tension"), m.info.npres)
    pF49 = [None] * m.info.ne
    F49 = [None] * m.info.ne
    g49 = [None] * m.info.ne
    tau49 = [None] * m.info.ne
    gd49 = [None] * m.info.ne
    u49 = [None] * m.info.nn
    for r in range(8):
        node_map, e0, ne = m.partition(r)
        _, un, b = pg.restart_parse(os.path.join(cp, "ref_out_tension", "box_%d_49.res" % r), pg.MODEL_CP,
                                    len(node_map), ne, 1)
        for i, n in enumerate(node_map):
            if u49[n] is None:
                u49[n] = un[i].tolist()
            assert max(abs(x - y) for x, y in zip(u49[n], un[i])) < 1e-12  # shared nodes agree
        for k in range(ne):
            blk = b[k, 0]
            F49[e0 + k] = blk[0:9].tolist()
            pF49[e0 + k] = blk[18:27].tolist()
            g49[e0 + k] = float(blk[60])
            tau49[e0 + k] = blk[36:48].tolist()
            gd49[e0 + k] = blk[48:60].tolist()
    d = dict(X=m.X.tolist(), conn=m.conn.tolist(), codes=m.codes.tolist(), defl=m.defl.tolist(),
             Ex=float(m.materials[0, 0]), nyz=float(m.materials[0, 6]), devPotFlag=int(m.dev_pot[0]),
             volPotFlag=int(m.vol_pot[0]), cp_params=list(mp.p)[:mp.np], euler_type=etype,
             angles=angles.tolist(), nor_min=sf.nor_min, times=times.tolist(),
             load_steps=load_steps[:NSTEPS].tolist(), load_incr=incr[:NSTEPS].tolist(),
             ref_step=49, ref_F=F49, ref_pF=pF49, ref_g=g49, ref_u=u49, ref_tau=tau49, ref_gdot=gd49,
             source="verification_tests/crystal_plasticity/{box_8CPU_tension/box_<r>.in, model_params.in, "
                    "CO/co_<r>.in, box_0.in.st_tension, ref_out_tension/box_<r>_49.res}")
    out = os.path.join(HERE, "cp_box_tension.json")
    with open(out, "w") as f:
        json.dump(d, f, indent=0)
    print(out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python %s <path of the PGFem3D source tree>" % sys.argv[0])
    main(sys.argv[1])
