"""Restart files in the reference's layout (host code, CPU): the formatter
and parser of one rank's file (src/restart.cc:187-300 with the HE and CP
and J2 write_restart blocks) round-trip bit-exactly through %.17e; files whose node,
element or point counts or model do not match are rejected (EFORMAT)."""
import numpy as np
import pytest

import pgfem_gpu as pg


@pytest.mark.parametrize("model,bs", [(pg.MODEL_HE, 18), (pg.MODEL_CP, 64), (pg.MODEL_J2, 47)])
def test_round_trip(tmp_path, model, bs):
    assert pg.restart_block_size(model) == bs
    rng = np.random.default_rng(model)
    nn, ne, nip = 14, 24, (1 if model == pg.MODEL_CP else 4)
    u1, u2 = rng.normal(size=(nn, 3)), rng.normal(size=(nn, 3))
    blocks = rng.normal(size=(ne, nip, bs)) * 10.0 ** rng.integers(-12, 12, size=(ne, nip, bs)).astype(float)
    if model == pg.MODEL_J2:  # the damage flag is an integer
        blocks[..., 46] = rng.integers(0, 2, size=(ne, nip))
    path = str(tmp_path / "box_0_7.res")
    pg.restart_format(path, model, u1, u2, blocks)
    lines = open(path).read().split("\n")
    assert len(lines[0].split()) == 6 and lines[nn].strip() == str(nip)
    a, b, c = pg.restart_parse(path, model, nn, ne, nip)
    assert np.array_equal(a, u1) and np.array_equal(b, u2) and np.array_equal(c, blocks)
    with pytest.raises(pg.PgfemError, match="EFORMAT.*point count"):
        pg.restart_parse(path, model, nn, ne, nip + 1)
    with pytest.raises(pg.PgfemError, match="EFORMAT"):
        pg.restart_parse(path, model, nn, ne + 1, nip)
    with pytest.raises(pg.PgfemError, match="EFORMAT.*trailing"):
        pg.restart_parse(path, model, nn, ne - 1, nip)
    for other in (pg.MODEL_HE, pg.MODEL_CP, pg.MODEL_J2):
        if other != model:
            with pytest.raises(pg.PgfemError, match="EFORMAT"):
                pg.restart_parse(path, other, nn, ne, nip)
    with pytest.raises(pg.PgfemError, match="EINVAL"):
        pg.restart_parse(path, 7, nn, ne, nip)


def test_j2_block_layout(tmp_path):
    """J2 block as CM_J2P_PARAM::write_restart writes it
    (src/cm_j2_plasticity.cc:784-808): four tensors of 9 on their own lines,
    the ten scalars w, X, H, ep, gam (n, n-1) on one line, the damage flag."""
    blocks = np.arange(47, dtype=float).reshape(1, 1, 47)
    blocks[0, 0, 46] = 1
    path = str(tmp_path / "j2_0_1.res")
    pg.restart_format(path, pg.MODEL_J2, np.zeros((1, 3)), np.zeros((1, 3)), blocks)
    lines = open(path).read().strip().split("\n")
    assert [len(x.split()) for x in lines] == [6, 1, 9, 9, 9, 9, 10, 1]
    assert lines[-1] == "1" and float(lines[6].split()[0]) == 36.0


def test_partition_files_of_a_merged_mesh(tmp_path):
    """Per-partition files (the reference's one file per rank) from a merged
    mesh: each holds its partition's nodes and elements; parsed back with the
    partition sizes they equal the merged arrays sliced by the node maps."""
    from input_files import material_line, write_partitions
    X, conn, _ = pg.mesh_box_tet(2, 4)
    parts = np.split(np.arange(conn.shape[0]), [17, 30])
    base = str(tmp_path / "box_")
    write_partitions(base, X, conn, np.zeros((X.shape[0], 3), dtype=np.int64), [], [material_line(2e5, 0.3, 1, 2)],
                     parts)
    m = pg.InputMesh(base, 3)
    rng = np.random.default_rng(3)
    nn, ne = m.info.nn, m.info.ne
    u1, u2 = rng.normal(size=(nn, 3)), rng.normal(size=(nn, 3))
    blocks = rng.normal(size=(ne, 1, 64))
    name = str(tmp_path / "box")
    pg.restart_write_partitions(m, name, 49, pg.MODEL_CP, u1, u2, blocks)
    for r in range(3):
        nm, e0, ne_r = m.partition(r)
        a, b, c = pg.restart_parse("%s_%d_49.res" % (name, r), pg.MODEL_CP, len(nm), ne_r, 1)
        assert np.array_equal(a, u1[nm]) and np.array_equal(b, u2[nm]) and np.array_equal(c, blocks[e0:e0 + ne_r])
