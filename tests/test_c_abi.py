"""The C ABI from C: tests/c/host_abi_demo.c, compiled with gcc against
include/pgfem_gpu.h and linked with libpgfem_gpu.so, calls the host entry
points (mesh, DOF ids, CSR pattern, mesh-file reader, restart files) the way a
C/C++ caller links them -- no Python bindings in between (CPU)."""
import os
import shutil
import subprocess

import pytest

from input_files import write_box_fixture

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "pgfem-3d_b200")


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_host_entry_points_from_c(tmp_path):
    exe = str(tmp_path / "host_abi_demo")
    subprocess.run(["gcc", "-std=c99", "-O1", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "host_abi_demo.c"), "-L" + LIBDIR, "-lpgfem_gpu",
                    "-Wl,-rpath," + LIBDIR, "-lm", "-o", exe], check=True)
    base = str(tmp_path / "box_")
    write_box_fixture(base, "LT")
    out = subprocess.run([exe, base, str(tmp_path / "box_0_1.res")], capture_output=True, text=True, timeout=120)
    lines = out.stdout.split("\n")
    assert out.returncode == 0, out.stdout + out.stderr
    assert sum(l.startswith("ok ") for l in lines) == 9 and "FAIL" not in out.stdout, out.stdout


@pytest.mark.gpu
@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_device_entry_points_from_c(gpu, tmp_path):
    """tests/c/device_abi_demo.c, built with gcc against the header and the
    library, runs create -> set_state -> assemble_RK -> get_state -> destroy
    on the GPU; its R, K and state equal the oracle's on the same mesh (1e-10)."""
    import numpy as np

    import oracle
    import pgfem_gpu as pg
    exe = str(tmp_path / "device_abi_demo")
    subprocess.run(["gcc", "-std=c99", "-O1", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "device_abi_demo.c"), "-L" + LIBDIR, "-lpgfem_gpu",
                    "-Wl,-rpath," + LIBDIR, "-lm", "-o", exe], check=True)
    out_path = str(tmp_path / "rk.bin")
    out = subprocess.run([exe, out_path], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert sum(l.startswith("ok ") for l in out.stdout.split("\n")) == 8, out.stdout
    raw = open(out_path, "rb").read()
    ndof, nnz = np.frombuffer(raw[:16], dtype=np.int64)
    v = np.frombuffer(raw[16:], dtype=np.float64)
    u, R, K, snp1 = v[:ndof], v[ndof:2 * ndof], v[2 * ndof:2 * ndof + nnz], v[2 * ndof + nnz:]
    X, conn, _ = pg.mesh_box_tet(3, 10)
    ids, nd = pg.generate_dof_ids(conn, X.shape[0], np.zeros((X.shape[0], 3), dtype=np.int64))
    Ap, Ai = pg.psparse_apai(conn, ids, nd)
    assert nd == ndof and len(Ai) == nnz
    P = oracle.Problem(X, conn, ids, nd, Ap, Ai)
    mat = oracle.material(oracle.J2, E=200e3, nu=0.3, sigma_y=250.0, H=2000.0)
    st = np.zeros((conn.shape[0] * 4, 10))
    st[:, [0, 4, 8]] = 1.0
    err, Ro, Ko, so = P.assemble(mat, u, state_n=st)
    assert err == 0 and (so[:, 9] > 0).any()
    assert np.linalg.norm(R - Ro) <= 1e-10 * np.linalg.norm(Ro)
    assert np.linalg.norm(K - Ko) <= 1e-10 * np.linalg.norm(Ko)
    assert np.abs(snp1.reshape(-1, 10) - so).max() <= 1e-10 * np.abs(so).max()
