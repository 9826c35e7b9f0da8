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
