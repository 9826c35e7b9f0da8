"""Builds the sm_100a assembly library libpgfem_gpu.so in place.

    python pgfem-3d_b200/build.py [--verbose]

The library is compiled with nvcc for sm_100a only (no PTX fallback, no
other architecture) and links the CUDA runtime statically, so it can be
loaded next to any other CUDA runtime in the process.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(HERE, "libpgfem_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

CU_SOURCES = ["pgfem_gpu.cu", "cp_kernels.cu", "mlp_kernels.cu", "rve_batch.cu", "solver.cu"]
CXX_SOURCES = ["setup_host.cpp", "input_reader.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _sources():
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES + CXX_SOURCES]
    return [s for s in srcs if os.path.exists(s)]


def _deps():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "pgfem_gpu.h")]


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in _deps())


def build(verbose=False, force=False):
    if not force and up_to_date():
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in _sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                               "-I" + INCLUDE, "-I" + CSRC, "-c", src, "-o", obj]
        if src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"] if verbose else []
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stdout.write(r.stdout)
            sys.stderr.write(r.stderr)
        if r.returncode:
            raise RuntimeError("nvcc failed on " + src)
        objs.append(obj)
    cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", OUT] + objs + ["-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return OUT


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(OUT)
