"""The C-ABI library loads and exports every entry point include/pgfem_gpu.h
declares; on a machine without an sm_100 device the device entry points fail
loudly (PGFEM_GPU_ENODEV) instead of falling back to a CPU path."""
import ctypes
import os
import re

import numpy as np
import pytest

import pgfem_gpu as pg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "pgfem_gpu.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(pgfem_\w+)\s*\(", hdr)))


def test_every_declared_symbol_is_exported():
    syms = declared_symbols()
    assert len(syms) >= 20
    L = ctypes.CDLL(pg.LIB_PATH)
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_build_recipe_targets_sm100a_only():
    """The library is compiled by build.py with exactly one -gencode, for
    sm_100a (no PTX, no other architecture)."""
    import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


@pytest.mark.gpu
def test_kernels_run_as_sm100_binaries(gpu):
    """The CUDA runtime reports the library's kernels as sm_100 binaries."""
    assert pg.binary_version() == 100


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_device_fails_loudly():
    import workloads as wl
    p = wl.he_p1(2)
    with pytest.raises(pg.PgfemError) as ei:
        p.context()
    assert ei.value.code in (-5, -2)
    F = np.tile(np.eye(3).ravel(), (2, 1))
    with pytest.raises(pg.PgfemError):
        pg.cm_integrate(pg.material(pg.MODEL_HE), F)
