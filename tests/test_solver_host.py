"""Host-side checks of the device solver entry points (no GPU needed):
argument and pattern validation come before any device work, and without an
sm_100 device solver creation fails with ENODEV instead of falling back."""
import numpy as np
import pytest

import pgfem_gpu as pg
import workloads as wl


def _create(Ap, Ai, n, **kw):
    return pg.Solver(Ap, Ai, n, **kw)


def test_bad_pattern_is_rejected_before_device_work():
    p = wl.tension(n=2, nne=4)
    Ai = p.Ai.copy()
    Ai[3] = p.ndof  # column id out of range
    with pytest.raises(pg.PgfemError) as e:
        _create(p.Ap, Ai, p.ndof)
    assert pg.ERRORS[e.value.code] == "EPATTERN"
    Ap = p.Ap.copy()
    Ap[2], Ap[1] = Ap[1], Ap[2] + 1  # decreasing row pointer
    with pytest.raises(pg.PgfemError) as e:
        _create(Ap, p.Ai, p.ndof)
    assert pg.ERRORS[e.value.code] == "EINVAL"
    for kw in (dict(maxit=0), dict(tol=0.0), dict(precond=7), dict(solver=3), dict(kdim=0)):
        with pytest.raises(pg.PgfemError) as e:
            _create(p.Ap, p.Ai, p.ndof, **kw)
        assert pg.ERRORS[e.value.code] == "EINVAL", kw
    with pytest.raises(pg.PgfemError) as e:
        _create(p.Ap, p.Ai, p.ndof, kdim=pg.GMRES_MAX_KDIM + 1)
    assert pg.ERRORS[e.value.code] == "ELIMIT"


def test_no_cpu_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = wl.tension(n=2, nne=4)
    with pytest.raises(pg.PgfemError) as e:
        _create(p.Ap, p.Ai, p.ndof)
    assert pg.ERRORS[e.value.code] == "ENODEV"
