"""The warm-start network's CPU oracle checked on its own: the FP64 backward
formulas against central differences of the loss, and the BF16 restatement
close to the FP64 network."""
import numpy as np

import mlp_oracle as MO


def _case(seed=1, n=9):
    rng = np.random.default_rng(seed)
    p = MO.init_params(seed).astype(np.float64)
    x = rng.normal(size=(n, 34))
    t = rng.normal(size=(n, 12)) * 1e-3
    xm = rng.normal(size=34) * 0.1
    xs = np.abs(rng.normal(size=34)) + 0.5
    ys = np.full(12, 1e-3)
    return p, x, t, xm, xs, ys


def test_parameter_count():
    assert MO.NPARAMS == 34 * 128 + 128 + 2 * (128 * 128 + 128) + 12 * 128 + 12 == 39052


def test_fp64_gradient_matches_central_differences():
    p, x, t, xm, xs, ys = _case()
    _, g = MO.loss_grad(p, x, t, xm, xs, ys, bf16_math=False)
    rng = np.random.default_rng(0)
    idx = rng.choice(len(p), 200, replace=False)
    fd = np.zeros(len(idx))
    h = 1e-6
    for j, i in enumerate(idx):
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = MO.loss_grad(pp, x, t, xm, xs, ys, bf16_math=False)
        lm, _ = MO.loss_grad(pm, x, t, xm, xs, ys, bf16_math=False)
        fd[j] = (lp - lm) / (2 * h)
    assert np.abs(fd - g[idx]).max() <= 1e-6 * np.abs(g[idx]).max()


def test_bf16_restatement_close_to_fp64():
    p, x, t, xm, xs, ys = _case(n=64)
    l64, g64 = MO.loss_grad(p, x, t, xm, xs, ys, bf16_math=False)
    l16, g16 = MO.loss_grad(p.astype(np.float32), x, t, xm, xs, ys, bf16_math=True)
    assert abs(l16 - l64) <= 1e-2 * l64
    assert np.linalg.norm(g16 - g64) <= 2e-2 * np.linalg.norm(g64)


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5], dtype=np.float32)
    r = MO.bf16(v)
    assert list(r) == [1.0, 1.0, 1.0 + 4 * 2 ** -8, 1.0, -2.5]
