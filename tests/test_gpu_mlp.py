"""Warm-start network kernels (tcgen05 BF16 GEMMs, FP32 accumulation) against the
numpy oracle that restates the same arithmetic (oracle/mlp_oracle.py):
forward outputs, the loss and every parameter gradient of the fused training
tile, and a training run that has to fit a smooth synthetic map.

Tolerances: the kernel and the oracle round the same FP32 values to BF16, but
their FP32 sums run in different orders, so an activation now and then lands
one BF16 step (2^-8 relative) apart; outputs agree to 1e-3 in norm, gradients
to 2e-3 per parameter block (measured: <= 2.5e-4) with cosine similarity above
0.99999."""
import numpy as np
import pytest

import mlp_oracle as MO
import pgfem_gpu as pg

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300))


def setup_model(n, seed=0):
    rng = np.random.default_rng(seed)
    m = pg.Mlp(seed=5)
    p = MO.init_params(seed)
    m.set_params(p)
    xm = (rng.normal(size=34) * 0.1).astype(np.float32)
    xs = (np.abs(rng.normal(size=34)) + 0.5).astype(np.float32)
    ys = np.full(12, 1e-3, np.float32)
    m.set_scaling(xm, xs, ys)
    x = (xm + xs * rng.normal(size=(n, 34))).astype(np.float32)
    t = (rng.normal(size=(n, 12)) * 1e-3).astype(np.float32)
    return m, p, x, t, xm, xs, ys


def test_params_round_trip(gpu):
    m = pg.Mlp(seed=3)
    assert pg.Mlp.num_params() == MO.NPARAMS == 39052
    p = MO.init_params(4)
    m.set_params(p)
    assert np.array_equal(m.params(), p)


@pytest.mark.parametrize("n", [1, 128, 333, 40000])
def test_forward_matches_oracle(gpu, n):
    m, p, x, t, xm, xs, ys = setup_model(n)
    y = m.predict(x)
    yo = MO.forward(p, x, xm, xs, ys)
    assert rel(y, yo) <= 1e-3
    assert np.abs(y - yo).max() <= 2e-2 * np.abs(yo).max()
    # and close to the exact FP64 network (BF16 operands cost well under a percent here)
    y64 = MO.forward(p.astype(np.float64), x.astype(np.float64), xm, xs, ys, bf16_math=False)
    assert rel(y, y64) <= 3e-2


@pytest.mark.parametrize("n", [128, 300])
def test_loss_and_gradients_match_oracle(gpu, n):
    m, p, x, t, xm, xs, ys = setup_model(n, seed=1)
    loss, g = m.loss_grad(x, t)
    lo, go = MO.loss_grad(p, x, t, xm, xs, ys)
    assert abs(loss - lo) <= 1e-4 * lo
    parts = MO.unpack(g)
    parts_o = MO.unpack(go)
    for name, _ in MO.SHAPES:
        assert rel(parts[name], parts_o[name]) <= 2e-3, name
    cos = float(np.dot(g, go) / (np.linalg.norm(g) * np.linalg.norm(go)))
    assert cos >= 0.99999


def test_training_fits_a_smooth_map(gpu):
    import torch
    rng = np.random.default_rng(7)
    n = 32768
    x = rng.normal(size=(n, 34)).astype(np.float32)
    A = rng.normal(size=(34, 12)) / np.sqrt(34)
    t = (np.tanh(x @ A) * 1e-3).astype(np.float32)
    dx = torch.from_numpy(x).cuda()
    dt = torch.from_numpy(t).cuda()
    m = pg.Mlp(seed=11)
    m.fit_scaling(n, dx.data_ptr(), dt.data_ptr())
    xm, xi, ys = m.scaling()
    assert np.allclose(xm, x.mean(0), atol=1e-3) and np.allclose(1 / xi, x.std(0), rtol=1e-3)
    assert np.allclose(ys, np.sqrt((t.astype(np.float64) ** 2).mean(0)), rtol=1e-3)
    l0, _ = m.loss_grad(x[:4096], t[:4096])
    hist = m.train_device(n, dx.data_ptr(), dt.data_ptr(), epochs=12, batch=1024, lr=3e-3, lr_min=1e-4)
    l1, _ = m.loss_grad(x[:4096], t[:4096])
    assert hist[-1] < hist[0]
    assert l1 < 0.05 * l0, (l0, l1, hist)
    # the trained network still matches the oracle with the trained parameters
    y = m.predict(x[:1000])
    yo = MO.forward(m.params(), x[:1000], xm, 1.0 / xi, ys)
    assert rel(y, yo) <= 1e-3
