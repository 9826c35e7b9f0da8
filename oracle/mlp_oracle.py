"""CPU oracle of the warm-start network (numpy).

TEST INFRASTRUCTURE ONLY: imported by tests/ and the CPU-baseline leg of
bench.py as the checker.  The product path never uses it.

The network has no counterpart in the reference; it produces the initial guess
of the crystal-plasticity local Newton (the reference starts that Newton from
the elastic predictor, src/plasticity_model.cc:1148-1224).

Architecture: 34 inputs -> 128 -> 128 -> 128 (GELU, exact erf form) -> 12.
Parameter vector (FP32), in this order: W1[128][34], b1[128], W2[128][128], b2,
W3[128][128], b3, W4[12][128], b4[12]  (39,052 values).

`forward`/`loss_grad` with bf16=True restate the device arithmetic: weights,
normalised inputs, hidden activations and output-layer error terms rounded to
bfloat16 (round to nearest even) before each matrix product, products
accumulated in FP32, biases and the nonlinearity in FP32, bias gradients summed
from the rounded error terms.  With bf16=False everything runs in FP64 (used to
check the backward formulas against central differences).
"""
import numpy as np

NIN, NH, NOUT = 34, 128, 12
SHAPES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)),
          ("W3", (NH, NH)), ("b3", (NH,)), ("W4", (NOUT, NH)), ("b4", (NOUT,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    out, o = {}, 0
    for name, s in SHAPES:
        n = int(np.prod(s))
        out[name] = p[o:o + n].reshape(s)
        o += n
    return out


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(x.shape)


def _erf(x):
    from scipy.special import erf
    return erf(x)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / np.sqrt(2.0)))


def gelu_prime(z):
    return 0.5 * (1.0 + _erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def _cast(a, lowp):
    return bf16(a) if lowp else a


def forward(p, x, xmean, xstd, ystd, bf16_math=True, keep=False):
    """Raw features x[n][34] -> raw slip increments y[n][12]."""
    P = unpack(np.asarray(p, dtype=np.float64 if not bf16_math else np.float32))
    ft = np.float32 if bf16_math else np.float64
    x = np.asarray(x, dtype=ft)
    xn = ((x - np.asarray(xmean, ft)) * (ft(1.0) / np.asarray(xstd, ft))).astype(ft)
    h = _cast(xn, bf16_math)
    acts, zs = [h], []
    for l in range(1, 4):
        W = _cast(P["W%d" % l].astype(ft), bf16_math)
        z = (h @ W.T).astype(ft) + P["b%d" % l].astype(ft)
        zs.append(z)
        h = _cast(gelu(z).astype(ft), bf16_math)
        acts.append(h)
    W4 = _cast(P["W4"].astype(ft), bf16_math)
    out = (h @ W4.T).astype(ft) + P["b4"].astype(ft)
    y = out * np.asarray(ystd, ft)
    if keep:
        return y, out, acts, zs
    return y


def loss_grad(p, x, t, xmean, xstd, ystd, bf16_math=True, batch=None):
    """Loss 1/(2B) sum (out - t/ystd)^2 over the batch (B rows, default all) and
    its gradient with respect to the parameter vector."""
    ft = np.float32 if bf16_math else np.float64
    y, out, acts, zs = forward(p, x, xmean, xstd, ystd, bf16_math, keep=True)
    P = unpack(np.asarray(p, dtype=ft))
    B = x.shape[0] if batch is None else batch
    tn = (np.asarray(t, ft) / np.asarray(ystd, ft)).astype(ft)
    r = (out - tn).astype(ft)
    loss = 0.5 * float(np.sum(r.astype(np.float64) ** 2)) / B
    g = {}
    dz = _cast((r / ft(B)).astype(ft), bf16_math)
    g["W4"] = (dz.T @ acts[3]).astype(ft)
    g["b4"] = dz.sum(axis=0, dtype=ft)
    W_next = _cast(P["W4"].astype(ft), bf16_math)
    for l in (3, 2, 1):
        dh = (dz @ W_next).astype(ft)
        dz = _cast((dh * gelu_prime(zs[l - 1]).astype(ft)).astype(ft), bf16_math)
        g["W%d" % l] = (dz.T @ acts[l - 1]).astype(ft)
        g["b%d" % l] = dz.sum(axis=0, dtype=ft)
        W_next = _cast(P["W%d" % l].astype(ft), bf16_math)
    grad = np.concatenate([g[name].ravel() for name, _ in SHAPES])
    return loss, grad


def init_params(seed):
    """Scaled-uniform initialisation used by the tests' reference models
    (any parameter vector works with forward/loss_grad)."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, s in SHAPES:
        if name.startswith("W"):
            lim = np.sqrt(6.0 / (s[0] + s[1]))
            parts.append(rng.uniform(-lim, lim, size=s).ravel())
        else:
            parts.append(rng.uniform(-0.1, 0.1, size=s))
    return np.concatenate(parts).astype(np.float32)
