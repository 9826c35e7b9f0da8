"""Learned warm start of the crystal-plasticity local Newton: training pairs and
training, driven through the C ABI (pgfem_gpu_cp_training_pairs,
pgfem_mlp_train_device).  Device buffers for the pairs are torch tensors
(plumbing only); every numerical step runs in libpgfem_gpu.so.

Training pairs come from the plain (cold-start) FP64 Newton on seeded CP
meshes: for seed index i the tension ramp runs to load step 1 + i mod 20 and
that step's (features, converged slip increments) pairs are kept, so the 20
seeds 100..119 cover the 20 load steps once each.
"""
import time

import numpy as np

import pgfem_gpu as pg
import workloads as wl

TRAIN_SEEDS = tuple(range(100, 120))


def generate_pairs(seeds=TRAIN_SEEDS, n=32, ngrains=512, device="cuda"):
    """(x, t, info): FP32 device tensors x [N][34], t [N][12]; only points whose
    plain Newton converged are kept."""
    import torch
    xs, ts = [], []
    t0 = time.time()
    dropped = 0
    for i, seed in enumerate(seeds):
        p = wl.cp_p1(n=n, seed=seed, ngrains=ngrains)
        ctx = p.context()
        target = 1 + i % wl.CP_STEPS
        for s in range(1, target + 1):
            R, st = ctx.assemble_R(p.displacement(s), dt=p.dt)
            if s == target:
                x = torch.empty((p.ne, pg.MLP_IN), dtype=torch.float32, device=device)
                t = torch.empty((p.ne, pg.MLP_OUT), dtype=torch.float32, device=device)
                ctx.cp_training_pairs(x.data_ptr(), t.data_ptr())
                it = ctx.cp_iterations()
                ok = torch.from_numpy((it < p.mat.cp_max_iter) & (it >= 0)).to(device)
                if st.nonconverged:
                    dropped += int((~ok).sum())
                xs.append(x[ok])
                ts.append(t[ok])
            ctx.commit_state()
        del ctx
    x = torch.cat(xs)
    t = torch.cat(ts)
    return x, t, {"pairs": int(x.shape[0]), "seeds": list(seeds), "n": n, "dropped": dropped,
                  "seconds": time.time() - t0}


def train(x, t, seed=0, epochs=30, batch=8192, lr=2e-3, lr_min=2e-5):
    """A fresh network fitted to the pairs on the GPU; returns (mlp, epoch_loss, seconds)."""
    import torch
    m = pg.Mlp(seed=seed)
    n = int(x.shape[0])
    m.fit_scaling(n, x.data_ptr(), t.data_ptr())
    torch.cuda.synchronize()
    t0 = time.time()
    hist = m.train_device(n, x.data_ptr(), t.data_ptr(), epochs=epochs, batch=batch, lr=lr, lr_min=lr_min,
                          seed=seed)
    return m, hist, time.time() - t0


def guess_from_prediction(p, y, state_n, points=None):
    """Newton guess (nqp x 10: M0 9, g0) from predicted slip increments y (nqp x 12),
    the same arithmetic as the device kernel k_cp_guess (numpy, FP64); with
    points, y and state_n are those of the listed points only."""
    s, n = wl.fcc_slip_systems()
    R = p.R_cp.reshape(-1, 3, 3)
    if points is not None:
        R = R[np.asarray(points)]
        state_n = np.asarray(state_n)[np.asarray(points)] if len(state_n) == p.R_cp.shape[0] else state_n
    rs = np.einsum("eij,aj->eai", R, s)
    rn = np.einsum("eij,aj->eai", R, n)
    P = np.einsum("eai,eaj->eaij", rs, rn)
    y = np.asarray(y, dtype=np.float64)
    M0 = np.eye(3)[None] - np.einsum("ea,eaij->eij", y, P)
    mat = p.mat
    c = mat.G0 * np.abs(y).sum(axis=1) / (mat.gs_0 - mat.g0)
    g0 = (state_n[:, 9] + c * mat.gs_0) / (1.0 + c)
    return np.concatenate([M0.reshape(-1, 9), g0[:, None]], axis=1)
