"""Training driver of the learned SPAI preconditioner.

The network and its forward/backward/Adam kernels live in the C ABI
(mclsgpu_spai_*); this module only decides what to train on and for how
long.  Training vectors for an operator A are

* residual snapshots of point-Jacobi MCSA on A x = b (the preconditioned
  residual after 1, 2, 4, ... iterations, taken with
  mclsgpu_domain_residual), i.e. the slowly damped modes MCSA leaves behind;
* random vectors (all modes), which keep the learned M from trading the
  high-frequency modes for the smooth ones.

Device vectors are torch tensors (plumbing only: every computation on them is
a library kernel).
"""
from __future__ import annotations

import numpy as np

from . import capi


def stencil_slots(A) -> int:
    """Number of distinct column offsets of A (the network's slot count)."""
    A = A.tocsr()
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    return int(np.unique(A.indices - rows).size)


def mcsa_residuals(ctx, op, b, iterations=(1, 2, 4, 8, 16, 32), seed=11, device=0):
    """Preconditioned residuals of point-Jacobi MCSA after each iteration count."""
    import torch

    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=seed,
                      estimator=capi.EXPECTED_VALUE, direction=capi.FORWARD, sample_ratio=1.0,
                      history_length=10)
    n = op.n
    bt = torch.tensor(np.asarray(b, np.float64), device=f"cuda:{device}")
    out = torch.empty((len(iterations), n), dtype=torch.float64, device=bt.device)
    for k, it in enumerate(iterations):
        x = torch.zeros_like(bt)
        dom.mcsa_solve_dev(bt.data_ptr(), x.data_ptr(), tolerance=0.0, max_iters=int(it))
        dom.residual(out[k].data_ptr())
    torch.cuda.synchronize(bt.device)
    dom.close()
    pc.close()
    return out


def training_vectors(ctx, op, b, n_random=8, seed=0, device=0, iterations=(1, 2, 4, 8, 16, 32)):
    """MCSA residual snapshots stacked over random vectors ([R, n], device)."""
    import torch

    res = mcsa_residuals(ctx, op, b, iterations=iterations, seed=seed + 11, device=device)
    g = torch.Generator(device=f"cuda:{device}")
    g.manual_seed(seed)
    rnd = torch.randn((n_random, op.n), dtype=torch.float64, device=res.device, generator=g)
    return torch.cat([res, rnd], 0).contiguous()


def onpolicy_vectors(net, op, count, iters, generator, device=0):
    """`count` random vectors smoothed by `iters` steps of the current
    I - M A: the modes the learned-preconditioner iteration (and so MCSA
    with it) leaves behind, i.e. its residual history from random starts."""
    import torch

    V = torch.randn((count, op.n), dtype=torch.float64, device=f"cuda:{device}",
                    generator=generator)
    net.smooth_vectors(op, V.data_ptr(), count, iters)
    return V


def train(net, samples, steps, lr=2e-3, lr_final=2e-4, grad_clip=0.0, log_every=0,
          refresh=0, adv_count=4, adv_iters=30, seed=0, device=0):
    """Adam over the (operator, vectors) samples in round robin with a
    cosine-decayed step size.  With refresh > 0, every `refresh` steps each
    sample also gets `adv_count` on-policy vectors (onpolicy_vectors) from
    the network as it stands, stacked over its fixed vectors.  Returns the
    per-step losses."""
    import torch

    gen = torch.Generator(device=f"cuda:{device}")
    gen.manual_seed(seed)
    adv = [None] * len(samples)
    losses = []
    for k in range(steps):
        j = k % len(samples)
        op, V = samples[j]
        if refresh > 0:
            if adv[j] is None or k % refresh < len(samples):
                adv[j] = torch.cat([onpolicy_vectors(net, op, adv_count, adv_iters, gen, device),
                                    V], 0).contiguous()
            V = adv[j]
        t = k / max(steps - 1, 1)
        step_lr = lr_final + 0.5 * (lr - lr_final) * (1.0 + np.cos(np.pi * t))
        loss = net.train_step(op, V.data_ptr(), V.shape[0], lr=step_lr, grad_clip=grad_clip)
        losses.append(loss)
        if log_every and k % log_every == 0:
            print(f"spai step {k}: loss {loss:.6f} lr {step_lr:.2e}", flush=True)
    return losses
