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

import json

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


def time_inference(ctx, net, grid, reps, device=0):
    """Device time of the forward MLP kernel over every row of a grid^3
    variable-coefficient diffusion operator (M values on A's pattern and the
    raw outputs into device arrays), after two warm-up launches."""
    import torch

    from . import problems as P

    A, _ = P.diffusion3d_varcoef(grid, seed=1)
    op = capi.Operator(ctx, A)
    n, nnz = A.shape[0], A.nnz
    dev = f"cuda:{device}"
    mv = torch.empty(nnz, dtype=torch.float64, device=dev)
    out = torch.empty((n, 16), dtype=torch.float32, device=dev)
    for _ in range(2):
        net.infer_dev(op, out.data_ptr(), mv.data_ptr())
    ms = [net.infer_dev(op, out.data_ptr(), mv.data_ptr()) for _ in range(reps)]
    per = float(np.mean(ms))
    # Bytes a row must move: its stencil values by diagonal (K x 8) and CSR
    # row pointer and columns (4 + 4 per entry) in, M on its pattern (8 per
    # entry) and the raw outputs (16 x 4) out.
    k = nnz / n
    row_bytes = 8 * k + 4 + 4 * k + 8 * k + 64
    flops = 2 * (16 * 64 + 64 * 64 + 64 * 16)
    op.close()
    return {"rows": n, "forward_ms": per, "rows_per_s": n / (per * 1e-3),
            "tflops": flops * n / (per * 1e-3) / 1e12, "bytes_per_row": row_bytes,
            "algorithmic_gbs": row_bytes * n / (per * 1e-3) / 1e9,
            "what": f"k_spai_forward over a {grid}^3 var-coef diffusion operator, mean of {reps} "
                    "launches after 2 warm-up launches"}


def main(argv=None):
    """Train a learned-SPAI network on seeded systems of one family and save
    its parameters (numpy .npy, FP32, the flat order of mclsgpu_spai_*)."""
    import argparse
    import time

    import torch

    from . import problems as P

    ap = argparse.ArgumentParser(prog="python -m mcls_b200.spai")
    ap.add_argument("--family", choices=["diffusion3d", "anisotropic2d"], default="diffusion3d")
    ap.add_argument("--grid", type=int, default=32, help="grid points per axis of each system")
    ap.add_argument("--systems", type=int, default=8)
    ap.add_argument("--steps", type=int, default=2000, help="0: no training (the initial network)")
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--seed", type=int, default=1000)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=None, help="where to save the parameters (.npy)")
    ap.add_argument("--infer-grid", type=int, default=0,
                    help="after training, time inference on an N^3 var-coef diffusion system")
    ap.add_argument("--infer-reps", type=int, default=10)
    args = ap.parse_args(argv)
    ctx = capi.Context(args.device)
    samples, slots = [], None
    t0 = time.perf_counter()
    for k in range(args.systems):
        if args.family == "diffusion3d":
            A, b = P.diffusion3d_varcoef(args.grid, seed=args.seed + k)
        else:
            A, b, _, _ = P.anisotropic2d_sample(args.grid, seed=args.seed + k)
        if slots is None:
            slots = stencil_slots(A)
        if stencil_slots(A) != slots:
            continue
        op = capi.Operator(ctx, A)
        if args.family == "diffusion3d":
            V = training_vectors(ctx, op, b, seed=k, n_random=4, iterations=(1, 4, 16),
                                 device=args.device)
        else:  # point-Jacobi MCSA may diverge on this family: random vectors only
            g = torch.Generator(device=f"cuda:{args.device}")
            g.manual_seed(k)
            V = torch.randn((4, op.n), dtype=torch.float64, device=f"cuda:{args.device}",
                            generator=g)
        samples.append((op, V))
    net = capi.SpaiNet(ctx, slots, seed=0)
    if args.steps > 0:
        losses = train(net, samples, steps=args.steps, lr=args.lr, lr_final=args.lr / 10,
                       refresh=25 if args.steps >= 100 else 0, adv_count=8, adv_iters=50,
                       device=args.device)
        torch.cuda.synchronize()
        print(f"{len(samples)} systems, {args.steps} steps, {time.perf_counter() - t0:.1f} s, "
              f"loss {np.mean(losses[:8]):.4f} -> {np.mean(losses[-8:]):.4f}", flush=True)
    if args.out:
        np.save(args.out, net.params)
    if args.infer_grid:
        print(json.dumps(time_inference(ctx, net, args.infer_grid, args.infer_reps, args.device)),
              flush=True)
    net.close()
    ctx.close()


if __name__ == "__main__":
    main()
