"""MCSA benchmark: time-to-1e-8 (and walk-steps/s) on one B200 per rank.

Workload (default): 3D 7-point variable-coefficient diffusion on 128^3
(2,097,152 unknowns; D log-uniform in [0.1, 10] per cell, absorption 0.01,
b ~ U(0,1), seed 0), point-Jacobi MCSA with the expected-value estimator,
FP32 walks/records/tallies, FP64 residual and update, 2^22 histories per
iteration (Sample Ratio 2), History Length 10, stop at |rp|/|PL b| <= 1e-8.

One step = one full MCSA solve from x = 0 on the same seed (identical work
each step).  `value` = seconds per solve to the tolerance with b and x
resident in HBM (CUDA events on the library stream; lower is better);
`e2e` = the same solves through the host-buffer C-ABI call (H2D of b and x0,
D2H of x inside the timed region).  Walk-steps/s is reported beside it.
Inputs are larger than L2 (working set ~0.4 GB).

Beside the timed solves the line carries: the error of the solution against
the oracle's FP64 conjugate-gradient solve, the FP32 walk's transition
agreement with the FP64 selection on the same draws, and the walk kernel's
HBM roofline on a 192^3 domain whose records exceed L2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mcls_b200|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MCSA time-to-1e-8 residual, learned vs Jacobi precond, one B200; walk-steps/sec"
UNIT = "s"
STEP_UNIT = "walk-steps/s"
CONFIGS = {
    "diffusion128": dict(workload="3D 7-pt variable-coefficient diffusion 128^3, Jacobi MCSA, forward "
                        "expected-value estimator, FP32 walks / FP64 tallies, residual and update, "
                        "2^22 histories per iteration",
               n=128, sample_ratio=2.0, estimator=1, history_length=10, direction=1),
    "blocks256": dict(workload="3D 7-pt diffusion-reaction 256^3, piecewise-constant D in "
                               "[0.5,5] and sigma_a in [0.001,0.1] on 8^3 random blocks, Jacobi "
                               "MCSA, forward expected-value estimator, FP32 walks / FP64 "
                               "tallies, residual and update, 2^24 histories per iteration",
                      n=256, sample_ratio=1.0, estimator=1, history_length=10, direction=1,
                      max_iters=60000),
    "batched": dict(workload="batched: 1024 systems (2D/3D Poisson and var-coef diffusion, N "
                             "log-uniform in [1e3, nmax] on square/cube grids), 1-16 right-hand "
                             "sides uniform(0,1) each, point-Jacobi forward expected-value MCSA, "
                             "FP32 walks shared by all right-hand sides, FP64 residuals, one "
                             "graph-captured loop, per-(system, rhs) convergence to 1e-8",
                    n=0, sample_ratio=1.0, estimator=1, history_length=10, direction=1),
    "poisson100": dict(workload="2D Poisson 5-pt 100x100, Jacobi MCSA, adjoint collision estimator, "
                        "FP64 walks, N histories per iteration, Weight Cutoff 1e-4 with a History "
                        "Length cap of 10",
               n=100, sample_ratio=1.0, estimator=0, history_length=10, direction=0,
               weight_cutoff=1e-4),
    "aniso512": dict(workload="2D anisotropic diffusion 512^2, 9-point stencil of K = R(theta) "
                              "diag(1, 1/a) R(theta)^T (one seeded system with rho(H_Jacobi) > "
                              "0.95), forward expected-value MCSA, FP32 walks / FP64 residual, 2 "
                              "histories per row per iteration: point Jacobi vs block Jacobi "
                              "(4 along x) vs learned SPAI (network trained on 2,000 seeded "
                              "systems of the family)",
                     n=512, sample_ratio=2.0, estimator=1, history_length=10, direction=1,
                     max_iters=100000),
}
# DRAM bytes (read + write) of one walk launch on each workload: ncu's
# dram__bytes_read.sum (83.90 MB) + dram__bytes_write.sum (7.82 MB) for the
# stencil forward expected-value walk32 launch at 128^3.
WALK_DRAM_BYTES_PER_LAUNCH = {"diffusion128": 91.72e6}
# The same for one walk32 launch of the 192^3 roofline domain (226 MB of
# records, more than L2): dram__bytes_read.sum (283.14 MB) +
# dram__bytes_write.sum (47.17 MB) of the 4-histories-per-lane x 256 launch
# (python -m mcls_b200.walkprof --n 192 --solves 2 --histories-per-lane 4).
HBM_WALK_DRAM_BYTES_PER_LAUNCH = 330.31e6
# The same capture's L2 and DRAM figures: what binds the walk (L2 throughput
# and latency, the records read from HBM about once per launch).
HBM_WALK_NCU = {"lts_throughput_pct_of_peak": 64.1, "lts_sector_hit_pct": 87.3,
                "dram_throughput_pct_of_peak": 8.8, "top_stall": "long scoreboard (L2 loads)",
                "capture": "ncu --set full, one walk32 launch, 192^3, 4 histories per lane x 256"}
# The oracle port's whole MCSA solve of a workload, run once to the end
# (FP64 forward expected-value walks on the counter stream, the workload's
# histories per iteration, seed 1234): its iteration count, which the
# reference arm multiplies by its timed seconds per iteration.
CPU_FULL_SOLVE = {
    "diffusion128": {"iterations": 6002,
                     "note": "run once to the tolerance on the 8-thread build container in "
                             "2,843 s: |b - A x|/|b| = 3.40e-8, error against the oracle CG "
                             "3.94e-8"},
}


def step_bytes(cfg, info):
    """Bytes one FP32 walk step must move: its state's record, plus (adjoint)
    an 8 B FP64 tally read-modify-write.

    Packed records hold k (CDF, column|sign) pairs and a {W, tally source}
    header; stencil records hold the header and one signed CDF slot per
    stencil offset (3D 7-point Jacobi: 2 + 6 words = 32 B).  The forward tally
    source rides in the record header, so the forward step is the record.
    """
    rec = info["record_bytes"]
    return rec if CONFIGS[cfg]["direction"] == 1 else rec + 16


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = self.rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def make_system(cfg):
    from mcls_b200 import problems as P

    c = CONFIGS[cfg]
    if cfg == "diffusion128":
        A, b = P.diffusion3d_varcoef(c["n"], seed=0)
    elif cfg == "blocks256":
        A, b = P.diffusion3d_blocks(c["n"], 8, seed=0)
    else:
        A = P.poisson2d(c["n"])
        b = np.ones(A.shape[0])
    return A, b


def dist_init(args):
    from mcls_b200 import dist

    return dist.init("nccl")


def barrier(pg):
    from mcls_b200 import dist

    dist.barrier(pg)


def allmax(pg, v):
    from mcls_b200 import dist

    return dist.allmax(pg, v)


def allsum(pg, v):
    from mcls_b200 import dist

    return dist.allsum(pg, v)


def _learned_threshold_run(args, ctx, op, pc, A, b, cfgd, thr, jacobi_ms):
    """Learned-SPAI MCSA with the composite operator M A filtered at `thr`
    ("Composite Operator Threshold": entries |v| <= thr * row max dropped
    before the domain is built), timed like the main learned solve."""
    import torch

    from mcls_b200 import capi

    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=args.seed,
                      estimator=cfgd["estimator"], sample_ratio=cfgd["sample_ratio"],
                      direction=cfgd["direction"], history_length=cfgd["history_length"],
                      composite_threshold=thr)
    mp = capi.mcsa_params(tolerance=1e-8, max_iters=args.max_iters)
    bt = torch.tensor(b, device=ctx_device(), dtype=torch.float64)
    xt = torch.zeros_like(bt)
    dom.autotune(bt.data_ptr(), reps=1)
    stats = []
    for k in range(1 + args.steps):
        dom.reseed(args.seed)
        xt.zero_()
        torch.cuda.synchronize()
        st = dom.mcsa_solve_dev(bt.data_ptr(), xt.data_ptr(), params=mp)
        if k >= 1:
            stats.append(st)
    ms = sum(s["solve_ms"] for s in stats) / len(stats)
    info = dom.info()
    out = {"composite_threshold": thr, "time_to_1e-8_s": ms / 1e3,
           "iterations": stats[-1]["iterations"], "converged": bool(stats[-1]["converged"]),
           "record_bytes": info["record_bytes"], "h_entries_per_row": info["max_row_entries"],
           "stencil_offsets": info["stencil_offsets"],
           "rel_residual_b_minus_Ax": float(np.linalg.norm(b - A @ xt.cpu().numpy()) /
                                            np.linalg.norm(b)),
           "speedup_vs_jacobi": jacobi_ms / ms}
    dom.close()
    return out


def learned_arm(args, ctx, op, A, b, cfgd, jacobi_ms):
    """Learned-SPAI MCSA on the same system: train the per-row network on the
    GPU (untimed set-up, reported), build the learned preconditioner and its
    domain, then time the same MCSA solve as the Jacobi arm."""
    import torch

    from mcls_b200 import capi
    from mcls_b200 import problems as P
    from mcls_b200 import spai

    t0 = time.perf_counter()
    samples = []
    for seed in range(8):
        if args.config == "blocks256":
            At, bt_ = P.diffusion3d_blocks(32, 4, seed=1000 + seed)
        else:
            At, bt_ = P.diffusion3d_varcoef(32, seed=1000 + seed)
        opt = capi.Operator(ctx, At)
        samples.append((opt, spai.training_vectors(ctx, opt, bt_, seed=seed, n_random=4,
                                                   iterations=(1, 4, 16))))
    net = capi.SpaiNet(ctx, spai.stencil_slots(A), seed=0)
    losses = spai.train(net, samples, steps=args.spai_steps, lr=3e-3, lr_final=3e-4,
                        refresh=25, adv_count=8, adv_iters=50)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    rl, rj = net.rho(op, iters=300)
    gate = {} if args.learned_rho_fallback is None else {"rho_fallback": args.learned_rho_fallback}
    pc = capi.Precond(ctx, op, capi.PREC_LEARNED_SPAI, net=net, **gate)
    thresholds = [float(t) for t in args.learned_threshold.split(",")]
    sweep = []
    for thr in thresholds[1:]:
        sweep.append(_learned_threshold_run(args, ctx, op, pc, A, b, cfgd, thr, jacobi_ms))
    mp = capi.mcsa_params(tolerance=1e-8, max_iters=args.max_iters,
                          host_loop=1 if args.host_loop else 0)
    bt = torch.tensor(b, device=ctx_device(), dtype=torch.float64)
    xt = torch.zeros_like(bt)
    # The FP32 stencil records of the 25-offset learned H (128 bytes) are timed
    # once beside the reported 16-bit-threshold records (64 bytes).
    fp32_rec = None
    if args.learned_format == "stencil16":
        d32 = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER,
                          seed=args.seed, estimator=cfgd["estimator"],
                          sample_ratio=cfgd["sample_ratio"], direction=cfgd["direction"],
                          history_length=cfgd["history_length"],
                          composite_threshold=thresholds[0], record_format=capi.RECORD_STENCIL)
        d32.autotune(bt.data_ptr(), reps=1)
        for k in range(2):
            d32.reseed(args.seed)
            xt.zero_()
            torch.cuda.synchronize()
            s32 = d32.mcsa_solve_dev(bt.data_ptr(), xt.data_ptr(), params=mp)
        fp32_rec = {"record_bytes": d32.info()["record_bytes"],
                    "time_to_1e-8_s": s32["solve_ms"] / 1e3, "iterations": s32["iterations"],
                    "walk_ms_per_launch": s32["walk_ms"] / max(s32["walk_launches"], 1),
                    "speedup_vs_jacobi": jacobi_ms / s32["solve_ms"]}
        d32.close()
    fmt = capi.RECORD_STENCIL16 if args.learned_format == "stencil16" else capi.RECORD_AUTO
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=args.seed,
                      estimator=cfgd["estimator"], sample_ratio=cfgd["sample_ratio"],
                      direction=cfgd["direction"], history_length=cfgd["history_length"],
                      composite_threshold=thresholds[0], record_format=fmt)
    tuned = dom.autotune(bt.data_ptr(), reps=1)
    stats = []
    for k in range(1 + args.steps):
        dom.reseed(args.seed)
        xt.zero_()
        torch.cuda.synchronize()
        st = dom.mcsa_solve_dev(bt.data_ptr(), xt.data_ptr(), params=mp)
        if k >= 1:
            stats.append(st)
    ms = sum(s["solve_ms"] for s in stats) / len(stats)
    steps = sum(s["walk_steps"] for s in stats)
    rel = float(np.linalg.norm(b - A @ xt.cpu().numpy()) / np.linalg.norm(b))
    info = dom.info()
    out = {"time_to_1e-8_s": ms / 1e3, "iterations": stats[-1]["iterations"],
           "converged": bool(stats[-1]["converged"]),
           "walk_steps_per_s": steps / (sum(s["solve_ms"] for s in stats) * 1e-3),
           "walk_ms_per_launch": sum(s["walk_ms"] for s in stats) /
                                 max(sum(s["walk_launches"] for s in stats), 1),
           "rel_residual_b_minus_Ax": rel, "rho_learned": rl, "rho_jacobi": rj,
           "fallback_taken": bool(stats[-1]["fallback_taken"]),
           "record_bytes": info["record_bytes"], "record_format": info["record_format"],
           "h_entries_per_row": info["max_row_entries"], "walk_launch": tuned,
           "train_s": train_s, "train_steps": args.spai_steps, "train_loss_first": float(np.mean(losses[:8])),
           "train_loss_last": float(np.mean(losses[-40:])),
           "train_systems": ("8 x 3D 7-pt diffusion-reaction 32^3 on 4^3 random blocks "
                             "(seeds 1000-1007)" if args.config == "blocks256" else
                             "8 x 3D 7-pt var-coef diffusion 32^3 (seeds 1000-1007)"),
           "speedup_vs_jacobi": jacobi_ms / ms,
           "composite_threshold": thresholds[0],
           "gate": {"rule": "point Jacobi replaces the learned M when rho(I - M A) >= 0.95 "
                            "and >= the Jacobi rho (both by 300 power iterations)",
                    "fell_back": bool(stats[-1]["fallback_taken"]),
                    "literal_rule": "rho >= 0.95 alone",
                    "literal_would_fall_back": bool(rl >= 0.95)}}
    if fp32_rec:
        out["fp32_stencil_records"] = fp32_rec
    if sweep:
        out["threshold_sweep"] = sweep
    if not args.no_anderson:
        M = pc.to_scipy(A.shape[0])
        depths = [int(d) for d in args.anderson_depth.split(",")]
        # The further seeds for the deepest store only (the accelerated arm).
        out["anderson"] = [anderson_arm(args, d, dom, bt, xt, A, b, args.seed, jacobi_ms, PL=M,
                                        seeds=args.learned_anderson_seeds
                                        if d == max(depths) else "")
                           for d in depths]
    dom.close()
    pc.close()
    net.close()
    return out


def anderson_arm(args, depth, dom, bt, xt, A, b, seed, jacobi_ms, PL=None, seeds=None):
    """Anderson-accelerated MCSA (the "Adjoint/Forward Anderson" managers) on
    an MCSA arm's domain and right-hand side: one untimed warm-up solve, then
    the timed solves, each from x = 0 on the same random stream.  PL: the
    domain's left preconditioner as a scipy matrix (point Jacobi if None)."""
    import torch

    # The Anderson status test divides by |b|_2, MCSA's by |PL b|_2; the
    # tolerance below stops both at the same |PL (b - A x)|_2.
    apply_pl = (lambda v: PL @ v) if PL is not None else (lambda v: v / A.diagonal())
    tol = 1e-8 * float(np.linalg.norm(apply_pl(b)) / np.linalg.norm(b))
    stats = []
    for k in range(1 + args.steps):
        dom.reseed(seed)
        xt.zero_()
        torch.cuda.synchronize()
        st = dom.anderson_solve_dev(bt.data_ptr(), xt.data_ptr(), tolerance=tol,
                                    max_iters=args.max_iters,
                                    storage_depth=depth, mixing=args.anderson_mixing,
                                    host_loop=1 if args.host_loop else 0)
        if k >= 1:
            stats.append(st)
    ms = sum(s["solve_ms"] for s in stats) / len(stats)
    rel = float(np.linalg.norm(b - A @ xt.cpu().numpy()) / np.linalg.norm(b))
    sweep = []
    for sd in [int(v) for v in (args.anderson_seeds if seeds is None else seeds).split(",") if v]:
        # One solve per further seed of the random stream: the spread of the
        # stochastic fixed-point map's acceleration.
        dom.reseed(sd)
        xs = torch.zeros_like(xt)
        torch.cuda.synchronize()
        sst = dom.anderson_solve_dev(bt.data_ptr(), xs.data_ptr(), tolerance=tol,
                                     max_iters=args.max_iters, storage_depth=depth,
                                     mixing=args.anderson_mixing,
                                     host_loop=1 if args.host_loop else 0)
        sweep.append({"seed": sd, "iterations": sst["iterations"],
                      "converged": bool(sst["converged"]),
                      "time_to_1e-8_s": sst["solve_ms"] / 1e3,
                      "speedup_vs_jacobi_mcsa": jacobi_ms / sst["solve_ms"] if jacobi_ms else None})
    out_seeds = {"seeds": sweep} if sweep else {}
    return {"time_to_1e-8_s": ms / 1e3, "iterations": stats[-1]["iterations"],
            "converged": bool(stats[-1]["converged"]), "storage_depth": depth,
            "mixing": args.anderson_mixing, **out_seeds,
            "criterion": "|PL (b - A x)|_2 < tol |b|_2, tol = 1e-8 |PL b|_2 / |b|_2 "
                         "(the MCSA arm's |PL (b - A x)|_2 <= 1e-8 |PL b|_2)",
            "tolerance": tol,
            "rel_prec_residual": float(np.linalg.norm(apply_pl(b - A @ xt.cpu().numpy())) /
                                       np.linalg.norm(apply_pl(b))),
            "walk_steps_per_s": sum(s["walk_steps"] for s in stats) /
                                (sum(s["solve_ms"] for s in stats) * 1e-3),
            "rel_residual_b_minus_Ax": rel,
            "speedup_vs_jacobi_mcsa": jacobi_ms / ms if jacobi_ms else None}


def partition_arm(args, ctx, A, b):
    """One adjoint-collision Monte Carlo solve (FP32 packed records, the
    Jacobi-preconditioned source) on the whole domain and on P row parts on
    this GPU (domain-decomposed transport: rounds of walks with the crossing
    histories handed between the parts).  Same histories, same transitions;
    the difference is the cost of the rounds and the hand-over."""
    import torch

    from mcls_b200 import capi, partition

    P = args.partition_parts
    n = A.shape[0]
    dinv = 1.0 / A.diagonal()
    mc = dict(precision=capi.FP32, rng_mode=capi.RNG_COUNTER, direction=capi.ADJOINT,
              estimator=capi.COLLISION, history_length=10, sample_ratio=1.0,
              record_format=capi.RECORD_PACKED, seed=args.seed)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, **mc)
    rt = torch.tensor(dinv * b, device=ctx_device(), dtype=torch.float64)
    xt = torch.zeros_like(rt)
    T = partition.transposed_composite(A, dinv)
    bounds = partition.row_bounds(n, P)
    parts = [partition.DevicePart(capi.Subdomain(ctx, n, bounds, q, T[bounds[q]:bounds[q + 1]],
                                                 params=capi.mc_params(**mc)),
                                  n // P + n // 4 + 1024, ctx_device())
             for q in range(P)]
    whole_ms, part_ms, steps, rounds, moved = [], [], 0, 0, 0
    for k in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        st = dom.mc_solve_dev(rt.data_ptr(), xt.data_ptr(), internal=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        xp, rounds, moved, steps = partition.solve_local(parts, rt)
        torch.cuda.synchronize()
        if k >= args.warmup:
            whole_ms.append(st["solve_ms"])
            part_ms.append((time.perf_counter() - t0) * 1e3)
    err = float((xp - xt).abs().max() / xt.abs().max())
    wm, pm = sum(whole_ms) / len(whole_ms), sum(part_ms) / len(part_ms)
    out = {"parts": P, "histories": int(st["histories"]), "walk_steps": int(steps),
           "whole_ms": wm, "parts_ms": pm, "whole_steps_per_s": steps / (wm * 1e-3),
           "parts_steps_per_s": steps / (pm * 1e-3), "rounds": rounds,
           "histories_handed_over": moved, "max_rel_diff_vs_whole": err,
           "timing": "whole: device time of the library call; parts: wall time of the "
                     "host-driven rounds (synchronised)"}
    for p in parts:
        p.sub.close()
    dom.close()
    pc.close()
    op.close()
    return out


def run_batched(args, world, rank, local, pg):
    """Batched workload: every step solves all (system, rhs) pairs to 1e-8."""
    import torch

    from mcls_b200 import capi
    from mcls_b200 import problems as P

    cfgd = CONFIGS["batched"]
    torch.cuda.set_device(local)
    systems, nrhs, rhs, kinds = P.batch_sample(args.batch_systems, 1e3, args.batch_nmax,
                                               seed=rank)
    ctx = capi.Context(local)
    seed = args.seed + rank
    bt = capi.Batch(ctx, systems, nrhs, direction=capi.FORWARD, estimator=cfgd["estimator"],
                    precision=capi.FP32, sample_ratio=cfgd["sample_ratio"],
                    history_length=cfgd["history_length"], seed=seed)
    Bh = bt.pack(rhs)
    B = torch.tensor(Bh, device=f"cuda:{local}").contiguous()
    X = torch.zeros_like(B)
    tuned = bt.autotune(B.data_ptr(), X.data_ptr(), reps=3)
    mp = capi.mcsa_params(tolerance=1e-8, max_iters=args.max_iters,
                          host_loop=1 if args.host_loop else 0)

    def step():
        bt.reseed(seed)
        X.zero_()
        torch.cuda.synchronize()
        return bt.mcsa_solve_dev(B.data_ptr(), X.data_ptr(), params=mp)

    for _ in range(args.warmup):
        step()
    clocks = ClockSampler(local)
    barrier(pg)
    torch.cuda.synchronize()
    clocks.start()
    t0 = time.perf_counter()
    res = [step() for _ in range(args.steps)]
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    barrier(pg)
    clk = clocks.stop()
    stats = [r[0] for r in res]
    dev_ms = sum(s["solve_ms"] for s in stats)
    dev_ms_max = allmax(pg, dev_ms)
    steps_all = allsum(pg, sum(s["walk_steps"] for s in stats))
    steps_per_s = steps_all / (dev_ms_max * 1e-3)
    # End to end: host right-hand sides in, host solutions out, every step.
    pinned_b = torch.tensor(Bh).pin_memory()
    pinned_x = torch.empty_like(pinned_b).pin_memory()
    e2e_ms = 0.0
    e2e_steps = 0
    barrier(pg)
    for _ in range(args.steps):
        bt.reseed(seed)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        B.copy_(pinned_b, non_blocking=True)
        X.zero_()
        st, _, _ = bt.mcsa_solve_dev(B.data_ptr(), X.data_ptr(), params=mp)
        pinned_x.copy_(X, non_blocking=True)
        torch.cuda.synchronize()
        e2e_ms += (time.perf_counter() - t1) * 1e3
        e2e_steps += st["walk_steps"]
    e2e_ms = allmax(pg, e2e_ms)
    e2e_steps_per_s = allsum(pg, e2e_steps) / (e2e_ms * 1e-3)
    s0, it, rr = res[-1]
    pairs = int(sum(nrhs))
    info = bt.domain_info()
    peak, peak_kind = load_peaks()
    walk_ms = sum(s["walk_ms"] for s in stats)
    launches = sum(s["walk_launches"] for s in stats)
    per_launch = walk_ms / max(launches, 1)
    # A step reads the record and its state's FP32 tally-source row (the
    # history's width class): the mean over histories of the row widths.
    mean_w = float((bt.n * bt.widths).sum()) / bt.rows
    bstep = info["record_bytes"] + 4 * mean_w
    walk_steps = sum(s["walk_steps"] for s in stats)
    achieved = (bstep * walk_steps / max(launches, 1)) / (per_launch * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": dev_ms_max / args.steps / 1e3, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": cfgd["workload"].replace("nmax", f"{args.batch_nmax:g}"),
                   "systems": args.batch_systems, "rows": bt.rows, "elements": bt.elements,
                   "max_rhs_width": bt.width, "mean_row_width": mean_w,
                   "pairs": pairs, "kinds": {k: kinds.count(k) for k in sorted(set(kinds))},
                   "parallelism": f"replicas x{world}" if world > 1 else "single batch",
                   "l2": "inputs larger than L2 (no flush)", "tolerance": 1e-8,
                   "max_iters": args.max_iters},
        "results": {"walk_launch": tuned, "time_to_1e-8_s": dev_ms_max / args.steps / 1e3,
                    "iterations": s0["iterations"], "pairs_converged": int((it >= 0).sum()),
                    "max_rel_residual": float(rr.max()), "walk_steps_per_s": steps_per_s,
                    "e2e_walk_steps_per_s": e2e_steps_per_s,
                    "median_pair_iterations":
                        float(np.median(it[it >= 0])) if (it >= 0).any() else None},
        "clocks": clk,
        "e2e": {"value": e2e_ms / args.steps / 1e3, "unit": UNIT,
                "h2d_bytes_per_step": int(Bh.nbytes), "d2h_bytes_per_step": int(Bh.nbytes)},
        "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "traffic": None,
                     "kernel": "walk32_multi", "peak_kind": peak_kind, "bytes_per_step": bstep,
                     "walk_ms_per_launch": per_launch,
                     "walk_share_of_solve": walk_ms / dev_ms if dev_ms else None},
        "wall_s": wall,
    }
    if rank == 0 and world == 1:
        line["results"]["err_vs_oracle"] = batch_oracle_error(bt, systems, rhs, X.cpu().numpy())
    if rank == 0:
        print(json.dumps(line))
    bt.close()
    ctx.close()


def oracle_error(A, b, x):
    """Relative error of x against the oracle's FP64 solve (diagonal-
    preconditioned conjugate gradients to |b - A x| <= 1e-12 |b|, all host
    threads), computed after the timed region as the checker."""
    from oracle import oracle as O

    O.set_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    r = O.pcg(O.Csr.from_scipy(A), b, tolerance=1e-12)
    secs = time.perf_counter() - t0
    xo = r["x"]
    return {"rel_error": float(np.linalg.norm(x - xo) / np.linalg.norm(xo)),
            "max_abs_error_rel": float(np.abs(x - xo).max() / np.abs(xo).max()),
            "oracle": "FP64 diagonal-preconditioned conjugate gradients (oracle/), "
                      "|b - A x_o|_2 <= 1e-12 |b|_2",
            "oracle_rel_residual": r["rel_residual"], "oracle_iterations": r["iters"],
            "oracle_s": secs}


def batch_oracle_error(bt, systems, rhs, X, sample_systems=8, sample_rhs=4):
    """Relative errors of the batch's solutions against the oracle's FP64
    solves of a sample of its pairs: `sample_systems` systems spaced evenly
    through the batch, their first `sample_rhs` right-hand sides each
    (diagonal-preconditioned conjugate gradients to 1e-12, all host threads;
    every system of the batch is symmetric positive definite)."""
    from oracle import oracle as O

    O.set_threads(os.cpu_count() or 1)
    blocks = bt.unpack(X)
    pick = sorted(set(np.linspace(0, len(systems) - 1, sample_systems).round().astype(int)))
    errs, rows = [], 0
    t0 = time.perf_counter()
    for s in pick:
        A = O.Csr.from_scipy(systems[s])
        rs = np.asarray(rhs[s]).reshape(systems[s].shape[0], -1)
        for r in range(min(sample_rhs, rs.shape[1])):
            xo = O.pcg(A, rs[:, r], tolerance=1e-12)["x"]
            errs.append(float(np.linalg.norm(blocks[s][:, r] - xo) / np.linalg.norm(xo)))
        rows += systems[s].shape[0]
    return {"max_rel_error": max(errs), "median_rel_error": float(np.median(errs)),
            "pairs_checked": len(errs), "systems_checked": len(pick), "rows_checked": rows,
            "sample": f"{len(pick)} systems spaced evenly through the batch, their first "
                      f"{sample_rhs} right-hand sides",
            "oracle": "FP64 diagonal-preconditioned conjugate gradients (oracle/), "
                      "|b - A x_o|_2 <= 1e-12 |b|_2", "oracle_s": time.perf_counter() - t0}


def walk_agreement(dom, histories, seed):
    """FP32 walk selections against the FP64 selections of the same draws."""
    hd, td = dom.walk_agreement(histories, seed=seed)
    L = dom.p.history_length
    return {"histories": histories, "transitions": histories * L,
            "histories_differing": hd, "transitions_differing": td,
            "history_rate": hd / histories, "transition_rate": td / (histories * L),
            "what": "history e starts at state e mod n on its counter stream; each transition "
                    "is selected by lower_bound over the FP64 CDF with the 53-bit uniform of "
                    "the draw (the reference's sampling) and, on the same draw, by the "
                    "production FP32 record search with its 24-bit uniform"}


def hbm_walk_roofline(args, ctx, n=192, reps=10):
    """walk32 on a domain whose records exceed L2: 3D 7-point var-coef
    diffusion n^3 (records 32 B x n^3: 226 MB at 192^3 against 126 MB of L2),
    Jacobi, forward expected value, 2 histories per row of 10 steps.  One
    Monte Carlo solve per repetition; the walk's launch time comes from the
    library's device timer (CUDA events, library stream)."""
    import torch

    from mcls_b200 import capi
    from mcls_b200 import problems as P

    A, b = P.diffusion3d_varcoef(n, seed=1)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=args.seed,
                      estimator=capi.EXPECTED_VALUE, sample_ratio=2.0, direction=capi.FORWARD,
                      history_length=10)
    rt = torch.tensor((1.0 / A.diagonal()) * b, device=ctx_device(), dtype=torch.float64)
    xt = torch.zeros_like(rt)
    torch.cuda.synchronize()
    tuned = dom.autotune(rt.data_ptr(), reps=2)
    for _ in range(3):
        dom.mc_solve_dev(rt.data_ptr(), xt.data_ptr(), internal=True)
    walk_ms = steps = launches = 0
    for _ in range(reps):
        st = dom.mc_solve_dev(rt.data_ptr(), xt.data_ptr(), internal=True)
        walk_ms += st["walk_ms"]
        steps += st["walk_steps"]
        launches += st["walk_launches"]
    info = dom.info()
    per_launch_ms = walk_ms / max(launches, 1)
    bstep = info["record_bytes"]
    bytes_per_launch = bstep * steps / max(launches, 1)
    dom.close()
    pc.close()
    op.close()
    return {"per_launch_ms": per_launch_ms, "bytes_per_launch": bytes_per_launch,
            "bytes_per_step": bstep, "steps_per_launch": steps / max(launches, 1),
            "records_bytes": bstep * A.shape[0], "walk_launch": tuned,
            "workload": f"walk32 alone: 3D 7-pt var-coef diffusion {n}^3 ({A.shape[0]} rows, "
                        f"{bstep * A.shape[0] / 1e6:.0f} MB of 32-byte stencil records, more "
                        f"than the 126 MB L2), Jacobi, forward expected value, 2 histories of "
                        f"10 steps per row, {reps} launches after 3 warm-up launches"}


def _aniso_solve(args, ctx, op, A, b, kind, cfgd, net=None, block=4, rho_fallback=2.0,
                 record_format=0, anderson_depth=0):
    """One timed MCSA solve of the anisotropic system (after one warm-up
    solve), and with anderson_depth the Anderson-accelerated solve on the same
    domain; divergence (non-finite weights or residual) is reported, not
    raised."""
    import torch

    from mcls_b200 import capi

    pc = capi.Precond(ctx, op, kind, block_size=block, net=net, rho_fallback=rho_fallback)

    def domain(fmt):
        return capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER,
                           seed=args.seed, estimator=cfgd["estimator"],
                           sample_ratio=cfgd["sample_ratio"], direction=cfgd["direction"],
                           history_length=cfgd["history_length"], record_format=fmt)

    try:
        dom = domain(record_format)
    except capi.MclsError as e:
        # More column offsets than 16-bit stencil records hold: the library's
        # own choice (FP32 stencil or packed records).
        if e.code != capi.ERR_UNSUPPORTED or record_format == capi.RECORD_AUTO:
            raise
        dom = domain(capi.RECORD_AUTO)
    mp = capi.mcsa_params(tolerance=1e-8, max_iters=args.max_iters)
    bt = torch.tensor(b, device=ctx_device(), dtype=torch.float64)
    xt = torch.zeros_like(bt)
    info = dom.info()
    out = {"record_bytes": info["record_bytes"], "record_format": info["record_format"]}
    try:
        for _ in range(2):
            dom.reseed(args.seed)
            xt.zero_()
            torch.cuda.synchronize()
            st = dom.mcsa_solve_dev(bt.data_ptr(), xt.data_ptr(), params=mp)
        x = xt.cpu().numpy()
        out.update({"converged": bool(st["converged"]), "iterations": st["iterations"],
                    "time_to_1e-8_s": st["solve_ms"] / 1e3 if st["converged"] else None,
                    "achieved_tol": st["achieved_tol"], "x": x,
                    "rel_residual_b_minus_Ax": float(np.linalg.norm(b - A @ x) /
                                                     np.linalg.norm(b)),
                    "walk_ms_per_launch": st["walk_ms"] / max(st["walk_launches"], 1)})
        if anderson_depth:
            try:
                aa = anderson_arm(args, anderson_depth, dom, bt, xt, A, b, args.seed,
                                  st["solve_ms"] if st["converged"] else None,
                                  PL=pc.to_scipy(A.shape[0]))
                aa["speedup_vs_this_mcsa"] = aa.pop("speedup_vs_jacobi_mcsa")
            except capi.MclsError as e:
                aa = {"converged": False, "storage_depth": anderson_depth, "error": str(e)}
            out["anderson"] = aa
    except capi.MclsError as e:
        out.update({"converged": False, "diverged": e.code == capi.ERR_DIVERGED,
                    "error": str(e), "time_to_1e-8_s": None})
    dom.close()
    pc.close()
    return out


def run_aniso(args, world, rank, local, pg):
    """The learned-preconditioner workload: train on 2,000 seeded systems of
    the family (32^2 grids, GPU kernels), then solve one seeded 512^2 system
    with point Jacobi, block Jacobi and the learned SPAI."""
    import torch

    from mcls_b200 import capi
    from mcls_b200 import problems as P
    from mcls_b200 import spai

    cfgd = CONFIGS["aniso512"]
    torch.cuda.set_device(local)
    ctx = capi.Context(local)
    # the solved system: the first seed from 7 whose Jacobi rho exceeds 0.95
    seed = 7
    while True:
        A, b, ratio, theta = P.anisotropic2d_sample(cfgd["n"], seed=seed)
        op = capi.Operator(ctx, A)
        probe = capi.SpaiNet(ctx, spai.stencil_slots(A), seed=0)
        _, rj = probe.rho(op, iters=300)
        probe.close()
        if rj > 0.95:
            break
        op.close()
        seed += 1
    slots = spai.stencil_slots(A)
    t0 = time.perf_counter()
    samples = []
    g = torch.Generator(device=ctx_device())
    g.manual_seed(0)
    for k in range(args.aniso_train_systems):
        At, _, _, _ = P.anisotropic2d_sample(32, seed=10000 + k)
        if spai.stencil_slots(At) != slots:
            continue
        opt = capi.Operator(ctx, At)
        V = torch.randn((4, opt.n), dtype=torch.float64, device=ctx_device(), generator=g)
        samples.append((opt, V))
    net = capi.SpaiNet(ctx, slots, seed=0)
    if args.spai_penalty > 0:
        net.set_penalty(args.spai_penalty, 1.0)
    losses = spai.train(net, samples, steps=args.aniso_train_steps, lr=3e-3, lr_final=3e-4,
                        refresh=25, adv_count=4, adv_iters=30)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    rl, rj = net.rho(op, iters=300)
    arms = {"jacobi": _aniso_solve(args, ctx, op, A, b, capi.PREC_POINT_JACOBI, cfgd),
            "block_jacobi": _aniso_solve(args, ctx, op, A, b, capi.PREC_BLOCK_JACOBI, cfgd,
                                         record_format=capi.RECORD_STENCIL16),
            "learned_spai": _aniso_solve(args, ctx, op, A, b, capi.PREC_LEARNED_SPAI, cfgd,
                                         net=net, record_format=capi.RECORD_STENCIL16,
                                         anderson_depth=0 if args.no_anderson else 6)}
    from oracle import oracle as O

    O.set_threads(os.cpu_count() or 1)
    ref = O.pcg(O.Csr.from_scipy(A), b, tolerance=1e-12)
    for arm in arms.values():
        x = arm.pop("x", None)
        if x is not None:
            arm["err_vs_oracle"] = float(np.linalg.norm(x - ref["x"]) / np.linalg.norm(ref["x"]))
    lt = arms["learned_spai"]["time_to_1e-8_s"]
    jt = arms["jacobi"]["time_to_1e-8_s"]
    line = {"metric": METRIC, "value": lt, "unit": UNIT, "n_gpus": world, "steps": 1,
            "warmup": 1, "ms_per_step": lt * 1e3 if lt else None, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": cfgd["workload"], "n": A.shape[0], "nnz": int(A.nnz),
                       "system_seed": seed, "anisotropy_ratio": ratio, "theta": theta,
                       "tolerance": 1e-8, "l2": "inputs larger than L2 (no flush)"},
            "results": {"arms": arms, "rho_jacobi": rj, "rho_learned": rl,
                        "gate": "disabled for the learned arm (rho_fallback 2): every system of "
                                "this family has rho >= 0.95 at 512^2, so the literal rule "
                                "'rho >= 0.95 falls back' would always take Jacobi",
                        "speedup_vs_jacobi": (jt / lt) if (jt and lt) else None,
                        "train_systems": len(samples), "train_steps": args.aniso_train_steps,
                        "train_grid": "32^2", "train_s": train_s,
                        "train_loss_first": float(np.mean(losses[:20])),
                        "train_loss_last": float(np.mean(losses[-100:])),
                        "oracle": {"solver": "FP64 diagonal-preconditioned CG (oracle/)",
                                   "rel_residual": ref["rel_residual"]}}}
    if rank == 0:
        print(json.dumps(line))
    net.close()
    op.close()
    ctx.close()


def ctx_device():
    import torch

    return f"cuda:{torch.cuda.current_device()}"


def workload_config(args, cfgd, n, nnz, world):
    """The workload as both arms run it (the same dictionary in both lines)."""
    per = int(np.ceil(cfgd["sample_ratio"]))
    hist = n * per if cfgd["direction"] == 1 else int(n * cfgd["sample_ratio"])
    return {"workload": cfgd["workload"], "n": n, "nnz": int(nnz),
            "histories_per_iteration": hist, "history_length": cfgd["history_length"],
            "tolerance": 1e-8, "weight_cutoff": cfgd.get("weight_cutoff", 0.0),
            "stopping_test": "|PL (b - A x)|_2 <= 1e-8 |PL b|_2 (MCSASolverManager's test)",
            "preconditioner": "point Jacobi",
            "parallelism": (f"multi-set x{world}: one set of the histories per GPU, "
                            "corrections summed by an NCCL all-reduce each iteration"
                            if world > 1 else "single domain"),
            "l2": ("inputs fit in L2 (small latency-bound solve; no flush)"
                   if args.config == "poisson100" else "inputs larger than L2 (no flush)")}


# MCSA iterations the CPU port times per sample of each workload.
CPU_SAMPLE_ITERATIONS = {"diffusion128": 8, "blocks256": 2, "poisson100": 0}


def cpu_mcsa(cfg, A, b, iterations, threads, seed=1234):
    """The oracle port's MCSA (FP64 walks on the counter stream, the
    workload's direction, estimator and histories) for `iterations`
    iterations, or to the tolerance when iterations is 0."""
    from oracle import oracle as O

    c = CONFIGS[cfg]
    O.set_threads(threads)
    Ao = O.Csr.from_scipy(A)
    r = O.mcsa_solve(Ao, b, PL=O.point_jacobi(Ao), tolerance=1e-8,
                     max_iters=iterations if iterations else 100000, rng_mode=1, seed=seed,
                     direction=c["direction"], estimator=c["estimator"],
                     sample_ratio=c["sample_ratio"], history_length=c["history_length"],
                     weight_cutoff=c.get("weight_cutoff", 0.0))
    return r


def cpu_time_to_solution(cfg, A, b, threads, gpu_iterations=None, seed=1234):
    """Seconds the port needs to reach the tolerance: the whole solve where it
    ends within a sample (small workloads), else the timed seconds per
    iteration of a sample of iterations times the iteration count of the
    port's own whole solve (CPU_FULL_SOLVE), or the GPU arm's count."""
    k = CPU_SAMPLE_ITERATIONS.get(cfg, 4)
    r = cpu_mcsa(cfg, A, b, k, threads, seed=seed)
    per_iter = r["loop_s"] / max(r["iters"], 1)
    out = {"setup_s": r["setup_s"], "seconds_per_iteration": per_iter,
           "sample_iterations": r["iters"], "walk_steps": int(r["steps"])}
    if k == 0:
        out.update(time_s=r["loop_s"], iterations=r["iters"], converged=bool(r["converged"]),
                   basis="the whole solve, timed")
        return out
    full = CPU_FULL_SOLVE.get(cfg)
    if full:
        n_it, basis = full["iterations"], (f"{r['iters']} timed iterations x the "
                                          f"{full['iterations']} iterations of the port's "
                                          f"whole solve ({full['note']})")
    elif gpu_iterations:
        n_it, basis = gpu_iterations, (f"{r['iters']} timed iterations x the GPU arm's "
                                      f"{gpu_iterations} iterations")
    else:
        n_it, basis = None, f"{r['iters']} timed iterations; no iteration count to project with"
    out.update(time_s=per_iter * n_it if n_it else None, iterations=n_it, basis=basis)
    return out


def cpu_baseline(cfg, A, b, gpu_iterations=None):
    """Oracle port on the host cores, all threads: time-to-1e-8 from a bounded
    sample of MCSA iterations, and its walk-steps/s on the same domain."""
    from oracle import oracle as O

    c = CONFIGS[cfg]
    threads = os.cpu_count() or 1
    t = cpu_time_to_solution(cfg, A, b, threads, gpu_iterations)
    Ao = O.Csr.from_scipy(A)
    mc = O.MC(Ao, PL=O.point_jacobi(Ao), history_length=c["history_length"], rng_mode=1,
              direction=c["direction"], estimator=c["estimator"])
    src = (1.0 / A.diagonal()) * b
    nh = 1 << 18
    steps, secs, _ = mc.bench_walks(src, nh, threads)
    nh2 = int(min(1 << 30, nh * max(1.0, 5.0 / max(secs, 1e-3))))
    steps, secs, _ = mc.bench_walks(src, nh2, threads)
    kind = ("forward " + ("expected-value" if c["estimator"] else "collision")
            if c["direction"] else "adjoint " + ("expected-value" if c["estimator"] else "collision"))
    return {"value": t["time_s"], "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"MCSA on the {A.shape[0]}-row workload, FP64 {kind} walks, "
                      f"{threads} threads: {t['basis']}",
            "mcsa": t,
            "walk_steps_per_s": steps / secs,
            "walk_sample": f"{nh2} {kind} histories x {c['history_length']} steps on the "
                           f"Jacobi domain, {secs:.1f} s"}


def run_reference(args, world, rank, pg):
    if rank != 0:
        return
    if args.config == "batched":
        print(json.dumps({"impl": "reference", "unavailable": "the CPU restatement solves one "
                          "system per call; the batched workload has no single-system "
                          "reference timing"}))
        return
    if args.config == "aniso512":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned "
                          "preconditioner, and its point-Jacobi MCSA does not converge on this "
                          "family (|H| row sums above 1)"}))
        return
    A, b = make_system(args.config)
    cfgd = CONFIGS[args.config]
    threads = os.cpu_count() or 1
    samples = []
    for i in range(args.warmup + args.steps):
        t = cpu_time_to_solution(args.config, A, b, threads, seed=1234 + i)
        if i >= args.warmup:
            samples.append(t)
    per_iter = float(np.mean([t["seconds_per_iteration"] for t in samples]))
    last = samples[-1]
    if last["iterations"] is None:
        print(json.dumps({"impl": "reference", "unavailable": "no iteration count of the "
                          "port's whole solve for this workload"}))
        return
    v = (float(np.mean([t["time_s"] for t in samples])) if CPU_SAMPLE_ITERATIONS.get(
        args.config, 4) == 0 else per_iter * last["iterations"])
    base = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"each step: {last['basis']}; {threads} threads",
            "seconds_per_iteration": per_iter, "iterations": last["iterations"],
            "setup_s": last["setup_s"]}
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": workload_config(args, cfgd, A.shape[0], A.nnz, 1),
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mcls_b200", choices=["mcls_b200", "reference"])
    ap.add_argument("--config", default="diffusion128", choices=sorted(CONFIGS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-hbm-roofline", action="store_true",
                    help="skip the walk roofline on the 192^3 domain whose records exceed L2")
    ap.add_argument("--max-iters", type=int, default=None,
                    help="iteration limit (default: the workload's own, else 20000)")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-learned", action="store_true",
                    help="skip the learned-SPAI arm (training + learned MCSA solves)")
    ap.add_argument("--walk-shape", default=None,
                    help="fixed walk launch shape 'histories_per_lane,block' (skips autotuning)")
    ap.add_argument("--host-loop", action="store_true",
                    help="host-driven MCSA loop (for profilers that cannot see kernels "
                         "inside conditional graph nodes)")
    ap.add_argument("--no-anderson", action="store_true",
                    help="skip the Anderson-accelerated MCSA arm")
    ap.add_argument("--anderson-mixing", type=float, default=1.0,
                    help="Anderson mixing parameter beta (NOX's default 1)")
    ap.add_argument("--anderson-seeds", default="",
                    help="comma-separated further seeds: one Anderson solve each")
    ap.add_argument("--learned-rho-fallback", type=float, default=None,
                    help="the learned preconditioner's rho gate (default: the library's 0.95; "
                         "2 disables it)")
    ap.add_argument("--learned-anderson-seeds", default="777,4242,99,2024",
                    help="further seeds for the Anderson solves on the learned domain")
    ap.add_argument("--anderson-depth", default="2,6",
                    help="Anderson storage depths to time, comma separated (NOX's default "
                         "is 2)")
    ap.add_argument("--partition-parts", type=int, default=0,
                    help="also time one Monte Carlo solve on this many row parts of the "
                         "domain (domain-decomposed transport) against the whole domain")
    ap.add_argument("--learned-threshold", default="0",
                    help="Composite Operator Threshold(s) of the learned-SPAI domain, comma "
                         "separated: the first is the reported learned solve, the others a "
                         "sweep")
    ap.add_argument("--seed", type=int, default=1234,
                    help="random-stream seed of the timed solves (rank r uses seed + r)")
    ap.add_argument("--spai-steps", type=int, default=2000,
                    help="training steps of the learned-SPAI network")
    ap.add_argument("--learned-format", default="stencil16", choices=["stencil16", "auto"],
                    help="walk records of the learned-SPAI domain: 16-bit CDF thresholds "
                         "(64 bytes for the 25-offset H) or the automatic FP32 choice")
    ap.add_argument("--aniso-train-systems", type=int, default=2000)
    ap.add_argument("--aniso-train-steps", type=int, default=4000)
    ap.add_argument("--spai-penalty", type=float, default=1.0,
                    help="weight of the |H| row-sum penalty in the anisotropic training loss")
    ap.add_argument("--batch-systems", type=int, default=1024)
    ap.add_argument("--batch-nmax", type=float, default=1e4,
                    help="largest system of the batched workload (5e5 for the full size)")
    args = ap.parse_args()
    if args.max_iters is None:
        args.max_iters = CONFIGS.get(args.config, {}).get("max_iters", 20000)
    world, rank, local, pg = dist_init(args)
    if args.impl == "mcls_b200" and args.config == "aniso512":
        run_aniso(args, world, rank, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.impl == "mcls_b200" and args.config == "batched":
        run_batched(args, world, rank, local, pg)
        if pg is not None:
            pg.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, world, rank, pg)
        if pg is not None:
            pg.destroy_process_group()
        return

    import torch

    from mcls_b200 import capi

    cfgd = CONFIGS[args.config]
    torch.cuda.set_device(local)
    A, b = make_system(args.config)
    n = A.shape[0]
    fp = capi.FP32 if args.config in ("diffusion128", "blocks256") else capi.FP64
    ctx = capi.Context(local)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    seed = args.seed + rank
    dom = capi.Domain(ctx, op, pc, precision=fp, rng_mode=capi.RNG_COUNTER, seed=seed,
                      estimator=cfgd["estimator"], sample_ratio=cfgd["sample_ratio"],
                      direction=cfgd["direction"],
                      history_length=cfgd["history_length"],
                      weight_cutoff=cfgd.get("weight_cutoff", 0.0))
    mp = capi.mcsa_params(tolerance=1e-8, max_iters=args.max_iters,
                          host_loop=1 if args.host_loop else 0)
    bt = torch.tensor(b, device=f"cuda:{local}", dtype=torch.float64)
    xt = torch.zeros_like(bt)
    tuned = None
    if args.walk_shape:
        hpl, blk = (int(v) for v in args.walk_shape.split(","))
        dom.set_launch(hpl, blk)
        tuned = {"histories_per_lane": hpl, "block_size": blk, "walk_ms": None}
    elif fp == capi.FP32 and not args.no_autotune:
        # Launch-shape autotuning on the workload's own right-hand side
        # (untimed set-up, like the domain build).
        dt = torch.tensor((1.0 / A.diagonal()) * b, device=f"cuda:{local}", dtype=torch.float64)
        torch.cuda.synchronize()
        tuned = dom.autotune(dt.data_ptr(), reps=2)
        del dt

    # More than one GPU: multi-set MCSA of the one system, one set per GPU,
    # the sets' corrections summed each iteration by the library's NCCL
    # communicator inside the device-side loop.
    sets = None
    if world > 1:
        uid = [capi.Comm.unique_id() if rank == 0 else None]
        pg.broadcast_object_list(uid, src=0)
        comm = capi.Comm(ctx, world, rank, uid[0])
        sets = comm.set_params()
        seed = capi.rank_seed(args.seed, rank)

    def device_step():
        dom.reseed(seed)
        xt.zero_()
        torch.cuda.synchronize()
        if sets is not None:
            return dom.mcsa_solve_sets_dev(sets, bt.data_ptr(), xt.data_ptr(), params=mp)[0]
        return dom.mcsa_solve_dev(bt.data_ptr(), xt.data_ptr(), params=mp)

    for _ in range(args.warmup):
        st = device_step()
    clocks = ClockSampler(local)
    barrier(pg)
    torch.cuda.synchronize()
    clocks.start()
    t0 = time.perf_counter()
    stats = [device_step() for _ in range(args.steps)]
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    barrier(pg)
    clk = clocks.stop()
    dev_ms = sum(s["solve_ms"] for s in stats)
    steps_total = sum(s["walk_steps"] for s in stats)
    dev_ms_max = allmax(pg, dev_ms)
    steps_all = allsum(pg, steps_total)
    value_steps = steps_all / (dev_ms_max * 1e-3)

    # End to end through the host-buffer call: H2D(b, x0) + solve + D2H(x).
    bh = np.ascontiguousarray(b)
    e2e_ms = 0.0
    e2e_steps = 0
    barrier(pg)
    for _ in range(args.steps):
        dom.reseed(seed)
        x0 = np.zeros(n)
        t1 = time.perf_counter()
        if sets is not None:
            x, st, _ = dom.mcsa_solve_sets(sets, bh, x0, params=mp)
        else:
            x, st = dom.mcsa_solve(bh, x0, params=mp)
        e2e_ms += (time.perf_counter() - t1) * 1e3
        e2e_steps += st["walk_steps"]
    barrier(pg)
    e2e_ms = allmax(pg, e2e_ms)
    e2e_steps_per_s = allsum(pg, e2e_steps) / (e2e_ms * 1e-3)

    s0 = stats[-1]
    x_dev = xt.cpu().numpy()
    rel = float(np.linalg.norm(b - A @ x_dev) / np.linalg.norm(b))
    peak, peak_kind = load_peaks()
    walk_ms = sum(s["walk_ms"] for s in stats)
    walk_launches = sum(s["walk_launches"] for s in stats)
    per_launch_ms = walk_ms / max(walk_launches, 1)
    info = dom.info()
    bstep = step_bytes(args.config, info)
    bytes_per_launch = bstep * steps_total / max(walk_launches, 1)
    achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9 if per_launch_ms > 0 else None
    traffic = WALK_DRAM_BYTES_PER_LAUNCH.get(args.config)
    solve_s = dev_ms_max / args.steps / 1e3
    config = workload_config(args, cfgd, n, A.nnz, world)
    results = {"time_to_1e-8_s": solve_s, "iterations": s0["iterations"],
               "converged": bool(s0["converged"]), "achieved_tol": s0["achieved_tol"],
               "rel_residual_b_minus_Ax": rel, "walk_steps_per_s": value_steps,
               "e2e_walk_steps_per_s": e2e_steps_per_s, "walk_launch": tuned,
               "dtype_detail": "FP32 walks, records and tallies reduced into FP64; FP64 "
                               "residual, update and norms" if fp == capi.FP32 else "FP64"}
    roofline_workload = {
        "bound": "l2" if traffic and traffic < 0.5 * bytes_per_launch else "hbm",
        "kernel": "walk32", "achieved": achieved, "unit": "GB/s",
        "frac_of_hbm_peak": achieved / peak if achieved else None, "peak": peak,
        "peak_kind": peak_kind, "traffic": traffic,
        "dram_gbs": traffic / (per_launch_ms * 1e-3) / 1e9 if traffic and per_launch_ms else None,
        "bytes_per_step": bstep, "walk_ms_per_launch": per_launch_ms,
        "walk_share_of_solve": walk_ms / dev_ms if dev_ms else None,
        "record_format": "stencil" if info["record_format"] == 2 else "packed",
        "note": "the timed workload's walk: its records fit L2, so the algorithmic bytes "
                "exceed what DRAM moves (traffic = ncu DRAM bytes per launch)"}
    line = {
        "metric": METRIC, "value": solve_s, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": False,
        "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "f32" if fp == capi.FP32 else "f64",
        "data": "synthetic", "config": config, "results": results,
        "clocks": clk,
        "e2e": {"value": e2e_ms / args.steps / 1e3, "unit": UNIT, "h2d_bytes_per_step": 2 * 8 * n,
                "d2h_bytes_per_step": 8 * n},
        "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
        "roofline_workload": roofline_workload,
        "wall_s": wall,
    }
    if rank == 0 and world == 1:
        line["results"]["err_vs_oracle"] = oracle_error(A, b, x_dev)
        if fp == capi.FP32:
            line["results"]["fp32_transition_agreement"] = walk_agreement(dom, 1 << 22,
                                                                          args.seed + 99)
    if world == 1 and not args.no_hbm_roofline:
        hr = hbm_walk_roofline(args, ctx)
        ach = hr["bytes_per_launch"] / (hr["per_launch_ms"] * 1e-3) / 1e9
        tr = HBM_WALK_DRAM_BYTES_PER_LAUNCH
        line["roofline"] = {
            "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
            "traffic": tr, "kernel": "walk32", "peak_kind": peak_kind,
            "dram_gbs": tr / (hr["per_launch_ms"] * 1e-3) / 1e9 if tr else None,
            "binding": "L2: the algorithmic bytes exceed the HBM peak because each record is "
                       "read from HBM about once per launch and its later reads hit L2",
            "ncu": HBM_WALK_NCU, **hr}
    else:
        line["roofline"] = dict(roofline_workload, frac=roofline_workload["frac_of_hbm_peak"])
    if world == 1 and args.partition_parts > 1:
        line["results"]["partitioned_mc"] = partition_arm(args, ctx, A, b)
    if world == 1 and not args.no_anderson:
        line["results"]["anderson"] = [
            anderson_arm(args, int(d), dom, bt, xt, A, b, seed, dev_ms_max / args.steps)
            for d in args.anderson_depth.split(",")]
    if world == 1 and args.config in ("diffusion128", "blocks256") and not args.no_learned:
        line["results"]["learned_spai"] = learned_arm(args, ctx, op, A, b, cfgd,
                                                      dev_ms_max / args.steps)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.config, A, b, gpu_iterations=s0["iterations"])
    if rank == 0:
        print(json.dumps(line))
    dom.close()
    pc.close()
    op.close()
    ctx.close()
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
