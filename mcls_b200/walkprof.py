"""A few Monte Carlo solves of one 3D variable-coefficient diffusion domain,
for profiling the FP32 walk kernel alone (ncu captures one walk32 launch).

    python -m mcls_b200.walkprof [--n 192] [--solves 4] [--format auto|stencil16]
        [--histories-per-lane 0|1|2|4] [--direction forward|adjoint]

Point-Jacobi walks of 10 steps, 2 histories per row: forward expected-value
(each history starts at its own row, neighbouring rows in neighbouring lanes)
or adjoint collision (start states drawn from the right-hand side, so
neighbouring lanes start at unrelated rows).  Prints the walk's device time
per launch and its algorithmic bandwidth (the record bytes of every step).
At n = 192 the records (32 bytes x n^3 = 226 MB) exceed the 126 MB L2.
"""
from __future__ import annotations

import argparse
import json


def main(argv=None):
    import torch

    from . import capi
    from . import problems as P

    ap = argparse.ArgumentParser(prog="python -m mcls_b200.walkprof")
    ap.add_argument("--n", type=int, default=192)
    ap.add_argument("--solves", type=int, default=4)
    ap.add_argument("--format", choices=["auto", "stencil16"], default="auto")
    ap.add_argument("--histories-per-lane", type=int, default=0,
                    help="0: autotune the launch shape")
    ap.add_argument("--l1", type=int, default=0, help="record loads allocated in L1 (fixed shape)")
    ap.add_argument("--direction", choices=["forward", "adjoint"], default="forward")
    args = ap.parse_args(argv)
    A, b = P.diffusion3d_varcoef(args.n, seed=1)
    ctx = capi.Context(0)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    fmt = capi.RECORD_STENCIL16 if args.format == "stencil16" else capi.RECORD_AUTO
    fwd = args.direction == "forward"
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=3,
                      estimator=capi.EXPECTED_VALUE if fwd else capi.COLLISION,
                      sample_ratio=2.0, direction=capi.FORWARD if fwd else capi.ADJOINT,
                      history_length=10, record_format=fmt)
    rt = torch.tensor((1.0 / A.diagonal()) * b, device="cuda:0", dtype=torch.float64)
    xt = torch.zeros_like(rt)
    torch.cuda.synchronize()
    if args.histories_per_lane:
        dom.set_launch(args.histories_per_lane, 256)
        dom.set_record_cache(args.l1)
        shape = {"histories_per_lane": args.histories_per_lane, "block_size": 256,
                 "record_cache_l1": args.l1}
    else:
        shape = dom.autotune(rt.data_ptr(), reps=1)
    ms = steps = launches = 0
    for _ in range(args.solves):
        st = dom.mc_solve_dev(rt.data_ptr(), xt.data_ptr(), internal=True)
        ms += st["walk_ms"]
        steps += st["walk_steps"]
        launches += st["walk_launches"]
    info = dom.info()
    per = ms / max(launches, 1)
    # A forward step reads its record (the tally source rides in it); an
    # adjoint step also reads and writes one FP64 tally.
    step_b = info["record_bytes"] + (0 if fwd else 16)
    print(json.dumps({"n": A.shape[0], "direction": args.direction, "record_bytes": info["record_bytes"],
                      "records_mb": info["record_bytes"] * A.shape[0] / 1e6,
                      "walk_ms_per_launch": per, "steps_per_launch": steps / max(launches, 1),
                      "step_bytes": step_b,
                      "algorithmic_gbs": step_b * steps / max(launches, 1) / (per * 1e-3) / 1e9,
                      "launch": shape}))
    dom.close()
    pc.close()
    op.close()
    ctx.close()


if __name__ == "__main__":
    main()
