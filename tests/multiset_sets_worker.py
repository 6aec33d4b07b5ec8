"""One set of the multi-set MCSA entry point (mclsgpu_mcsa_solve_sets), run
as one of several processes on one GPU by tests/test_multiset_sets_gpu.py.
The sets' corrections are summed over gloo on host copies (the host-loop
form of the entry point; no kernel waits on another process)."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from mcls_b200 import capi, dist, multiset  # noqa: E402
from mcls_b200 import problems as P  # noqa: E402


def main(out):
    import torch

    world, rank, _, pg = dist.init("gloo", timeout_s=120)
    A = P.poisson2d(20)
    b = np.linspace(0.1, 1.0, A.shape[0])
    ctx = capi.Context(0)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    seed = capi.rank_seed(99, rank)
    # Forward expected-value walks, one history per row (bit-reproducible
    # corrections; the test compares with an emulation in one process).
    dom = capi.Domain(ctx, op, pc, precision=capi.FP64, rng_mode=capi.RNG_COUNTER, seed=seed,
                      estimator=capi.EXPECTED_VALUE, direction=capi.FORWARD, sample_ratio=1.0,
                      history_length=10)
    sets = multiset.torch_set_params(pg, world, "cuda:0", host_copy=True)
    x, st, on_device = dom.mcsa_solve_sets(sets, b, tolerance=1e-8, max_iters=5000)
    # Anderson-accelerated sets on their own domain and streams.
    da = capi.Domain(ctx, op, pc, precision=capi.FP64, rng_mode=capi.RNG_COUNTER,
                     seed=capi.rank_seed(17, rank), estimator=capi.EXPECTED_VALUE,
                     direction=capi.FORWARD, sample_ratio=1.0, history_length=10)
    xa, sa = da.anderson_solve_sets(sets, b, tolerance=1e-10, max_iters=2000, storage_depth=3)
    da.close()
    pg.barrier()
    with open(out, "w") as f:
        json.dump({"rank": rank, "seed": seed, "x": x.tolist(), "iters": st["iterations"],
                   "converged": st["converged"], "device_loop": on_device,
                   "aa_x": xa.tolist(), "aa_iters": sa["iterations"],
                   "aa_converged": sa["converged"]}, f)
    dom.close()
    pc.close()
    op.close()
    ctx.close()
    pg.destroy_process_group()


if __name__ == "__main__":
    main(sys.argv[1])
