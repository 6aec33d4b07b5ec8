"""Walk launch-shape autotuner and the explicit launch-shape entry point."""
import numpy as np
import pytest

from mcls_b200 import capi
from mcls_b200 import problems as P

pytestmark = pytest.mark.gpu


def test_launch_shapes_give_identical_forward_solves(ctx):
    # Histories per lane and block size change the schedule, not the
    # histories: each history's stream and path depend only on its index.
    A, b = P.diffusion3d_varcoef(12, seed=2)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    xs = []
    for hpl, blk, l1 in ((1, 256, 0), (2, 256, 0), (1, 128, 0), (2, 128, 0), (4, 256, 0),
                         (4, 128, 0), (8, 256, 0), (8, 128, 0), (2, 256, 1), (4, 256, 1)):
        dom = capi.Domain(ctx, op, pc, precision=capi.FP32, direction=capi.FORWARD,
                          estimator=capi.EXPECTED_VALUE, sample_ratio=2.0, seed=9)
        dom.set_launch(hpl, blk)
        dom.set_record_cache(l1)
        info = dom.info()
        assert (info["histories_per_lane"], info["block_size"], info["record_cache_l1"]) == \
            (hpl, blk, l1)
        x, st = dom.mcsa_solve(b, tolerance=0.0, max_iters=15)
        xs.append(x)
    for x in xs[1:]:
        assert np.array_equal(x, xs[0])


def test_autotune_picks_a_shape_and_restores_the_stream(ctx):
    torch = pytest.importorskip("torch")
    A, b = P.diffusion3d_varcoef(16, seed=2)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    kw = dict(precision=capi.FP32, direction=capi.FORWARD, estimator=capi.EXPECTED_VALUE,
              sample_ratio=2.0, seed=4)
    d1 = capi.Domain(ctx, op, pc, **kw)
    d2 = capi.Domain(ctx, op, pc, **kw)
    src = torch.tensor((1.0 / A.diagonal()) * b, device="cuda:0", dtype=torch.float64)
    torch.cuda.synchronize()
    t = d1.autotune(src.data_ptr(), reps=1)
    assert t["histories_per_lane"] in (1, 2, 4, 8) and t["block_size"] in (128, 256)
    assert t["walk_ms"] > 0
    # the tuned domain continues the same stream as an untuned one
    x1, s1 = d1.mcsa_solve(b, tolerance=0.0, max_iters=10)
    x2, s2 = d2.mcsa_solve(b, tolerance=0.0, max_iters=10)
    assert np.array_equal(x1, x2)


def test_bad_launch_shape_rejected(ctx):
    A = P.poisson2d(8)
    op = capi.Operator(ctx, A)
    dom = capi.Domain(ctx, op, None, precision=capi.FP32)
    with pytest.raises(capi.MclsError):
        dom.set_launch(3, 256)
    with pytest.raises(capi.MclsError):
        dom.set_launch(1, 512)
