"""Step-wise MCSA entry points on the GPU (the multi-set building blocks).

* One set through mcls_b200.multiset.solve (begin / correction / apply /
  finish) converges like the one-call MCSA solve.
* Two sets emulated in one process on one GPU: two domains with different
  streams, corrections averaged on the device between the steps (what the
  all-reduce does across GPUs); both sets keep the same iterate and reach
  the direct solution.
* The same for the Anderson-accelerated solve's step-wise entry points
  (mclsgpu_anderson_begin / _correction / _apply / _finish), whose single-set
  steps follow the one-call solve's.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from mcls_b200 import capi, multiset
from mcls_b200 import problems as P

pytestmark = pytest.mark.gpu


def _domain(ctx, op, pc, seed, **kw):
    return capi.Domain(ctx, op, pc, precision=kw.pop("precision", capi.FP64),
                       rng_mode=capi.RNG_COUNTER, seed=seed,
                       estimator=kw.pop("estimator", capi.COLLISION),
                       direction=kw.pop("direction", capi.ADJOINT), sample_ratio=1.0,
                       history_length=10, **kw)


@pytest.mark.parametrize("direction", [capi.ADJOINT, capi.FORWARD])
def test_one_set_steps_match_the_one_call_solve(ctx, direction):
    A = P.poisson2d(20)
    b = np.linspace(0.1, 1.0, A.shape[0])
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = _domain(ctx, op, pc, 7, direction=direction)
    x1, s1 = dom.mcsa_solve(b, tolerance=1e-8, max_iters=5000)
    dom2 = _domain(ctx, op, pc, 7, direction=direction)
    eng = multiset.DeviceEngine(dom2, A.shape[0])
    x2, it, conv, rel, st = multiset.solve(eng, b, np.zeros_like(b), tolerance=1e-8,
                                           max_iters=5000)
    x2 = x2.cpu().numpy()
    assert conv and rel <= 1e-8 and st["walk_steps"] > 0
    assert abs(it - s1["iterations"]) <= max(3, 0.1 * s1["iterations"])
    xs = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x2 - xs) <= 1e-6 * np.linalg.norm(xs)
    assert np.linalg.norm(x1 - xs) <= 1e-6 * np.linalg.norm(xs)


def test_two_sets_on_one_gpu_average_their_corrections(ctx):
    import torch

    A, b = P.diffusion3d_varcoef(10, seed=3)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    engines = [multiset.DeviceEngine(_domain(ctx, op, pc, capi.rank_seed(99, r)), A.shape[0])
               for r in range(2)]
    params = capi.mcsa_params(tolerance=1e-8, max_iters=5000)
    norms = [e.begin(b, np.zeros_like(b), params) for e in engines]
    crit = 1e-8 * norms[0][1]
    it = 0
    rn = norms[0][0]
    while rn > crit and it < 5000:
        it += 1
        d = [e.correction().clone() for e in engines]
        assert not torch.equal(d[0], d[1])  # independent histories per set
        total = d[0] + d[1]
        rns = [e.apply(total, 0.5) for e in engines]
        assert rns[0] == rns[1]
        rn = rns[0]
    xs = [e.finish()[0].cpu().numpy() for e in engines]
    assert np.array_equal(xs[0], xs[1])
    ref = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(xs[0] - ref) <= 1e-6 * np.linalg.norm(ref)


def test_anderson_steps_follow_the_one_call_solve(ctx):
    # FP64 walks on the reference stream: the step-wise path takes the
    # one-call solve's steps (the same kernels, F with scale 1).
    A = P.poisson2d(12)
    b = np.linspace(0.1, 1.0, A.shape[0])
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)

    def dom():
        return capi.Domain(ctx, op, pc, precision=capi.FP64, rng_mode=capi.RNG_REFERENCE,
                           seed=31, history_length=10)

    x1, s1 = dom().anderson_solve(b, tolerance=0.0, max_iters=8, storage_depth=3)
    eng = multiset.DeviceEngine(dom(), A.shape[0])
    x2, it, conv, rel, st = multiset.solve_anderson(eng, b, np.zeros_like(b), tolerance=0.0,
                                                    max_iters=8, storage_depth=3)
    assert it == s1["iterations"] == st["iterations"] == 8
    assert np.allclose(x2.cpu().numpy(), x1, rtol=1e-9, atol=1e-14)


def test_two_anderson_sets_on_one_gpu(ctx):
    import torch

    A, b = P.diffusion3d_varcoef(10, seed=3)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    engines = [multiset.DeviceEngine(_domain(ctx, op, pc, capi.rank_seed(17, r)), A.shape[0])
               for r in range(2)]
    params = capi.anderson_params(tolerance=1e-10, max_iters=2000, storage_depth=3)
    starts = [e.aa_begin(b, np.zeros_like(b), params) for e in engines]
    done = starts[0][2]
    steps = 0
    while not done:
        steps += 1
        d = [e.aa_correction().clone() for e in engines]
        assert not torch.equal(d[0], d[1])  # independent histories per set
        total = d[0] + d[1]
        out = [e.aa_apply(total, 0.5) for e in engines]
        assert out[0] == out[1]
        done = out[0][1]
    xs = [e.aa_finish()[0].cpu().numpy() for e in engines]
    assert np.array_equal(xs[0], xs[1])
    assert steps < 2000
    ref = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(xs[0] - ref) <= 1e-5 * np.linalg.norm(ref)
