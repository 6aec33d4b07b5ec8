"""Anderson-accelerated MCSA on the GPU (through the C ABI) against the oracle.

With FP64 walks on the reference Xorshift stream the device takes the
oracle's Monte Carlo corrections; the least-squares fits then agree to the
rounding of inner products summed in another order, so iterates are compared
to relative 1e-7 and iteration counts to within one.  FP32 walks are checked
for convergence to the MCSA status test |PL (b - A x)|_2 < tol |b|_2.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from mcls_b200 import capi
from mcls_b200 import problems as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _parity_pair(ctx, A, b, jacobi, seed, stratified=False, **aa):
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI) if jacobi else None
    dom = capi.Domain(ctx, op, pc, precision=capi.FP64, rng_mode=capi.RNG_REFERENCE, seed=seed,
                      history_length=10,
                      source_sampling=capi.SOURCE_STRATIFIED if stratified else capi.SOURCE_RANDOM)
    x, st = dom.anderson_solve(b, **aa)
    Ao = O.Csr.from_scipy(A)
    aa.pop("host_loop", None)
    r = O.anderson_solve(Ao, b, PL=O.point_jacobi(Ao) if jacobi else None, rng_mode=0,
                         seed=seed, stratified=int(stratified), **aa)
    return x, st, r


@pytest.mark.parametrize("aa", [
    dict(storage_depth=2),
    dict(storage_depth=0, mixing=0.8),
    dict(storage_depth=3, start_iteration=3),
    dict(storage_depth=4, adjust_condition=1, drop_tolerance=1e-3),
    dict(storage_depth=2, smoother_steps=2),
    dict(storage_depth=2, host_loop=1),
    # no smoothing: the random source's variance stalls the plain map, as it
    # stalls MCSA without smoothing; the stratified source converges
    dict(storage_depth=2, smoother_steps=0, stratified=True),
])
def test_anderson_follows_oracle_on_reference_stream(ctx, aa):
    A = P.tridiag_test(10)
    b = np.full(10, -1.0)
    x, st, r = _parity_pair(ctx, A, b, False, 4242, tolerance=1e-8, max_iters=40, **aa)
    assert st["converged"] == 1 and r["converged"]
    assert abs(st["iterations"] - r["iters"]) <= 1
    assert np.allclose(x, r["x"], rtol=1e-7, atol=1e-12)
    assert np.all(x < 0)


def test_anderson_jacobi_poisson_follows_oracle(ctx):
    # The first steps follow the oracle's.  The least-squares fits amplify
    # the last-bit differences of atomically summed tallies from step to
    # step, so within a few more steps a history count or a sampled source
    # state can change, after which the two runs are independent samples of
    # the same solve: they still reach the same solution.
    A = P.poisson2d(9)
    b = np.linspace(0.5, 1.5, 81)
    x, st, r = _parity_pair(ctx, A, b, True, 99, tolerance=0.0, max_iters=3, storage_depth=3)
    assert st["iterations"] == r["iters"] == 3
    assert np.allclose(x, r["x"], rtol=1e-7, atol=1e-12 * np.abs(r["x"]).max())
    x, st, r = _parity_pair(ctx, A, b, True, 99, tolerance=1e-8, max_iters=200,
                            storage_depth=3)
    assert st["converged"] == 1 and r["converged"]
    assert abs(st["iterations"] - r["iters"]) <= 5
    # independent runs stopped at |PL r| < 1e-8 |b| differ by about 2e-6 here
    assert np.allclose(x, r["x"], rtol=1e-5, atol=0)


@pytest.mark.parametrize("direction", [capi.ADJOINT, capi.FORWARD])
def test_anderson_fp32_converges(ctx, direction):
    A, b = P.diffusion3d_varcoef(10, seed=6)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=5,
                      direction=direction, estimator=capi.EXPECTED_VALUE, sample_ratio=1.0)
    x, st = dom.anderson_solve(b, tolerance=1e-8, max_iters=2000, storage_depth=2)
    assert st["converged"] == 1
    assert np.linalg.norm((b - A @ x) / A.diagonal()) < 1e-8 * np.linalg.norm(b) * 1.0001
    # The error is the residual times the conditioning (D spans 0.1..10).
    xs = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x - xs) <= 1e-5 * np.linalg.norm(xs)
    # The host-driven loop (FP32 tallies are summed by atomics, so the
    # iterates match the graph loop's statistically, not bit for bit).
    x2, st2 = dom.anderson_solve(b, tolerance=1e-8, max_iters=2000, storage_depth=2,
                                 host_loop=1)
    assert st2["converged"] == 1
    assert np.linalg.norm(x2 - xs) <= 1e-5 * np.linalg.norm(xs)


def test_anderson_device_vectors_and_stats(ctx):
    import torch

    A = P.poisson2d(16)
    n = A.shape[0]
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, seed=3, sample_ratio=2.0)
    b = torch.ones(n, dtype=torch.float64, device="cuda:0")
    x = torch.zeros_like(b)
    st = dom.anderson_solve_dev(b.data_ptr(), x.data_ptr(), tolerance=1e-8, max_iters=500)
    assert st["converged"] == 1 and st["iterations"] > 0
    assert st["histories"] >= st["iterations"] * n and st["walk_steps"] > 0
    assert st["achieved_tol"] < 1e-8
    # error <= cond(A) (about 120 here) x the relative residual
    xs = spla.spsolve(A.tocsc(), np.ones(n))
    assert np.linalg.norm(x.cpu().numpy() - xs) <= 1e-5 * np.linalg.norm(xs)


def test_converged_initial_guess_takes_no_step(ctx):
    A = P.tridiag_test(10)
    xs = np.linalg.solve(A.toarray(), np.ones(10))
    dom = capi.Domain(ctx, capi.Operator(ctx, A), None, precision=capi.FP64, seed=1)
    x, st = dom.anderson_solve(np.ones(10), x0=xs, tolerance=1e-8)
    assert st["converged"] == 1 and st["iterations"] == 0 and st["histories"] == 0
    assert np.array_equal(x, xs)


def test_anderson_parameter_checks(ctx):
    A = P.poisson2d(6)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, seed=1)
    for bad in (dict(storage_depth=17), dict(start_iteration=0), dict(max_iters=0)):
        with pytest.raises(capi.MclsError):
            dom.anderson_solve(np.ones(36), **bad)
    # The model evaluator applies no right preconditioner.
    dr = capi.Domain(ctx, op, pc, right=pc, precision=capi.FP32, seed=1)
    with pytest.raises(capi.MclsError) as e:
        dr.anderson_solve(np.ones(36))
    assert e.value.code == capi.ERR_UNSUPPORTED


@pytest.mark.parametrize("solver", ["anderson", "mcsa"])
def test_reseed_reaches_the_captured_loop(ctx, solver):
    # The seed is baked into the walk launches of the captured device-side
    # loop: a reseed must rebuild it.  Forward expected-value walks with one
    # history per row (every tally one addition onto zero) give the same bits
    # for the same seed, so a second seed must differ and the first seed,
    # set again, must come back exactly.
    A, b = P.diffusion3d_varcoef(10, seed=6)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=5,
                      direction=capi.FORWARD, estimator=capi.EXPECTED_VALUE, sample_ratio=1.0)

    def run(seed):
        dom.reseed(seed)
        if solver == "anderson":
            return dom.anderson_solve(b, tolerance=0.0, max_iters=12, storage_depth=3)[0]
        return dom.mcsa_solve(b, tolerance=0.0, max_iters=12)[0]

    x1 = run(11)
    x2 = run(12)
    x1b = run(11)
    assert not np.array_equal(x1, x2)
    assert np.array_equal(x1, x1b)
