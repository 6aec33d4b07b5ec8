"""Fixed-point iterations on the GPU (through the C ABI) against the oracle.

* FixedPointSolverManager: the reference's known answers
  (tpetra/test/tstTpetraFixedPointSolverManager.cpp: 15 Richardson
  iterations, solution sign, PL = PR = I), and the iterates of every
  "Fixed Point Type" against the oracle's restatement (inner products are
  summed in another order, so the bar is relative 1e-10, not bit equality).
* The MCSA smoother with each type: the oracle's steps on the reference
  Xorshift stream (FP64 walks), and convergence to 1e-8 with FP32 walks.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from mcls_b200 import capi
from mcls_b200 import problems as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TYPES = ["Richardson", "Steepest Descent", "MINRES", "RNSD"]


def _identity_precond(ctx, op, n):
    I = sp.identity(n, format="csr")
    return capi.Precond(ctx, op, capi.PREC_USER_CSR, user=I)


@pytest.mark.parametrize("b", [-1.0, 2.0, -2.0])
@pytest.mark.parametrize("prec", [False, True])
def test_fixed_point_reference_known_answer(ctx, b, prec):
    A = P.fixed_point_test(10)
    op = capi.Operator(ctx, A)
    I = _identity_precond(ctx, op, 10) if prec else None
    x, st = capi.fixed_point_solve(ctx, op, np.full(10, b), left=I, right=I, tolerance=1e-8,
                                   max_iters=100)
    assert st["converged"] == 1 and st["iterations"] == 15 and st["achieved_tol"] > 0
    assert np.all(np.sign(x) == np.sign(b))


@pytest.mark.parametrize("kind", TYPES)
@pytest.mark.parametrize("prec", [None, "jacobi"])
def test_fixed_point_iterates_match_oracle(ctx, kind, prec):
    A = P.anisotropic2d(9, 8.0, 0.4)
    n = A.shape[0]
    b = np.linspace(-1.0, 2.0, n)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI) if prec else None
    Ao = O.Csr.from_scipy(A)
    PL = O.point_jacobi(Ao) if prec else None
    t = capi.FIXED_POINT_TYPES[kind]
    its = 25
    x, st = capi.fixed_point_solve(ctx, op, b, left=pc, tolerance=0.0, max_iters=its,
                                   fixed_point_type=t, richardson_omega=0.9)
    r = O.fixed_point_solve(Ao, b, PL=PL, tolerance=0.0, max_iters=its, fixed_point_type=t,
                            richardson_omega=0.9)
    assert st["iterations"] == its == r["iters"]
    assert np.allclose(x, r["x"], rtol=1e-10, atol=1e-12 * np.abs(r["x"]).max())
    assert st["residual_norm"] == pytest.approx(r["residuals"][-1], rel=1e-8)


def test_rnsd_with_general_left_and_right_preconditioners(ctx):
    # Block-Jacobi on both sides: the transposes of A, PL and PR are formed
    # on the device for RNSD's transposed composite operator.
    A = P.anisotropic2d(8, 5.0, 0.3)
    n = A.shape[0]
    b = np.cos(np.arange(n))
    op = capi.Operator(ctx, A)
    L = capi.Precond(ctx, op, capi.PREC_BLOCK_JACOBI, block_size=4)
    R = capi.Precond(ctx, op, capi.PREC_BLOCK_JACOBI, block_size=2)
    Ao = O.Csr.from_scipy(A)
    PL, PR = O.block_jacobi(Ao, 4), O.block_jacobi(Ao, 2)
    x, st = capi.fixed_point_solve(ctx, op, b, left=L, right=R, tolerance=0.0, max_iters=30,
                                   fixed_point_type="RNSD")
    r = O.fixed_point_solve(Ao, b, PL=PL, PR=PR, tolerance=0.0, max_iters=30,
                            fixed_point_type=3)
    assert np.allclose(x, r["x"], rtol=1e-10, atol=1e-12 * np.abs(r["x"]).max())


@pytest.mark.parametrize("kind", ["Steepest Descent", "MINRES"])
def test_fixed_point_converges_to_direct_solve(ctx, kind):
    A = P.poisson2d(12)
    n = A.shape[0]
    b = np.ones(n)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    x, st = capi.fixed_point_solve(ctx, op, b, left=pc, tolerance=1e-10, max_iters=20000,
                                   fixed_point_type=kind)
    assert st["converged"] == 1
    xs = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x - xs) <= 1e-7 * np.linalg.norm(xs)
    # host loop: the same iterations
    x2, st2 = capi.fixed_point_solve(ctx, op, b, left=pc, tolerance=1e-10, max_iters=20000,
                                     fixed_point_type=kind, host_loop=1)
    assert st2["iterations"] == st["iterations"] and np.array_equal(x, x2)


@pytest.mark.parametrize("kind", TYPES[1:])
def test_zero_residual_takes_a_zero_step(ctx, kind):
    # Homogeneous system from x = 0: rp = 0, the step length's denominator
    # is 0 and the step is 0 (the reference would divide 0 by 0); the
    # criterion falls back to the tolerance itself.
    A = P.poisson2d(6)
    op = capi.Operator(ctx, A)
    x, st = capi.fixed_point_solve(ctx, op, np.zeros(36), tolerance=1e-12, max_iters=5,
                                   fixed_point_type=kind)
    assert st["converged"] == 1 and st["iterations"] == 1
    assert np.all(x == 0.0)


def test_fixed_point_rejects_unknown_type(ctx):
    op = capi.Operator(ctx, P.poisson2d(4))
    with pytest.raises(capi.MclsError):
        capi.fixed_point_solve(ctx, op, np.ones(16), fixed_point_type=7)


@pytest.mark.parametrize("kind", TYPES[1:])
def test_mcsa_smoother_types_follow_oracle_in_parity_mode(ctx, kind):
    # FP64 walks on the reference stream: the smoother's iterates and the
    # Monte Carlo corrections follow the oracle's.
    A = P.tridiag_test(10)
    b = np.full(10, -1.0)
    op = capi.Operator(ctx, A)
    dom = capi.Domain(ctx, op, None, precision=capi.FP64, rng_mode=capi.RNG_REFERENCE, seed=77,
                      history_length=10)
    t = capi.FIXED_POINT_TYPES[kind]
    x, st = dom.mcsa_solve(b, tolerance=1e-8, max_iters=20, fixed_point_type=t)
    r = O.mcsa_solve(O.Csr.from_scipy(A), b, tolerance=1e-8, max_iters=20, rng_mode=0, seed=77,
                     fixed_point_type=t)
    assert st["converged"] == 1 and r["converged"]
    assert abs(st["iterations"] - r["iters"]) <= 1
    assert np.allclose(x, r["x"], rtol=1e-7, atol=1e-12)


@pytest.mark.parametrize("kind", TYPES[1:])
def test_mcsa_smoother_types_converge_fp32(ctx, kind):
    A, b = P.diffusion3d_varcoef(10, seed=6)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=4,
                      estimator=capi.EXPECTED_VALUE, sample_ratio=1.0)
    x, st = dom.mcsa_solve(b, tolerance=1e-8, max_iters=3000,
                           fixed_point_type=capi.FIXED_POINT_TYPES[kind])
    assert st["converged"] == 1
    Dinv = 1.0 / A.diagonal()
    assert np.linalg.norm(Dinv * (b - A @ x)) <= 1e-8 * np.linalg.norm(Dinv * b) * 1.0001


def test_step_api_with_minres_smoother(ctx):
    import torch

    A = P.poisson2d(10)
    n = A.shape[0]
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=8,
                      sample_ratio=2.0)
    b = torch.ones(n, dtype=torch.float64, device="cuda:0")
    x = torch.zeros_like(b)
    d = torch.zeros_like(b)
    rn, bn = dom.mcsa_begin(b.data_ptr(), x.data_ptr(), tolerance=1e-8,
                            fixed_point_type=capi.FIXED_POINT_MINRES)
    for _ in range(400):
        dom.mcsa_correction(d.data_ptr())
        rn = dom.mcsa_apply(d.data_ptr(), 1.0)
        if rn <= 1e-8 * bn:
            break
    dom.mcsa_finish(x.data_ptr())
    assert rn <= 1e-8 * bn
    xs = spla.spsolve(A.tocsc(), np.ones(n))
    assert np.linalg.norm(x.cpu().numpy() - xs) <= 1e-6 * np.linalg.norm(xs)
