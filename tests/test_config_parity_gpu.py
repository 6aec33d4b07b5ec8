"""Parity on the benchmark workloads' own generators, at sizes that run in
seconds, and the pieces of the path that only those workloads exercise.

* MCSA solutions of the 3D variable-coefficient diffusion generator (48^3)
  and of the block diffusion-reaction generator (64^3, 8^3 material blocks):
  FP32 forward expected-value walks, FP64 residual and update, stopped by the
  reference's test |PL r|_2 <= 1e-8 |PL b|_2.  Each solution is compared with
  the oracle's FP64 conjugate-gradient solve to |b - A x|_2 <= 1e-13 |b|_2.
  Bars: the stopping test holds; the error against the oracle is within the
  bound the reached residual allows, |x - x_o| <= |A^-1| |b - A x| with
  |A^-1| = 1/lambda_min(A) (A is symmetric positive definite); and, solved to
  1e-9 instead, |b - A x|_2 / |b|_2 <= 1e-8.
* FP32 transition agreement: the production FP32 walk's selections against
  the FP64 selections of the same random draws on the 48^3 domain; the rate
  must stay within the rounding width of FP32 CDFs and 24-bit uniforms.
* "Composite Operator Threshold": the filtered domain (signed row maximum,
  tpetra/src/MCLS_TpetraHelpers.hpp:196-259) equals the oracle's bit for bit.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from mcls_b200 import capi
from mcls_b200 import problems as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = {
    # workload: generator, sample ratio (histories per row)
    "varcoef48": (lambda: P.diffusion3d_varcoef(48, seed=0), 2.0),
    "blocks64": (lambda: P.diffusion3d_blocks(64, 8, seed=0), 1.0),
}


def _lambda_min(A):
    # Smallest eigenvalue of the SPD operator (shift-invert Lanczos).
    return float(spla.eigsh(A.tocsc(), k=1, sigma=0.0, which="LM",
                            return_eigenvectors=False)[0])


def _solve(ctx, A, b, ratio, tol, seed=11):
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=seed,
                      direction=capi.FORWARD, estimator=capi.EXPECTED_VALUE, history_length=10,
                      sample_ratio=ratio)
    x, st = dom.mcsa_solve(b, tolerance=tol, max_iters=40000)
    dom.close()
    pc.close()
    op.close()
    return x, st


@pytest.mark.parametrize("name", sorted(CASES))
def test_workload_solution_against_fp64_oracle(ctx, name):
    gen, ratio = CASES[name]
    A, b = gen()
    xo = O.pcg(O.Csr.from_scipy(A), b, tolerance=1e-13)
    assert xo["converged"]
    xo = xo["x"]
    x, st = _solve(ctx, A, b, ratio, 1e-8)
    assert st["converged"] == 1
    dinv = 1.0 / A.diagonal()
    assert np.linalg.norm(dinv * (b - A @ x)) <= 1e-8 * np.linalg.norm(dinv * b) * 1.0001
    r = b - A @ x
    err = np.linalg.norm(x - xo) / np.linalg.norm(xo)
    bound = np.linalg.norm(r) / _lambda_min(A) / np.linalg.norm(xo)
    print(f"{name}: {st['iterations']} iterations, |b-Ax|/|b| = "
          f"{np.linalg.norm(r) / np.linalg.norm(b):.3e}, |x-x_o|/|x_o| = {err:.3e} "
          f"(bound {bound:.3e})")
    assert err <= bound * 1.001 + 1e-13
    assert err <= 1e-6
    # To a tighter stopping level the unpreconditioned relative residual
    # reaches 1e-8.
    x9, st9 = _solve(ctx, A, b, ratio, 1e-9)
    assert st9["converged"] == 1
    assert np.linalg.norm(b - A @ x9) <= 1e-8 * np.linalg.norm(b)
    assert np.linalg.norm(x9 - xo) / np.linalg.norm(xo) <= 1e-7


def test_fp32_transition_agreement_rate(ctx):
    A, b = P.diffusion3d_varcoef(48, seed=0)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=3,
                      direction=capi.FORWARD, estimator=capi.EXPECTED_VALUE, history_length=10,
                      sample_ratio=2.0)
    nh = 1 << 22
    hd, td = dom.walk_agreement(nh, seed=5)
    L = 10
    # A transition can only differ when a CDF boundary lies within the FP32
    # rounding of the CDF (half an ulp, <= 2^-25) or within the 24-bit
    # truncation of the uniform (< 2^-24) of u: at most (6 + 1) * 2^-24 per
    # transition on this 6-neighbour domain, averaged over u.
    rate = td / (nh * L)
    print(f"FP32 vs FP64 selection: {td} of {nh * L} transitions ({rate:.3e}), "
          f"{hd} of {nh} histories")
    assert rate <= 7 * 2.0 ** -24
    assert hd <= td
    assert hd / nh <= L * 7 * 2.0 ** -24
    dom.close()
    pc.close()
    op.close()


def _threshold_cases():
    A3, _ = P.diffusion3d_varcoef(6, seed=4)
    Aa = P.anisotropic2d(8, 20.0, 0.6)
    # A left preconditioner -D^-1 (user CSR): rows of the composite operator
    # then have a negative diagonal, so the signed row maximum (the
    # reference's) is the largest positive off-diagonal entry, not the
    # largest magnitude.
    neg = sp.diags(-1.0 / Aa.diagonal(), format="csr")
    return [("varcoef_jacobi", A3, "jacobi", 0.02), ("aniso_jacobi", Aa, "jacobi", 0.15),
            ("aniso_negated_jacobi", Aa, neg, 0.5)]


@pytest.mark.parametrize("case", range(3))
@pytest.mark.parametrize("direction", [0, 1])
def test_composite_threshold_domain_matches_oracle(ctx, case, direction):
    name, A, prec, thr = _threshold_cases()[case]
    Ao = O.Csr.from_scipy(A)
    op = capi.Operator(ctx, A)
    if isinstance(prec, str):
        pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
        PL = O.point_jacobi(Ao)
    else:
        pc = capi.Precond(ctx, op, capi.PREC_USER_CSR, user=prec)
        PL = O.Csr.from_scipy(prec)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP64, direction=direction,
                      composite_threshold=thr)
    g = dom.export()
    o = O.MC(Ao, PL=PL, direction=direction, composite_threshold=thr).domain()
    unfiltered = O.MC(Ao, PL=PL, direction=direction).domain()
    assert len(o["col"]) < len(unfiltered["col"]), "the threshold must drop entries"
    for key in ("rowptr", "col", "h", "cdf", "weights"):
        assert np.array_equal(g[key], o[key]), (name, key)
    dom.close()
    pc.close()
    op.close()


@pytest.mark.parametrize("direction", [0, 1])
def test_composite_threshold_that_empties_rows_is_reported(ctx, direction):
    # Filtering away every off-diagonal entry of a row leaves H's row empty
    # (H = I - M with M's row reduced to its unit diagonal): the reference
    # trips MCLS_CHECK(num_entries > 0), the oracle refuses the domain and
    # the device build reports MCLSGPU_ERR_DEGENERATE.
    A, _ = P.diffusion3d_varcoef(6, seed=4)
    Ao = O.Csr.from_scipy(A)
    with pytest.raises(RuntimeError):
        O.MC(Ao, PL=O.point_jacobi(Ao), direction=direction, composite_threshold=0.2)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    with pytest.raises(capi.MclsError) as e:
        capi.Domain(ctx, op, pc, precision=capi.FP64, direction=direction,
                    composite_threshold=0.2)
    assert e.value.code == capi.ERR_DEGENERATE
    pc.close()
    op.close()
