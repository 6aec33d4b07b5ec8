"""FP32 walk record formats: packed (column, CDF) pairs vs stencil slots.

Both formats hold the same FP32 CDF values and compare them with the same
uniforms, so they select the same transitions: with the collision estimator
the forward MCSA iterates agree bit for bit.  With the expected-value
estimator the stencil path rebuilds H b from the FP32 record (W times CDF
differences) instead of the FP64 domain, so the iterates agree to FP32
rounding of the tally source.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from mcls_b200 import capi
from mcls_b200 import problems as P

pytestmark = pytest.mark.gpu


def _solve(ctx, A, b, fmt, **kw):
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=5,
                      record_format=fmt, **kw)
    return dom.mcsa_solve(b, tolerance=0.0, max_iters=20)


@pytest.mark.parametrize("name", ["varcoef3d", "poisson2d", "aniso9pt"])
@pytest.mark.parametrize("estimator", [capi.COLLISION, capi.EXPECTED_VALUE])
def test_stencil_and_packed_records_walk_identically(ctx, name, estimator):
    if name == "varcoef3d":
        A, b = P.diffusion3d_varcoef(12, seed=3)
    elif name == "poisson2d":
        A = P.poisson2d(30)
        b = np.linspace(0.1, 1.0, A.shape[0])
    else:
        A = P.anisotropic2d(24, 15.0, 0.4)
        b = np.linspace(-1.0, 1.0, A.shape[0])
    kw = dict(direction=capi.FORWARD, estimator=estimator, sample_ratio=2.0)
    x1, s1 = _solve(ctx, A, b, capi.RECORD_PACKED, **kw)
    x2, s2 = _solve(ctx, A, b, capi.RECORD_STENCIL, **kw)
    assert s1["walk_steps"] == s2["walk_steps"] > 0
    if estimator == capi.COLLISION:
        assert np.array_equal(x1, x2)
    else:
        assert np.allclose(x1, x2, rtol=1e-5, atol=1e-6 * np.abs(x1).max())


@pytest.mark.parametrize("direction", [capi.FORWARD, capi.ADJOINT])
def test_wide_stencil_records_walk_like_packed(ctx, direction):
    """A left preconditioner on A's 7-point pattern makes H = I - M A a
    25-offset stencil: 128-byte stencil records (2 + 25 words, padded)
    against 256-byte packed records."""
    import scipy.sparse as sp

    A, b = P.diffusion3d_varcoef(10, seed=4)
    d = 1.0 / A.diagonal()
    N = sp.diags(d) @ (sp.diags(A.diagonal()) - A)  # D^-1 (D - A), off-diagonal
    M = (sp.diags(d) @ (sp.identity(A.shape[0]) + 0.3 * N)).tocsr()
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_USER_CSR, user=M)
    out = {}
    for fmt in (capi.RECORD_PACKED, capi.RECORD_STENCIL):
        dom = capi.Domain(ctx, op, pc, precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=5,
                          record_format=fmt, direction=direction, estimator=capi.COLLISION,
                          sample_ratio=2.0)
        info = dom.info()
        x, st = dom.mcsa_solve(b, tolerance=0.0, max_iters=15)
        out[fmt] = (x, st, info)
    (x1, s1, i1), (x2, s2, i2) = out[capi.RECORD_PACKED], out[capi.RECORD_STENCIL]
    assert i2["record_format"] == capi.RECORD_STENCIL and i2["stencil_offsets"] == 25
    assert i2["record_bytes"] == 128 and i1["record_bytes"] == 256
    assert s1["walk_steps"] == s2["walk_steps"] > 0
    if direction == capi.FORWARD:
        assert np.array_equal(x1, x2)
    else:  # adjoint tallies: FP64 atomics from many histories, any order
        assert np.linalg.norm(x1 - x2) <= 1e-9 * np.linalg.norm(x1)


def test_domain_query_reports_layouts(ctx):
    A, _ = P.diffusion3d_varcoef(8, seed=1)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    d1 = capi.Domain(ctx, op, pc, precision=capi.FP32, direction=capi.FORWARD)
    i1 = d1.info()
    assert i1["record_format"] == capi.RECORD_STENCIL and i1["record_bytes"] == 32
    assert i1["stencil_offsets"] == 6 and i1["operator_dia"] == 7
    d2 = capi.Domain(ctx, op, pc, precision=capi.FP32, direction=capi.FORWARD,
                     record_format=capi.RECORD_PACKED)
    i2 = d2.info()
    assert i2["record_format"] == capi.RECORD_PACKED and i2["record_bytes"] == 64
    assert i1["entries"] == i2["entries"] == i1["rows"] * 6 - 6 * 8 * 8


def test_stencil_records_rejected_for_irregular_rows(ctx):
    # A random sparse pattern has far more than 14 distinct column offsets.
    import scipy.sparse as sp

    rng = np.random.Generator(np.random.PCG64(1))
    n = 400
    R = sp.random(n, n, density=0.02, random_state=3, format="csr")
    A = (R + R.T + sp.diags(np.full(n, 20.0))).tocsr()
    op = capi.Operator(ctx, A)
    with pytest.raises(capi.MclsError) as e:
        capi.Domain(ctx, op, None, precision=capi.FP32, record_format=capi.RECORD_STENCIL)
    assert e.value.code == capi.ERR_UNSUPPORTED
    # automatic selection falls back to packed records and solves
    dom = capi.Domain(ctx, op, None, precision=capi.FP32, direction=capi.FORWARD,
                      sample_ratio=4.0)
    x, st = dom.mc_solve(rng.uniform(0, 1, n))
    assert np.all(np.isfinite(x))


@pytest.mark.parametrize("direction", [capi.ADJOINT, capi.FORWARD])
def test_fp32_weight_cutoff_walks(ctx, direction):
    # Variable-length histories take the lane-refill loop: fewer steps than
    # the History Length cap, and an unbiased estimate of the same quantity.
    A = P.poisson2d(20)
    b = np.linspace(0.5, 1.5, A.shape[0])
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    kw = dict(precision=capi.FP32, direction=direction, sample_ratio=8.0, history_length=60)
    d_cut = capi.Domain(ctx, op, pc, weight_cutoff=0.2, **kw)
    x, st = d_cut.mc_solve(b)
    nh = st["histories"]
    assert 0 < st["walk_steps"] < 60 * nh
    assert np.all(np.isfinite(x))
    d_full = capi.Domain(ctx, op, pc, **kw)
    xf, sf = d_full.mc_solve(b)
    assert sf["walk_steps"] == 60 * sf["histories"]
    # Jacobi-Poisson interior weights stay 1, so the cutoff only trims walks
    # that lose weight at the boundary: the two estimates agree to MC noise.
    assert np.linalg.norm(x - xf) / np.linalg.norm(xf) < 0.2


def _wide_preconditioner(A, beta=0.3):  # noqa: D103
    import scipy.sparse as sp

    d = 1.0 / A.diagonal()
    N = sp.diags(d) @ (sp.diags(A.diagonal()) - A)
    return (sp.diags(d) @ (sp.identity(A.shape[0]) + beta * N)).tocsr()


def test_stencil16_record_layouts(ctx):
    # 25 offsets (H = I - M A, M on A's 7-point pattern): 64 bytes instead of
    # 128; the 9-point Jacobi H (8 offsets): 32 bytes instead of 64.
    A, _ = P.diffusion3d_varcoef(10, seed=4)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_USER_CSR, user=_wide_preconditioner(A))
    d = capi.Domain(ctx, op, pc, precision=capi.FP32, direction=capi.FORWARD,
                    record_format=capi.RECORD_STENCIL16)
    i = d.info()
    assert i["record_format"] == capi.RECORD_STENCIL16
    assert i["stencil_offsets"] == 25 and i["record_bytes"] == 64
    Aa = P.anisotropic2d(24, 15.0, 0.4)
    opa = capi.Operator(ctx, Aa)
    pca = capi.Precond(ctx, opa, capi.PREC_POINT_JACOBI)
    da = capi.Domain(ctx, opa, pca, precision=capi.FP32, direction=capi.FORWARD,
                     record_format=capi.RECORD_STENCIL16)
    ia = da.info()
    assert ia["stencil_offsets"] == 8 and ia["record_bytes"] == 32


@pytest.mark.parametrize("case", ["wide", "aniso9pt"])
def test_stencil16_selection_rate_and_solution(ctx, case):
    # 16-bit CDF thresholds: a transition can differ from the FP64 selection
    # only when u falls within 2^-16 of a CDF boundary (plus the FP32 rounding
    # the other formats have), at most (K + 1) 2^-16 per transition; MCSA
    # (forward expected value, the production estimator) still converges to
    # the tolerance, the residual being FP64, in about the FP32 records'
    # iteration count.
    if case == "wide":
        A, b = P.diffusion3d_varcoef(12, seed=6)
        op = capi.Operator(ctx, A)
        M = _wide_preconditioner(A, beta=0.15)
        pc = capi.Precond(ctx, op, capi.PREC_USER_CSR, user=M)
        K = 25
    else:
        A = P.anisotropic2d(24, 2.0, 0.3)
        b = np.linspace(0.1, 1.0, A.shape[0])
        op = capi.Operator(ctx, A)
        M = None
        pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
        K = 8
    kw = dict(precision=capi.FP32, direction=capi.FORWARD, estimator=capi.EXPECTED_VALUE,
              sample_ratio=2.0, seed=9)
    d16 = capi.Domain(ctx, op, pc, record_format=capi.RECORD_STENCIL16, **kw)
    nh = 1 << 20
    hd, td = d16.walk_agreement(nh, seed=3)
    assert td / (nh * 10) <= (K + 1) * 2.0 ** -16
    x, st = d16.mcsa_solve(b, tolerance=1e-8, max_iters=5000)
    assert st["converged"] == 1
    Pl = M if M is not None else sp.diags(1.0 / A.diagonal())
    r = Pl @ (b - A @ x)
    assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(Pl @ b) * 1.0001
    d32 = capi.Domain(ctx, op, pc, record_format=capi.RECORD_STENCIL, **kw)
    x32, st32 = d32.mcsa_solve(b, tolerance=1e-8, max_iters=5000)
    assert st32["converged"] == 1
    assert abs(st["iterations"] - st32["iterations"]) <= 0.2 * st32["iterations"] + 3
