"""Edge cases of the C ABI on the GPU: malformed operators, the homogeneous
system, a one-row system, unsorted and duplicate CSR entries, and a batch
of one system against the single-system path."""
import numpy as np
import pytest
import scipy.sparse as sp

from mcls_b200 import capi
from mcls_b200 import problems as P

pytestmark = pytest.mark.gpu


def _raw_upload(ctx, n, rp, ci, v):
    import ctypes as C

    rp = np.ascontiguousarray(rp, np.int64)
    ci = np.ascontiguousarray(ci, np.int64)
    v = np.ascontiguousarray(v, np.float64)
    h = C.c_void_p()
    rc = ctx.L.mclsgpu_operator_upload(ctx.h, n, rp.ctypes.data, ci.ctypes.data,
                                       v.ctypes.data, C.byref(h))
    if rc == capi.OK:
        ctx.L.mclsgpu_operator_destroy(h)
    return rc


def test_malformed_operators_are_rejected(ctx):
    assert _raw_upload(ctx, 0, [0], [0], [1.0]) == capi.ERR_INVALID_ARG          # empty
    assert _raw_upload(ctx, 2, [0, 1, 2], [0, 2], [1.0, 1.0]) == capi.ERR_INVALID_ARG  # column
    assert _raw_upload(ctx, 2, [0, 1, 2], [0, 1], [1.0, np.nan]) == capi.ERR_INVALID_ARG
    assert _raw_upload(ctx, 2, [0, 2, 1], [0, 1], [1.0, 1.0]) == capi.ERR_INVALID_ARG  # rowptr
    assert _raw_upload(ctx, 2, [1, 2, 3], [0, 1, 1], [1, 1, 1.0]) == capi.ERR_INVALID_ARG


@pytest.mark.parametrize("direction", [capi.ADJOINT, capi.FORWARD])
@pytest.mark.parametrize("sampling", [capi.SOURCE_RANDOM, capi.SOURCE_STRATIFIED])
def test_homogeneous_system_converges_at_zero(ctx, direction, sampling):
    # b = 0 and x0 = 0: the residual and the Monte Carlo source are zero; the
    # solve must stay at x = 0 and report convergence, not a divergence.
    A = P.poisson2d(10)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, direction=direction,
                      source_sampling=sampling, sample_ratio=1.0)
    x, st = dom.mcsa_solve(np.zeros(A.shape[0]), tolerance=1e-8, max_iters=20)
    assert st["converged"] == 1
    assert np.all(x == 0.0)


def test_exact_initial_guess_stays_exact(ctx):
    import scipy.sparse.linalg as spla

    A = P.poisson2d(10)
    b = np.linspace(0.1, 1.0, A.shape[0])
    xs = spla.spsolve(A.tocsc(), b)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP64, sample_ratio=1.0)
    x, st = dom.mcsa_solve(b, xs, tolerance=1e-8, max_iters=20)
    assert st["converged"] == 1
    assert np.linalg.norm(x - xs) <= 1e-12 * np.linalg.norm(xs)


def test_one_row_system_is_degenerate_like_the_reference(ctx):
    # With Jacobi, H = I - D^-1 A has no retained entry in the only row; the
    # reference's domain build rejects that row (MCLS_CHECK num_entries > 0).
    op = capi.Operator(ctx, sp.csr_matrix(np.array([[2.0]])))
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    with pytest.raises(capi.MclsError) as e:
        capi.Domain(ctx, op, pc, precision=capi.FP64)
    assert e.value.code == capi.ERR_DEGENERATE


def test_unsorted_duplicate_entries_are_summed(ctx):
    A = P.poisson2d(6).tocoo()
    # split every entry in two halves, shuffle the order inside the rows
    rng = np.random.default_rng(0)
    rows = np.concatenate([A.row, A.row])
    cols = np.concatenate([A.col, A.col])
    vals = np.concatenate([0.5 * A.data, 0.5 * A.data])
    order = np.lexsort((rng.random(rows.size), rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rp = np.zeros(A.shape[0] + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    rp = np.cumsum(rp)
    import ctypes as C

    h = C.c_void_p()
    ci = np.ascontiguousarray(cols, np.int64)
    va = np.ascontiguousarray(vals, np.float64)
    ctx.check(ctx.L.mclsgpu_operator_upload(ctx.h, A.shape[0], rp.ctypes.data, ci.ctypes.data,
                                            va.ctypes.data, C.byref(h)))
    x = np.linspace(-1.0, 1.0, A.shape[0])
    y = np.empty_like(x)
    ctx.check(ctx.L.mclsgpu_operator_apply(h, x.ctypes.data, y.ctypes.data))
    ctx.L.mclsgpu_operator_destroy(h)
    np.testing.assert_allclose(y, A.tocsr() @ x, rtol=1e-14, atol=1e-12)


def test_batch_of_one_system_matches_single(ctx):
    import torch

    A, b = P.diffusion3d_varcoef(8, seed=4)
    bt = capi.Batch(ctx, [A], [1], direction=capi.FORWARD, estimator=capi.EXPECTED_VALUE,
                    precision=capi.FP32, sample_ratio=2.0)
    B = torch.tensor(bt.pack([b[:, None]]), device="cuda:0").contiguous()
    X = torch.zeros_like(B)
    st, it, rr = bt.mcsa_solve_dev(B.data_ptr(), X.data_ptr(), tolerance=1e-8, max_iters=5000)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, direction=capi.FORWARD,
                      estimator=capi.EXPECTED_VALUE, sample_ratio=2.0)
    x1, s1 = dom.mcsa_solve(b, tolerance=1e-8, max_iters=5000)
    assert st["converged"] == 1 and s1["converged"] == 1
    np.testing.assert_allclose(bt.unpack(X.cpu().numpy())[0][:, 0], x1, rtol=1e-6,
                               atol=1e-9 * np.abs(x1).max())
