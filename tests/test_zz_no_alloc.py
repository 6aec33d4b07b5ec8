"""mclsgpu_operator_apply_static: y = A x through the library's static device
staging array (no device allocation), checked against mclsgpu_operator_apply.

Both entry points run the same CSR SpMV kernel, so the results must agree to
the last bit; the tolerance below is a relative 1e-15 for safety.  The file
is named to be collected last so the static array is exercised after every
other test has used the device, and it also passes alone in a fresh process.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from mcls_b200 import capi
from mcls_b200 import problems as P

RTOL = 1e-15


def _check(ctx, A, seeds):
    op = capi.Operator(ctx, A)
    try:
        for s in seeds:  # calls in a row share (and overwrite) the staging array
            x = np.random.default_rng(s).standard_normal(A.shape[0])
            y_static = op.apply_static(x)
            y_alloc = op.apply(x)
            np.testing.assert_allclose(y_static, y_alloc, rtol=RTOL, atol=0)
            np.testing.assert_allclose(y_static, A @ x, rtol=1e-12, atol=1e-12)
    finally:
        op.close()


@pytest.mark.gpu
def test_static_apply_matches_allocating_apply(ctx):
    A, _ = P.diffusion3d_varcoef(24, seed=3)
    _check(ctx, A, seeds=[1, 2])


@pytest.mark.gpu
def test_static_apply_smaller_operator_after_larger(ctx):
    # A smaller operator after a larger one: rows beyond n keep the previous
    # call's values and must not leak into the result.
    _check(ctx, P.diffusion3d_varcoef(20, seed=4)[0], seeds=[5])
    _check(ctx, P.poisson2d(30), seeds=[6, 7])


@pytest.mark.gpu
def test_static_apply_makes_no_device_allocation(ctx):
    # The library counts every cudaMalloc/cudaFree it makes.  The allocating
    # apply moves the counters (which shows they count); repeated static
    # applies after the first must leave them where they were.
    A, _ = P.diffusion3d_varcoef(16, seed=8)
    op = capi.Operator(ctx, A)
    try:
        x = np.random.default_rng(9).standard_normal(A.shape[0])
        a0, f0 = capi.device_allocations()
        op.apply(x)
        a1, f1 = capi.device_allocations()
        assert a1 - a0 == 2 and f1 - f0 == 2
        first = op.apply_static(x)
        a2, f2 = capi.device_allocations()
        for _ in range(5):
            np.testing.assert_array_equal(op.apply_static(x), first)
        assert capi.device_allocations() == (a2, f2)
        assert (a2, f2) == (a1, f1)
    finally:
        op.close()


@pytest.mark.gpu
def test_static_apply_rejects_operator_above_limit(ctx):
    n = (1 << 20) + 1
    A = sp.identity(n, format="csr")
    op = capi.Operator(ctx, A)
    try:
        with pytest.raises(capi.MclsError) as ei:
            op.apply_static(np.ones(n))
        assert ei.value.code == capi.ERR_INVALID_ARG
        assert "static staging array" in str(ei.value)
        np.testing.assert_array_equal(op.apply(np.ones(n)), np.ones(n))
    finally:
        op.close()
