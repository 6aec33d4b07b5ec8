"""FP32 walk record formats: packed (column, CDF) pairs vs stencil slots.

Both formats hold the same FP32 CDF values and compare them with the same
uniforms, so they select the same transitions: the walks, and therefore the
forward-estimator MCSA iterates, agree bit for bit.
"""
import numpy as np
import pytest

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
def test_stencil_and_packed_records_walk_identically(ctx, name):
    if name == "varcoef3d":
        A, b = P.diffusion3d_varcoef(12, seed=3)
    elif name == "poisson2d":
        A = P.poisson2d(30)
        b = np.linspace(0.1, 1.0, A.shape[0])
    else:
        A = P.anisotropic2d(24, 15.0, 0.4)
        b = np.linspace(-1.0, 1.0, A.shape[0])
    kw = dict(direction=capi.FORWARD, estimator=capi.EXPECTED_VALUE, sample_ratio=2.0)
    x1, s1 = _solve(ctx, A, b, capi.RECORD_PACKED, **kw)
    x2, s2 = _solve(ctx, A, b, capi.RECORD_STENCIL, **kw)
    assert s1["walk_steps"] == s2["walk_steps"] > 0
    assert np.array_equal(x1, x2)


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
