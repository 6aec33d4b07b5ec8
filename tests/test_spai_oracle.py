"""The learned-SPAI oracle (oracle/spai_oracle.py) on the CPU.

The learned preconditioner has no reference counterpart, so its oracle is
pinned by mathematics: the analytic gradient of the loss through the network
(FP64, no rounding) against central finite differences, Jacobi at a zero
output layer, and the BF16 rounding rule.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from mcls_b200 import problems as P
from oracle import spai_oracle as so


def _system(n=8, seed=3):
    A, _, _, _ = P.anisotropic2d_sample(n, seed)
    return A


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, -2.5e-3, 3.0e38],
                 dtype=np.float32)
    r = so.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0  # 1 + 2^-8 is a tie between 1 and 1 + 2^-7; 1 is even
    assert r[2] == np.float32(1.0 + 2 ** -7)  # above the tie
    assert r[3] == 1.0  # below the tie
    assert abs(r[4] - x[4]) <= abs(x[4]) * 2 ** -8
    assert np.isfinite(r[5])


def test_zero_output_layer_is_point_jacobi():
    A = _system()
    p = so.init_params(1, zero_last=True)
    out, _ = so.forward(p, so.features(A))
    assert np.all(out == 0)
    m = so.mvalues(A, out)
    M = sp.csr_matrix((m, A.indices, A.indptr), shape=A.shape)
    np.testing.assert_array_equal(M.toarray(), np.diag(1.0 / A.diagonal()))


def test_features_of_constant_coefficient_stencil():
    A = P.poisson2d(6)
    X = so.features(A)
    i = 6 * 2 + 3  # interior row
    a = X[i, 0:8:2]
    d = X[i, 1:8:2]
    np.testing.assert_allclose(a, -0.25, rtol=1e-7)
    np.testing.assert_array_equal(d, 0.0)
    assert np.all(X[:, 8:] == 0)
    # Boundary row 0 has no west/south neighbour: those slots are zero.
    assert X[0, 0] == 0 and X[0, 2] == 0


@pytest.mark.parametrize("pen_w", [0.0, 5.0])
def test_analytic_gradient_matches_finite_differences(pen_w):
    A = _system(n=7, seed=5)
    rng = np.random.default_rng(0)
    V = rng.standard_normal((3, A.shape[0]))
    p = so.init_params(2, zero_last=False).astype(np.float64)
    kw = dict(rounded=False, pen_w=pen_w, pen_c=0.9)
    loss, g = so.loss_and_gradient(p, A, V, **kw)
    assert loss > 0
    idx = np.concatenate([rng.choice(np.arange(so.W1, so.B1), 8, replace=False),
                          rng.choice(np.arange(so.B1, so.W2), 4, replace=False),
                          rng.choice(np.arange(so.W2, so.B2), 8, replace=False),
                          rng.choice(np.arange(so.B2, so.W3), 4, replace=False),
                          rng.choice(np.arange(so.W3, so.B3), 8, replace=False),
                          np.arange(so.B3, so.B3 + 4)])
    eps = 1e-6
    for k in idx:
        q = p.copy()
        q[k] += eps
        lp, _ = so.loss_and_gradient(q, A, V, **kw)
        q[k] -= 2 * eps
        lm, _ = so.loss_and_gradient(q, A, V, **kw)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)) + 1e-5 * abs(g).max(), (k, fd, g[k])


def test_loss_of_jacobi_equals_jacobi_damping():
    # With M = D^-1 the loss is the mean of |(I - D^-1 A) v|^2 / |v|^2.
    A = _system()
    rng = np.random.default_rng(1)
    V = rng.standard_normal((4, A.shape[0]))
    p = so.init_params(1, zero_last=True)
    loss, _ = so.loss_and_gradient(p, A, V)
    Hj = np.eye(A.shape[0]) - np.diag(1.0 / A.diagonal()) @ A.toarray()
    ref = np.mean([np.sum((Hj @ v) ** 2) / np.sum(v * v) for v in V])
    np.testing.assert_allclose(loss, ref, rtol=1e-12)


def test_row_sum_penalty_is_active_and_zero_below_threshold():
    A = _system()
    V = np.random.default_rng(2).standard_normal((2, A.shape[0]))
    p = so.init_params(4, zero_last=False)
    l0, _ = so.loss_and_gradient(p, A, V)
    l1, _ = so.loss_and_gradient(p, A, V, pen_w=3.0, pen_c=0.5)
    l2, _ = so.loss_and_gradient(p, A, V, pen_w=3.0, pen_c=100.0)
    assert l1 > l0
    assert l2 == l0
