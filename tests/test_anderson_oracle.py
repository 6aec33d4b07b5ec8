"""The Anderson-acceleration oracle (oracle/mcls_oracle.cpp, Anderson) on the CPU.

NOX, which holds the reference's Anderson solver, is not part of the
reference tree, so the restatement is pinned by mathematics:

* against an independent least-squares statement of the same iteration
  (numpy lstsq on the stored differences, Walker & Ni 2011 eq. (2.1)-(2.3))
  for several storage depths, mixing parameters and start iterations;
* Walker & Ni 2011, Theorem 2.2: untruncated Anderson with mixing 1 on a
  linear map g(x) = G x + c gives x_{k+1} = g(x_k^GMRES);
* depth 0 is the damped fixed-point iteration x += beta F;
* dropping columns for the condition number down to one column is depth 1;
* the Anderson-accelerated MCSA reaches the MCSA status test
  |PL (b - A x)|_2 < tol |b|_2 on the reference's tridiagonal test system.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from mcls_b200 import problems as P
from oracle import oracle as O


def _linear(n=30, seed=1, scale=0.3):
    M = sp.csr_matrix(sp.random(n, n, density=0.2, random_state=seed) * scale)
    M.sort_indices()
    c = np.random.default_rng(seed).standard_normal(n)
    return M, c


def _anderson_lstsq(M, c, m, beta, start, iters):
    x = np.zeros(c.size)
    xs, Fs, Xs = [x.copy()], [], []
    for k in range(iters):
        F = M @ x + c - x
        Xs.append(x.copy())
        Fs.append(F.copy())
        if m > 0 and k >= start:
            first = max(start - 1, k - m)
            dF = np.column_stack([Fs[j + 1] - Fs[j] for j in range(first, k)])
            dX = np.column_stack([Xs[j + 1] - Xs[j] for j in range(first, k)])
            g = np.linalg.lstsq(dF, F, rcond=None)[0]
            x = x + beta * F - (dX + beta * dF) @ g
        else:
            x = x + beta * F
        xs.append(x.copy())
    return np.array(xs)


@pytest.mark.parametrize("m,beta,start", [(1, 1.0, 1), (2, 1.0, 1), (3, 0.7, 1), (2, 1.0, 3),
                                          (5, 0.9, 2)])
def test_matches_least_squares_statement(m, beta, start):
    M, c = _linear()
    _, its, _, X = O.anderson_linear(O.Csr.from_scipy(M), c, tolerance=0.0, max_iters=12,
                                     storage_depth=m, mixing=beta, start_iteration=start)
    R = _anderson_lstsq(M.toarray(), c, m, beta, start, 12)
    assert its == 12
    assert np.abs(X - R).max() <= 1e-12 * np.abs(R).max()


def test_untruncated_anderson_is_gmres_then_g():
    M, c = _linear(seed=4)
    G = M.toarray()
    A = np.eye(c.size) - G
    _, _, _, X = O.anderson_linear(O.Csr.from_scipy(M), c, tolerance=0.0, max_iters=7,
                                   storage_depth=16)
    for k in range(1, 7):
        K = np.column_stack([np.linalg.matrix_power(A, j) @ c for j in range(k)])
        xg = K @ np.linalg.lstsq(A @ K, c, rcond=None)[0]
        assert np.abs(X[k + 1] - (G @ xg + c)).max() <= 1e-10 * np.abs(X[k + 1]).max()


def test_depth_zero_is_damped_fixed_point():
    M, c = _linear(seed=2)
    _, _, _, X = O.anderson_linear(O.Csr.from_scipy(M), c, tolerance=0.0, max_iters=10,
                                   storage_depth=0, mixing=0.6)
    x = np.zeros(c.size)
    for k in range(10):
        x = x + 0.6 * (M @ x + c - x)
        assert np.allclose(X[k + 1], x, rtol=1e-13, atol=1e-15)


def test_condition_drop_to_one_column_is_depth_one():
    M, c = _linear(seed=3)
    Mo = O.Csr.from_scipy(M)
    _, _, _, X1 = O.anderson_linear(Mo, c, tolerance=0.0, max_iters=10, storage_depth=1)
    _, _, _, Xd = O.anderson_linear(Mo, c, tolerance=0.0, max_iters=10, storage_depth=4,
                                    adjust_condition=1, drop_tolerance=2.0)
    assert np.allclose(Xd, X1, rtol=1e-11, atol=1e-14)


def test_acceleration_beats_the_plain_fixed_point():
    # A contraction with rho(G) = 0.95: both converge, Anderson far sooner.
    M, c = _linear(n=60, seed=5)
    M = sp.csr_matrix(M * (0.95 / max(abs(np.linalg.eigvals(M.toarray())))))
    M.sort_indices()
    Mo = O.Csr.from_scipy(M)
    _, it_aa, conv_aa, _ = O.anderson_linear(Mo, c, tolerance=1e-10, max_iters=2000,
                                             storage_depth=5)
    _, it_fp, conv_fp, _ = O.anderson_linear(Mo, c, tolerance=1e-10, max_iters=2000,
                                             storage_depth=0)
    assert conv_aa and conv_fp and 3 * it_aa < it_fp


@pytest.mark.parametrize("b", [-1.0, 2.0])
@pytest.mark.parametrize("direction", [0, 1])
def test_anderson_mcsa_tridiagonal(b, direction):
    A = O.Csr.from_scipy(P.tridiag_test(10))
    r = O.anderson_solve(A, np.full(10, b), tolerance=1e-8, max_iters=50, seed=11,
                         direction=direction, sample_ratio=10.0 if direction else 1.0)
    assert r["converged"] and r["iters"] < 20
    assert np.all(np.sign(r["x"]) == np.sign(b))
    assert r["achieved"] < 1e-8


def test_anderson_mcsa_already_converged_takes_no_step():
    A = P.tridiag_test(10)
    xs = np.linalg.solve(A.toarray(), np.ones(10))
    r = O.anderson_solve(O.Csr.from_scipy(A), np.ones(10), x0=xs, tolerance=1e-8, seed=2)
    assert r["converged"] and r["iters"] == 0 and r["steps"] == 0
