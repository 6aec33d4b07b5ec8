"""The CPU baseline walks (oracle/mcls_oracle.cpp orc_bench_walks) that
bench.py times beside the GPU: they walk the workload's own direction and
estimator, so the baseline's walk steps are the GPU's.

* Forward, H = -I (A = 2I): every transition stays put and flips the sign,
  so each estimate is exact and equals the oracle's forward solve.
* Forward collision and expected value on a small contraction: the mean
  over many histories matches the truncated Neumann sums
  sum_{k<L} H^k b and b + sum_{k<L} H^{k+1} b.
* Adjoint: nh histories of L steps each, and the adjoint solve's mean over
  independent streams within 5 standard errors of the Neumann sums.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from mcls_b200 import problems as P
from oracle import oracle as O


@pytest.mark.parametrize("L", [1, 2, 3])
@pytest.mark.parametrize("threads", [1, 3])
def test_forward_walks_on_minus_identity_are_exact(L, threads):
    n = 8
    b = np.linspace(-1.0, 2.0, n)
    A = O.Csr.from_scipy(sp.csr_matrix(2.0 * sp.identity(n)))
    for est in (0, 1):
        mc = O.MC(A, history_length=L, direction=1, estimator=est)
        steps, _, x = mc.bench_walks(b, 5 * n, threads)
        xs, _ = mc.solve(b)
        assert steps == 5 * n * L
        assert np.allclose(x, xs, rtol=0, atol=1e-15)


@pytest.mark.parametrize("est", [0, 1])
def test_forward_walk_means_are_the_neumann_sums(est):
    A = P.poisson2d(4)
    n = A.shape[0]
    b = np.linspace(0.5, 1.5, n)
    Ao = O.Csr.from_scipy(A)
    L = 4
    mc = O.MC(Ao, PL=O.point_jacobi(Ao), history_length=L, direction=1, estimator=est)
    d = mc.domain()
    H = sp.csr_matrix((d["h"], d["col"], d["rowptr"]), shape=(n, n)).toarray()
    terms = [np.linalg.matrix_power(H, k + est) @ b for k in range(L)]
    want = sum(terms) + (b if est else 0.0)
    steps, _, x = mc.bench_walks(b, 20000 * n, 4)
    assert steps == 20000 * n * L
    assert np.abs(x - want).max() <= 0.02 * np.abs(want).max()


def test_adjoint_walk_steps():
    A = P.tridiag_test(10)
    Ao = O.Csr.from_scipy(A)
    mc = O.MC(Ao, history_length=7)
    steps, secs, x = mc.bench_walks(np.ones(10), 1000, 2)
    assert steps == 7000 and secs >= 0.0 and np.all(np.isfinite(x))


@pytest.mark.parametrize("est", [0, 1])
def test_adjoint_solve_means_are_the_neumann_sums(est):
    # The oracle's adjoint solve is unbiased: over 30 independent streams the
    # mean of x lies within 5 standard errors of sum_{k<L} H^k PL b
    # (collision) or sum_{k<=L} H^k PL b (expected value) in every entry.
    A = P.poisson2d(4)
    n = A.shape[0]
    b = np.linspace(0.5, 1.5, n)
    Ao = O.Csr.from_scipy(A)
    L = 4
    D = np.diag(1.0 / A.diagonal())
    H = np.eye(n) - D @ A.toarray()
    src = D @ b
    want = sum(np.linalg.matrix_power(H, k) @ src for k in range(L + est))
    E = np.array([O.MC(Ao, PL=O.point_jacobi(Ao), history_length=L, sample_ratio=50.0,
                       seed=100 + s, rng_mode=1, estimator=est).solve(b)[0]
                  for s in range(30)])
    se = E.std(0, ddof=1) / np.sqrt(len(E))
    assert np.all(np.abs(E.mean(0) - want) <= 5.0 * se)


def test_oracle_cg_matches_direct_solve():
    # The FP64 solve MCSA results are measured against: conjugate gradients
    # to 1e-13 agree with a sparse direct solve, with one or several threads.
    import scipy.sparse.linalg as spla

    from mcls_b200 import problems as P
    from oracle import oracle as O

    A, b = P.diffusion3d_varcoef(42, seed=2)  # 74,088 rows: the threaded loops run
    xs = spla.spsolve(A.tocsc(), b)
    for threads in (1, 4):
        O.set_threads(threads)
        r = O.pcg(O.Csr.from_scipy(A), b, tolerance=1e-13)
        assert r["converged"] and r["rel_residual"] <= 1e-13
        assert np.linalg.norm(r["x"] - xs) / np.linalg.norm(xs) < 1e-11
    O.set_threads(1)


def test_threaded_forward_walks_equal_one_thread():
    # The oracle's forward counter-stream walks partitioned over threads give
    # the one-thread result bit for bit (histories grouped by start state).
    from mcls_b200 import problems as P
    from oracle import oracle as O

    A, b = P.diffusion3d_varcoef(42, seed=1)
    Ao = O.Csr.from_scipy(A)
    out = []
    for threads in (1, 8):
        O.set_threads(threads)
        r = O.mcsa_solve(Ao, b, PL=O.point_jacobi(Ao), tolerance=1e-8, max_iters=3,
                         estimator=1, direction=1, sample_ratio=2.0, rng_mode=1, seed=3)
        out.append(r)
    O.set_threads(1)
    assert np.array_equal(out[0]["x"], out[1]["x"])
    assert out[0]["steps"] == out[1]["steps"]
