"""The oracle pinned against the reference's own code and known answers.

* RNG stream and CDF sampler: golden vectors written by the reference's own
  Xorshift<>, RNGTraits and SamplingTools compiled from its sources
  (tests/golden/make_golden.py via oracle/_ref).
* test/tstSamplingTools.cpp:65-101 known-answer table.
* tpetra/test/tstTpetraAlmostOptimalDomain.cpp:204-259 (Diagonal),
  tpetra/test/tstTpetraDomainTransporter.cpp:97-172 (Cutoff) and :175-242
  (Boundary, as trajectories leaving their block of rows),
  tpetra/test/tstTpetraAdjointTally.cpp:83-167 (normalize),
  tpetra/test/tstTpetraUniformAdjointSource.cpp:75-240 (counts, weight;
  nh_not_set and nh_set),
  tpetra/test/tstTpetraUniformForwardSource.cpp:75-260 (counts, weight 1),
  tpetra/test/tstTpetraForwardTally.cpp:83-235 (tally, finalize, normalize),
  tpetra/test/tstTpetraMCSASolverManager.cpp:72-510 (MCSA < 20 iterations:
  adjoint, forward, PL = PR = I),
  tpetra/test/tstTpetraFixedPointSolverManager.cpp:72-345 (Richardson: 15
  iterations, solution sign), tpetra/test/tstTpetraMCSolver.cpp:68-156
  (signs on one domain), tpetra/test/tstTpetraPointJacobiPreconditioner.cpp,
  tpetra/test/tstTpetraBlockJacobiPreconditioner.cpp
  and test/tstBlockInversion.cpp:46-105 (block inverses).
"""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from mcls_b200 import problems as P
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden", "reference_rng.json")


def _gold():
    with open(GOLD) as f:
        return json.load(f)


def test_golden_uniform_streams():
    g = _gold()
    for st in g["streams"]:
        u = O.xorshift_uniforms(st["seed"], len(st["uniforms_hex"]))
        want = np.array([float.fromhex(h) for h in st["uniforms_hex"]])
        assert np.array_equal(u, want), st["seed"]


def test_golden_sampler():
    for case in _gold()["sampling"]:
        cdf = np.array([float.fromhex(h) for h in case["cdf_hex"]])
        for uh, b in zip(case["u_hex"], case["bin"]):
            assert O.sample_cdf(cdf, float.fromhex(uh)) == b


def test_reference_harness_matches_oracle_live():
    R = O.ref_lib()
    if R is None:
        pytest.skip("oracle/_ref not built here (no reference tree)")
    for seed in (3, 99, 2**40 + 5):
        a = O.xorshift_uniforms(seed, 1000)
        b = np.empty(1000)
        R.ref_xorshift_uniforms(seed, 1000, b)
        assert np.array_equal(a, b)


def test_sampling_tools_known_answers():
    # test/tstSamplingTools.cpp:65-101
    cdf = np.array([0.13, 0.27, 0.44, 0.69, 1.00])
    table = [(0.13, 0), (0.27, 1), (0.44, 2), (0.69, 3), (1.00, 4), (0.00, 0),
             (0.12999999, 0), (0.13000001, 1), (0.26999999, 1), (0.27000001, 2),
             (0.43999999, 2), (0.44000001, 3), (0.68999999, 3), (0.69000001, 4),
             (0.99999999, 4)]
    for u, b in table:
        assert O.sample_cdf(cdf, u) == b
    for u in (0.13, 0.27, 0.44, 0.69, 1.0):
        assert O.sample_cdf(np.array([1.0]), u) == 0


def test_diagonal_transition_known_answer():
    # A = 3I: H = 1 - 3 = -2 on the diagonal; one transition keeps the state
    # and multiplies the weight by W * sign = -2 (w = -3*(3-1) for w0 = 3).
    A = O.Csr.from_scipy(sp.identity(8, format="csr") * 3.0)
    mc = O.MC(A, history_length=1, stratified=1)
    d = mc.domain()
    assert np.all(d["h"] == -2.0) and np.all(d["weights"] == 2.0) and np.all(d["cdf"] == 1.0)
    b = np.full(8, 0.375)  # |b|_1 = 3 exactly, one history per state (stratified)
    x, nh, tr = mc.solve(b, trace=8)
    assert nh == 8
    assert np.all(tr["states"][:, 1] == tr["states"][:, 0])
    assert np.all(tr["final_weight"] == -3.0 * (3 - 1))


def test_cutoff_known_answer():
    # A = 0.5 I, History Length 1: x_i = 3 before normalisation, final weight
    # 1.5, event CUTOFF.
    A = O.Csr.from_scipy(sp.identity(8, format="csr") * 0.5)
    mc = O.MC(A, history_length=1, stratified=1)
    x, nh, tr = mc.solve(np.full(8, 0.375), trace=8)
    assert nh == 8
    assert np.all(tr["final_weight"] == 1.5)
    assert np.all(tr["events"] == 2)
    assert np.allclose(x * nh, 3.0, rtol=0, atol=1e-15)


@pytest.mark.parametrize("mult", [1, 10])
def test_adjoint_source_counts_and_weight(mult):
    # tstTpetraUniformAdjointSource nh_not_set / nh_set (Sample Ratio mult):
    # b = -1 gives mult * N histories, all local states, weight -|b|_1 = -N.
    # The reference's operator has no entry in row 0 and keeps the identity
    # only where A has a diagonal entry.
    n = 10
    A = sp.lil_matrix((n, n))
    for i in range(1, n):
        A[i, i - 1] = -0.5
    A[n - 1, n - 1] = -0.5
    mc = O.MC(O.Csr.from_scipy(sp.csr_matrix(A)), history_length=1, sample_ratio=float(mult))
    d = mc.domain()
    # Row i of A^T holds A(i+1, i) = -0.5 -> h = +0.5 (no identity term: the
    # diagonal is absent); the last row holds A(n-1,n-1) -> h = 1 + 0.5.
    assert np.all(d["h"][:-1] == 0.5) and d["h"][-1] == 1.5
    # b > 0: nh = mult * N histories, weight +|b|_1 = N.
    x, nh, tr = mc.solve(np.full(n, 1.0), trace=mult * n)
    assert nh == mult * n
    W = d["weights"][tr["start"]]
    assert np.all(tr["final_weight"] == float(n) * W)
    # b = -1: the source code seeds its CDF with the signed b[0]
    # (src/MCLS_UniformAdjointSource_impl.hpp:185), so cdf.back() = N - 2 and
    # nh = int(mult * N * (N-2)/N) = 8 mult, and state 0 is never sampled.
    # The reference unit test still expects mult * N here; it predates that
    # code (it also builds the source before setting its RNG) and is stale --
    # the oracle follows the source code.
    x, nh, tr = mc.solve(np.full(n, -1.0), trace=mult * n)
    assert nh == mult * (n - 2)
    assert np.all(tr["start"] >= 1)
    W = d["weights"][tr["start"]]
    assert np.all(tr["final_weight"] == -float(n) * W)


@pytest.mark.parametrize("mult", [1, 10])
def test_forward_source_counts_and_weight(mult):
    # tstTpetraUniformForwardSource nh_not_set / nh_set: Sample Ratio = mult
    # gives mult * N histories, mult starting in every state, each of weight
    # 1 (the forward source does not scale by |b|_1).  History Length 1: the
    # final weight is W_i times the sign of the one transition's entry.  The
    # reference builds its forward domain from A^T; the forward oracle walks
    # the rows of the operator it is given, so it is given A^T.
    n = 10
    A = sp.lil_matrix((n, n))
    for i in range(1, n):
        A[i, i - 1] = -0.5
    A[n - 1, n - 1] = -0.5
    mc = O.MC(O.Csr.from_scipy(sp.csr_matrix(A.T)), history_length=1, direction=1,
              sample_ratio=float(mult))
    x, nh, tr = mc.solve(np.full(n, -1.0), trace=mult * n)
    assert nh == mult * n
    assert np.array_equal(np.bincount(tr["start"], minlength=n), np.full(n, mult))
    d = mc.domain()
    W = d["weights"][tr["start"]]
    assert np.allclose(np.abs(tr["final_weight"]), W, rtol=0, atol=0)


@pytest.mark.parametrize("L", [1, 2, 3, 4])
def test_forward_tally_known_answer(L):
    # tstTpetraForwardTally TallyHistory / Normalize: a history tallies
    # weight x b at each state it visits before its cutoff, the sum goes to
    # its starting state, finalize divides by the histories per state and
    # normalize leaves the forward result alone.  A = 2 I gives H = -I
    # (W = 1, every transition flips the sign and stays put), so L steps
    # give x = sum_{k<L} (-1)^k b: b for odd L, 0 for even L.
    n = 8
    A = sp.csr_matrix(2.0 * sp.identity(n))
    b = np.linspace(-1.0, 2.0, n)
    for ratio in (1.0, 3.0):
        mc = O.MC(O.Csr.from_scipy(A), history_length=L, direction=1, sample_ratio=ratio)
        x, nh = mc.solve(b)
        assert nh == int(ratio) * n
        # sum / count: exact for one history per state, one rounding for 3
        assert np.allclose(x, b if L % 2 else np.zeros(n), rtol=1e-15, atol=0)


@pytest.mark.parametrize("b", [-1.0, 2.0, -2.0])
def test_mcsa_tridiagonal_converges(b):
    # tstTpetraMCSASolverManager adjoint: 1 / -0.14 tridiagonal, tol 1e-8,
    # fewer than 20 iterations, solution sign follows the source.
    A = O.Csr.from_scipy(P.tridiag_test(10))
    r = O.mcsa_solve(A, np.full(10, b), tolerance=1e-8, max_iters=20, seed=11)
    assert r["converged"] and r["iters"] < 20 and r["achieved"] > 0
    assert np.all(np.sign(r["x"]) == np.sign(b))


def test_mcsa_tridiagonal_prec_identity():
    # prec_adjoint variant: PL = PR = I.
    A = O.Csr.from_scipy(P.tridiag_test(10))
    I = O.Csr.from_scipy(sp.identity(10, format="csr"))
    r = O.mcsa_solve(A, np.full(10, -1.0), PL=I, PR=I, tolerance=1e-8, max_iters=20, seed=5)
    assert r["converged"] and r["iters"] < 20
    assert np.all(r["x"] < 0)


@pytest.mark.parametrize("b", [-1.0, 2.0])
def test_mcsa_forward_tridiagonal(b):
    A = O.Csr.from_scipy(P.tridiag_test(10))
    r = O.mcsa_solve(A, np.full(10, b), tolerance=1e-8, max_iters=20, seed=3, direction=1)
    assert r["converged"] and r["iters"] < 20
    assert np.all(np.sign(r["x"]) == np.sign(b))


def test_mcsa_forward_prec_identity_successive_solves():
    # tstTpetraMCSASolverManager prec_forward (:391-510): forward, PL = PR =
    # I, Sample Ratio 1, four solves from x = 0 with b = -1, 2, 2, -2: each
    # converges in fewer than 20 iterations with the sign of b.  (The
    # reference runs them on one manager, one continuing stream; each solve
    # here starts a stream of its own.)
    A = O.Csr.from_scipy(P.tridiag_test(10))
    I = O.Csr.from_scipy(sp.identity(10, format="csr"))
    for k, b in enumerate((-1.0, 2.0, 2.0, -2.0)):
        r = O.mcsa_solve(A, np.full(10, b), PL=I, PR=I, tolerance=1e-8, max_iters=20,
                         seed=17 + k, direction=1, sample_ratio=1.0)
        assert r["converged"] and r["iters"] < 20 and r["achieved"] > 0, b
        assert np.all(np.sign(r["x"]) == np.sign(b))


@pytest.mark.parametrize("b", [-1.0, 2.0, -2.0])
@pytest.mark.parametrize("prec", [False, True])
def test_fixed_point_richardson_known_answer(b, prec):
    # tstTpetraFixedPointSolverManager one_by_one and one_by_one_prec
    # (PL = PR = I): Richardson, tolerance 1e-8, exactly 15 iterations.
    A = O.Csr.from_scipy(P.fixed_point_test(10))
    I = O.Csr.from_scipy(sp.identity(10, format="csr")) if prec else None
    r = O.fixed_point_solve(A, np.full(10, b), PL=I, PR=I, tolerance=1e-8, max_iters=100)
    assert r["converged"] and r["iters"] == 15 and r["achieved"] > 0
    assert np.all(np.sign(r["x"]) == np.sign(b))


@pytest.mark.parametrize("kind", [1, 2, 3])
def test_fixed_point_iterations_minimise_their_residuals(kind):
    # Steepest descent and MINRES take the step that makes the new residual
    # orthogonal to r (SD) or to A r (MINRES); RNSD to A A^T r.  One step
    # from x = 0 on a nonsymmetric system checks each against its
    # Petrov-Galerkin condition.
    rng = np.random.default_rng(kind)
    n = 12
    M = sp.random(n, n, density=0.3, random_state=3) + sp.identity(n) * 4.0
    M = sp.csr_matrix(M)
    M.sort_indices()
    b = rng.standard_normal(n)
    r = O.fixed_point_solve(O.Csr.from_scipy(M), b, tolerance=0.0, max_iters=1,
                            fixed_point_type=kind)
    r1 = b - M @ r["x"]
    Md = M.toarray()
    w = {1: b, 2: Md @ b, 3: Md @ (Md.T @ b)}[kind]
    assert abs(w @ r1) <= 1e-12 * np.linalg.norm(w) * np.linalg.norm(b)


def test_monte_carlo_solve_sign():
    # tstTpetraMonteCarloSolverManager: Sample Ratio 10, solution sign.
    A = O.Csr.from_scipy(P.tridiag_test(10))
    for direction in (0, 1):
        mc = O.MC(A, sample_ratio=10.0, direction=direction, seed=9)
        for b in (-1.0, 2.0):
            x, _ = mc.solve(np.full(10, b))
            assert np.all(np.sign(x) == np.sign(b))


def test_mc_solver_signs_on_one_source():
    # tpetra/test/tstTpetraMCSolver.cpp:68-156: Sample Ratio 100, the
    # reference's own stream ("Reproducible MC Mode"), b = -2 then b = 2 on
    # the same domain: the solution takes b's sign, whatever x held before.
    A = O.Csr.from_scipy(P.tridiag_test(10))
    # The source's CDF starts from the signed b[0]
    # (src/MCLS_UniformAdjointSource_impl.hpp:185), so b = -2 draws
    # 1000 * (-2 + 9 * 2) / 20 = 800 histories and b = 2 all 1000.
    mc = O.MC(A, sample_ratio=100.0, rng_mode=0, seed=5)
    x, nh = mc.solve(np.full(10, -2.0))
    assert nh == 800 and np.all(x < 0.0)
    x, nh = mc.solve(np.full(10, 2.0))
    assert nh == 1000 and np.all(x > 0.0)


@pytest.mark.parametrize("parts", [2, 4])
def test_long_histories_leave_their_part(parts):
    # tpetra/test/tstTpetraDomainTransporter.cpp:175-242 (Boundary): on the
    # 1 / -0.499 tridiagonal with History Length 10000, every history started
    # in a rank's rows ends in a BOUNDARY event.  One domain here (the
    # adjoint one, on A^T as the reference builds it; stratified, so one
    # history starts in every row), so the pin is on the trajectories: each
    # one reaches a row outside the block of 10 rows it started in.
    n = 10 * parts
    rows = np.arange(n)
    A = sp.lil_matrix(P.tridiag_test(n, off=-0.499))
    A[0, 1] = A[0, 2] = -0.499  # the reference's first and last rows
    A[n - 1, n - 3] = A[n - 1, n - 2] = -0.499
    A = sp.csr_matrix(A)
    A.eliminate_zeros()
    L = 10000
    mc = O.MC(O.Csr.from_scipy(A), history_length=L, stratified=1, seed=3)
    _, nh, tr = mc.solve(np.ones(n), trace=n)
    assert nh == n
    for h in range(n):
        states = tr["states"][h]
        block = tr["start"][h] // 10
        assert np.any(states // 10 != block), h
    assert np.array_equal(np.sort(tr["start"]), rows)


@pytest.mark.parametrize("tridiagonal", [False, True])
def test_point_jacobi_known_answers(tridiagonal):
    # tpetra/test/tstTpetraPointJacobiPreconditioner.cpp diag_matrix /
    # tridiag_matrix: every entry 2 (the first and last rows hold only their
    # diagonal) gives M^-1 = diag(1/2), diagonal only.
    n = 10
    A = sp.lil_matrix((n, n))
    for i in range(n):
        cols = [i] if not tridiagonal or i in (0, n - 1) else [i - 1, i, i + 1]
        for c in cols:
            A[i, c] = 2.0
    M = O.point_jacobi(O.Csr.from_scipy(sp.csr_matrix(A))).to_scipy()
    assert M.nnz == n and np.array_equal(M.toarray(), np.diag(np.full(n, 0.5)))


def test_point_jacobi_and_composite():
    A = P.poisson2d(6)
    Ao = O.Csr.from_scipy(A)
    PL = O.point_jacobi(Ao).to_scipy()
    assert np.allclose(PL.diagonal(), 1.0 / A.diagonal(), rtol=0, atol=0)
    M = O.composite(Ao, O.point_jacobi(Ao), transpose_=True).to_scipy()
    ref = (A.T @ sp.diags(1.0 / A.diagonal())).tocsr()
    assert abs(M - ref).max() == 0.0


def test_block_jacobi_known_answers():
    # tstTpetraBlockJacobiPreconditioner: blocks of a tridiagonal matrix.
    A = sp.csr_matrix(np.array([[2.0, -1, 0, 0], [-1, 2, -1, 0], [0, -1, 2, -1], [0, 0, -1, 2]]))
    Pm = O.block_jacobi(O.Csr.from_scipy(A), 2).to_scipy().toarray()
    blk = np.linalg.inv(np.array([[2.0, -1], [-1, 2]]))
    want = np.zeros((4, 4))
    want[:2, :2] = blk
    want[2:, 2:] = blk
    assert np.allclose(Pm, want, rtol=1e-14, atol=1e-14)


# test/tstBlockInversion.cpp:46-105: a 4x4 block and its GETRF/GETRI inverse.
BLOCK_INVERSION = (
    [[3.2, -1.43, 2.98, 0.32], [-4.12, -7.53, 1.44, -3.72], [4.24, -6.42, 1.82, 2.67],
     [-0.23, 5.8, 1.13, -3.73]],
    [[-0.461356423424245, -0.060920073472551, 0.547244760641934, 0.412904055961420],
     [0.154767451798665, -0.056225122550555, -0.174451348828054, -0.055523340725809],
     [0.848746201780808, 0.045927762119214, -0.618485718805259, -0.415712965073367],
     [0.526232280383953, -0.069757566407458, -0.492378815120724, -0.505833501236923]])


def test_block_inversion_known_answer():
    # One block of size 4 is the whole matrix: the preconditioner is its
    # inverse, to the reference's relative 1e-14.
    B, want = (np.array(m) for m in BLOCK_INVERSION)
    Pm = O.block_jacobi(O.Csr.from_scipy(sp.csr_matrix(B)), 4).to_scipy().toarray()
    assert np.all(np.abs(Pm - want) <= 1e-14 * np.abs(want))


def test_filter_relative_threshold():
    # TpetraMatrixHelpers::filter: drop |v| <= threshold * (signed row max).
    A = sp.csr_matrix(np.array([[4.0, 0.1, -0.3], [0.2, 1.0, 0.05], [1.0, 1.0, 1.0]]))
    I = O.Csr.from_scipy(sp.identity(3, format="csr"))
    C = O.multiply(O.Csr.from_scipy(A), I, 0.05).to_scipy().toarray()
    assert C[0, 1] == 0.0 and C[0, 2] == -0.3   # 0.1 <= 0.2 dropped, 0.3 kept
    assert C[1, 2] == 0.0 and C[1, 0] == 0.2
    assert np.all(C[2] == 1.0)


def test_composite_threshold_uses_the_signed_row_maximum():
    # tpetra/src/MCLS_TpetraHelpers.hpp:226-233 takes the row maximum of the
    # signed values.  With PL = -D^-1 every row of the composite operator has
    # a negative diagonal, so the signed maximum is the largest positive
    # off-diagonal entry and the filter keeps more than a magnitude-based
    # threshold would.
    A = P.anisotropic2d(8, 20.0, 0.6)
    thr = 0.3
    neg = sp.diags(-1.0 / A.diagonal(), format="csr")
    M = (neg @ A).T.tocsr()  # transposed composite operator (adjoint)
    kept_signed = kept_abs = 0
    for i in range(M.shape[0]):
        v = M.data[M.indptr[i]:M.indptr[i + 1]]
        kept_signed += int(np.sum(np.abs(v) > thr * v.max()))
        kept_abs += int(np.sum(np.abs(v) > thr * np.abs(v).max()))
    assert kept_signed > kept_abs
    o = O.MC(O.Csr.from_scipy(A), PL=O.Csr.from_scipy(neg), direction=0,
             composite_threshold=thr).domain()
    # H = I - M keeps every retained entry of M (its diagonal becomes 2).
    assert len(o["col"]) == kept_signed
