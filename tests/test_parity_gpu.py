"""Parity of the CUDA path (through the C ABI) with the oracle.

Bars:
* domain (H, CDFs, weights): bit-exact against the oracle's restatement of
  AlmostOptimalDomain::addMatrixToDomain;
* walk trajectories (states per step, final weight, termination event,
  starting state): bit-exact with the FP64 walk, for the reference Xorshift
  stream and for the counter-based stream;
* FP64 tallies: equal to the oracle up to atomic summation order (rel 1e-12);
* FP32 tallies: per-component replica means within a z = 4 confidence
  interval of the oracle's FP64 replica means;
* MCSA: relative residual <= 1e-8 and agreement with a direct FP64 solve.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from mcls_b200 import capi
from mcls_b200 import problems as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _systems():
    A3, b3 = P.diffusion3d_varcoef(6, seed=4)
    return {
        "tridiag": (P.tridiag_test(10), np.full(10, -1.0)),
        "poisson2d": (P.poisson2d(9), np.ones(81)),
        "varcoef3d": (A3, b3),
        "aniso9pt": (P.anisotropic2d(8, 20.0, 0.6), np.linspace(-1, 1, 64)),
    }


def _gpu_domain(ctx, A, prec=None, block=2, **kw):
    op = capi.Operator(ctx, A)
    pc = None
    if prec == "jacobi":
        pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    elif prec == "block":
        pc = capi.Precond(ctx, op, capi.PREC_BLOCK_JACOBI, block_size=block)
    dom = capi.Domain(ctx, op, pc, **kw)
    return dom, op, pc


def _oracle_mc(A, prec=None, block=2, **kw):
    Ao = O.Csr.from_scipy(A)
    PL = None
    if prec == "jacobi":
        PL = O.point_jacobi(Ao)
    elif prec == "block":
        PL = O.block_jacobi(Ao, block)
    return O.MC(Ao, PL=PL, **kw), Ao, PL


@pytest.mark.parametrize("name", ["tridiag", "poisson2d", "varcoef3d", "aniso9pt"])
@pytest.mark.parametrize("prec", [None, "jacobi", "block"])
@pytest.mark.parametrize("direction", [0, 1])
def test_domain_bit_exact(ctx, name, prec, direction):
    A, _ = _systems()[name]
    if prec == "block" and A.shape[0] % 2:
        pytest.skip("block size must divide n")
    try:
        mc, _, _ = _oracle_mc(A, prec, direction=direction)
    except RuntimeError:
        # Every entry of some row of H falls below epsilon (a block-Jacobi
        # block that inverts its rows exactly): the reference trips
        # MCLS_CHECK(num_entries > 0); the device build reports it.
        with pytest.raises(capi.MclsError) as e:
            _gpu_domain(ctx, A, prec, direction=direction, precision=capi.FP64)
        assert e.value.code == capi.ERR_DEGENERATE
        return
    dom, op, pc = _gpu_domain(ctx, A, prec, direction=direction, precision=capi.FP64)
    g, o = dom.export(), mc.domain()
    assert np.array_equal(g["rowptr"], o["rowptr"])
    assert np.array_equal(g["col"], o["col"])
    if prec == "block":
        # Block inverses come from the same algorithm but not the same
        # LAPACK code, and the composite sums several products per entry.
        assert np.allclose(g["h"], o["h"], rtol=1e-12, atol=1e-14)
        assert np.allclose(g["cdf"], o["cdf"], rtol=1e-12, atol=1e-14)
    else:
        assert np.array_equal(g["h"], o["h"])
        assert np.array_equal(g["cdf"], o["cdf"])
        assert np.array_equal(g["weights"], o["weights"])


def _trace_compare(ctx, A, b, prec, solves=3, **kw):
    L = kw.get("history_length", 10)
    dom, op, pc = _gpu_domain(ctx, A, prec, precision=capi.FP64, **kw)
    okw = dict(kw)
    okw["rng_mode"] = okw.pop("rng_mode", capi.RNG_COUNTER)
    if "source_sampling" in okw:
        okw["stratified"] = okw.pop("source_sampling")
    mc, _, _ = _oracle_mc(A, prec, **okw)
    for rep in range(solves):
        rhs = b * (1.0 + 0.25 * rep)
        xg, nhg, tg = dom.mc_trace(rhs, 100000)
        xo, nho, to = mc.solve(rhs, trace=100000)
        assert nhg == nho
        assert np.array_equal(tg["start"], to["start"])
        assert np.array_equal(tg["states"], to["states"])
        assert np.array_equal(tg["events"], to["events"])
        if okw["rng_mode"] == capi.RNG_REFERENCE:
            assert np.array_equal(tg["final_weight"], to["final_weight"])
        else:
            # Outside the reproducible mode |b|_1 (the starting weight) is a
            # parallel tree sum: the weights agree to its rounding.
            assert np.allclose(tg["final_weight"], to["final_weight"], rtol=1e-13, atol=0)
        assert tg["states"].shape[1] == L + 1
        scale = np.abs(xo).max()
        assert np.allclose(xg, xo, rtol=1e-12, atol=1e-12 * scale)


@pytest.mark.parametrize("name", ["tridiag", "poisson2d", "varcoef3d", "aniso9pt"])
def test_trajectories_reference_stream(ctx, name):
    A, b = _systems()[name]
    _trace_compare(ctx, A, b, "jacobi", rng_mode=capi.RNG_REFERENCE, seed=12345,
                   history_length=10, sample_ratio=2.0)


@pytest.mark.parametrize("name", ["tridiag", "poisson2d", "varcoef3d"])
@pytest.mark.parametrize("estimator", [0, 1])
def test_trajectories_counter_stream(ctx, name, estimator):
    A, b = _systems()[name]
    _trace_compare(ctx, A, b, "jacobi", rng_mode=capi.RNG_COUNTER, seed=777, estimator=estimator,
                   history_length=7)


def test_trajectories_stratified_and_unpreconditioned(ctx):
    A, b = _systems()["tridiag"]
    _trace_compare(ctx, A, b, None, rng_mode=capi.RNG_REFERENCE, seed=99, source_sampling=1,
                   history_length=5, sample_ratio=3.0)


@pytest.mark.parametrize("estimator", [0, 1])
def test_trajectories_forward(ctx, estimator):
    A, b = _systems()["poisson2d"]
    _trace_compare(ctx, A, b, "jacobi", rng_mode=capi.RNG_REFERENCE, seed=5, direction=1,
                   estimator=estimator, history_length=6, sample_ratio=2.0)


def test_reference_signed_first_source_element(ctx):
    # b[0] < 0: the source CDF starts at the signed b[0] (quirk kept).
    A = P.tridiag_test(10)
    b = np.full(10, -1.0)
    _trace_compare(ctx, A, b, None, rng_mode=capi.RNG_REFERENCE, seed=3, history_length=4)


def test_weight_cutoff_trajectories(ctx):
    A, b = _systems()["varcoef3d"]
    _trace_compare(ctx, A, b, "jacobi", rng_mode=capi.RNG_COUNTER, seed=21, history_length=200,
                   weight_cutoff=0.05)


@pytest.mark.parametrize("direction,estimator", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_fp32_tally_mean_within_ci(ctx, direction, estimator):
    A, _ = _systems()["varcoef3d"]
    n = A.shape[0]
    rng = np.random.Generator(np.random.PCG64(8))
    b = rng.uniform(0.1, 1.0, n)
    reps = 24
    kw = dict(direction=direction, estimator=estimator, history_length=8, sample_ratio=4.0)
    dom, op, pc = _gpu_domain(ctx, A, "jacobi", precision=capi.FP32, rng_mode=capi.RNG_COUNTER,
                              seed=1, **kw)
    mc, _, _ = _oracle_mc(A, "jacobi", rng_mode=1, seed=2, **kw)
    xs_g = np.array([dom.mc_solve(b)[0] for _ in range(reps)])
    xs_o = np.array([mc.solve(b)[0] for _ in range(reps)])
    mg, mo = xs_g.mean(0), xs_o.mean(0)
    se = np.sqrt(xs_g.var(0, ddof=1) / reps + xs_o.var(0, ddof=1) / reps) + 1e-12 * np.abs(mo).max()
    z = np.abs(mg - mo) / se
    assert np.mean(z > 4.0) <= 0.01, z.max()
    # and the whole difference vector is within 4 pooled standard errors
    assert np.linalg.norm(mg - mo) <= 4.0 * np.linalg.norm(se)


def test_mc_solve_unpreconditioned_reference_sign(ctx):
    # tstTpetraMonteCarloSolverManager: Sample Ratio 10, solution sign.
    A = P.tridiag_test(10)
    for direction in (0, 1):
        dom, op, pc = _gpu_domain(ctx, A, None, direction=direction, sample_ratio=10.0,
                                  precision=capi.FP32)
        for bval in (-1.0, 2.0, -2.0):
            x, st = dom.mc_solve(np.full(10, bval))
            assert np.all(np.sign(x) == np.sign(bval))
            assert st["walk_steps"] > 0


@pytest.mark.parametrize("precision", [capi.FP64, capi.FP32])
@pytest.mark.parametrize("direction", [0, 1])
def test_mcsa_tridiagonal_reference_test(ctx, precision, direction):
    # tstTpetraMCSASolverManager: tol 1e-8, < 20 iterations, four solves with
    # b = -1, 2, 2 (same operator re-set), -2; solution sign follows b.
    A = P.tridiag_test(10)
    dom, op, pc = _gpu_domain(ctx, A, None, direction=direction, precision=precision,
                              sample_ratio=1.0, seed=17)
    for bval in (-1.0, 2.0, 2.0, -2.0):
        x, st = dom.mcsa_solve(np.full(10, bval), tolerance=1e-8, max_iters=20)
        assert st["converged"] == 1 and st["iterations"] < 20 and st["achieved_tol"] > 0
        assert np.all(np.sign(x) == np.sign(bval))
        r = np.full(10, bval) - A @ x
        assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(np.full(10, bval)) * 1.0001


@pytest.mark.parametrize("precision", [capi.FP64, capi.FP32])
def test_mcsa_poisson_jacobi_solution(ctx, precision):
    A = P.poisson2d(24)
    b = np.ones(A.shape[0])
    dom, op, pc = _gpu_domain(ctx, A, "jacobi", precision=precision, seed=3, history_length=10)
    x, st = dom.mcsa_solve(b, tolerance=1e-8, max_iters=5000)
    assert st["converged"] == 1
    Dinv = 1.0 / A.diagonal()
    assert np.linalg.norm(Dinv * (b - A @ x)) <= 1e-8 * np.linalg.norm(Dinv * b) * 1.0001
    xs = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-6


def test_mcsa_varcoef_expected_value_fp32(ctx):
    A, b = P.diffusion3d_varcoef(12, seed=1)
    dom, op, pc = _gpu_domain(ctx, A, "jacobi", precision=capi.FP32, estimator=1,
                              sample_ratio=2.0, seed=3)
    x, st = dom.mcsa_solve(b, tolerance=1e-8, max_iters=3000)
    assert st["converged"] == 1
    xs = spla.spsolve(A.tocsc(), b)
    rel = np.linalg.norm(b - A @ x) / np.linalg.norm(b)
    assert rel < 1e-6
    assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-6
    # the oracle restatement converges on the same system
    r = O.mcsa_solve(O.Csr.from_scipy(A), b, PL=O.point_jacobi(O.Csr.from_scipy(A)),
                     tolerance=1e-8, max_iters=3000, estimator=1, sample_ratio=2.0, rng_mode=1,
                     seed=3)
    assert r["converged"]


def test_mcsa_matches_oracle_iterates_in_parity_mode(ctx):
    # FP64 walks on the reference stream: the MCSA loop takes the oracle's
    # steps.  The residual SpMV rounds differently (fused multiply-add), so a
    # source count can differ by one in a late iteration and the two iterates
    # agree to the solve tolerance, not bit for bit.
    A = P.tridiag_test(10)
    b = np.full(10, 2.0)
    dom, op, pc = _gpu_domain(ctx, A, None, precision=capi.FP64, rng_mode=capi.RNG_REFERENCE,
                              seed=4242, history_length=10)
    x, st = dom.mcsa_solve(b, tolerance=1e-8, max_iters=20)
    r = O.mcsa_solve(O.Csr.from_scipy(A), b, tolerance=1e-8, max_iters=20, rng_mode=0, seed=4242)
    assert abs(st["iterations"] - r["iters"]) <= 1
    assert np.allclose(x, r["x"], rtol=1e-7, atol=1e-12)


def test_block_jacobi_matches_oracle(ctx):
    A = P.anisotropic2d(8, 10.0, 0.3)
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_BLOCK_JACOBI, block_size=4)
    G = pc.to_scipy(A.shape[0]).toarray()
    Po = O.block_jacobi(O.Csr.from_scipy(A), 4).to_scipy().toarray()
    assert np.allclose(G, Po, rtol=1e-13, atol=1e-15)


def test_spectral_radius_matches_dense_eigensolve(ctx):
    A, _ = P.diffusion3d_varcoef(5, seed=2)
    dom, op, pc = _gpu_domain(ctx, A, "jacobi", precision=capi.FP64)
    d = dom.export()
    n = A.shape[0]
    H = sp.csr_matrix((d["h"], d["col"], d["rowptr"]), shape=(n, n)).toarray()
    for which, M in ((0, H), (1, np.abs(H)), (2, np.abs(H) * d["weights"][:, None])):
        rho = dom.spectral_radius(which, max_iters=4000, tol=1e-10)
        want = np.abs(np.linalg.eigvals(M)).max()
        assert abs(rho - want) <= 1e-4 * want, (which, rho, want)


@pytest.mark.parametrize("name", ["varcoef3d", "aniso9pt"])
def test_convergence_criteria_match_dense_computation(ctx, name):
    # AlmostOptimalDomain::computeConvergenceCriteria
    # (src/MCLS_AlmostOptimalDomain_impl.hpp:437-635): spectral radii of H,
    # |H| and H*, |H|_inf, the smallest row sum and the balance parameters
    # max_j |h_ij| / max_j |h_ji|.
    A, _ = _systems()[name]
    dom, op, pc = _gpu_domain(ctx, A, "jacobi", precision=capi.FP64)
    c = dom.convergence_criteria(max_iters=4000, tol=1e-10)
    d = dom.export()
    n = A.shape[0]
    H = sp.csr_matrix((d["h"], d["col"], d["rowptr"]), shape=(n, n)).toarray()
    Hp = np.abs(H)
    for key, M in (("rho_h", H), ("rho_abs", Hp), ("rho_star", Hp * d["weights"][:, None])):
        want = np.abs(np.linalg.eigvals(M)).max()
        assert abs(c[key] - want) <= 1e-4 * want, (key, c[key], want)
    rs = Hp.sum(1)
    assert c["row_sum_max"] == pytest.approx(rs.max(), rel=1e-14)
    assert c["row_sum_min"] == pytest.approx(rs.min(), rel=1e-14)
    colmax = Hp.max(0)
    keep = colmax > 0
    ratio = Hp.max(1)[keep] / colmax[keep]
    assert c["balance_min"] == pytest.approx(ratio.min(), rel=1e-14)
    assert c["balance_max"] == pytest.approx(ratio.max(), rel=1e-14)
    assert c["balance_ave"] == pytest.approx(ratio.mean(), rel=1e-12)


def test_degenerate_row_is_reported(ctx):
    A = sp.lil_matrix((4, 4))
    A[0, 0] = 1.0
    A[1, 1] = 1.0  # H row = 1 - 1 = 0 -> dropped -> empty row
    A[2, 2] = 2.0
    A[3, 3] = 2.0
    op = capi.Operator(ctx, sp.csr_matrix(A))
    with pytest.raises(capi.MclsError) as e:
        capi.Domain(ctx, op, None, precision=capi.FP32)
    assert e.value.code == capi.ERR_DEGENERATE


def test_invalid_operator_is_rejected(ctx):
    bad = sp.csr_matrix((np.array([1.0, np.nan]), np.array([0, 1]), np.array([0, 1, 2])),
                        shape=(2, 2))
    with pytest.raises(capi.MclsError) as e:
        capi.Operator(ctx, bad)
    assert e.value.code == capi.ERR_INVALID_ARG


def test_reference_stream_weight_cutoff_needs_fp64(ctx):
    # Variable-length histories on the reference stream are walked by the
    # FP64 parity walk only.
    A = P.poisson2d(4)
    op = capi.Operator(ctx, A)
    with pytest.raises(capi.MclsError) as e:
        capi.Domain(ctx, op, None, rng_mode=capi.RNG_REFERENCE, weight_cutoff=1e-4,
                    precision=capi.FP32)
    assert e.value.code == capi.ERR_UNSUPPORTED


@pytest.mark.parametrize("name,L,cutoff", [("tridiag", 10, 1e-4), ("varcoef3d", 200, 0.05),
                                           ("poisson2d", 40, 1e-4), ("aniso9pt", 30, 1e-3)])
def test_weight_cutoff_trajectories_reference_stream(ctx, name, L, cutoff):
    # "Weight Cutoff" with "Reproducible MC Mode": histories end at different
    # steps, so each history's draws start where the previous one's ended in
    # the reference's single stream; trajectories, events and final weights
    # are bit-exact against the oracle over successive solves.
    A, b = _systems()[name]
    _trace_compare(ctx, A, b, "jacobi", rng_mode=capi.RNG_REFERENCE, seed=31, history_length=L,
                   weight_cutoff=cutoff, sample_ratio=2.0)


@pytest.mark.parametrize("direction", [0, 1])
def test_mcsa_weight_cutoff_reference_stream_matches_oracle(ctx, direction):
    # MCSA with the cutoff in the reproducible mode follows the oracle's
    # iterates (the residual rounds differently, as in the fixed-length test).
    A = P.poisson2d(10)
    b = np.ones(A.shape[0])
    kw = dict(history_length=20, weight_cutoff=1e-3, sample_ratio=4.0)
    dom, op, pc = _gpu_domain(ctx, A, "jacobi", precision=capi.FP64,
                              rng_mode=capi.RNG_REFERENCE, seed=77, direction=direction, **kw)
    x, st = dom.mcsa_solve(b, tolerance=1e-8, max_iters=400)
    Ao = O.Csr.from_scipy(A)
    r = O.mcsa_solve(Ao, b, PL=O.point_jacobi(Ao), tolerance=1e-8, max_iters=400, rng_mode=0,
                     seed=77, direction=direction, **kw)
    assert st["converged"] == 1 and r["converged"]
    assert abs(st["iterations"] - r["iters"]) <= 1
    assert np.allclose(x, r["x"], rtol=1e-7, atol=1e-12 * np.abs(r["x"]).max())


def test_device_vectors_entry_point(ctx):
    torch = pytest.importorskip("torch")
    A = P.poisson2d(16)
    b = np.ones(A.shape[0])
    dom, op, pc = _gpu_domain(ctx, A, "jacobi", precision=capi.FP32, seed=9)
    bt = torch.tensor(b, device="cuda:0", dtype=torch.float64)
    xt = torch.zeros_like(bt)
    torch.cuda.synchronize()
    st = dom.mcsa_solve_dev(bt.data_ptr(), xt.data_ptr(), tolerance=1e-8, max_iters=5000)
    assert st["converged"] == 1
    x = xt.cpu().numpy()
    assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-6


@pytest.mark.parametrize("direction,estimator", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_fused_iteration_matches_unfused(ctx, direction, estimator):
    # Point Jacobi runs the fused iteration (Richardson+residual, correction+
    # residual+norm+check); the same diagonal passed as a user CSR matrix runs
    # the kernel-per-operation path.  After a fixed number of iterations the
    # iterates agree bit for bit (the two residual-norm reductions associate
    # differently, so the stopping test is kept out of the comparison).
    A, b = P.diffusion3d_varcoef(10, seed=5)
    op = capi.Operator(ctx, A)
    pj = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    pu = capi.Precond(ctx, op, capi.PREC_USER_CSR, user=sp.diags(1.0 / A.diagonal()).tocsr())
    kw = dict(precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=11, direction=direction,
              estimator=estimator, sample_ratio=2.0)
    d1 = capi.Domain(ctx, op, pj, **kw)
    d2 = capi.Domain(ctx, op, pu, **kw)
    # Forward: each state receives exactly two history sums (Sample Ratio 2)
    # and a + b == b + a, so the unordered FP64 reductions are still
    # deterministic and 25 iterations compare bit for bit.  Adjoint: many
    # unordered per-step reductions per state round in run-dependent order,
    # so one iteration is compared to round-off.
    its = 25 if direction == 1 else 1
    x1, s1 = d1.mcsa_solve(b, tolerance=0.0, max_iters=its)
    x2, s2 = d2.mcsa_solve(b, tolerance=0.0, max_iters=its)
    assert s1["iterations"] == s2["iterations"] == its
    d1.reseed(11)
    x3, s3 = d1.mcsa_solve(b, tolerance=0.0, max_iters=its, host_loop=1)
    assert s3["iterations"] == its
    if direction == 1:
        assert np.array_equal(x1, x2) and np.array_equal(x1, x3)
    else:
        assert np.allclose(x1, x2, rtol=1e-12, atol=0)
        assert np.allclose(x1, x3, rtol=1e-12, atol=0)
    assert abs(s1["residual_norm"] - s2["residual_norm"]) <= 1e-10 * s2["residual_norm"]


@pytest.mark.parametrize("direction", [capi.FORWARD, capi.ADJOINT])
def test_fused_learned_iteration_matches_unfused(ctx, direction):
    # A learned left preconditioner kept on A's pattern runs the fused
    # iteration with M applied by diagonals; the same M given as a user CSR
    # matrix runs the kernel-per-operation path.
    import torch

    from mcls_b200 import spai

    A, b = P.diffusion3d_varcoef(10, seed=5)
    op = capi.Operator(ctx, A)
    net = capi.SpaiNet(ctx, spai.stencil_slots(A), seed=1)
    V = torch.randn((6, A.shape[0]), dtype=torch.float64, device="cuda:0")
    spai.train(net, [(op, V)], steps=150, lr=3e-3)
    rl, rj = net.rho(op)
    assert rl < min(rj, 1.0)
    pl = capi.Precond(ctx, op, capi.PREC_LEARNED_SPAI, net=net)
    M = pl.to_scipy(A.shape[0])
    assert M.nnz == A.nnz  # kept on A's pattern, not the Jacobi fallback
    pu = capi.Precond(ctx, op, capi.PREC_USER_CSR, user=M)
    kw = dict(precision=capi.FP32, rng_mode=capi.RNG_COUNTER, seed=11, direction=direction,
              estimator=capi.EXPECTED_VALUE if direction == capi.FORWARD else capi.COLLISION,
              sample_ratio=2.0)
    d1 = capi.Domain(ctx, op, pl, **kw)
    d2 = capi.Domain(ctx, op, pu, **kw)
    its = 20 if direction == capi.FORWARD else 1
    x1, s1 = d1.mcsa_solve(b, tolerance=0.0, max_iters=its)
    x2, s2 = d2.mcsa_solve(b, tolerance=0.0, max_iters=its)
    assert s1["iterations"] == s2["iterations"] == its
    assert s1["kernel_launches"] < s2["kernel_launches"]
    if direction == capi.FORWARD:
        assert np.array_equal(x1, x2)
    else:
        assert np.allclose(x1, x2, rtol=1e-12, atol=0)


def test_smoother_steps_and_relaxation(ctx):
    A = P.poisson2d(20)
    b = np.ones(A.shape[0])
    dom, op, pc = _gpu_domain(ctx, A, "jacobi", precision=capi.FP32, seed=2,
                              neumann_relaxation=0.9)
    x, st = dom.mcsa_solve(b, tolerance=1e-8, max_iters=5000, smoother_steps=2,
                           richardson_omega=0.8)
    assert st["converged"] == 1
    Dinv = 1.0 / A.diagonal()
    assert np.linalg.norm(Dinv * (b - A @ x)) <= 1e-8 * np.linalg.norm(Dinv * b) * 1.0001


@pytest.mark.parametrize("name", ["tridiag", "poisson2d", "varcoef3d", "aniso9pt", "nonsym"])
def test_stencil_residual_is_bitwise_the_csr_one(ctx, name):
    # The MCSA residual kernels read a symmetric stencil operator through its
    # diagonal and upper diagonals only (the lower ones are the upper ones'
    # mirror); the sums must equal the CSR product's bit for bit, with the
    # full diagonal layout for a nonsymmetric operator.
    import torch

    systems = _systems()
    if name == "nonsym":
        A = sp.csr_matrix(P.poisson2d(9) + 0.1 * sp.eye(81, k=1))
    else:
        A = systems[name][0]
    n = A.shape[0]
    rng = np.random.default_rng(3)
    x = rng.standard_normal(n)
    b = rng.standard_normal(n)
    dom, op, pc = _gpu_domain(ctx, A, "jacobi", precision=capi.FP32)
    bt = torch.tensor(b, device="cuda:0")
    xt = torch.tensor(x, device="cuda:0")
    rp = torch.empty_like(bt)
    dom.mcsa_begin(bt.data_ptr(), xt.data_ptr(), tolerance=1e-8)
    dom.residual(rp.data_ptr())
    dom.mcsa_finish(xt.data_ptr())
    ref = (1.0 / A.diagonal()) * (b - op.apply(x))
    assert np.array_equal(rp.cpu().numpy(), ref)
