"""Batched MCSA: systems of uneven size with several right-hand sides each in
one loop (shared forward FP32 walks), checked pair by pair against scipy
direct solves and against the single-system path."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from mcls_b200 import capi
from mcls_b200 import problems as P

pytestmark = pytest.mark.gpu


def _systems():
    A1 = P.poisson2d(15)
    A2, _ = P.diffusion3d_varcoef(8, seed=2)
    A3 = P.poisson2d(30, 20)
    A4, _ = P.diffusion3d_varcoef(10, seed=5)
    return [A1, A2, A3, A4], [1, 3, 2, 4]


def _solve(ctx, systems, nrhs, B_blocks, estimator=capi.EXPECTED_VALUE, tol=1e-8):
    import torch

    bt = capi.Batch(ctx, systems, nrhs, direction=capi.FORWARD, estimator=estimator,
                    precision=capi.FP32, sample_ratio=2.0, history_length=10, seed=3)
    B = torch.tensor(bt.pack(B_blocks), device="cuda:0").contiguous()
    X = torch.zeros_like(B)
    st, it, rr = bt.mcsa_solve_dev(B.data_ptr(), X.data_ptr(), tolerance=tol, max_iters=20000)
    return bt, bt.unpack(X.cpu().numpy()), st, it, rr


@pytest.mark.parametrize("estimator", [capi.EXPECTED_VALUE, capi.COLLISION])
def test_batch_pairs_converge_to_direct_solutions(ctx, estimator):
    systems, nrhs = _systems()
    rng = np.random.default_rng(0)
    Bb = [rng.uniform(0, 1, (A.shape[0], r)) for A, r in zip(systems, nrhs)]
    bt, X, st, it, rr = _solve(ctx, systems, nrhs, Bb, estimator)
    assert st["converged"] == 1 and st["walk_steps"] > 0
    for s, (A, r) in enumerate(zip(systems, nrhs)):
        assert np.all(it[s, :r] > 0), (s, it[s])
        assert np.all(it[s, r:] == -1)
        assert np.all(rr[s, :r] <= 1e-8), (s, rr[s])
        for k in range(r):
            xs = spla.spsolve(A.tocsc(), Bb[s][:, k])
            err = np.linalg.norm(X[s][:, k] - xs) / np.linalg.norm(xs)
            assert err <= 1e-6, (s, k, err)
    bt.close()


def test_duplicate_columns_share_walks_exactly(ctx):
    # Every right-hand side rides the same histories: equal columns give
    # equal solutions bit for bit.
    A, b = P.diffusion3d_varcoef(9, seed=1)
    B = np.stack([b, b, 2 * b], 1)
    bt, X, st, it, rr = _solve(ctx, [A], [3], [B])
    assert np.array_equal(X[0][:, 0], X[0][:, 1])
    np.testing.assert_allclose(X[0][:, 2], 2 * X[0][:, 0], rtol=1e-6)
    bt.close()


def test_batch_matches_single_system_iterations(ctx):
    import torch

    A, b = P.diffusion3d_varcoef(10, seed=7)
    bt, X, st, it, rr = _solve(ctx, [A, P.poisson2d(12)], [1, 1],
                               [b[:, None], np.ones((144, 1))])
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP32, direction=capi.FORWARD,
                      estimator=capi.EXPECTED_VALUE, sample_ratio=2.0, history_length=10)
    x1, s1 = dom.mcsa_solve(b, tolerance=1e-8, max_iters=20000)
    assert abs(int(it[0, 0]) - s1["iterations"]) <= max(3, 0.1 * s1["iterations"])
    np.testing.assert_allclose(X[0][:, 0], x1, rtol=1e-6, atol=1e-9 * np.abs(x1).max())
    bt.close()


def test_batch_autotune_and_layout(ctx):
    import torch

    systems, nrhs = _systems()  # right-hand sides 1, 3, 2, 4 -> widths 1, 4, 2, 4
    bt = capi.Batch(ctx, systems, nrhs, direction=capi.FORWARD, estimator=capi.EXPECTED_VALUE,
                    precision=capi.FP32, sample_ratio=1.0, history_length=10)
    assert bt.width == 4 and bt.rows == sum(A.shape[0] for A in systems)
    assert list(bt.widths) == [1, 4, 2, 4]
    # Grouped by width: the one-column system first, then the two-column one,
    # then the four-column ones in argument order; groups start on 16-element
    # boundaries and the blocks do not overlap.
    order = np.argsort(bt.elem_offsets)
    assert list(order) == [0, 2, 1, 3]
    ends = bt.elem_offsets + bt.n * bt.widths
    assert np.all(bt.elem_offsets[order][1:] >= ends[order][:-1])
    assert bt.elem_offsets[2] % 16 == 0 and bt.elem_offsets[1] % 16 == 0
    assert bt.elements >= ends.max() and bt.elements % 16 == 0
    B = torch.ones(bt.elements, dtype=torch.float64, device="cuda:0")
    X = torch.zeros_like(B)
    tuned = bt.autotune(B.data_ptr(), X.data_ptr(), reps=2)
    assert tuned["block_size"] in (128, 256) and tuned["grab"] in (1, 2, 4)
    assert tuned["walk_ms"] > 0
    bt.close()


@pytest.mark.parametrize("grab", [1, 4])
def test_batch_launch_shapes_agree(ctx, grab):
    # The walk's queue grab changes which warp runs a history, not its draws:
    # every shape gives the same solutions up to the order of the FP64 tally
    # additions.
    import torch

    systems, nrhs = _systems()
    rng = np.random.default_rng(1)
    Bb = [rng.uniform(0, 1, (A.shape[0], r)) for A, r in zip(systems, nrhs)]
    out = []
    for blk in (256, 128):
        bt = capi.Batch(ctx, systems, nrhs, direction=capi.FORWARD,
                        estimator=capi.EXPECTED_VALUE, precision=capi.FP32, sample_ratio=2.0,
                        history_length=10, seed=3)
        bt.set_launch(blk, grab)
        B = torch.tensor(bt.pack(Bb), device="cuda:0")
        X = torch.zeros_like(B)
        st, it, rr = bt.mcsa_solve_dev(B.data_ptr(), X.data_ptr(), tolerance=1e-8,
                                       max_iters=20000)
        assert st["converged"] == 1
        out.append(bt.unpack(X.cpu().numpy()))
        bt.close()
    for a, b in zip(*out):
        np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-10 * np.abs(b).max())


def test_batch_rejects_adjoint_and_too_many_rhs(ctx):
    A = P.poisson2d(8)
    with pytest.raises(capi.MclsError) as e:
        capi.Batch(ctx, [A], [1], direction=capi.ADJOINT, precision=capi.FP32)
    assert e.value.code == capi.ERR_UNSUPPORTED
    with pytest.raises(capi.MclsError) as e:
        capi.Batch(ctx, [A], [17], direction=capi.FORWARD, precision=capi.FP32)
    assert e.value.code == capi.ERR_INVALID_ARG
