"""Learned SPAI on the GPU against its CPU oracle (oracle/spai_oracle.py).

Forward outputs and parameter gradients of the tensor-core kernels are
compared with the oracle's BF16-rounded restatement.  Tolerances: outputs
within 2e-2 relative (+ 2e-3 of the largest output) -- BF16 activations can
round differently when FP32 accumulation orders differ; each parameter
block's gradient within 3e-2 relative L2 error; M values exactly as the
formula (delta + out) / A_ii gives them from the device outputs.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from mcls_b200 import capi
from mcls_b200 import problems as P
from mcls_b200 import spai
from oracle import spai_oracle as so

BLOCKS = {"W1": (so.W1, so.B1), "b1": (so.B1, so.W2), "W2": (so.W2, so.B2),
          "b2": (so.B2, so.W3), "W3": (so.W3, so.B3), "b3": (so.B3, so.NPARAMS)}


def _op_and_net(ctx, A, p):
    op = capi.Operator(ctx, A)
    net = capi.SpaiNet(ctx, spai.stencil_slots(A), seed=1)
    net.params = p
    return op, net


@pytest.mark.gpu
@pytest.mark.parametrize("n", [30, 32])
def test_forward_matches_oracle(ctx, n):
    A, _, _, _ = P.anisotropic2d_sample(n, seed=4)
    p = so.init_params(7, zero_last=False)
    op, net = _op_and_net(ctx, A, p)
    out, m = net.infer(op, A.nnz)
    ref, _ = so.forward(p, so.features(A))
    k = spai.stencil_slots(A)
    np.testing.assert_allclose(out[:, :k], ref[:, :k], rtol=2e-2,
                               atol=2e-3 * np.abs(ref[:, :k]).max())
    np.testing.assert_allclose(m, so.mvalues(A, out), rtol=1e-12, atol=0)


@pytest.mark.gpu
def test_zero_output_layer_gives_point_jacobi(ctx):
    A, _, _, _ = P.anisotropic2d_sample(20, seed=2)
    op, net = _op_and_net(ctx, A, so.init_params(3, zero_last=True))
    out, m = net.infer(op, A.nnz)
    assert np.all(out == 0)
    M = sp.csr_matrix((m, A.indices, A.indptr), shape=A.shape)
    np.testing.assert_array_equal(M.diagonal(), 1.0 / A.diagonal())
    assert np.count_nonzero(M.toarray() - np.diag(M.diagonal())) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("n,seed,pen_w", [(30, 4, 0.0), (40, 9, 0.0), (30, 4, 5.0)])
def test_gradient_matches_oracle(ctx, n, seed, pen_w):
    import torch

    A, _, _, _ = P.anisotropic2d_sample(n, seed=seed)
    p = so.init_params(5, zero_last=False)
    op, net = _op_and_net(ctx, A, p)
    net.set_penalty(pen_w, 0.9)
    V = np.random.default_rng(seed).standard_normal((3, A.shape[0]))
    Vt = torch.tensor(V, device="cuda:0").contiguous()
    loss, g = net.gradient(op, Vt.data_ptr(), 3)
    loss_o, g_o = so.loss_and_gradient(p, A, V, rounded=True, pen_w=pen_w, pen_c=0.9)
    np.testing.assert_allclose(loss, loss_o, rtol=5e-3)
    for name, (lo, hi) in BLOCKS.items():
        err = np.linalg.norm(g[lo:hi] - g_o[lo:hi]) / np.linalg.norm(g_o[lo:hi])
        assert err < 3e-2, (name, err)


@pytest.mark.gpu
def test_adam_steps_lower_the_loss(ctx):
    import torch

    A, _, _, _ = P.anisotropic2d_sample(24, seed=6)
    op, net = _op_and_net(ctx, A, so.init_params(8, zero_last=True))
    V = torch.randn((4, A.shape[0]), dtype=torch.float64, device="cuda:0")
    l0 = net.gradient(op, V.data_ptr(), 4)[0]
    for _ in range(30):
        net.train_step(op, V.data_ptr(), 4, lr=2e-3)
    l1 = net.gradient(op, V.data_ptr(), 4)[0]
    assert l1 < l0


@pytest.mark.gpu
def test_gate_falls_back_to_jacobi(ctx):
    A, _, _, _ = P.anisotropic2d_sample(24, seed=3)
    op = capi.Operator(ctx, A)
    net = capi.SpaiNet(ctx, spai.stencil_slots(A), seed=1)
    # Zero output layer: M is point Jacobi, rho equal -> the plain one is kept.
    pc = capi.Precond(ctx, op, capi.PREC_LEARNED_SPAI, net=net)
    J = pc.to_scipy(A.shape[0])
    np.testing.assert_array_equal(J.toarray(), np.diag(1.0 / A.diagonal()))
    # A network that inflates M: rho(I - M A) > 1, fallback taken.
    p = net.params
    p[so.B3:so.NPARAMS] = 4.0
    net.params = p
    rl, rj = net.rho(op)
    assert rl > 1.0 > rj
    pc2 = capi.Precond(ctx, op, capi.PREC_LEARNED_SPAI, net=net)
    np.testing.assert_array_equal(pc2.to_scipy(A.shape[0]).toarray(), J.toarray())
    # Without a stencil network at all: Jacobi.
    pc3 = capi.Precond(ctx, op, capi.PREC_LEARNED_SPAI)
    np.testing.assert_array_equal(pc3.to_scipy(A.shape[0]).toarray(), J.toarray())


def _mcsa_iterations(ctx, op, A, b, kind, net, max_iters):
    """MCSA iterations to 1e-8 (adjoint collision, FP64 walks); max_iters + 1
    when the solve diverges or does not converge."""
    pc = capi.Precond(ctx, op, kind, net=net if kind == capi.PREC_LEARNED_SPAI else None)
    dom = capi.Domain(ctx, op, pc, precision=capi.FP64, rng_mode=capi.RNG_COUNTER, seed=5,
                      estimator=capi.COLLISION, direction=capi.ADJOINT, sample_ratio=4.0,
                      history_length=10)
    try:
        x, st = dom.mcsa_solve(b, np.zeros_like(b), tolerance=1e-8, max_iters=max_iters)
    except capi.MclsError as e:
        assert e.code == capi.ERR_DIVERGED, e
        return max_iters + 1, None
    finally:
        dom.close()
        pc.close()
    if not st["converged"]:
        return max_iters + 1, None
    return st["iterations"], x


@pytest.mark.gpu
def test_trained_network_beats_jacobi(ctx):
    """What the trained network gains on held-out anisotropic systems: lower
    rho(I - M A) than point Jacobi and fewer MCSA iterations to 1e-8 (point
    Jacobi MCSA may not converge at all: its |H| row sums exceed 1 where the
    cross terms are strong)."""
    n = 24
    slots = None
    samples = []
    for seed in range(6):
        A, b, _, _ = P.anisotropic2d_sample(n, seed=100 + seed)
        slots = slots or spai.stencil_slots(A)
        if spai.stencil_slots(A) != slots:
            continue
        op = capi.Operator(ctx, A)
        samples.append((op, spai.training_vectors(ctx, op, b, seed=seed)))
    net = capi.SpaiNet(ctx, slots, seed=0)
    losses = spai.train(net, samples, steps=600, lr=3e-3)
    assert np.mean(losses[-20:]) < 0.5 * np.mean(losses[:6])
    checked = 0
    for seed in (200, 201, 202):
        A, b, _, _ = P.anisotropic2d_sample(n, seed=seed)
        if spai.stencil_slots(A) != slots:
            continue
        op = capi.Operator(ctx, A)
        rl, rj = net.rho(op)
        assert rl < rj
        its_l, x = _mcsa_iterations(ctx, op, A, b, capi.PREC_LEARNED_SPAI, net, 3000)
        assert x is not None, "learned-SPAI MCSA did not converge"
        assert np.linalg.norm(b - A @ x) <= 1e-6 * np.linalg.norm(b)
        its_j, _ = _mcsa_iterations(ctx, op, A, b, capi.PREC_POINT_JACOBI, None, 3000)
        assert its_j > 1.5 * its_l, (seed, its_j, its_l)
        checked += 1
    assert checked >= 2
