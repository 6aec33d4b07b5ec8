"""Failure detection without a GPU fault: a bounded device wait that runs out.

The learned-SPAI kernels wait on tensor-core completion barriers with a
bounded number of polls.  A host-set limit of 0 polls makes every such wait
give up at once (the barrier is never observed, as if nothing had set it).
The kernel then issues no further MMA, lets the one phase it committed
finish before releasing tensor memory, records the timeout in the context's
status word and returns; the call reports MCLSGPU_ERR_TIMEOUT and the
context stays usable: with the default limit restored, the same calls match
their oracle again.
"""
import numpy as np
import pytest

from mcls_b200 import capi
from mcls_b200 import problems as P
from mcls_b200 import spai
from oracle import spai_oracle as so


def _setup(ctx):
    A, _, _, _ = P.anisotropic2d_sample(24, seed=6)
    op = capi.Operator(ctx, A)
    net = capi.SpaiNet(ctx, spai.stencil_slots(A), seed=1)
    p = so.init_params(5, zero_last=False)
    net.params = p
    return A, op, net, p


@pytest.mark.gpu
def test_forward_wait_timeout_reports_and_recovers(ctx):
    A, op, net, p = _setup(ctx)
    try:
        ctx.set_wait_limit(0)
        try:
            with pytest.raises(capi.MclsError) as ei:
                net.infer(op, A.nnz)
            assert ei.value.code == capi.ERR_TIMEOUT
        finally:
            ctx.set_wait_limit(-1)
        out, _ = net.infer(op, A.nnz)
        ref, _ = so.forward(p, so.features(A))
        k = spai.stencil_slots(A)
        np.testing.assert_allclose(out[:, :k], ref[:, :k], rtol=2e-2,
                                   atol=2e-3 * np.abs(ref[:, :k]).max())
    finally:
        net.close()
        op.close()


@pytest.mark.gpu
def test_backward_wait_timeout_reports_and_recovers(ctx):
    import torch

    A, op, net, p = _setup(ctx)
    try:
        n = A.shape[0]
        V = torch.tensor(np.random.default_rng(3).standard_normal((2, n)), device="cuda:0")
        ctx.set_wait_limit(0)
        try:
            with pytest.raises(capi.MclsError) as ei:
                net.gradient(op, V.data_ptr(), 2)
            assert ei.value.code == capi.ERR_TIMEOUT
        finally:
            ctx.set_wait_limit(-1)
        loss, g = net.gradient(op, V.data_ptr(), 2)
        loss_ref, g_ref = so.loss_and_gradient(p, A, V.cpu().numpy(), rounded=True)
        np.testing.assert_allclose(loss, loss_ref, rtol=5e-3)
        assert np.linalg.norm(g - g_ref) <= 3e-2 * np.linalg.norm(g_ref)
    finally:
        net.close()
        op.close()
