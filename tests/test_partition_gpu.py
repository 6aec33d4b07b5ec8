"""Domain-decomposed transport on the GPU: a row-partitioned domain gives the
whole domain's Monte Carlo solve.

Two to four parts share one GPU (mcls_b200.partition.solve_local drives the
rounds and moves the histories between the parts' outboxes and inboxes).
Every history takes the transitions the whole-domain FP32 walk takes -- the
random stream travels with it -- so the parts' tallies equal the whole
domain's up to the order of the FP64 additions, and the walk-step totals are
equal.  Adjoint collision and forward (expected value, collision) walks, of
fixed length or ended by the weight cutoff; a forward history's sum goes
home to its start row's part when it ends elsewhere.
"""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from mcls_b200 import capi, partition
from mcls_b200 import problems as P

pytestmark = pytest.mark.gpu

MC = dict(precision=capi.FP32, rng_mode=capi.RNG_COUNTER, direction=capi.ADJOINT,
          estimator=capi.COLLISION, history_length=10, sample_ratio=2.0,
          record_format=capi.RECORD_PACKED)


def _parts(ctx, A, nparts, seed, capacity=None, **kw):
    n = A.shape[0]
    dinv = 1.0 / A.diagonal()
    if kw.get("direction", MC["direction"]) == capi.FORWARD:
        T = partition.composite(A, dinv)
    else:
        T = partition.transposed_composite(A, dinv)
    bounds = partition.row_bounds(n, nparts)
    p = capi.mc_params(seed=seed, **{**MC, **kw})
    cap = capacity or int(n * 2 + 64)
    return [partition.DevicePart(capi.Subdomain(ctx, n, bounds, q, T[bounds[q]:bounds[q + 1]],
                                                params=p), cap, "cuda:0")
            for q in range(nparts)]


def _whole(ctx, A, seed, **kw):
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    return capi.Domain(ctx, op, pc, seed=seed, **{**MC, **kw}), op, pc


WALKS = {
    "adjoint": {},
    "adjoint_cutoff": dict(weight_cutoff=0.6),
    "forward_ev": dict(direction=capi.FORWARD, estimator=capi.EXPECTED_VALUE),
    "forward_collision": dict(direction=capi.FORWARD, estimator=capi.COLLISION),
    "forward_ev_cutoff": dict(direction=capi.FORWARD, estimator=capi.EXPECTED_VALUE,
                              weight_cutoff=0.6),
    # Stencil records: column offsets from the global row, on the whole domain
    # and in every part.
    "adjoint_stencil": dict(record_format=capi.RECORD_STENCIL),
    "forward_ev_stencil": dict(direction=capi.FORWARD, estimator=capi.EXPECTED_VALUE,
                               record_format=capi.RECORD_STENCIL),
    "forward_ev_stencil16": dict(direction=capi.FORWARD, estimator=capi.EXPECTED_VALUE,
                                 record_format=capi.RECORD_STENCIL16),
}


@pytest.mark.parametrize("walks", sorted(WALKS))
@pytest.mark.parametrize("nparts", [2, 3, 4])
@pytest.mark.parametrize("name", ["varcoef3d", "poisson2d"])
def test_parts_give_the_whole_domain_solve(ctx, nparts, name, walks):
    import torch

    kw = WALKS[walks]
    if name == "varcoef3d":
        A, b = P.diffusion3d_varcoef(12, seed=7)
    else:
        A = P.poisson2d(30)
        b = np.linspace(-1.0, 2.0, A.shape[0])
    r = b / A.diagonal()  # the preconditioned residual an MCSA loop hands over
    dom, op, pc = _whole(ctx, A, 4242, **kw)
    parts = _parts(ctx, A, nparts, 4242, **kw)
    rt = torch.tensor(r, device="cuda:0")
    for solve in range(2):  # successive solves continue on the streams
        xw, st = dom.mc_solve(r, internal=True)
        xp, rounds, moved, steps = partition.solve_local(parts, rt)
        xp = xp.cpu().numpy()
        assert rounds >= 2 and moved > 0
        assert np.allclose(xp, xw, rtol=0, atol=1e-12 * np.abs(xw).max()), solve
        assert parts[0].sub.record_bytes == dom.info()["record_bytes"]
        assert steps == st["walk_steps"]
        if "weight_cutoff" in kw:
            assert steps < st["histories"] * 10  # some histories ended early
        else:
            assert steps == st["histories"] * 10


def test_parts_split_the_source(ctx):
    import torch

    A, b = P.diffusion3d_varcoef(10, seed=2)
    parts = _parts(ctx, A, 3, 99)
    rt = torch.tensor(b / A.diagonal(), device="cuda:0")
    starts = [p.begin(rt) for p in parts]
    total = starts[0][1]
    assert all(s[1] == total for s in starts) and sum(s[0] for s in starts) == total
    for p in parts:
        p.finish()


def test_small_outbox_is_reported(ctx):
    import torch

    A, b = P.diffusion3d_varcoef(8, seed=1)
    parts = _parts(ctx, A, 4, 3, capacity=1)
    rt = torch.tensor(b / A.diagonal(), device="cuda:0")
    with pytest.raises(capi.MclsError):
        partition.solve_local(parts, rt)


def test_partitioned_mc_drives_mcsa(ctx):
    # MCSA with the Monte Carlo correction from three parts: Richardson,
    # residual, partitioned correction, update; converges to the solution.
    # (2D Poisson: the adjoint collision estimator's variance makes MCSA
    # diverge on the strongly varying 3D coefficients, whole domain or not.)
    import torch

    A = P.poisson2d(20)
    b = np.ones(A.shape[0])
    n = A.shape[0]
    dinv = 1.0 / A.diagonal()
    parts = _parts(ctx, A, 3, 11)
    x = np.zeros(n)
    rp = dinv * (b - A @ x)
    crit = 1e-8 * np.linalg.norm(dinv * b)
    it = 0
    while np.linalg.norm(rp) > crit and it < 500:
        it += 1
        x = x + rp
        rp = dinv * (b - A @ x)
        d = partition.solve_local(parts, torch.tensor(rp, device="cuda:0"))[0]
        x = x + d.cpu().numpy()
        rp = dinv * (b - A @ x)
    assert np.linalg.norm(rp) <= crit
    xs = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x - xs) <= 1e-6 * np.linalg.norm(xs)
