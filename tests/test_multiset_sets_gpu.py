"""Multi-set MCSA through the C ABI (mclsgpu_mcsa_solve_sets), the drop-in
form of MCSASolverManager on a MultiSetLinearProblem with several sets.

* Two sets in two processes on one GPU, corrections summed over gloo on host
  copies: both sets end with the same iterate and iteration count, equal
  bit for bit to the step-wise two-set emulation in one process (the same
  per-set streams), and the direct solution; the same for the
  Anderson-accelerated solve (mclsgpu_anderson_solve_sets).
* One set through the library's NCCL communicator (a one-rank clique): the
  loop with the ncclAllReduce runs inside the captured device-side WHILE
  loop and gives the host-loop result bit for bit.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import scipy.sparse.linalg as spla

from mcls_b200 import capi, multiset
from mcls_b200 import problems as P

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _domain(ctx, op, pc, seed):
    # Forward expected-value walks, one history per row: each row's tally is
    # one addition onto zero, so a set's correction is the same bits on every
    # run (adjoint tallies of several histories into one row are FP64 atomic
    # sums whose order, and last bits, vary from run to run).
    return capi.Domain(ctx, op, pc, precision=capi.FP64, rng_mode=capi.RNG_COUNTER, seed=seed,
                       estimator=capi.EXPECTED_VALUE, direction=capi.FORWARD, sample_ratio=1.0,
                       history_length=10)


def _emulated_two_sets(ctx, A, b):
    engines = []
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    engines = [multiset.DeviceEngine(_domain(ctx, op, pc, capi.rank_seed(99, r)), A.shape[0])
               for r in range(2)]
    params = capi.mcsa_params(tolerance=1e-8, max_iters=5000)
    norms = [e.begin(b, np.zeros_like(b), params) for e in engines]
    crit = 1e-8 * norms[0][1]
    it, rn = 0, norms[0][0]
    while rn > crit and it < 5000:
        it += 1
        d = [e.correction().clone() for e in engines]
        total = d[0] + d[1]
        rn = [e.apply(total, 0.5) for e in engines][0]
    return engines[0].finish()[0].cpu().numpy(), it


def _emulated_two_anderson_sets(ctx, A, b):  # noqa: D103
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    engines = [multiset.DeviceEngine(_domain(ctx, op, pc, capi.rank_seed(17, r)), A.shape[0])
               for r in range(2)]
    params = capi.anderson_params(tolerance=1e-10, max_iters=2000, storage_depth=3)
    done = [e.aa_begin(b, np.zeros_like(b), params) for e in engines][0][2]
    steps = 0
    while not done:
        steps += 1
        d = [e.aa_correction().clone() for e in engines]
        total = d[0] + d[1]
        done = [e.aa_apply(total, 0.5) for e in engines][0][1]
    return engines[0].aa_finish()[0].cpu().numpy(), steps


def test_two_processes_sum_their_corrections(ctx, tmp_path):
    A = P.poisson2d(20)
    b = np.linspace(0.1, 1.0, A.shape[0])
    port = _free_port()
    procs, outs = [], []
    for r in range(2):
        out = str(tmp_path / f"set{r}.json")
        outs.append(out)
        env = dict(os.environ, RANK=str(r), LOCAL_RANK="0", WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.join(ROOT, "tests",
                                                                    "multiset_sets_worker.py"),
                                       out], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT))
    logs = []
    for p in procs:
        try:
            o, _ = p.communicate(timeout=600)
        except subprocess.TimeoutExpired:
            p.kill()
            o, _ = p.communicate()
        logs.append(o.decode(errors="replace"))
    for p in procs:
        assert p.returncode == 0, "\n".join(logs)
    r0, r1 = [json.load(open(o)) for o in outs]
    assert r0["seed"] != r1["seed"]
    assert r0["converged"] and r1["converged"] and r0["iters"] == r1["iters"]
    assert not r0["device_loop"]  # a host reduction runs the loop from the host
    x0, x1 = np.array(r0["x"]), np.array(r1["x"])
    assert np.array_equal(x0, x1)
    xe, ite = _emulated_two_sets(ctx, A, b)
    assert ite == r0["iters"]
    assert np.array_equal(x0, xe)
    xs = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x0 - xs) <= 1e-6 * np.linalg.norm(xs)
    # Anderson-accelerated sets (mclsgpu_anderson_solve_sets)
    assert r0["aa_converged"] and r1["aa_converged"] and r0["aa_iters"] == r1["aa_iters"]
    a0, a1 = np.array(r0["aa_x"]), np.array(r1["aa_x"])
    assert np.array_equal(a0, a1)
    xa, steps = _emulated_two_anderson_sets(ctx, A, b)
    assert steps == r0["aa_iters"] and np.array_equal(a0, xa)
    assert np.linalg.norm(a0 - xs) <= 1e-5 * np.linalg.norm(xs)


def _one_set_steps(ctx, op, pc, A, b, seed):
    eng = multiset.DeviceEngine(_domain(ctx, op, pc, seed), A.shape[0])
    x, it, conv, rel, st = multiset.solve(eng, b, np.zeros_like(b), tolerance=1e-8,
                                          max_iters=5000)
    return x.cpu().numpy(), it


def test_one_set_with_an_identity_reducer_is_the_step_wise_loop(ctx):
    # One set whose reducer leaves the correction as it is: the one-call
    # multi-set loop takes the step-wise loop's steps bit for bit.
    A = P.poisson2d(20)
    b = np.linspace(0.1, 1.0, A.shape[0])
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    calls = []
    sets = capi.set_params(1, lambda ptr, n, stream: calls.append(n))
    x, st, on_device = _domain(ctx, op, pc, 41).mcsa_solve_sets(sets, b, tolerance=1e-8,
                                                                max_iters=5000)
    assert not on_device and st["converged"] == 1
    assert len(calls) == st["iterations"] and calls[0] == A.shape[0]
    xs, its = _one_set_steps(ctx, op, pc, A, b, 41)
    assert its == st["iterations"]
    assert np.array_equal(x, xs)


def test_nccl_one_rank_runs_on_the_device(ctx):
    A = P.poisson2d(20)
    b = np.linspace(0.1, 1.0, A.shape[0])
    op = capi.Operator(ctx, A)
    pc = capi.Precond(ctx, op, capi.PREC_POINT_JACOBI)
    comm = capi.Comm(ctx, 1, 0, capi.Comm.unique_id())
    sets = comm.set_params()
    assert sets.num_sets == 1 and sets.capturable == 1
    x_host, st_host, on_dev2 = _domain(ctx, op, pc, 41).mcsa_solve_sets(
        sets, b, tolerance=1e-8, max_iters=5000, host_loop=1)
    assert not on_dev2 and st_host["converged"] == 1
    x_dev, st_dev, on_device = _domain(ctx, op, pc, 41).mcsa_solve_sets(
        sets, b, tolerance=1e-8, max_iters=5000)
    assert on_device and st_dev["converged"] == 1
    assert st_dev["iterations"] == st_host["iterations"]
    assert np.array_equal(x_dev, x_host)
    xs, its = _one_set_steps(ctx, op, pc, A, b, 41)
    assert its == st_dev["iterations"] and np.array_equal(x_dev, xs)
    comm.close()
