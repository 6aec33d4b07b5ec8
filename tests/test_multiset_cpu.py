"""Multi-set MCSA host logic across two processes over gloo (CPU).

Two ranks, one set each (the CPU oracle as each set's Monte Carlo engine,
per-rank seeds as PRNG(rank) derives them), corrections summed by the
product's multi-set drivers (MCSA and Anderson-accelerated MCSA).  Checks: both ranks end with the same iterate
and iteration count, the solution matches a direct solve, and the
reduction helpers the benchmark's timing uses (max / sum over ranks) work.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import scipy.sparse.linalg as spla

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_ranks(tmp_path, world=2):
    port = _free_port()
    procs = []
    outs = []
    for r in range(world):
        out = str(tmp_path / f"rank{r}.json")
        outs.append(out)
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(ROOT, "tests",
                                                                    "multiset_worker.py"), out],
                                      env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT))
    logs = []
    for p in procs:
        try:
            o, _ = p.communicate(timeout=300)
        except subprocess.TimeoutExpired:
            p.kill()
            o, _ = p.communicate()
        logs.append(o.decode(errors="replace"))
        assert p.returncode == 0, "\n".join(logs)
    return [json.load(open(o)) for o in outs]


def test_two_sets_agree_and_converge(tmp_path):
    from mcls_b200 import problems as P

    res = _run_ranks(tmp_path)
    r0, r1 = res
    assert r0["world"] == r1["world"] == 2
    assert r0["seed"] != r1["seed"]  # independent streams per set
    assert r0["converged"] and r1["converged"]
    assert r0["iters"] == r1["iters"]
    assert np.array_equal(np.array(r0["x"]), np.array(r1["x"]))
    A = P.poisson2d(12)
    b = np.linspace(0.5, 1.5, A.shape[0])
    xs = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(np.array(r0["x"]) - xs) <= 1e-7 * np.linalg.norm(xs)
    assert r0["allmax"] == r1["allmax"] == 2.0
    assert r0["allsum"] == r1["allsum"] == 2.0
    # Anderson-accelerated: the sets take identical steps to the solution.
    assert r0["aa_converged"] and r1["aa_converged"]
    assert r0["aa_iters"] == r1["aa_iters"] and r0["aa_iters"] < r0["iters"]
    assert np.array_equal(np.array(r0["aa_x"]), np.array(r1["aa_x"]))
    assert np.linalg.norm(np.array(r0["aa_x"]) - xs) <= 1e-7 * np.linalg.norm(xs)
