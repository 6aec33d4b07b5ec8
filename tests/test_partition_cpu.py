"""Domain-decomposed transport host logic across processes over gloo (CPU).

Two and three ranks each own a block of rows and walk a deterministic toy
history set (adjoint tallies where the history stands; forward sums that go
home to their start row) in the library's 32-byte history records; the
product's driver
(mcls_b200.partition.solve_distributed) runs the rounds, the all-to-all
exchanges and the termination test.  The ranks' tallies, put together, must
equal the same walk done in one piece, and histories must have crossed.
"""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("mode", ["adjoint", "forward"])
@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_walk_equals_whole_walk(tmp_path, world, mode):
    port = _free_port()
    procs, outs = [], []
    for r in range(world):
        out = str(tmp_path / f"rank{r}.json")
        outs.append(out)
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(ROOT, "tests",
                                                                    "partition_worker.py"), out, mode],
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
    res = sorted((json.load(open(o)) for o in outs), key=lambda r: r["rank"])
    x = np.concatenate([r["x"] for r in res])
    whole = np.array(res[0]["whole"])
    assert np.allclose(x, whole, rtol=1e-15, atol=0)
    assert all(r["rounds"] == res[0]["rounds"] for r in res) and res[0]["rounds"] >= 3
    assert sum(r["sent"] for r in res) > 0


def test_host_composite_rows_match_the_oracle():
    # The host helper that forms a part's rows: (PL A)^T with point Jacobi,
    # entry (i, j) = A_ji * (1 / A_jj), against the oracle's restatement of
    # LinearProblem's composite operator (exact values, zeros aside).
    import scipy.sparse as sp

    from mcls_b200 import partition
    from mcls_b200 import problems as P
    from oracle import oracle as O

    A, _ = P.diffusion3d_varcoef(6, seed=3)
    T = partition.transposed_composite(A, 1.0 / A.diagonal())
    Ao = O.Csr.from_scipy(A)
    ref = O.composite(Ao, PL=O.point_jacobi(Ao), transpose_=True).to_scipy()
    D = (T - ref).tocsr()
    D.eliminate_zeros()
    assert D.nnz == 0
    b = partition.row_bounds(A.shape[0], 5)
    assert b[0] == 0 and b[-1] == A.shape[0] and np.all(np.diff(b) > 0)
    assert isinstance(T, sp.csr_matrix) and T.has_sorted_indices
