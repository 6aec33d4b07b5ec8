"""One rank of the CPU multi-set MCSA check (started twice by
tests/test_multiset_cpu.py with RANK / WORLD_SIZE / MASTER_* set).

Each rank is one set: a point-Jacobi Monte Carlo engine from the CPU oracle
(test infrastructure) with its own random stream, seeded as the reference's
PRNG(rank) derives per-rank seeds.  The product's multi-set driver
(mcls_b200.multiset.solve) sums the corrections over the ranks with gloo.
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from mcls_b200 import dist, multiset  # noqa: E402
from mcls_b200 import problems as P  # noqa: E402
from oracle import oracle as O  # noqa: E402


class OracleEngine:
    def __init__(self, A, seed):
        import torch

        self.torch = torch
        self.A = A
        self.dinv = 1.0 / A.diagonal()
        Ao = O.Csr.from_scipy(A)
        self.mc = O.MC(Ao, PL=O.point_jacobi(Ao), direction=0, estimator=0, history_length=10,
                       sample_ratio=1.0, rng_mode=0, seed=seed)

    def _rp(self):
        return self.dinv * (self.b - self.A @ self.x)

    def begin(self, b, x0, params):
        self.b = np.asarray(b, np.float64)
        self.x = np.array(x0, np.float64)
        self.omega = params.richardson_omega
        self.steps = params.smoother_steps
        self.rp = self._rp()
        return float(np.linalg.norm(self.rp)), float(np.linalg.norm(self.dinv * self.b))

    def correction(self):
        for _ in range(self.steps):
            self.x = self.x + self.omega * self.rp
            self.rp = self._rp()
        delta, _ = self.mc.solve(self.rp, internal=True)
        return self.torch.tensor(delta)

    def apply(self, delta, scale):
        self.x = self.x + scale * delta.numpy()
        self.rp = self._rp()
        return float(np.linalg.norm(self.rp))

    def finish(self):
        return self.x, {}

    # Anderson-accelerated steps: the same map and acceleration in numpy
    # (least squares on the stored differences, Walker & Ni 2011).
    def aa_begin(self, b, x0, params):
        self.b = np.asarray(b, np.float64)
        self.x = np.array(x0, np.float64)
        self.p = params
        self.k = 0
        self.Fs, self.Xs = [], []
        self.rp = self._rp()
        rn, bn = float(np.linalg.norm(self.rp)), float(np.linalg.norm(self.b))
        return rn, bn, rn < params.tolerance * bn

    def aa_correction(self):
        self.f = self.x.copy()
        r = self.rp
        for _ in range(self.p.smoother_steps):
            self.f = self.f + r
            r = self.dinv * (self.b - self.A @ self.f)
        delta, _ = self.mc.solve(r, internal=True)
        return self.torch.tensor(delta)

    def aa_apply(self, delta, scale):
        p = self.p
        F = self.f + scale * delta.numpy() - self.x
        self.Fs.append(F)
        self.Xs.append(self.x.copy())
        k = self.k
        if p.storage_depth > 0 and k >= p.start_iteration:
            first = max(p.start_iteration - 1, k - p.storage_depth)
            dF = np.column_stack([self.Fs[j + 1] - self.Fs[j] for j in range(first, k)])
            dX = np.column_stack([self.Xs[j + 1] - self.Xs[j] for j in range(first, k)])
            g = np.linalg.lstsq(dF, F, rcond=None)[0]
            self.x = self.x + p.mixing * F - (dX + p.mixing * dF) @ g
        else:
            self.x = self.x + p.mixing * F
        self.k += 1
        self.rp = self._rp()
        rn = float(np.linalg.norm(self.rp))
        return rn, rn < p.tolerance * np.linalg.norm(self.b) or self.k >= p.max_iters

    def aa_finish(self):
        return self.x, {}


def main(out_path):
    world, rank, _, pg = dist.init("gloo", timeout_s=60)
    A = P.poisson2d(12)
    b = np.linspace(0.5, 1.5, A.shape[0])
    seed = O.rank_seed(433494437, rank)
    eng = OracleEngine(A, seed)
    x, it, conv, rel, _ = multiset.solve(eng, b, np.zeros_like(b), group=pg, tolerance=1e-8,
                                         max_iters=3000)
    eng_aa = OracleEngine(A, seed)
    xa, ita, conva, rela, _ = multiset.solve_anderson(eng_aa, b, np.zeros_like(b), group=pg,
                                                      tolerance=1e-10, max_iters=500,
                                                      storage_depth=3)
    res = {"rank": rank, "world": world, "iters": it, "converged": bool(conv), "rel": rel,
           "x": list(map(float, x)), "seed": int(seed),
           "aa_iters": ita, "aa_converged": bool(conva), "aa_rel": rela,
           "aa_x": list(map(float, xa)),
           "allmax": dist.allmax(pg, rank + 1.0), "allsum": dist.allsum(pg, 1.0)}
    dist.barrier(pg)
    with open(out_path, "w") as f:
        json.dump(res, f)
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main(sys.argv[1])
