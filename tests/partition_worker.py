"""One rank of the CPU check of the domain-decomposed transport driver
(started by tests/test_partition_cpu.py with RANK / WORLD_SIZE / MASTER_*).

Each rank owns a block of rows and runs a small deterministic walker with
the library's history record layout (partition.WIRE_DTYPE): history h starts
at state h with weight 1, each step halves the weight and moves to
(7 s + 3) mod n.  Adjoint mode (argv[2] "adjoint"): a step tallies the weight
at the state it leaves (from the second step on, as the device walk does).
Forward mode ("forward"): a step adds w (s + 1) at the state it leaves to the
history's sum, which belongs to its start row h; a sum that ends away from
h's rank goes home as a tally return (state -1), as the device walk sends it.
The product's driver (partition.solve_distributed) exchanges the records over
gloo; the test compares the ranks' tallies with the same walk done in one
piece.
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from mcls_b200 import dist, partition  # noqa: E402

N, L = 97, 6


def next_state(s):
    return (7 * s + 3) % N


def whole_walk(mode):
    y = np.zeros(N)
    for h in range(N):
        s, w, acc = h, 1.0, 0.0
        for k in range(L):
            if mode == "forward":
                acc += w * (s + 1)
            elif k > 0:
                y[s] += w
            w *= 0.5
            s = next_state(s)
        if mode == "forward":
            y[h] += acc
    return y


class ToyPart:
    def __init__(self, bounds, part, mode):
        self.mode = mode
        import torch

        self.torch = torch
        self.bounds = bounds
        self.P = len(bounds) - 1
        self.lo, self.hi = int(bounds[part]), int(bounds[part + 1])
        self.y = np.zeros(self.hi - self.lo)
        self.cap = N

    def begin(self, rhs):
        return self.hi - self.lo, N

    def _owner(self, s):
        return int(np.searchsorted(self.bounds, s, side="right") - 1)

    def transport(self, inbox, n_in):
        fwd = self.mode == "forward"
        if inbox is None:
            hist = [(h, 0, 1.0, h, 0.0) for h in range(self.lo, self.hi)]
        else:
            rec = np.frombuffer(inbox.numpy().tobytes(), dtype=partition.WIRE_DTYPE)
            hist = [(int(r["state"]), int(r["step"]), float(r["weight"]), int(r["id"]),
                     float(r["acc"])) for r in rec]
        out = [[] for _ in range(self.P)]
        for s, k, w, hid, acc in hist:
            if s < 0:  # a forward tally return
                assert fwd and self.lo <= hid < self.hi
                self.y[hid - self.lo] += acc
                continue
            assert self.lo <= s < self.hi
            while k < L:
                if fwd:
                    acc += w * (s + 1)
                elif k > 0:
                    self.y[s - self.lo] += w
                w *= 0.5
                s = next_state(s)
                k += 1
                if k < L and not (self.lo <= s < self.hi):
                    out[self._owner(s)].append((0, s, k, w, hid, acc, 0.0))
                    break
            if k == L and fwd:
                if self.lo <= hid < self.hi:
                    self.y[hid - self.lo] += acc
                else:
                    out[self._owner(hid)].append((0, -1, k, w, hid, acc, 0.0))
        self.out = [np.array(o, dtype=partition.WIRE_DTYPE) for o in out]
        return np.array([len(o) for o in out], np.int64)

    def departures(self, q, count):
        b = np.frombuffer(self.out[q][:count].tobytes(), dtype=np.uint8).copy()
        return self.torch.from_numpy(b).view(count, partition.WIRE_BYTES)

    def finish(self):
        return self.torch.from_numpy(self.y.copy()), {}


def main(out_path, mode):
    import torch

    world, rank, _, pg = dist.init("gloo", timeout_s=60)
    bounds = partition.row_bounds(N, world)
    part = ToyPart(bounds, rank, mode)
    x, rounds, sent = partition.solve_distributed(part, torch.zeros(N, dtype=torch.float64), pg)
    res = {"rank": rank, "lo": int(bounds[rank]), "x": x.tolist(), "rounds": rounds,
           "sent": sent, "whole": whole_walk(mode).tolist()}
    dist.barrier(pg)
    with open(out_path, "w") as f:
        json.dump(res, f)
    pg.destroy_process_group()


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2] if len(sys.argv) > 2 else "adjoint")
