"""Domain-decomposed Monte Carlo transport: the domain's rows split into
parts (one per GPU), histories handed between parts as they cross.

The reference decomposes the domain over MPI ranks and moves histories that
leave a rank's rows to the owning rank through buffered messages
(src/MCLS_DomainTransporter_impl.hpp:70-119,
src/MCLS_DomainCommunicator_impl.hpp, src/MCLS_SourceTransporter_impl.hpp).
Here a part is a `capi.Subdomain`; one Monte Carlo solve is

    begin       adjoint: every part builds the global source of the
                residual and keeps the histories that start in its rows;
                forward: every part takes the histories of its own rows and
                the tally source of its rows
    rounds      every part walks its histories until they end or cross;
                the departures (32-byte history records; forward sums of
                histories that ended away from their start row go home as
                tally returns) are exchanged -- all-to-all between ranks,
                device copies between the parts of one process -- and
                walked by their new owners, until no part has departures in
                a round
    finish      every part normalises the tallies of its rows.

Every rank takes the same collective steps in the same order (two
all-to-alls and one all-reduce per round).  `solve_local` drives all parts
from one process (the parts may share one GPU); `solve_distributed` drives
one part per rank of a torch.distributed group.  An MCSA loop calls either
in place of the whole-domain Monte Carlo solve.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import capi

#: mclsgpu_history_wire (32 bytes).
WIRE_DTYPE = np.dtype([("rng", "<u8"), ("state", "<i4"), ("step", "<i4"), ("weight", "<f4"),
                       ("id", "<i4"), ("acc", "<f4"), ("comp", "<f4")])
WIRE_BYTES = WIRE_DTYPE.itemsize


def row_bounds(n: int, nparts: int):
    """Contiguous row blocks of nearly equal size."""
    return np.array([(n * q) // nparts for q in range(nparts + 1)], np.int64)


def transposed_composite(A, left_diag_inv=None):
    """(PL A)^T on the host as the library's adjoint domain build forms it:
    with a point-Jacobi PL (left_diag_inv = 1 / diag(A)) the columns of A^T
    are scaled, entry (i, j) = A_ji * (1 / A_jj)."""
    T = sp.csr_matrix(A.T)
    if left_diag_inv is not None:
        T = sp.csr_matrix(T.multiply(np.asarray(left_diag_inv)[None, :]))
    T.sort_indices()
    return T


def composite(A, left_diag_inv=None):
    """PL A on the host as the library's forward domain build forms it: with
    a point-Jacobi PL (left_diag_inv = 1 / diag(A)) row i is scaled,
    entry (i, j) = (1 / A_ii) * A_ij."""
    M = sp.csr_matrix(A, copy=True)
    if left_diag_inv is not None:
        M = sp.csr_matrix(sp.diags(np.asarray(left_diag_inv)) @ M)
    M.sort_indices()
    return M


class DevicePart:
    """One part on one device, with its outbox ([nparts][capacity] records)."""

    def __init__(self, sub: "capi.Subdomain", capacity: int, device: str):
        import torch

        self.sub = sub
        self.cap = int(capacity)
        self.dev = device
        self.out = torch.empty((sub.nparts, self.cap, WIRE_BYTES), dtype=torch.uint8,
                               device=device)
        self.x = torch.empty(sub.rows, dtype=torch.float64, device=device)

    def begin(self, rhs):
        return self.sub.begin(rhs.data_ptr())

    def transport(self, inbox, n_in):
        """inbox None: the part's starting histories; else a uint8 tensor of
        n_in records.  Returns the departures per destination part."""
        ptr = inbox.data_ptr() if inbox is not None else None
        return self.sub.transport(ptr, n_in, self.out.data_ptr(), self.cap)

    def departures(self, q, count):
        return self.out[q, :count]

    def finish(self):
        return self.x, self.sub.finish(self.x.data_ptr())


def solve_local(parts, rhs, max_rounds=10 ** 6):
    """One Monte Carlo solve over all parts driven from this process.
    Returns (x over all rows, rounds, histories exchanged, walk steps)."""
    import torch

    P = len(parts)
    for p in parts:
        p.begin(rhs)
    counts = [p.transport(None, 0) for p in parts]
    rounds, moved = 1, 0
    while any(int(c.sum()) for c in counts) and rounds < max_rounds:
        inboxes = []
        for q in range(P):
            pieces = [parts[r].departures(q, int(counts[r][q])).to(parts[q].dev)
                      for r in range(P) if counts[r][q]]
            inboxes.append(torch.cat(pieces) if pieces else None)
        moved += sum(int(c.sum()) for c in counts)
        counts = [parts[q].transport(inboxes[q], inboxes[q].shape[0])
                  if inboxes[q] is not None else np.zeros(P, np.int64) for q in range(P)]
        rounds += 1
    done = [p.finish() for p in parts]
    xs = [d[0] for d in done]
    steps = sum(d[1]["walk_steps"] for d in done)
    return torch.cat([x.to(xs[0].device) for x in xs]), rounds, moved, steps


def solve_distributed(part, rhs, group, max_rounds=10 ** 6):
    """One Monte Carlo solve with one part per rank of `group`.  Returns
    (this part's rows of x, rounds, histories this rank sent)."""
    import torch

    P = group.get_world_size()
    dev = rhs.device
    part.begin(rhs)
    counts = part.transport(None, 0)
    rounds, sent = 1, 0
    while rounds < max_rounds:
        send_n = torch.tensor(counts, dtype=torch.int64, device=dev)
        total = send_n.sum().clone()
        group.all_reduce(total)
        if int(total.item()) == 0:
            break
        recv_n = torch.empty_like(send_n)
        group.all_to_all_single(recv_n, send_n)
        rn = [int(v) for v in recv_n.tolist()]
        send = torch.cat([part.departures(q, int(counts[q])) for q in range(P)])
        recv = torch.empty((sum(rn), WIRE_BYTES), dtype=torch.uint8, device=dev)
        group.all_to_all_single(recv.view(-1), send.reshape(-1),
                                output_split_sizes=[c * WIRE_BYTES for c in rn],
                                input_split_sizes=[int(c) * WIRE_BYTES for c in counts])
        sent += int(send_n.sum().item())
        counts = part.transport(recv, recv.shape[0]) if recv.shape[0] else np.zeros(P, np.int64)
        rounds += 1
    x, _ = part.finish()
    return x, rounds, sent
