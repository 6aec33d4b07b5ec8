"""Multi-set MCSA: one set (one domain, its own random streams) per process,
the Monte Carlo corrections summed over the sets by an all-reduce and
divided by the set count -- the loop of MCSASolverManager::solve with
MultiSetLinearProblem::blockConstantVectorSum
(src/MCLS_MCSASolverManager_impl.hpp:344-400,
src/MCLS_MultiSetLinearProblem_impl.hpp:102-120) -- and the same for the
Anderson-accelerated solve, whose model evaluator sums the sets' corrections
before forming F (src/MCLS_MCSAModelEvaluator_impl.hpp:338-345).

The driver is written against a small engine interface so that the same
host logic runs on GPUs (DeviceEngine: the library's step-wise MCSA entry
points, NCCL all-reduce) and, in the tests, on CPU processes over gloo.
Every rank takes the same collective steps in the same order: one
all-reduce of the correction and one of the residual norm per iteration.
"""
from __future__ import annotations

import os

from . import capi


class DeviceEngine:
    """One set on one GPU through mclsgpu_mcsa_begin/_correction/_apply/_finish."""

    def __init__(self, domain: "capi.Domain", n: int, device: int = 0):
        import torch

        self.dom = domain
        self.n = n
        self.dev = f"cuda:{device}"
        self.delta = torch.zeros(n, dtype=torch.float64, device=self.dev)

    def begin(self, b, x0, params):
        import torch

        self.b = torch.as_tensor(b, dtype=torch.float64, device=self.dev).contiguous()
        self.x = torch.as_tensor(x0, dtype=torch.float64, device=self.dev).clone().contiguous()
        return self.dom.mcsa_begin(self.b.data_ptr(), self.x.data_ptr(), params=params)

    def correction(self):
        self.dom.mcsa_correction(self.delta.data_ptr())
        return self.delta

    def apply(self, delta, scale):
        return self.dom.mcsa_apply(delta.data_ptr(), scale)

    def finish(self):
        stats = self.dom.mcsa_finish(self.x.data_ptr())
        return self.x, stats

    # Anderson-accelerated MCSA (mclsgpu_anderson_begin/_correction/_apply/_finish)
    def aa_begin(self, b, x0, params):
        import torch

        self.b = torch.as_tensor(b, dtype=torch.float64, device=self.dev).contiguous()
        self.x = torch.as_tensor(x0, dtype=torch.float64, device=self.dev).clone().contiguous()
        return self.dom.anderson_begin(self.b.data_ptr(), self.x.data_ptr(), params=params)

    def aa_correction(self):
        self.dom.anderson_correction(self.delta.data_ptr())
        return self.delta

    def aa_apply(self, delta, scale):
        return self.dom.anderson_apply(delta.data_ptr(), scale)

    def aa_finish(self):
        stats = self.dom.anderson_finish(self.x.data_ptr())
        return self.x, stats


def solve(engine, b, x0, group=None, tolerance=1e-8, max_iters=1000, check_freq=1,
          smoother_steps=1, richardson_omega=1.0):
    """Multi-set MCSA on every rank of `group` (torch.distributed module or
    None for one set).  Returns (x, iterations, converged, |rp|/|PL b|, stats)."""
    import torch

    world = group.get_world_size() if group is not None else 1
    params = capi.mcsa_params(tolerance=tolerance, max_iters=max_iters, check_freq=check_freq,
                              smoother_steps=smoother_steps, richardson_omega=richardson_omega)
    rnorm, bnorm = engine.begin(b, x0, params)
    crit = tolerance * (bnorm if bnorm > 0.0 else 1.0)
    it = 0
    converged = rnorm <= crit
    while not converged and it < max_iters:
        it += 1
        delta = engine.correction()
        if world > 1:
            group.all_reduce(delta)  # blockConstantVectorSum over the sets
        rnorm = engine.apply(delta, 1.0 / world)
        if world > 1:
            # Identical x on every rank gives identical norms; the MAX keeps
            # the stopping decision common to all ranks regardless.
            t = torch.tensor([rnorm], dtype=torch.float64, device=delta.device)
            group.all_reduce(t, op=group.ReduceOp.MAX)
            rnorm = float(t.item())
        if it % check_freq == 0:
            converged = rnorm <= crit
    x, stats = engine.finish()
    return x, it, converged, rnorm / (bnorm if bnorm > 0.0 else 1.0), stats


def solve_anderson(engine, b, x0, group=None, tolerance=1e-8, max_iters=1000, smoother_steps=1,
                   storage_depth=2, mixing=1.0, start_iteration=1, adjust_condition=0,
                   drop_tolerance=1e-12):
    """Multi-set Anderson-accelerated MCSA on every rank of `group`: each step
    sums the sets' Monte Carlo corrections (blockConstantVectorSum) and
    scales by 1 / number of sets before the accelerated update.  Stops on
    |PL (b - A x)|_2 < tolerance |b|_2 or max_iters steps.  Returns
    (x, steps, converged, |PL (b - A x)|_2 / |b|_2, stats)."""
    import torch

    world = group.get_world_size() if group is not None else 1
    params = capi.anderson_params(tolerance=tolerance, max_iters=max_iters,
                                  smoother_steps=smoother_steps, storage_depth=storage_depth,
                                  mixing=mixing, start_iteration=start_iteration,
                                  adjust_condition=adjust_condition,
                                  drop_tolerance=drop_tolerance)
    rnorm, bnorm, done = engine.aa_begin(b, x0, params)
    steps = 0
    while not done:
        steps += 1
        delta = engine.aa_correction()
        if world > 1:
            group.all_reduce(delta)  # blockConstantVectorSum over the sets
        rnorm, done = engine.aa_apply(delta, 1.0 / world)
        if world > 1:
            # Identical iterates give identical decisions; the MAX keeps the
            # stopping decision common to all ranks regardless.
            t = torch.tensor([rnorm, float(done)], dtype=torch.float64, device=delta.device)
            group.all_reduce(t, op=group.ReduceOp.MAX)
            rnorm, done = float(t[0].item()), bool(t[1].item())
    x, stats = engine.aa_finish()
    return x, steps, rnorm < tolerance * bnorm, rnorm / (bnorm if bnorm > 0.0 else 1.0), stats


class _DeviceArray:
    """A device vector of n doubles at ptr, seen by torch through the CUDA
    array interface (no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8",
                                         "data": (ptr, False), "version": 2}


def _cudart():
    """The CUDA runtime the process has loaded (torch's), for the host-copy
    reducer's stream synchronisation and copies."""
    import ctypes
    import glob

    import torch  # noqa: F401  (loads its CUDA runtime)

    for name in ("libcudart.so.12", "libcudart.so"):
        try:
            return ctypes.CDLL(name)
        except OSError:
            pass
    for path in glob.glob(os.path.join(os.path.dirname(torch.__file__), "..", "nvidia",
                                       "cuda_runtime", "lib", "libcudart.so*")):
        return ctypes.CDLL(path)
    raise OSError("CUDA runtime not found")


def torch_set_params(pg, num_sets: int, device: str, host_copy: bool):
    """Set params for mclsgpu_mcsa_solve_sets whose reducer is a
    torch.distributed all-reduce (sum) of the set's correction: with
    host_copy over a CPU backend (gloo) on a host copy (the library's stream
    synchronised, the vector copied out and back), otherwise over NCCL on the
    device vector on the library's stream.  The loop then runs from the host;
    the library's own NCCL communicator (capi.Comm) runs it on the device."""
    import ctypes

    import numpy as np
    import torch

    rt = _cudart() if host_copy else None

    def reduce(ptr, n, stream):
        if host_copy:
            h = np.empty(n, np.float64)
            nbytes = ctypes.c_size_t(8 * n)
            st = ctypes.c_void_p(stream)
            # Both copies on the library's stream, each completed before the
            # host goes on (that stream does not synchronise with the legacy
            # default stream, so a plain cudaMemcpy could still be landing
            # when the next kernel reads the vector).
            if (rt.cudaMemcpyAsync(ctypes.c_void_p(h.ctypes.data), ctypes.c_void_p(ptr), nbytes,
                                   2, st) or rt.cudaStreamSynchronize(st)):
                raise RuntimeError("cudaMemcpyAsync D2H")
            t = torch.from_numpy(h)
            pg.all_reduce(t)
            if (rt.cudaMemcpyAsync(ctypes.c_void_p(ptr), ctypes.c_void_p(h.ctypes.data), nbytes,
                                   1, st) or rt.cudaStreamSynchronize(st)):
                raise RuntimeError("cudaMemcpyAsync H2D")
            return
        t = torch.as_tensor(_DeviceArray(ptr, n), device=device)
        ext = torch.cuda.ExternalStream(stream, device=device)
        with torch.cuda.stream(ext):
            pg.all_reduce(t)

    return capi.set_params(num_sets, reduce, capturable=False)
