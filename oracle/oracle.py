"""Python binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the checker for the CUDA product path: a plain FP64 C++
restatement of the reference MCLS hot path (oracle/mcls_oracle.cpp).  Only the
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
import this module; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import scipy.sparse as sp

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")


class MCParams(C.Structure):
    _fields_ = [
        ("direction", C.c_int),
        ("estimator", C.c_int),
        ("history_length", C.c_int),
        ("weight_cutoff", C.c_double),
        ("sample_ratio", C.c_double),
        ("stratified", C.c_int),
        ("neumann_relaxation", C.c_double),
        ("composite_threshold", C.c_double),
        ("rng_mode", C.c_int),
        ("seed", C.c_uint64),
    ]


class MCSAParams(C.Structure):
    _fields_ = [
        ("tolerance", C.c_double),
        ("max_iters", C.c_int),
        ("check_freq", C.c_int),
        ("smoother_steps", C.c_int),
        ("richardson_omega", C.c_double),
        ("fixed_point_type", C.c_int),
    ]


class AndersonParams(C.Structure):
    _fields_ = [
        ("tolerance", C.c_double),
        ("max_iters", C.c_int),
        ("smoother_steps", C.c_int),
        ("storage_depth", C.c_int),
        ("mixing", C.c_double),
        ("start_iteration", C.c_int),
        ("adjust_condition", C.c_int),
        ("drop_tolerance", C.c_double),
    ]


def anderson_params(tolerance=1e-8, max_iters=1000, smoother_steps=1, storage_depth=2,
                    mixing=1.0, start_iteration=1, adjust_condition=0, drop_tolerance=1e-12):
    return AndersonParams(tolerance, max_iters, smoother_steps, storage_depth, mixing,
                          start_iteration, adjust_condition, drop_tolerance)


def build():
    """Compile liboracle.so, and oracle/_ref when the environment variable
    MCLS_REFERENCE_ROOT names an MCLS source tree."""
    subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    ref = os.environ.get("MCLS_REFERENCE_ROOT", "")
    if ref and os.path.isdir(os.path.join(ref, "src")):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", "REF_ROOT=" + ref], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P = C.c_void_p
        L.orc_xorshift_uniforms.argtypes = [C.c_uint64, C.c_int64, f64p]
        L.orc_rank_seed.argtypes = [C.c_uint64, C.c_int]
        L.orc_rank_seed.restype = C.c_uint64
        L.orc_counter_uniforms.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_int64, C.c_int64, f64p]
        L.orc_sample_discrete_cdf.argtypes = [f64p, C.c_int, C.c_double]
        L.orc_sample_discrete_cdf.restype = C.c_int
        L.orc_csr_create.argtypes = [C.c_int64, i64p, i64p, f64p]
        L.orc_csr_create.restype = P
        L.orc_csr_free.argtypes = [P]
        L.orc_csr_n.argtypes = [P]
        L.orc_csr_n.restype = C.c_int64
        L.orc_csr_nnz.argtypes = [P]
        L.orc_csr_nnz.restype = C.c_int64
        L.orc_csr_copy.argtypes = [P, i64p, i64p, f64p]
        for name in ("orc_transpose", "orc_point_jacobi"):
            getattr(L, name).argtypes = [P]
            getattr(L, name).restype = P
        L.orc_multiply.argtypes = [P, P, C.c_double]
        L.orc_multiply.restype = P
        L.orc_composite.argtypes = [P, P, P, C.c_int, C.c_double]
        L.orc_composite.restype = P
        L.orc_block_jacobi.argtypes = [P, C.c_int]
        L.orc_block_jacobi.restype = P
        L.orc_spmv.argtypes = [P, f64p, f64p]
        L.orc_mc_create.argtypes = [P, P, P, C.POINTER(MCParams)]
        L.orc_mc_create.restype = P
        L.orc_mc_free.argtypes = [P]
        L.orc_mc_domain_nnz.argtypes = [P]
        L.orc_mc_domain_nnz.restype = C.c_int64
        L.orc_mc_domain_copy.argtypes = [P, i64p, i64p, f64p, f64p, f64p]
        L.orc_mc_solve.argtypes = [P, f64p, f64p, C.c_int, C.c_int64, P, P, P, P]
        L.orc_mc_solve.restype = C.c_int64
        L.orc_mc_stream_position.argtypes = [P]
        L.orc_mc_stream_position.restype = C.c_uint64
        L.orc_mc_total_steps.argtypes = [P]
        L.orc_mc_total_steps.restype = C.c_int64
        L.orc_mcsa_solve.argtypes = [P, P, P, C.POINTER(MCParams), C.POINTER(MCSAParams),
                                     f64p, f64p, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                     C.c_int, P, C.POINTER(C.c_int64)]
        L.orc_mcsa_solve.restype = C.c_int
        L.orc_fixed_point_solve.argtypes = [P, P, P, C.POINTER(MCSAParams), f64p, f64p,
                                            C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int,
                                            P]
        L.orc_fixed_point_solve.restype = C.c_int
        L.orc_anderson_solve.argtypes = [P, P, C.POINTER(MCParams), C.POINTER(AndersonParams),
                                         f64p, f64p, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                         C.c_int, P, C.POINTER(C.c_int64)]
        L.orc_anderson_solve.restype = C.c_int
        L.orc_anderson_linear.argtypes = [P, f64p, C.POINTER(AndersonParams), f64p,
                                          C.POINTER(C.c_int), C.c_int, P]
        L.orc_anderson_linear.restype = C.c_int
        L.orc_bench_walks.argtypes = [P, f64p, C.c_int64, C.c_int, P, C.POINTER(C.c_double)]
        L.orc_bench_walks.restype = C.c_int64
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_mcsa_last_timing.argtypes = [C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_pcg.argtypes = [P, f64p, f64p, C.c_double, C.c_int, C.POINTER(C.c_int),
                              C.POINTER(C.c_double)]
        L.orc_pcg.restype = C.c_int
        _LIB = L
    return _LIB


def ref_lib():
    """The reference's own RNG/sampler compiled into oracle/_ref, or None."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libmcls_ref.so")
        if not os.path.exists(path):
            return None
        R = C.CDLL(path)
        R.ref_xorshift_uniforms.argtypes = [C.c_uint64, C.c_int64, f64p]
        R.ref_xorshift_raw.argtypes = [C.c_uint64, C.c_int64, u64p]
        R.ref_sample_discrete_cdf.argtypes = [f64p, C.c_int, C.c_double]
        R.ref_sample_discrete_cdf.restype = C.c_int
        _REF = R
    return _REF


# ---------------------------------------------------------------- RNG ----
def xorshift_uniforms(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, np.float64)
    lib().orc_xorshift_uniforms(seed, n, out)
    return out


def counter_uniforms(seed: int, epoch: int, kind: int, idx: int, n: int) -> np.ndarray:
    out = np.empty(n, np.float64)
    lib().orc_counter_uniforms(seed, epoch, kind, idx, n, out)
    return out


def rank_seed(master: int, rank: int) -> int:
    return int(lib().orc_rank_seed(master, rank))


def sample_cdf(cdf, u: float) -> int:
    cdf = np.ascontiguousarray(cdf, np.float64)
    return int(lib().orc_sample_discrete_cdf(cdf, len(cdf), u))


# ---------------------------------------------------------------- CSR ----
class Csr:
    """Owning handle around an oracle CSR matrix."""

    def __init__(self, handle):
        if not handle:
            raise RuntimeError("oracle returned no matrix")
        self.h = handle

    def __del__(self):
        if getattr(self, "h", None) and _LIB is not None:
            _LIB.orc_csr_free(self.h)
            self.h = None

    @classmethod
    def from_scipy(cls, A):
        A = sp.csr_matrix(A)
        A.sort_indices()
        rp = np.ascontiguousarray(A.indptr, np.int64)
        ci = np.ascontiguousarray(A.indices, np.int64)
        v = np.ascontiguousarray(A.data, np.float64)
        return cls(lib().orc_csr_create(A.shape[0], rp, ci, v))

    @classmethod
    def from_arrays(cls, n, rp, ci, v):
        return cls(lib().orc_csr_create(n, np.ascontiguousarray(rp, np.int64),
                                        np.ascontiguousarray(ci, np.int64),
                                        np.ascontiguousarray(v, np.float64)))

    def arrays(self):
        L = lib()
        n, nnz = L.orc_csr_n(self.h), L.orc_csr_nnz(self.h)
        rp = np.empty(n + 1, np.int64)
        ci = np.empty(max(nnz, 1), np.int64)
        v = np.empty(max(nnz, 1), np.float64)
        L.orc_csr_copy(self.h, rp, ci, v)
        return n, rp, ci[:nnz], v[:nnz]

    def to_scipy(self):
        n, rp, ci, v = self.arrays()
        return sp.csr_matrix((v, ci, rp), shape=(n, n))

    def spmv(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty_like(x)
        lib().orc_spmv(self.h, x, y)
        return y


def _h(m):
    return m.h if m is not None else None


def transpose(A: Csr) -> Csr:
    return Csr(lib().orc_transpose(A.h))


def multiply(A: Csr, B: Csr, threshold: float = 0.0) -> Csr:
    return Csr(lib().orc_multiply(A.h, B.h, threshold))


def composite(A: Csr, PL=None, PR=None, transpose_: bool = True, threshold: float = 0.0) -> Csr:
    return Csr(lib().orc_composite(A.h, _h(PL), _h(PR), int(transpose_), threshold))


def point_jacobi(A: Csr) -> Csr:
    return Csr(lib().orc_point_jacobi(A.h))


def block_jacobi(A: Csr, block_size: int) -> Csr:
    return Csr(lib().orc_block_jacobi(A.h, block_size))


# ---------------------------------------------------------- Monte Carlo --
def mc_params(direction=0, estimator=0, history_length=10, weight_cutoff=0.0,
              sample_ratio=-1.0, stratified=0, neumann_relaxation=-1.0,
              composite_threshold=0.0, rng_mode=0, seed=1) -> MCParams:
    return MCParams(direction, estimator, history_length, weight_cutoff, sample_ratio,
                    stratified, neumann_relaxation, composite_threshold, rng_mode, seed)


class MC:
    """Monte Carlo solver over one operator (domain + PRNG position)."""

    def __init__(self, A: Csr, PL=None, PR=None, params: MCParams | None = None, **kw):
        self.p = params if params is not None else mc_params(**kw)
        self.n = lib().orc_csr_n(A.h)
        self.h = lib().orc_mc_create(A.h, _h(PL), _h(PR), C.byref(self.p))
        if not self.h:
            raise RuntimeError("oracle domain build failed (empty or zero-weight row)")

    def __del__(self):
        if getattr(self, "h", None) and _LIB is not None:
            _LIB.orc_mc_free(self.h)
            self.h = None

    def domain(self):
        L = lib()
        nnz = L.orc_mc_domain_nnz(self.h)
        rp = np.empty(self.n + 1, np.int64)
        col = np.empty(nnz, np.int64)
        h = np.empty(nnz, np.float64)
        cdf = np.empty(nnz, np.float64)
        w = np.empty(self.n, np.float64)
        L.orc_mc_domain_copy(self.h, rp, col, h, cdf, w)
        return dict(rowptr=rp, col=col, h=h, cdf=cdf, weights=w)

    def solve(self, rhs, internal=False, trace=0):
        rhs = np.ascontiguousarray(rhs, np.float64)
        x = np.empty_like(rhs)
        L = self.p.history_length
        if trace:
            ts = np.empty(trace * (L + 1), np.int64)
            fw = np.empty(trace, np.float64)
            ev = np.empty(trace, np.int32)
            st = np.empty(trace, np.int64)
            nh = lib().orc_mc_solve(self.h, rhs, x, int(internal), trace,
                                    ts.ctypes.data, fw.ctypes.data, ev.ctypes.data, st.ctypes.data)
            k = min(trace, nh)
            return x, nh, dict(states=ts.reshape(trace, L + 1)[:k], final_weight=fw[:k],
                               events=ev[:k], start=st[:k])
        nh = lib().orc_mc_solve(self.h, rhs, x, int(internal), 0, None, None, None, None)
        return x, nh

    @property
    def stream_position(self):
        return int(lib().orc_mc_stream_position(self.h))

    @property
    def total_steps(self):
        return int(lib().orc_mc_total_steps(self.h))

    def bench_walks(self, rhs, nh, threads):
        rhs = np.ascontiguousarray(rhs, np.float64)
        secs = C.c_double(0.0)
        x = np.empty_like(rhs)
        steps = lib().orc_bench_walks(self.h, rhs, nh, threads, x.ctypes.data, C.byref(secs))
        return int(steps), secs.value, x


def mcsa_solve(A: Csr, b, x0=None, PL=None, PR=None, mc: MCParams | None = None,
               tolerance=1e-8, max_iters=1000, check_freq=1, smoother_steps=1,
               richardson_omega=1.0, fixed_point_type=0, **mckw):
    mp = mc if mc is not None else mc_params(**mckw)
    spp = MCSAParams(tolerance, max_iters, check_freq, smoother_steps, richardson_omega,
                     fixed_point_type)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64)
    iters = C.c_int(0)
    ach = C.c_double(0.0)
    steps = C.c_int64(0)
    hist = np.zeros(max_iters, np.float64)
    rc = lib().orc_mcsa_solve(A.h, _h(PL), _h(PR), C.byref(mp), C.byref(spp), b, x,
                              C.byref(iters), C.byref(ach), max_iters, hist.ctypes.data,
                              C.byref(steps))
    if rc < 0:
        raise RuntimeError("oracle MCSA failed")
    t_setup, t_loop = C.c_double(), C.c_double()
    lib().orc_mcsa_last_timing(C.byref(t_setup), C.byref(t_loop))
    return dict(x=x, converged=bool(rc), iters=iters.value, achieved=ach.value,
                residuals=hist[: iters.value], steps=steps.value, setup_s=t_setup.value,
                loop_s=t_loop.value)


def set_threads(threads: int):
    """Host threads of the oracle's SpMVs and counter-stream forward walks
    (results do not depend on the count)."""
    lib().orc_set_threads(int(threads))


def pcg(A: Csr, b, x0=None, tolerance=1e-12, max_iters=100000):
    """FP64 diagonal-preconditioned conjugate gradients (SPD A): the oracle
    solve MCSA solutions are measured against."""
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64)
    it = C.c_int(0)
    rr = C.c_double(0.0)
    rc = lib().orc_pcg(A.h, b, x, tolerance, max_iters, C.byref(it), C.byref(rr))
    if rc < 0:
        raise RuntimeError("oracle CG: non-positive diagonal")
    return dict(x=x, converged=bool(rc), iters=it.value, rel_residual=rr.value)


def fixed_point_solve(A: Csr, b, x0=None, PL=None, PR=None, tolerance=1.0, max_iters=1000,
                      check_freq=1, richardson_omega=1.0, fixed_point_type=0):
    """FixedPointSolverManager::solve restatement (no Monte Carlo)."""
    spp = MCSAParams(tolerance, max_iters, check_freq, 1, richardson_omega, fixed_point_type)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64)
    iters = C.c_int(0)
    ach = C.c_double(0.0)
    hist = np.zeros(max_iters, np.float64)
    rc = lib().orc_fixed_point_solve(A.h, _h(PL), _h(PR), C.byref(spp), b, x, C.byref(iters),
                                     C.byref(ach), max_iters, hist.ctypes.data)
    return dict(x=x, converged=bool(rc), iters=iters.value, achieved=ach.value,
                residuals=hist[: iters.value])


def anderson_solve(A: Csr, b, x0=None, PL=None, mc: MCParams | None = None,
                   aa: AndersonParams | None = None, **kw):
    """Anderson-accelerated MCSA restatement.  Keywords go to anderson_params
    when they name one of its fields, else to mc_params."""
    akeys = {f for f, _ in AndersonParams._fields_}
    ap = aa if aa is not None else anderson_params(**{k: v for k, v in kw.items() if k in akeys})
    mp = mc if mc is not None else mc_params(**{k: v for k, v in kw.items() if k not in akeys})
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64)
    iters = C.c_int(0)
    ach = C.c_double(0.0)
    steps = C.c_int64(0)
    hist = np.zeros(max(ap.max_iters, 1), np.float64)
    rc = lib().orc_anderson_solve(A.h, _h(PL), C.byref(mp), C.byref(ap), b, x, C.byref(iters),
                                  C.byref(ach), ap.max_iters, hist.ctypes.data, C.byref(steps))
    if rc < 0:
        raise RuntimeError("oracle Anderson failed")
    return dict(x=x, converged=bool(rc), iters=iters.value, achieved=ach.value,
                residuals=hist[: iters.value], steps=steps.value)


def anderson_linear(M: Csr, c, x0=None, **kw):
    """Anderson acceleration of g(x) = M x + c: (x, iterations, converged,
    iterates x_0..x_k)."""
    ap = anderson_params(**kw)
    c = np.ascontiguousarray(c, np.float64)
    x = np.zeros_like(c) if x0 is None else np.array(x0, np.float64)
    its = np.zeros((ap.max_iters + 1, c.size), np.float64)
    iters = C.c_int(0)
    rc = lib().orc_anderson_linear(M.h, c, C.byref(ap), x, C.byref(iters), ap.max_iters,
                                   its.ctypes.data)
    return x, iters.value, bool(rc), its[: iters.value + 1]
