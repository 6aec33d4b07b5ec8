"""ctypes binding of libmclsgpu.so (the C ABI in include/mclsgpu.h).

This is what the tests and bench.py call: every solve goes through the same
extern "C" entry points a C++, cgo or JNI caller would bind.  Loading fails
loudly when the library is missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmclsgpu.so")

OK, ERR_INVALID_ARG, ERR_CUDA, ERR_DIVERGED, ERR_TIMEOUT, ERR_NOT_CONVERGED, \
    ERR_DEGENERATE, ERR_NO_DEVICE, ERR_UNSUPPORTED = range(9)
ADJOINT, FORWARD = 0, 1
COLLISION, EXPECTED_VALUE = 0, 1
SOURCE_RANDOM, SOURCE_STRATIFIED = 0, 1
FP64, FP32 = 0, 1
RNG_REFERENCE, RNG_COUNTER = 0, 1
RECORD_AUTO, RECORD_PACKED, RECORD_STENCIL, RECORD_STENCIL16 = 0, 1, 2, 3
PREC_NONE, PREC_POINT_JACOBI, PREC_BLOCK_JACOBI, PREC_LEARNED_SPAI, PREC_USER_CSR = range(5)
FIXED_POINT_RICHARDSON, FIXED_POINT_STEEPEST_DESCENT, FIXED_POINT_MINRES, FIXED_POINT_RNSD = range(4)
#: "Fixed Point Type" names (FixedPointIterationFactory) to the C enum.
FIXED_POINT_TYPES = {"Richardson": FIXED_POINT_RICHARDSON,
                     "Steepest Descent": FIXED_POINT_STEEPEST_DESCENT,
                     "MINRES": FIXED_POINT_MINRES, "RNSD": FIXED_POINT_RNSD}


class McParams(C.Structure):
    _fields_ = [
        ("size", C.c_uint32),
        ("direction", C.c_int32),
        ("estimator", C.c_int32),
        ("history_length", C.c_int32),
        ("weight_cutoff", C.c_double),
        ("sample_ratio", C.c_double),
        ("source_sampling", C.c_int32),
        ("precision", C.c_int32),
        ("neumann_relaxation", C.c_double),
        ("composite_threshold", C.c_double),
        ("rng_mode", C.c_int32),
        ("record_format", C.c_int32),
        ("seed", C.c_uint64),
    ]


class McsaParams(C.Structure):
    _fields_ = [
        ("size", C.c_uint32),
        ("max_iters", C.c_int32),
        ("tolerance", C.c_double),
        ("check_freq", C.c_int32),
        ("smoother_steps", C.c_int32),
        ("richardson_omega", C.c_double),
        ("print_freq", C.c_int32),
        ("verbose", C.c_int32),
        ("host_loop", C.c_int32),
        ("fixed_point_type", C.c_int32),
    ]


class AndersonParams(C.Structure):
    _fields_ = [
        ("size", C.c_uint32),
        ("max_iters", C.c_int32),
        ("tolerance", C.c_double),
        ("smoother_steps", C.c_int32),
        ("storage_depth", C.c_int32),
        ("mixing", C.c_double),
        ("start_iteration", C.c_int32),
        ("adjust_condition", C.c_int32),
        ("drop_tolerance", C.c_double),
        ("host_loop", C.c_int32),
        ("reserved0", C.c_int32),
    ]


class PrecondParams(C.Structure):
    _fields_ = [
        ("size", C.c_uint32),
        ("kind", C.c_int32),
        ("block_size", C.c_int32),
        ("reserved0", C.c_int32),
        ("user_n", C.c_int64),
        ("user_rowptr", C.c_void_p),
        ("user_colind", C.c_void_p),
        ("user_values", C.c_void_p),
        ("spai_net", C.c_void_p),
        ("rho_fallback", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("size", C.c_uint32),
        ("iterations", C.c_int32),
        ("converged", C.c_int32),
        ("fallback_taken", C.c_int32),
        ("achieved_tol", C.c_double),
        ("residual_norm", C.c_double),
        ("histories", C.c_int64),
        ("walk_steps", C.c_int64),
        ("solve_ms", C.c_double),
        ("walk_ms", C.c_double),
        ("rho", C.c_double),
        ("walk_launches", C.c_int64),
        ("kernel_launches", C.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "size"}


class SpaiAdam(C.Structure):
    _fields_ = [
        ("size", C.c_uint32),
        ("lr", C.c_double),
        ("beta1", C.c_double),
        ("beta2", C.c_double),
        ("eps", C.c_double),
        ("grad_clip", C.c_double),
    ]


class DomainInfo(C.Structure):
    _fields_ = [
        ("size", C.c_uint32),
        ("record_format", C.c_int32),
        ("rows", C.c_int64),
        ("entries", C.c_int64),
        ("record_bytes", C.c_int32),
        ("max_row_entries", C.c_int32),
        ("stencil_offsets", C.c_int32),
        ("operator_dia", C.c_int32),
        ("histories_per_lane", C.c_int32),
        ("block_size", C.c_int32),
        ("record_cache_l1", C.c_int32),
        ("reserved0", C.c_int32),
    ]


class Criteria(C.Structure):
    _fields_ = [
        ("size", C.c_uint32),
        ("reserved0", C.c_int32),
        ("rho_h", C.c_double),
        ("rho_abs", C.c_double),
        ("rho_star", C.c_double),
        ("row_sum_max", C.c_double),
        ("row_sum_min", C.c_double),
        ("balance_min", C.c_double),
        ("balance_max", C.c_double),
        ("balance_ave", C.c_double),
    ]


#: Multi-set reducer: (user, data_dev, n, cudaStream_t) -> status.
SET_REDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p)


class SetParams(C.Structure):
    _fields_ = [
        ("size", C.c_uint32),
        ("num_sets", C.c_int32),
        ("reduce", C.c_void_p),
        ("user", C.c_void_p),
        ("capturable", C.c_int32),
        ("reserved0", C.c_int32),
    ]


#: Every entry point declared in include/mclsgpu.h.
EXPORTS = [
    "mclsgpu_abi_version", "mclsgpu_build_info", "mclsgpu_context_create",
    "mclsgpu_context_destroy", "mclsgpu_last_error", "mclsgpu_context_sync",
    "mclsgpu_operator_upload", "mclsgpu_operator_destroy", "mclsgpu_operator_rows",
    "mclsgpu_operator_nnz", "mclsgpu_operator_apply", "mclsgpu_precond_build",
    "mclsgpu_precond_destroy", "mclsgpu_precond_export", "mclsgpu_domain_build",
    "mclsgpu_domain_destroy", "mclsgpu_domain_export", "mclsgpu_domain_reseed",
    "mclsgpu_rank_seed", "mclsgpu_mc_solve", "mclsgpu_mc_solve_dev", "mclsgpu_mc_trace",
    "mclsgpu_mcsa_solve", "mclsgpu_mcsa_solve_dev", "mclsgpu_domain_spectral_radius",
    "mclsgpu_domain_query", "mclsgpu_domain_set_launch", "mclsgpu_domain_autotune",
    "mclsgpu_operator_apply_static", "mclsgpu_spai_num_params", "mclsgpu_spai_create",
    "mclsgpu_spai_destroy", "mclsgpu_spai_get_params", "mclsgpu_spai_set_params",
    "mclsgpu_spai_infer", "mclsgpu_spai_infer_dev", "mclsgpu_spai_gradient", "mclsgpu_spai_train_step", "mclsgpu_spai_rho",
    "mclsgpu_domain_residual", "mclsgpu_spai_smooth_vectors", "mclsgpu_spai_set_penalty",
    "mclsgpu_batch_build", "mclsgpu_batch_destroy", "mclsgpu_batch_layout",
    "mclsgpu_batch_domain", "mclsgpu_batch_set_launch", "mclsgpu_batch_autotune",
    "mclsgpu_batch_mcsa_solve_dev", "mclsgpu_mcsa_begin", "mclsgpu_mcsa_correction",
    "mclsgpu_mcsa_apply", "mclsgpu_mcsa_finish", "mclsgpu_fixed_point_solve",
    "mclsgpu_fixed_point_solve_dev", "mclsgpu_anderson_solve", "mclsgpu_anderson_solve_dev",
    "mclsgpu_anderson_begin", "mclsgpu_anderson_correction", "mclsgpu_anderson_apply",
    "mclsgpu_anderson_finish", "mclsgpu_history_wire_size", "mclsgpu_subdomain_build",
    "mclsgpu_subdomain_destroy", "mclsgpu_subdomain_info", "mclsgpu_subdomain_begin",
    "mclsgpu_subdomain_transport", "mclsgpu_subdomain_finish",
    "mclsgpu_debug_device_allocations", "mclsgpu_set_wait_limit",
    "mclsgpu_domain_walk_agreement", "mclsgpu_mcsa_solve_sets", "mclsgpu_mcsa_solve_sets_dev",
    "mclsgpu_comm_unique_id", "mclsgpu_comm_create", "mclsgpu_comm_destroy",
    "mclsgpu_comm_set_params", "mclsgpu_domain_convergence_criteria",
    "mclsgpu_anderson_solve_sets", "mclsgpu_domain_set_record_cache",
]

_LIB = None


class MclsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mclsgpu error {code}: {msg}")
        self.code = code


def load(path: str = LIB_PATH):
    """Load libmclsgpu.so; raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise ImportError(f"{path} not built: run `python -m mcls_b200.build`")
    L = C.CDLL(path)
    P = C.c_void_p
    PP = C.POINTER(C.c_void_p)
    d = C.c_double
    i64 = C.c_int64
    L.mclsgpu_abi_version.restype = C.c_int
    L.mclsgpu_build_info.restype = C.c_char_p
    L.mclsgpu_context_create.argtypes = [C.c_int, PP]
    L.mclsgpu_context_destroy.argtypes = [P]
    L.mclsgpu_last_error.argtypes = [P]
    L.mclsgpu_last_error.restype = C.c_char_p
    L.mclsgpu_context_sync.argtypes = [P]
    L.mclsgpu_debug_device_allocations.argtypes = [C.POINTER(i64), C.POINTER(i64)]
    L.mclsgpu_set_wait_limit.argtypes = [P, C.c_int32]
    L.mclsgpu_operator_upload.argtypes = [P, i64, P, P, P, PP]
    L.mclsgpu_operator_destroy.argtypes = [P]
    L.mclsgpu_operator_rows.argtypes = [P]
    L.mclsgpu_operator_rows.restype = i64
    L.mclsgpu_operator_nnz.argtypes = [P]
    L.mclsgpu_operator_nnz.restype = i64
    L.mclsgpu_operator_apply.argtypes = [P, P, P]
    L.mclsgpu_operator_apply_static.argtypes = [P, P, P]
    L.mclsgpu_precond_build.argtypes = [P, P, C.POINTER(PrecondParams), PP]
    L.mclsgpu_precond_destroy.argtypes = [P]
    L.mclsgpu_precond_export.argtypes = [P, C.POINTER(i64), P, P, P]
    L.mclsgpu_domain_build.argtypes = [P, P, P, P, C.POINTER(McParams), PP]
    L.mclsgpu_domain_destroy.argtypes = [P]
    L.mclsgpu_domain_export.argtypes = [P, C.POINTER(i64), P, P, P, P, P]
    L.mclsgpu_domain_reseed.argtypes = [P, C.c_uint64]
    L.mclsgpu_domain_walk_agreement.argtypes = [P, i64, C.c_uint64, C.POINTER(i64),
                                                C.POINTER(i64)]
    L.mclsgpu_mcsa_solve_sets.argtypes = [P, C.POINTER(SetParams), P, P, C.POINTER(McsaParams),
                                          C.POINTER(Stats), C.POINTER(C.c_int32)]
    L.mclsgpu_mcsa_solve_sets_dev.argtypes = [P, C.POINTER(SetParams), P, P,
                                              C.POINTER(McsaParams), C.POINTER(Stats),
                                              C.POINTER(C.c_int32)]
    L.mclsgpu_comm_unique_id.argtypes = [P]
    L.mclsgpu_comm_create.argtypes = [P, C.c_int, C.c_int, P, PP]
    L.mclsgpu_comm_destroy.argtypes = [P]
    L.mclsgpu_comm_set_params.argtypes = [P, C.POINTER(SetParams)]
    L.mclsgpu_anderson_solve_sets.argtypes = [P, C.POINTER(SetParams), P, P,
                                              C.POINTER(AndersonParams), C.POINTER(Stats)]
    L.mclsgpu_domain_convergence_criteria.argtypes = [P, C.c_int, d, C.c_uint64,
                                                      C.POINTER(Criteria)]
    L.mclsgpu_domain_query.argtypes = [P, C.POINTER(DomainInfo)]
    L.mclsgpu_domain_set_launch.argtypes = [P, C.c_int, C.c_int]
    L.mclsgpu_domain_set_record_cache.argtypes = [P, C.c_int]
    L.mclsgpu_domain_autotune.argtypes = [P, P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                          C.POINTER(d)]
    L.mclsgpu_rank_seed.argtypes = [C.c_uint64, C.c_int]
    L.mclsgpu_rank_seed.restype = C.c_uint64
    L.mclsgpu_mc_solve.argtypes = [P, P, P, C.c_int, C.POINTER(Stats)]
    L.mclsgpu_mc_solve_dev.argtypes = [P, P, P, C.c_int, C.POINTER(Stats)]
    L.mclsgpu_mc_trace.argtypes = [P, P, P, C.c_int, i64, P, P, P, P, C.POINTER(i64)]
    L.mclsgpu_mcsa_solve.argtypes = [P, P, P, C.POINTER(McsaParams), C.POINTER(Stats)]
    L.mclsgpu_mcsa_solve_dev.argtypes = [P, P, P, C.POINTER(McsaParams), C.POINTER(Stats)]
    L.mclsgpu_domain_spectral_radius.argtypes = [P, C.c_int, C.c_int, d, C.c_uint64,
                                                 C.POINTER(d)]
    L.mclsgpu_domain_residual.argtypes = [P, P]
    L.mclsgpu_mcsa_begin.argtypes = [P, P, P, C.POINTER(McsaParams), C.POINTER(d), C.POINTER(d)]
    L.mclsgpu_mcsa_correction.argtypes = [P, P]
    L.mclsgpu_mcsa_apply.argtypes = [P, P, d, C.POINTER(d)]
    L.mclsgpu_mcsa_finish.argtypes = [P, P, C.POINTER(Stats)]
    L.mclsgpu_anderson_solve.argtypes = [P, P, P, C.POINTER(AndersonParams), C.POINTER(Stats)]
    L.mclsgpu_anderson_solve_dev.argtypes = [P, P, P, C.POINTER(AndersonParams),
                                             C.POINTER(Stats)]
    L.mclsgpu_anderson_begin.argtypes = [P, P, P, C.POINTER(AndersonParams), C.POINTER(d),
                                         C.POINTER(d), C.POINTER(C.c_int32)]
    L.mclsgpu_anderson_correction.argtypes = [P, P]
    L.mclsgpu_anderson_apply.argtypes = [P, P, d, C.POINTER(d), C.POINTER(C.c_int32)]
    L.mclsgpu_anderson_finish.argtypes = [P, P, C.POINTER(Stats)]
    L.mclsgpu_history_wire_size.restype = C.c_int32
    L.mclsgpu_subdomain_build.argtypes = [P, i64, C.c_int32, P, C.c_int32, P, P, P,
                                          C.POINTER(McParams), PP]
    L.mclsgpu_subdomain_destroy.argtypes = [P]
    L.mclsgpu_subdomain_info.argtypes = [P, C.POINTER(i64), C.POINTER(i64),
                                         C.POINTER(C.c_int32)]
    L.mclsgpu_subdomain_begin.argtypes = [P, P, C.POINTER(i64), C.POINTER(i64)]
    L.mclsgpu_subdomain_transport.argtypes = [P, P, i64, P, i64, P]
    L.mclsgpu_subdomain_finish.argtypes = [P, P, C.POINTER(Stats)]
    L.mclsgpu_fixed_point_solve.argtypes = [P, P, P, P, P, P, C.POINTER(McsaParams),
                                            C.POINTER(Stats)]
    L.mclsgpu_fixed_point_solve_dev.argtypes = [P, P, P, P, P, P, C.POINTER(McsaParams),
                                                C.POINTER(Stats)]
    L.mclsgpu_spai_num_params.restype = C.c_int
    L.mclsgpu_spai_create.argtypes = [P, C.c_int, C.c_uint64, PP]
    L.mclsgpu_spai_destroy.argtypes = [P]
    L.mclsgpu_spai_get_params.argtypes = [P, P]
    L.mclsgpu_spai_set_params.argtypes = [P, P]
    L.mclsgpu_spai_infer.argtypes = [P, P, P, P]
    L.mclsgpu_spai_infer_dev.argtypes = [P, P, P, P, C.POINTER(C.c_float)]
    L.mclsgpu_spai_gradient.argtypes = [P, P, P, C.c_int, C.POINTER(d), P]
    L.mclsgpu_spai_train_step.argtypes = [P, P, P, C.c_int, C.POINTER(SpaiAdam), C.POINTER(d)]
    L.mclsgpu_spai_rho.argtypes = [P, P, C.c_int, C.POINTER(d), C.POINTER(d)]
    L.mclsgpu_spai_smooth_vectors.argtypes = [P, P, P, C.c_int, C.c_int]
    L.mclsgpu_spai_set_penalty.argtypes = [P, d, d]
    L.mclsgpu_batch_build.argtypes = [P, C.c_int, P, P, P, P, P, C.POINTER(McParams), PP]
    L.mclsgpu_batch_destroy.argtypes = [P]
    L.mclsgpu_batch_layout.argtypes = [P, P, P, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]
    L.mclsgpu_batch_domain.argtypes = [P, PP]
    L.mclsgpu_batch_set_launch.argtypes = [P, C.c_int, C.c_int]
    L.mclsgpu_batch_autotune.argtypes = [P, P, P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(d)]
    L.mclsgpu_batch_mcsa_solve_dev.argtypes = [P, P, P, C.POINTER(McsaParams), P, P,
                                               C.POINTER(Stats)]
    _LIB = L
    return L


def _torch_ready():
    """Device vectors handed to the library are often torch tensors written by
    kernels on torch's current stream; the library works on its own
    non-blocking stream, so wait for torch's stream first."""
    import sys

    torch = sys.modules.get("torch")
    if torch is not None and torch.cuda.is_available() and torch.cuda.is_initialized():
        torch.cuda.current_stream().synchronize()


def _ptr(a):
    return a.ctypes.data if a is not None else None


def _stats():
    st = Stats()
    st.size = C.sizeof(Stats)
    return st


class Context:
    """One device context.  Handles created on it are released before it is:
    the C ABI requires every operator, preconditioner and domain of a context
    to be destroyed before the context itself."""

    def __init__(self, device: int = 0):
        self.L = load()
        h = C.c_void_p()
        rc = self.L.mclsgpu_context_create(device, C.byref(h))
        if rc != OK:
            raise MclsError(rc, "context create failed")
        self.h = h
        self._children = []  # weak references, released in reverse order

    def check(self, rc):
        if rc != OK:
            raise MclsError(rc, self.L.mclsgpu_last_error(self.h).decode())

    def set_wait_limit(self, polls: int):
        """Polls a bounded device wait makes before it gives up (< 0: the
        default)."""
        self.check(self.L.mclsgpu_set_wait_limit(self.h, int(polls)))

    def _adopt(self, child):
        import weakref

        self._children.append(weakref.ref(child))

    def close(self):
        if getattr(self, "h", None):
            for ref in reversed(self._children):
                child = ref()
                if child is not None:
                    child.close()
            self._children = []
            self.L.mclsgpu_context_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def _csr64(A):
    A = sp.csr_matrix(A)
    rp = np.ascontiguousarray(A.indptr, np.int64)
    ci = np.ascontiguousarray(A.indices, np.int64)
    v = np.ascontiguousarray(A.data, np.float64)
    return A.shape[0], rp, ci, v


class Operator:
    def __init__(self, ctx: Context, A):
        self.ctx = ctx
        n, rp, ci, v = _csr64(A)
        self.n = n
        h = C.c_void_p()
        ctx.check(ctx.L.mclsgpu_operator_upload(ctx.h, n, _ptr(rp), _ptr(ci), _ptr(v), C.byref(h)))
        self.h = h
        ctx._adopt(self)

    def apply(self, x):
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty_like(x)
        self.ctx.check(self.ctx.L.mclsgpu_operator_apply(self.h, _ptr(x), _ptr(y)))
        return y

    def apply_static(self, x):
        """y = A x staged through the library's static device array: no
        device allocation, at most 1,048,576 rows, calls must not overlap."""
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty_like(x)
        self.ctx.check(self.ctx.L.mclsgpu_operator_apply_static(self.h, _ptr(x), _ptr(y)))
        return y

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.mclsgpu_operator_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class Precond:
    def __init__(self, ctx: Context, op: Operator, kind: int, block_size: int = 1, user=None,
                 rho_fallback: float = 0.95, net=None):
        self.ctx = ctx
        p = PrecondParams()
        p.size = C.sizeof(PrecondParams)
        p.kind = kind
        p.block_size = block_size
        p.rho_fallback = rho_fallback
        keep = []
        if user is not None:
            n, rp, ci, v = _csr64(user)
            keep = [rp, ci, v]
            p.user_n = n
            p.user_rowptr, p.user_colind, p.user_values = _ptr(rp), _ptr(ci), _ptr(v)
        if net is not None:
            p.spai_net = net.h if isinstance(net, SpaiNet) else net
        h = C.c_void_p()
        ctx.check(ctx.L.mclsgpu_precond_build(ctx.h, op.h, C.byref(p), C.byref(h)))
        del keep
        self.h = h
        ctx._adopt(self)

    def to_scipy(self, n):
        nnz = C.c_int64()
        L = self.ctx.L
        self.ctx.check(L.mclsgpu_precond_export(self.h, C.byref(nnz), None, None, None))
        rp = np.empty(n + 1, np.int64)
        ci = np.empty(max(nnz.value, 1), np.int64)
        v = np.empty(max(nnz.value, 1), np.float64)
        self.ctx.check(L.mclsgpu_precond_export(self.h, C.byref(nnz), _ptr(rp), _ptr(ci), _ptr(v)))
        return sp.csr_matrix((v[: nnz.value], ci[: nnz.value], rp), shape=(n, n))

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.mclsgpu_precond_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def mc_params(direction=ADJOINT, estimator=COLLISION, history_length=10, weight_cutoff=0.0,
              sample_ratio=-1.0, source_sampling=SOURCE_RANDOM, precision=FP32,
              neumann_relaxation=-1.0, composite_threshold=0.0, rng_mode=RNG_COUNTER, seed=1,
              record_format=0):
    p = McParams()
    p.size = C.sizeof(McParams)
    p.record_format = record_format
    p.direction = direction
    p.estimator = estimator
    p.history_length = history_length
    p.weight_cutoff = weight_cutoff
    p.sample_ratio = sample_ratio
    p.source_sampling = source_sampling
    p.precision = precision
    p.neumann_relaxation = neumann_relaxation
    p.composite_threshold = composite_threshold
    p.rng_mode = rng_mode
    p.seed = seed
    return p


def mcsa_params(tolerance=1e-8, max_iters=1000, check_freq=1, smoother_steps=1,
                richardson_omega=1.0, print_freq=10, verbose=0, host_loop=0,
                fixed_point_type=FIXED_POINT_RICHARDSON):
    if isinstance(fixed_point_type, str):
        fixed_point_type = FIXED_POINT_TYPES[fixed_point_type]
    p = McsaParams()
    p.size = C.sizeof(McsaParams)
    p.tolerance = tolerance
    p.max_iters = max_iters
    p.check_freq = check_freq
    p.smoother_steps = smoother_steps
    p.richardson_omega = richardson_omega
    p.print_freq = print_freq
    p.verbose = verbose
    p.host_loop = host_loop
    p.fixed_point_type = fixed_point_type
    return p


def anderson_params(tolerance=1e-8, max_iters=1000, smoother_steps=1, storage_depth=2,
                    mixing=1.0, start_iteration=1, adjust_condition=0, drop_tolerance=1e-12,
                    host_loop=0):
    p = AndersonParams()
    p.size = C.sizeof(AndersonParams)
    p.tolerance = tolerance
    p.max_iters = max_iters
    p.smoother_steps = smoother_steps
    p.storage_depth = storage_depth
    p.mixing = mixing
    p.start_iteration = start_iteration
    p.adjust_condition = adjust_condition
    p.drop_tolerance = drop_tolerance
    p.host_loop = host_loop
    return p


def fixed_point_solve(ctx: Context, op: Operator, b, x0=None, left: Precond | None = None,
                      right: Precond | None = None, params: McsaParams | None = None, **kw):
    """FixedPointSolverManager::solve on the GPU: (x, stats).  Keywords as
    mcsa_params; the reference's default tolerance here is 1.0."""
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64)
    kw.setdefault("tolerance", 1.0)
    p = params if params is not None else mcsa_params(**kw)
    st = Stats()
    st.size = C.sizeof(Stats)
    ctx.check(ctx.L.mclsgpu_fixed_point_solve(ctx.h, op.h, left.h if left else None,
                                              right.h if right else None, _ptr(b), _ptr(x),
                                              C.byref(p), C.byref(st)))
    return x, st.as_dict()


class Domain:
    def __init__(self, ctx: Context, op: Operator, left: Precond | None = None,
                 right: Precond | None = None, params: McParams | None = None, **kw):
        self.ctx = ctx
        self.op = op
        self.left = left
        self.right = right
        self.p = params if params is not None else mc_params(**kw)
        self.n = op.n
        h = C.c_void_p()
        ctx.check(ctx.L.mclsgpu_domain_build(ctx.h, op.h, left.h if left else None,
                                             right.h if right else None, C.byref(self.p),
                                             C.byref(h)))
        self.h = h
        ctx._adopt(self)

    def export(self):
        L = self.ctx.L
        nnz = C.c_int64()
        self.ctx.check(L.mclsgpu_domain_export(self.h, C.byref(nnz), None, None, None, None, None))
        k = nnz.value
        rp = np.empty(self.n + 1, np.int64)
        col = np.empty(max(k, 1), np.int64)
        h = np.empty(max(k, 1), np.float64)
        cdf = np.empty(max(k, 1), np.float64)
        w = np.empty(self.n, np.float64)
        self.ctx.check(L.mclsgpu_domain_export(self.h, C.byref(nnz), _ptr(rp), _ptr(col), _ptr(h),
                                               _ptr(cdf), _ptr(w)))
        return dict(rowptr=rp, col=col[:k], h=h[:k], cdf=cdf[:k], weights=w)

    def info(self):
        d = DomainInfo()
        d.size = C.sizeof(DomainInfo)
        self.ctx.check(self.ctx.L.mclsgpu_domain_query(self.h, C.byref(d)))
        return {k: getattr(d, k) for k, _ in d._fields_ if k != "size"}

    def set_launch(self, histories_per_lane, block_size):
        self.ctx.check(self.ctx.L.mclsgpu_domain_set_launch(self.h, histories_per_lane,
                                                            block_size))

    def autotune(self, rhs_dev_ptr, reps=3):
        """Pick the fastest FP32 walk launch shape on a device right-hand side."""
        _torch_ready()
        hpl, blk, ms = C.c_int(), C.c_int(), C.c_double()
        self.ctx.check(self.ctx.L.mclsgpu_domain_autotune(self.h, C.c_void_p(rhs_dev_ptr), reps,
                                                          C.byref(hpl), C.byref(blk),
                                                          C.byref(ms)))
        return {"histories_per_lane": hpl.value, "block_size": blk.value, "walk_ms": ms.value,
                "record_cache_l1": self.info()["record_cache_l1"]}

    def set_record_cache(self, allocate_l1: bool):
        """FP32 walk record loads allocated in L1 or bypassing it."""
        self.ctx.check(self.ctx.L.mclsgpu_domain_set_record_cache(self.h, int(bool(allocate_l1))))

    def mcsa_solve_sets_dev(self, sets: "SetParams", b_ptr, x_ptr,
                            params: McsaParams | None = None, **kw):
        """Multi-set MCSA with device vectors: (stats, ran on the device)."""
        _torch_ready()
        p = params if params is not None else mcsa_params(**kw)
        st = _stats()
        dl = C.c_int32(0)
        self.ctx.check(self.ctx.L.mclsgpu_mcsa_solve_sets_dev(
            self.h, C.byref(sets), C.c_void_p(b_ptr), C.c_void_p(x_ptr), C.byref(p),
            C.byref(st), C.byref(dl)))
        return st.as_dict(), bool(dl.value)

    def mcsa_solve_sets(self, sets: "SetParams", b, x0=None, params: McsaParams | None = None,
                        **kw):
        """Multi-set MCSA with host vectors: (x, stats, ran on the device)."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64)
        p = params if params is not None else mcsa_params(**kw)
        st = _stats()
        dl = C.c_int32(0)
        self.ctx.check(self.ctx.L.mclsgpu_mcsa_solve_sets(self.h, C.byref(sets), _ptr(b), _ptr(x),
                                                          C.byref(p), C.byref(st),
                                                          C.byref(dl)))
        return x, st.as_dict(), bool(dl.value)

    def anderson_solve_sets(self, sets: "SetParams", b, x0=None,
                            params: AndersonParams | None = None, **kw):
        """Multi-set Anderson-accelerated MCSA with host vectors: (x, stats)."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64)
        p = params if params is not None else anderson_params(**kw)
        st = _stats()
        self.ctx.check(self.ctx.L.mclsgpu_anderson_solve_sets(self.h, C.byref(sets), _ptr(b),
                                                              _ptr(x), C.byref(p), C.byref(st)))
        return x, st.as_dict()

    def walk_agreement(self, histories, seed=1):
        """FP32 walk against the FP64 selection on the same draws: (histories
        with a differing transition, differing transitions)."""
        h, t = C.c_int64(), C.c_int64()
        self.ctx.check(self.ctx.L.mclsgpu_domain_walk_agreement(self.h, int(histories), seed,
                                                                C.byref(h), C.byref(t)))
        return h.value, t.value

    def reseed(self, seed):
        self.ctx.check(self.ctx.L.mclsgpu_domain_reseed(self.h, seed))

    def mc_solve(self, rhs, internal=False):
        rhs = np.ascontiguousarray(rhs, np.float64)
        x = np.empty_like(rhs)
        st = Stats()
        st.size = C.sizeof(Stats)
        self.ctx.check(self.ctx.L.mclsgpu_mc_solve(self.h, _ptr(rhs), _ptr(x), int(internal),
                                                   C.byref(st)))
        return x, st.as_dict()

    def mc_solve_dev(self, rhs_ptr, x_ptr, internal=False):
        """Device-pointer Monte Carlo solve (mclsgpu_mc_solve_dev)."""
        _torch_ready()
        st = Stats()
        st.size = C.sizeof(Stats)
        self.ctx.check(self.ctx.L.mclsgpu_mc_solve_dev(self.h, C.c_void_p(rhs_ptr),
                                                       C.c_void_p(x_ptr), int(internal),
                                                       C.byref(st)))
        return st.as_dict()

    def mc_trace(self, rhs, max_trace, internal=False):
        rhs = np.ascontiguousarray(rhs, np.float64)
        x = np.empty_like(rhs)
        L = self.p.history_length
        states = np.empty(max(max_trace, 1) * (L + 1), np.int64)
        fw = np.empty(max(max_trace, 1), np.float64)
        ev = np.empty(max(max_trace, 1), np.int32)
        st = np.empty(max(max_trace, 1), np.int64)
        nh = C.c_int64()
        self.ctx.check(self.ctx.L.mclsgpu_mc_trace(self.h, _ptr(rhs), _ptr(x), int(internal),
                                                   max_trace, _ptr(states), _ptr(fw), _ptr(ev),
                                                   _ptr(st), C.byref(nh)))
        k = min(nh.value, max_trace)
        return x, nh.value, dict(states=states.reshape(-1, L + 1)[:k], final_weight=fw[:k],
                                 events=ev[:k], start=st[:k])

    def mcsa_solve(self, b, x0=None, params: McsaParams | None = None, **kw):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64)
        p = params if params is not None else mcsa_params(**kw)
        st = Stats()
        st.size = C.sizeof(Stats)
        self.ctx.check(self.ctx.L.mclsgpu_mcsa_solve(self.h, _ptr(b), _ptr(x), C.byref(p),
                                                     C.byref(st)))
        return x, st.as_dict()

    def mcsa_solve_dev(self, b_ptr, x_ptr, params: McsaParams | None = None, **kw):
        """Device-pointer variant (e.g. torch tensors' data_ptr())."""
        _torch_ready()
        p = params if params is not None else mcsa_params(**kw)
        st = Stats()
        st.size = C.sizeof(Stats)
        self.ctx.check(self.ctx.L.mclsgpu_mcsa_solve_dev(self.h, C.c_void_p(b_ptr),
                                                         C.c_void_p(x_ptr), C.byref(p),
                                                         C.byref(st)))
        return st.as_dict()

    def anderson_solve(self, b, x0=None, params: AndersonParams | None = None, **kw):
        """Anderson-accelerated MCSA (AndersonSolverManager::solve)."""
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64)
        p = params if params is not None else anderson_params(**kw)
        st = Stats()
        st.size = C.sizeof(Stats)
        self.ctx.check(self.ctx.L.mclsgpu_anderson_solve(self.h, _ptr(b), _ptr(x), C.byref(p),
                                                         C.byref(st)))
        return x, st.as_dict()

    def anderson_solve_dev(self, b_ptr, x_ptr, params: AndersonParams | None = None, **kw):
        _torch_ready()
        p = params if params is not None else anderson_params(**kw)
        st = Stats()
        st.size = C.sizeof(Stats)
        self.ctx.check(self.ctx.L.mclsgpu_anderson_solve_dev(self.h, C.c_void_p(b_ptr),
                                                             C.c_void_p(x_ptr), C.byref(p),
                                                             C.byref(st)))
        return st.as_dict()

    def anderson_begin(self, b_ptr, x0_ptr, params: AndersonParams | None = None, **kw):
        """Step-wise Anderson MCSA: (|PL (b - A x0)|_2, |b|_2, done)."""
        _torch_ready()
        p = params if params is not None else anderson_params(**kw)
        rn, bn, done = C.c_double(), C.c_double(), C.c_int32()
        self.ctx.check(self.ctx.L.mclsgpu_anderson_begin(self.h, C.c_void_p(b_ptr),
                                                         C.c_void_p(x0_ptr), C.byref(p),
                                                         C.byref(rn), C.byref(bn),
                                                         C.byref(done)))
        return rn.value, bn.value, bool(done.value)

    def anderson_correction(self, delta_ptr):
        _torch_ready()
        self.ctx.check(self.ctx.L.mclsgpu_anderson_correction(self.h, C.c_void_p(delta_ptr)))

    def anderson_apply(self, delta_ptr, scale=1.0):
        """Returns (|PL (b - A x)|_2 after the step, done)."""
        _torch_ready()
        rn, done = C.c_double(), C.c_int32()
        self.ctx.check(self.ctx.L.mclsgpu_anderson_apply(self.h, C.c_void_p(delta_ptr), scale,
                                                         C.byref(rn), C.byref(done)))
        return rn.value, bool(done.value)

    def anderson_finish(self, x_ptr):
        _torch_ready()
        st = Stats()
        st.size = C.sizeof(Stats)
        self.ctx.check(self.ctx.L.mclsgpu_anderson_finish(self.h, C.c_void_p(x_ptr),
                                                          C.byref(st)))
        return st.as_dict()

    def mcsa_begin(self, b_ptr, x0_ptr, params: McsaParams | None = None, **kw):
        """Step-wise MCSA: initial residual; returns (|rp|_2, |PL b|_2)."""
        _torch_ready()
        p = params if params is not None else mcsa_params(**kw)
        rn, bn = C.c_double(), C.c_double()
        self.ctx.check(self.ctx.L.mclsgpu_mcsa_begin(self.h, C.c_void_p(b_ptr), C.c_void_p(x0_ptr),
                                                     C.byref(p), C.byref(rn), C.byref(bn)))
        return rn.value, bn.value

    def mcsa_correction(self, delta_ptr):
        _torch_ready()
        self.ctx.check(self.ctx.L.mclsgpu_mcsa_correction(self.h, C.c_void_p(delta_ptr)))

    def mcsa_apply(self, delta_ptr, scale=1.0):
        _torch_ready()
        rn = C.c_double()
        self.ctx.check(self.ctx.L.mclsgpu_mcsa_apply(self.h, C.c_void_p(delta_ptr), scale,
                                                     C.byref(rn)))
        return rn.value

    def mcsa_finish(self, x_ptr):
        _torch_ready()
        st = Stats()
        st.size = C.sizeof(Stats)
        self.ctx.check(self.ctx.L.mclsgpu_mcsa_finish(self.h, C.c_void_p(x_ptr), C.byref(st)))
        return st.as_dict()

    def residual(self, rp_dev_ptr):
        """Copy the last MCSA solve's preconditioned residual to a device vector."""
        _torch_ready()
        self.ctx.check(self.ctx.L.mclsgpu_domain_residual(self.h, C.c_void_p(rp_dev_ptr)))

    def convergence_criteria(self, max_iters=2000, tol=1e-8, seed=7):
        """AlmostOptimalDomain::computeConvergenceCriteria's report."""
        c = Criteria()
        c.size = C.sizeof(Criteria)
        self.ctx.check(self.ctx.L.mclsgpu_domain_convergence_criteria(self.h, max_iters, tol,
                                                                      seed, C.byref(c)))
        return {k: getattr(c, k) for k, _ in c._fields_ if k not in ("size", "reserved0")}

    def spectral_radius(self, which=0, max_iters=2000, tol=1e-8, seed=7):
        rho = C.c_double()
        self.ctx.check(self.ctx.L.mclsgpu_domain_spectral_radius(self.h, which, max_iters, tol,
                                                                 seed, C.byref(rho)))
        return rho.value

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.mclsgpu_domain_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class SpaiNet:
    """The learned-SPAI network (16 -> 64 -> 64 -> 16) on a context."""

    def __init__(self, ctx: Context, slots: int, seed: int = 0):
        self.ctx = ctx
        self.slots = slots
        self.nparams = int(ctx.L.mclsgpu_spai_num_params())
        h = C.c_void_p()
        ctx.check(ctx.L.mclsgpu_spai_create(ctx.h, slots, seed, C.byref(h)))
        self.h = h
        ctx._adopt(self)

    def set_penalty(self, weight, threshold=1.0):
        """Row-sum penalty of the training loss (weight 0 = off)."""
        self.ctx.check(self.ctx.L.mclsgpu_spai_set_penalty(self.h, weight, threshold))

    @property
    def params(self):
        p = np.empty(self.nparams, np.float32)
        self.ctx.check(self.ctx.L.mclsgpu_spai_get_params(self.h, _ptr(p)))
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparams
        self.ctx.check(self.ctx.L.mclsgpu_spai_set_params(self.h, _ptr(p)))

    def infer(self, op: Operator, nnz: int):
        """(raw outputs [n, 16], M values on A's pattern)."""
        out = np.empty((op.n, 16), np.float32)
        m = np.empty(nnz, np.float64)
        self.ctx.check(self.ctx.L.mclsgpu_spai_infer(self.h, op.h, _ptr(out), _ptr(m)))
        return out, m

    def infer_dev(self, op: Operator, out_ptr=None, mvals_ptr=None):
        """Inference into device arrays; returns the forward kernel's device
        time in ms."""
        _torch_ready()
        ms = C.c_float()
        self.ctx.check(self.ctx.L.mclsgpu_spai_infer_dev(
            self.h, op.h, C.c_void_p(out_ptr) if out_ptr else None,
            C.c_void_p(mvals_ptr) if mvals_ptr else None, C.byref(ms)))
        return ms.value

    def gradient(self, op: Operator, v_dev_ptr, nvec):
        """(loss, FP32 parameter gradient) for nvec device vectors."""
        _torch_ready()
        loss = C.c_double()
        g = np.empty(self.nparams, np.float32)
        self.ctx.check(self.ctx.L.mclsgpu_spai_gradient(self.h, op.h, C.c_void_p(v_dev_ptr), nvec,
                                                        C.byref(loss), _ptr(g)))
        return loss.value, g

    def train_step(self, op: Operator, v_dev_ptr, nvec, lr=1e-3, beta1=0.9, beta2=0.999,
                   eps=1e-8, grad_clip=0.0):
        _torch_ready()
        a = SpaiAdam()
        a.size = C.sizeof(SpaiAdam)
        a.lr, a.beta1, a.beta2, a.eps, a.grad_clip = lr, beta1, beta2, eps, grad_clip
        loss = C.c_double()
        self.ctx.check(self.ctx.L.mclsgpu_spai_train_step(self.h, op.h, C.c_void_p(v_dev_ptr),
                                                          nvec, C.byref(a), C.byref(loss)))
        return loss.value

    def smooth_vectors(self, op: Operator, v_dev_ptr, nvec, iters):
        """In place: iters applications of I - M A (normalised) to each vector."""
        _torch_ready()
        self.ctx.check(self.ctx.L.mclsgpu_spai_smooth_vectors(self.h, op.h, C.c_void_p(v_dev_ptr),
                                                              nvec, iters))

    def rho(self, op: Operator, iters=200):
        """(rho(I - M A) learned, rho(I - D^-1 A) point Jacobi)."""
        rl, rj = C.c_double(), C.c_double()
        self.ctx.check(self.ctx.L.mclsgpu_spai_rho(self.h, op.h, iters, C.byref(rl), C.byref(rj)))
        return rl.value, rj.value

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.mclsgpu_spai_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class Batch:
    """Many systems with 1..16 right-hand sides each in one MCSA loop
    (forward FP32 walks shared by every right-hand side).  Device vectors are
    flat FP64 arrays of `elements` entries: system s owns the row-major
    [n_s, widths[s]] block at elem_offsets[s] (widths[s] = its right-hand-side
    count rounded up to a power of two); pack/unpack convert."""

    def __init__(self, ctx: Context, systems, nrhs, params: McParams | None = None, **kw):
        self.ctx = ctx
        p = params if params is not None else mc_params(**kw)
        mats = [_csr64(A) for A in systems]
        self.nsys = len(mats)
        n = np.array([m[0] for m in mats], np.int64)
        rp = (C.c_void_p * self.nsys)(*[m[1].ctypes.data for m in mats])
        ci = (C.c_void_p * self.nsys)(*[m[2].ctypes.data for m in mats])
        va = (C.c_void_p * self.nsys)(*[m[3].ctypes.data for m in mats])
        self.nrhs = np.ascontiguousarray(nrhs, np.int32)
        h = C.c_void_p()
        ctx.check(ctx.L.mclsgpu_batch_build(ctx.h, self.nsys, _ptr(n), rp, ci, va,
                                            _ptr(self.nrhs), C.byref(p), C.byref(h)))
        del mats
        self.h = h
        off = np.empty(self.nsys, np.int64)
        wid = np.empty(self.nsys, np.int32)
        ne, w = C.c_int64(), C.c_int32()
        ctx.check(ctx.L.mclsgpu_batch_layout(self.h, _ptr(off), _ptr(wid), C.byref(ne),
                                             C.byref(w)))
        self.elem_offsets, self.widths, self.elements, self.width = off, wid, ne.value, w.value
        self.n = n
        self.rows = int(n.sum())
        ctx._adopt(self)

    def block(self, X, s):
        """System s's [n_s, widths[s]] view of a flat element array."""
        o = int(self.elem_offsets[s])
        return X[o:o + int(self.n[s]) * int(self.widths[s])].reshape(int(self.n[s]),
                                                                      int(self.widths[s]))

    def pack(self, vectors):
        """Flat element array from per-system [n_s, nrhs_s] blocks."""
        out = np.zeros(self.elements)
        for s, v in enumerate(vectors):
            v = np.asarray(v, np.float64).reshape(int(self.n[s]), -1)
            self.block(out, s)[:, : v.shape[1]] = v
        return out

    def unpack(self, X):
        X = np.asarray(X).reshape(-1)
        return [self.block(X, s)[:, : self.nrhs[s]] for s in range(self.nsys)]

    def domain_info(self):
        hd = C.c_void_p()
        self.ctx.check(self.ctx.L.mclsgpu_batch_domain(self.h, C.byref(hd)))
        d = DomainInfo()
        d.size = C.sizeof(DomainInfo)
        self.ctx.check(self.ctx.L.mclsgpu_domain_query(hd, C.byref(d)))
        return {k: getattr(d, k) for k, _ in d._fields_ if k != "size"}

    def reseed(self, seed):
        hd = C.c_void_p()
        self.ctx.check(self.ctx.L.mclsgpu_batch_domain(self.h, C.byref(hd)))
        self.ctx.check(self.ctx.L.mclsgpu_domain_reseed(hd, seed))

    def set_launch(self, block_size, grab=1):
        self.ctx.check(self.ctx.L.mclsgpu_batch_set_launch(self.h, block_size, grab))

    def autotune(self, b_ptr, x_ptr, reps=3):
        _torch_ready()
        blk, grab, ms = C.c_int(), C.c_int(), C.c_double()
        self.ctx.check(self.ctx.L.mclsgpu_batch_autotune(self.h, C.c_void_p(b_ptr),
                                                         C.c_void_p(x_ptr), reps, C.byref(blk),
                                                         C.byref(grab), C.byref(ms)))
        return {"block_size": blk.value, "grab": grab.value, "walk_ms": ms.value}

    def mcsa_solve_dev(self, b_ptr, x_ptr, params: McsaParams | None = None, **kw):
        """Solve in place on device element arrays; returns (stats, per-pair
        convergence iterations [nsys, width], final relative preconditioned
        residuals [nsys, width]), width the widest system's."""
        _torch_ready()
        p = params if params is not None else mcsa_params(**kw)
        st = Stats()
        st.size = C.sizeof(Stats)
        it = np.empty((self.nsys, self.width), np.int32)
        rr = np.empty((self.nsys, self.width), np.float64)
        self.ctx.check(self.ctx.L.mclsgpu_batch_mcsa_solve_dev(self.h, C.c_void_p(b_ptr),
                                                               C.c_void_p(x_ptr), C.byref(p),
                                                               _ptr(it), _ptr(rr), C.byref(st)))
        return st.as_dict(), it, rr

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.mclsgpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class Subdomain:
    """One part of a row-partitioned domain (mclsgpu_subdomain_*).

    `rows` is the part's rows of the composite operator the walks follow --
    (PL A PR)^T for adjoint walks, PL A PR for forward walks -- with global
    column indices (scipy CSR, n_global columns)."""

    def __init__(self, ctx: Context, n_global: int, bounds, part: int, rows,
                 params: McParams | None = None, **kw):
        self.ctx = ctx
        self.p = params if params is not None else mc_params(**kw)
        self.bounds = np.ascontiguousarray(bounds, np.int64)
        self.nparts = len(self.bounds) - 1
        self.part = part
        R = sp.csr_matrix(rows)
        R.sort_indices()
        rp = np.ascontiguousarray(R.indptr, np.int64)
        ci = np.ascontiguousarray(R.indices, np.int64)
        v = np.ascontiguousarray(R.data, np.float64)
        h = C.c_void_p()
        ctx.check(ctx.L.mclsgpu_subdomain_build(ctx.h, n_global, self.nparts, _ptr(self.bounds),
                                                part, _ptr(rp), _ptr(ci), _ptr(v),
                                                C.byref(self.p), C.byref(h)))
        self.h = h
        ctx._adopt(self)
        b, r, rb = C.c_int64(), C.c_int64(), C.c_int32()
        ctx.check(ctx.L.mclsgpu_subdomain_info(self.h, C.byref(b), C.byref(r), C.byref(rb)))
        self.row_begin, self.rows, self.record_bytes = b.value, r.value, rb.value

    def begin(self, rhs_ptr):
        """Returns (histories starting in this part, histories in the solve)."""
        _torch_ready()
        ns, nt = C.c_int64(), C.c_int64()
        self.ctx.check(self.ctx.L.mclsgpu_subdomain_begin(self.h, C.c_void_p(rhs_ptr),
                                                          C.byref(ns), C.byref(nt)))
        return ns.value, nt.value

    def transport(self, inbox_ptr, n_in, outbox_ptr, capacity):
        """One round; returns the departures per destination part."""
        _torch_ready()
        counts = np.zeros(self.nparts, np.int64)
        self.ctx.check(self.ctx.L.mclsgpu_subdomain_transport(
            self.h, C.c_void_p(inbox_ptr) if inbox_ptr else None, n_in, C.c_void_p(outbox_ptr),
            capacity, _ptr(counts)))
        return counts

    def finish(self, x_ptr):
        _torch_ready()
        st = Stats()
        st.size = C.sizeof(Stats)
        self.ctx.check(self.ctx.L.mclsgpu_subdomain_finish(self.h, C.c_void_p(x_ptr),
                                                           C.byref(st)))
        return st.as_dict()

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.mclsgpu_subdomain_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class Comm:
    """The library's NCCL communicator of `nranks` sets (multi-set MCSA)."""

    @staticmethod
    def unique_id() -> bytes:
        buf = (C.c_uint8 * 128)()
        rc = load().mclsgpu_comm_unique_id(buf)
        if rc != OK:
            raise MclsError(rc, "NCCL unique id")
        return bytes(buf)

    def __init__(self, ctx: Context, nranks: int, rank: int, uid: bytes):
        self.ctx = ctx
        buf = (C.c_uint8 * 128).from_buffer_copy(uid)
        h = C.c_void_p()
        ctx.check(ctx.L.mclsgpu_comm_create(ctx.h, nranks, rank, buf, C.byref(h)))
        self.h = h
        ctx._adopt(self)

    def set_params(self) -> SetParams:
        sp = SetParams()
        self.ctx.check(self.ctx.L.mclsgpu_comm_set_params(self.h, C.byref(sp)))
        return sp

    def close(self):
        if getattr(self, "h", None):
            self.ctx.L.mclsgpu_comm_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def set_params(num_sets: int, reduce, capturable: bool = False) -> SetParams:
    """Set params around a Python reducer reduce(data_ptr, n, stream_ptr) ->
    None that sums the n doubles at data_ptr over the sets in place.  The
    returned structure keeps the callback alive."""

    def _cb(user, data, n, stream):
        try:
            reduce(int(data or 0), int(n), int(stream or 0))
            return 0
        except Exception:  # reported to the library as a failed reduction
            import traceback

            traceback.print_exc()
            return ERR_INVALID_ARG

    fn = SET_REDUCE_FN(_cb)
    sp = SetParams()
    sp.size = C.sizeof(SetParams)
    sp.num_sets = num_sets
    sp.reduce = C.cast(fn, C.c_void_p).value
    sp.user = None
    sp.capturable = 1 if capturable else 0
    sp._keep = fn
    return sp


def device_allocations():
    """(allocations, releases) of device memory the library has made."""
    L = load()
    a, f = C.c_int64(), C.c_int64()
    L.mclsgpu_debug_device_allocations(C.byref(a), C.byref(f))
    return a.value, f.value


def rank_seed(master: int, rank: int) -> int:
    return int(load().mclsgpu_rank_seed(master, rank))
