// capi.cu -- context, operator, preconditioner and domain entry points of the
// C ABI, plus the error plumbing shared by the other translation units.
#include <algorithm>
#include <cstdarg>
#include <cmath>
#include <cstring>
#include <limits>
#include <random>
#include <vector>

#include "internal.h"
#include "rng.cuh"

namespace mclsgpu {

std::atomic<long long> g_device_allocs{0};
std::atomic<long long> g_device_frees{0};

int set_error(mclsgpu_context* ctx, int code, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->err = buf;
    }
    return code;
}

int cuda_fail(mclsgpu_context* ctx, cudaError_t e, const char* what) {
    return set_error(ctx, MCLSGPU_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int check_device_status(mclsgpu_context* ctx) {
    cudaError_t e = cudaMemcpyAsync(ctx->h_status, ctx->d_status, sizeof(int),
                                    cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "device status");
    const int st = *ctx->h_status;
    if (!st) return MCLSGPU_OK;
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream);
    if (st & DEV_ERR_DEGENERATE)
        return set_error(ctx, MCLSGPU_ERR_DEGENERATE,
                         "domain row with no retained entries or zero weight");
    if (st & DEV_ERR_CAPACITY)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "more histories than the domain was sized for");
    if (st & DEV_ERR_NONFINITE)
        return set_error(ctx, MCLSGPU_ERR_DIVERGED, "non-finite source, weight or residual");
    if (st & DEV_ERR_TIMEOUT) return set_error(ctx, MCLSGPU_ERR_TIMEOUT, "bounded device wait expired");
    return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "device index check failed (status %d)", st);
}

void prepare_walk(mclsgpu_domain* dom);
int walk_agreement(mclsgpu_domain* dom, long long histories, uint64_t seed, long long* hist_diff,
                   long long* trans_diff);
void prepare_source(mclsgpu_domain* dom);
int spai_build(mclsgpu_context* ctx, mclsgpu_operator* op, const mclsgpu_precond_params* p,
               mclsgpu_precond* pc);

namespace {

inline int grid_for(long long work, int threads = 256, int cap = 148 * 16) {
    long long g = (work + threads - 1) / threads;
    if (g < 1) g = 1;
    return int(g > cap ? cap : g);
}

__global__ void k_i32_to_i64(const int* a, long long* b, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        b[i] = a[i];
}

// y = M x where M is the domain with values h, |h| or |h| * W_row.
__global__ void k_domain_spmv(const int* rp, const int* ci, const double* h, const double* W,
                              int n, int mode, const double* x, double* y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            double v = h[k];
            if (mode == 1) v = fabs(v);
            if (mode == 2) v = fabs(v) * W[i];
            s = fma(v, x[ci[k]], s);
        }
        y[i] = s;
    }
}

// Balance parameters of |H|: rmax[i] = max_j |h_ij|, cmax[j] = max_i |h_ij|
// (non-negative doubles order like their bit patterns).
__global__ void k_row_col_max(const int* rp, const double* h, const int* ci, int n, double* rmax,
                              unsigned long long* cmax) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double m = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const double a = fabs(h[k]);
            m = fmax(m, a);
            atomicMax(&cmax[ci[k]], (unsigned long long)__double_as_longlong(a));
        }
        rmax[i] = m;
    }
}

__global__ void k_fill_random(double* x, int n, uint64_t seed) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = 0.5 + canonical64(splitmix64(seed ^ splitmix64(uint64_t(i))));
}

__global__ void k_scale(double* x, int n, const double* sumsq) {
    const double inv = 1.0 / sqrt(*sumsq);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] *= inv;
}

struct XsEngine {  // Xorshift(13,7,17) as a UniformRandomBitGenerator
    typedef uint64_t result_type;
    uint64_t x;
    static constexpr uint64_t min() { return 0; }
    static constexpr uint64_t max() { return ~uint64_t(0); }
    uint64_t operator()() { return x = xs_step(x); }
};

int copy_csr_out(mclsgpu_context* ctx, const DevCsr& A, int64_t* nnz_out, int64_t* rowptr,
                 int64_t* colind, double* values) {
    if (nnz_out) *nnz_out = A.nnz;
    cudaStream_t s = ctx->stream;
    long long* tmp = nullptr;
    cudaError_t e = dmalloc(&tmp, size_t(A.nnz > A.n + 1 ? A.nnz : A.n + 1));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    if (rowptr) {
        k_i32_to_i64<<<grid_for(A.n + 1), 256, 0, s>>>(A.rp, tmp, A.n + 1);
        cudaMemcpyAsync(rowptr, tmp, (A.n + 1) * sizeof(long long), cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
    }
    if (colind) {
        k_i32_to_i64<<<grid_for(A.nnz), 256, 0, s>>>(A.ci, tmp, A.nnz);
        cudaMemcpyAsync(colind, tmp, A.nnz * sizeof(long long), cudaMemcpyDeviceToHost, s);
        cudaStreamSynchronize(s);
    }
    if (values) cudaMemcpyAsync(values, A.v, A.nnz * sizeof(double), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    dfree(tmp);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(ctx, e, "export");
}

void release_domain(mclsgpu_domain* d) {
    release_anderson(d);
    d->D.release();
    d->DS.release();
    d->DT.release();
    dfree(d->cdf);
    dfree(d->w);
    dfree(d->dt_h32);
    dfree(d->rec);
    dfree(d->d_jump);
    dfree(d->d_pos);
    dfree(d->hoff);
    dfree(d->hlen);
    dfree(d->hoff2);
    dfree(d->y_save);
    dfree(d->delta);
    if (d->set_graph) cudaGraphExecDestroy(d->set_graph);
    d->set_graph = nullptr;
    dfree(d->d_epoch);
    dfree(d->src);
    dfree(d->scdf);
    dfree(d->guide);
    dfree(d->counts);
    dfree(d->offs);
    dfree(d->start);
    dfree(d->y64);
    dfree(d->c32);
    dfree(d->c64);
    dfree(d->d_nh);
    dfree(d->d_counter);
    dfree(d->d_scalars);
    dfree(d->d_steps);
    dfree(d->d_tim);
    dfree(d->d_hist);
    dfree(d->part);
    dfree(d->ipart);
    dfree(d->x);
    dfree(d->b);
    dfree(d->rp);
    dfree(d->tmp);
    dfree(d->tmp2);
    dfree(d->x2);
    dfree(d->rp2);
    dfree(d->d_ticket);
    dfree(d->d_state);
    dfree(d->d_resid);
    if (d->h_state) cudaFreeHost(d->h_state);
    d->h_state = nullptr;
    if (d->graph) cudaGraphExecDestroy(d->graph);
    d->graph = nullptr;
}

}  // namespace
}  // namespace mclsgpu

using namespace mclsgpu;

extern "C" {

int mclsgpu_abi_version(void) { return MCLSGPU_ABI_VERSION; }

const char* mclsgpu_build_info(void) {
    return "mclsgpu sm_100a; walk records FP32 {4,8,12,16,24,32} slots; FP64 parity walk";
}

int mclsgpu_debug_device_allocations(int64_t* allocs, int64_t* frees) {
    if (allocs) *allocs = g_device_allocs.load(std::memory_order_relaxed);
    if (frees) *frees = g_device_frees.load(std::memory_order_relaxed);
    return MCLSGPU_OK;
}

int mclsgpu_context_create(int device, mclsgpu_context** out) {
    if (!out) return MCLSGPU_ERR_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return MCLSGPU_ERR_NO_DEVICE;
    }
    if (device < 0) cudaGetDevice(&device);
    if (device >= count) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = new mclsgpu_context;
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = dmalloc(&ctx->d_status, 1);
    if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void**>(&ctx->h_status), sizeof(int));
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        delete ctx;
        return MCLSGPU_ERR_CUDA;
    }
    *out = ctx;
    return MCLSGPU_OK;
}

int mclsgpu_context_destroy(mclsgpu_context* ctx) {
    if (!ctx) return MCLSGPU_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    dfree(ctx->d_status);
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return MCLSGPU_OK;
}

const char* mclsgpu_last_error(const mclsgpu_context* ctx) {
    return ctx ? ctx->err.c_str() : "null context";
}

int mclsgpu_context_sync(mclsgpu_context* ctx) {
    if (!ctx) return MCLSGPU_ERR_INVALID_ARG;
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "sync");
    return check_device_status(ctx);
}

// ---- operator --------------------------------------------------------------
int mclsgpu_operator_upload(mclsgpu_context* ctx, int64_t n, const int64_t* rowptr,
                            const int64_t* colind, const double* values, mclsgpu_operator** out) {
    if (!ctx || !out) return MCLSGPU_ERR_INVALID_ARG;
    *out = nullptr;
    static uint64_t serial = 0;
    mclsgpu_operator* op = new mclsgpu_operator;
    op->ctx = ctx;
    op->serial = ++serial;
    int rc = upload_csr(ctx, n, rowptr, colind, values, op->A);
    if (!rc) rc = csr_to_sell(ctx, op->A, op->S);
    // Stencil operators also get diagonal-offset storage (no column indices)
    // when it holds at most 25% more values than the CSR arrays.
    int K = 0;
    if (!rc) rc = collect_offsets(ctx, op->A, 16, op->dia_off, &K);
    if (!rc && K > 0 && double(K) * op->A.n <= 1.25 * op->A.nnz + op->A.n) {
        rc = csr_to_dia(ctx, op->A, K, op->dia_off, &op->dia_val);
        if (!rc) op->dia_k = K;
        if (!rc && K <= 9)
            rc = dia_symmetric(ctx, op->A.n, K, op->dia_off, op->dia_val, &op->sym_val,
                               &op->sym_h, op->sym_off);
    }
    if (rc) {
        op->A.release();
        op->S.release();
        dfree(op->dia_val);
        dfree(op->sym_val);
        delete op;
        return rc;
    }
    *out = op;
    return MCLSGPU_OK;
}

int mclsgpu_operator_destroy(mclsgpu_operator* op) {
    if (!op) return MCLSGPU_OK;
    op->A.release();
    op->AT.release();
    op->S.release();
    dfree(op->dia_val);
    dfree(op->sym_val);
    dfree(op->dinv);
    delete op;
    return MCLSGPU_OK;
}

int64_t mclsgpu_operator_rows(const mclsgpu_operator* op) { return op ? op->A.n : -1; }
int64_t mclsgpu_operator_nnz(const mclsgpu_operator* op) { return op ? op->A.nnz : -1; }

int mclsgpu_operator_apply(mclsgpu_operator* op, const double* x, double* y) {
    if (!op || !x || !y) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = op->ctx;
    const size_t bytes = size_t(op->A.n) * sizeof(double);
    double *dx = nullptr, *dy = nullptr;
    cudaError_t e;
    if ((e = dmalloc(&dx, op->A.n)) != cudaSuccess || (e = dmalloc(&dy, op->A.n)) != cudaSuccess) {
        dfree(dx);
        return cuda_fail(ctx, e, "cudaMalloc");
    }
    const char* what = "copy x";
    e = cudaMemcpyAsync(dx, x, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) {
        spmv(ctx->stream, op->A, dx, dy);
        what = "apply: spmv launch";
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        what = "copy y";
        e = cudaMemcpyAsync(y, dy, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    }
    if (e == cudaSuccess) {
        what = "apply";
        e = cudaStreamSynchronize(ctx->stream);
    }
    dfree(dx);
    dfree(dy);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(ctx, e, what);
}

// ---- preconditioner ----------------------------------------------------------
int mclsgpu_precond_build(mclsgpu_context* ctx, mclsgpu_operator* op,
                          const mclsgpu_precond_params* p, mclsgpu_precond** out) {
    if (!ctx || !op || !p || !out) return MCLSGPU_ERR_INVALID_ARG;
    if (p->size < sizeof(mclsgpu_precond_params))
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "precond params: size mismatch");
    *out = nullptr;
    mclsgpu_precond* pc = new mclsgpu_precond;
    pc->ctx = ctx;
    pc->kind = p->kind;
    int rc = MCLSGPU_OK;
    cudaError_t e;
    switch (p->kind) {
        case MCLSGPU_PREC_POINT_JACOBI:
            if ((e = dmalloc(&pc->diag, op->A.n)) != cudaSuccess) {
                rc = cuda_fail(ctx, e, "cudaMalloc");
                break;
            }
            rc = reciprocal_diagonal(ctx, op->A, pc->diag);
            if (!rc) rc = point_jacobi_csr(ctx, op->A.n, pc->diag, pc->P);
            break;
        case MCLSGPU_PREC_BLOCK_JACOBI:
            pc->block_size = p->block_size;
            rc = block_jacobi(ctx, op->A, p->block_size, pc->P);
            break;
        case MCLSGPU_PREC_USER_CSR:
            if (p->user_n != op->A.n)
                rc = set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "user preconditioner size mismatch");
            else
                rc = upload_csr(ctx, p->user_n, p->user_rowptr, p->user_colind, p->user_values, pc->P);
            break;
        case MCLSGPU_PREC_LEARNED_SPAI:
            rc = spai_build(ctx, op, p, pc);
            break;
        default:
            rc = set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "unknown preconditioner kind %d", p->kind);
    }
    if (!rc) {
        e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "precond build");
    }
    if (rc) {
        pc->P.release();
        dfree(pc->diag);
        dfree(pc->mdia);
        delete pc;
        return rc;
    }
    *out = pc;
    return MCLSGPU_OK;
}

int mclsgpu_precond_destroy(mclsgpu_precond* pc) {
    if (!pc) return MCLSGPU_OK;
    pc->P.release();
    pc->PT.release();
    dfree(pc->diag);
    dfree(pc->mdia);
    delete pc;
    return MCLSGPU_OK;
}

int mclsgpu_precond_export(mclsgpu_precond* pc, int64_t* nnz_out, int64_t* rowptr,
                           int64_t* colind, double* values) {
    if (!pc) return MCLSGPU_ERR_INVALID_ARG;
    return copy_csr_out(pc->ctx, pc->P, nnz_out, rowptr, colind, values);
}

// ---- domain --------------------------------------------------------------------
uint64_t mclsgpu_rank_seed(uint64_t master_seed, int rank) {
    // PRNG<RNG>::PRNG (src/MCLS_PRNG_impl.hpp:56-75): master engine, then the
    // (rank+1)-th uniform_int_distribution<int>(0, INT_MAX) draw.
    XsEngine master{master_seed};
    std::uniform_int_distribution<int> dist(0, std::numeric_limits<int>::max());
    int seed = 0;
    for (int i = -1; i < rank; ++i) seed = dist(master);
    return uint64_t(seed);
}

int mclsgpu_domain_build(mclsgpu_context* ctx, mclsgpu_operator* op, mclsgpu_precond* left,
                         mclsgpu_precond* right, const mclsgpu_mc_params* p,
                         mclsgpu_domain** out) {
    if (!ctx || !op || !p || !out) return MCLSGPU_ERR_INVALID_ARG;
    *out = nullptr;
    if (p->size < sizeof(mclsgpu_mc_params))
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "mc params: size mismatch");
    if (p->history_length < 1)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "History Length must be >= 1");
    if (p->direction != MCLSGPU_ADJOINT && p->direction != MCLSGPU_FORWARD)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "bad direction");
    if (p->precision != MCLSGPU_FP64 && p->precision != MCLSGPU_FP32)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "bad precision");
    if (p->rng_mode != MCLSGPU_RNG_REFERENCE && p->rng_mode != MCLSGPU_RNG_COUNTER)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "bad rng mode");
    if (p->rng_mode == MCLSGPU_RNG_REFERENCE && p->weight_cutoff > 0.0 &&
        p->precision != MCLSGPU_FP64)
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED,
                         "a Weight Cutoff on the reference stream needs the FP64 walk");
    if ((left && left->P.n != op->A.n) || (right && right->P.n != op->A.n))
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "preconditioner size mismatch");
    if (left && left->kind == MCLSGPU_PREC_NONE) left = nullptr;
    if (right && right->kind == MCLSGPU_PREC_NONE) right = nullptr;
    cudaSetDevice(ctx->device);
    mclsgpu_domain* dom = new mclsgpu_domain;
    dom->ctx = ctx;
    dom->op = op;
    dom->left = left;
    dom->right = right;
    dom->p = *p;
    dom->n = op->A.n;
    dom->seed = p->seed;
    const int n = dom->n;
    int rc = MCLSGPU_OK;
    cudaError_t e = cudaSuccess;
    // Composite operator (src/MCLS_LinearProblem_impl.hpp:143-221).
    const bool adj = p->direction == MCLSGPU_ADJOINT;
    const double thr = p->composite_threshold;
    DevCsr M;
    const DevCsr* PL = left ? &left->P : nullptr;
    const DevCsr* PR = right ? &right->P : nullptr;
    if (!PL && !PR) {
        rc = adj ? csr_transpose(ctx, op->A, M) : csr_copy(ctx, op->A, M);
    } else if (adj && PL && !PR && left->kind == MCLSGPU_PREC_POINT_JACOBI) {
        // A^T * PL^T with a diagonal PL: column j of A^T scaled by 1/a_jj.
        DevCsr T;
        rc = csr_transpose(ctx, op->A, T);
        if (!rc) {
            csr_scale_cols(ctx, T, left->diag);
            rc = csr_filter(ctx, T, thr, M);
        }
        T.release();
    } else if (adj) {
        DevCsr AT, PLT, PRT, tmp;
        rc = csr_transpose(ctx, op->A, AT);
        if (!rc && PL) rc = csr_transpose(ctx, *PL, PLT);
        if (!rc && PR) rc = csr_transpose(ctx, *PR, PRT);
        if (!rc) {
            if (PL && PR) {
                rc = csr_multiply(ctx, AT, PLT, thr, tmp);
                if (!rc) rc = csr_multiply(ctx, PRT, tmp, thr, M);
            } else if (PR) {
                rc = csr_multiply(ctx, PRT, AT, thr, M);
            } else {
                rc = csr_multiply(ctx, AT, PLT, thr, M);
            }
        }
        AT.release();
        PLT.release();
        PRT.release();
        tmp.release();
    } else {
        DevCsr tmp;
        if (PL && PR) {
            rc = csr_multiply(ctx, op->A, *PR, thr, tmp);
            if (!rc) rc = csr_multiply(ctx, *PL, tmp, thr, M);
        } else if (PL) {
            rc = csr_multiply(ctx, *PL, op->A, thr, M);
        } else {
            rc = csr_multiply(ctx, op->A, *PR, thr, M);
        }
        tmp.release();
    }
    const double relax = p->neumann_relaxation > 0.0 ? p->neumann_relaxation : 1.0;
    if (!rc) rc = build_domain_arrays(ctx, M, relax, dom);
    M.release();
    // Work buffers.
    int64_t nh_req = p->sample_ratio > 0.0 ? int64_t(double(n) * p->sample_ratio) : n;
    if (!adj)
        dom->nh_cap = int64_t(n) * int64_t(p->sample_ratio > 0.0 ? std::ceil(p->sample_ratio) : 1.0);
    else
        dom->nh_cap = nh_req + (p->source_sampling == MCLSGPU_SOURCE_STRATIFIED ? n : 0);
    if (!rc && (dom->nh_cap >= (int64_t(1) << 31) - (int64_t(1) << 24) || nh_req < 0))
        rc = set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "too many histories per solve (%lld)",
                       (long long)dom->nh_cap);
    if (!rc && p->precision == MCLSGPU_FP32 && dom->slots == 0)
        rc = set_error(ctx, MCLSGPU_ERR_UNSUPPORTED,
                       "domain rows longer than 31 entries need the FP64 walk");
    // Partials: one per scan tile (scans) and one per block of the fused
    // residual kernels, whose grid is at most 8 blocks per SM.
    const int fused_blocks = ctx->num_sms * 8;
    const int scan_parts = scan_partials_needed(n);
    const int parts = (scan_parts > fused_blocks ? scan_parts : fused_blocks) + 8;
    if (!rc) {
        if ((e = dmalloc(&dom->src, n)) != cudaSuccess || (e = dmalloc(&dom->scdf, n)) != cudaSuccess ||
            (e = dmalloc(&dom->guide, n)) != cudaSuccess || (e = dmalloc(&dom->counts, n)) != cudaSuccess ||
            (e = dmalloc(&dom->offs, n)) != cudaSuccess ||
            (e = dmalloc(&dom->start, size_t(dom->nh_cap) + 1)) != cudaSuccess ||
            (e = dmalloc(&dom->y64, n)) != cudaSuccess ||
            (e = dmalloc(&dom->c32, n)) != cudaSuccess || (e = dmalloc(&dom->c64, n)) != cudaSuccess ||
            (e = dmalloc(&dom->d_nh, 1)) != cudaSuccess || (e = dmalloc(&dom->d_counter, 1)) != cudaSuccess ||
            (e = dmalloc(&dom->d_scalars, 16)) != cudaSuccess ||
            (e = dmalloc(&dom->d_steps, 1)) != cudaSuccess || (e = dmalloc(&dom->d_hist, 1)) != cudaSuccess ||
            (e = dmalloc(&dom->d_tim, 4)) != cudaSuccess ||
            (e = dmalloc(&dom->d_pos, 1)) != cudaSuccess || (e = dmalloc(&dom->d_epoch, 1)) != cudaSuccess ||
            (e = dmalloc(&dom->part, parts)) != cudaSuccess || (e = dmalloc(&dom->ipart, parts)) != cudaSuccess ||
            (e = dmalloc(&dom->x, n)) != cudaSuccess || (e = dmalloc(&dom->b, n)) != cudaSuccess ||
            (e = dmalloc(&dom->rp, n)) != cudaSuccess || (e = dmalloc(&dom->tmp, n)) != cudaSuccess ||
            (e = dmalloc(&dom->tmp2, n)) != cudaSuccess || (e = dmalloc(&dom->d_state, 1)) != cudaSuccess ||
            (e = dmalloc(&dom->x2, n)) != cudaSuccess || (e = dmalloc(&dom->rp2, n)) != cudaSuccess ||
            (e = dmalloc(&dom->d_ticket, 1)) != cudaSuccess ||
            (e = cudaMallocHost(reinterpret_cast<void**>(&dom->h_state), sizeof(McsaState))) != cudaSuccess)
            rc = cuda_fail(ctx, e, "cudaMalloc domain buffers");
    }
    if (!rc) {
        dom->part_cap = parts;
        cudaMemsetAsync(dom->d_pos, 0, sizeof(unsigned long long), ctx->stream);
        cudaMemsetAsync(dom->d_epoch, 0, sizeof(unsigned long long), ctx->stream);
        cudaMemsetAsync(dom->d_steps, 0, sizeof(unsigned long long), ctx->stream);
        cudaMemsetAsync(dom->d_hist, 0, sizeof(unsigned long long), ctx->stream);
        cudaMemsetAsync(dom->d_ticket, 0, sizeof(unsigned int), ctx->stream);
        cudaMemsetAsync(dom->d_counter, 0, sizeof(int), ctx->stream);
        cudaMemsetAsync(dom->d_scalars, 0, 16 * sizeof(double), ctx->stream);
        const unsigned long long tim0[4] = {~0ULL, 0ULL, 0ULL, 0ULL};
        cudaMemcpyAsync(dom->d_tim, tim0, sizeof(tim0), cudaMemcpyHostToDevice, ctx->stream);
        cudaStreamSynchronize(ctx->stream);
        if (!rc && walk_needs_rounds(dom) &&
            ((e = dmalloc(&dom->hoff, size_t(dom->nh_cap) + 1)) != cudaSuccess ||
             (e = dmalloc(&dom->hlen, size_t(dom->nh_cap) + 1)) != cudaSuccess ||
             (e = dmalloc(&dom->hoff2, size_t(dom->nh_cap) + 2)) != cudaSuccess ||
             (e = dmalloc(&dom->y_save, n)) != cudaSuccess))
            rc = cuda_fail(ctx, e, "cudaMalloc history offsets");
        if (p->rng_mode == MCLSGPU_RNG_REFERENCE) {
            std::vector<uint64_t> tab(64 * 64);
            xs_jump_tables(tab.data());
            if ((e = dmalloc(&dom->d_jump, tab.size())) != cudaSuccess)
                rc = cuda_fail(ctx, e, "cudaMalloc");
            else
                cudaMemcpyAsync(dom->d_jump, tab.data(), tab.size() * sizeof(uint64_t),
                                cudaMemcpyHostToDevice, ctx->stream);
        }
    }
    if (!rc) {
        prepare_walk(dom);
        prepare_source(dom);
        e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "domain build");
    }
    if (rc) {
        release_domain(dom);
        delete dom;
        return rc;
    }
    *out = dom;
    return MCLSGPU_OK;
}

int mclsgpu_domain_destroy(mclsgpu_domain* dom) {
    if (!dom) return MCLSGPU_OK;
    cudaStreamSynchronize(dom->ctx->stream);
    release_domain(dom);
    delete dom;
    return MCLSGPU_OK;
}

int mclsgpu_domain_export(mclsgpu_domain* dom, int64_t* nnz_out, int64_t* rowptr, int64_t* col,
                          double* h, double* cdf, double* weights) {
    if (!dom) return MCLSGPU_ERR_INVALID_ARG;
    int rc = copy_csr_out(dom->ctx, dom->D, nnz_out, rowptr, col, h);
    if (rc) return rc;
    cudaStream_t s = dom->ctx->stream;
    if (cdf) cudaMemcpyAsync(cdf, dom->cdf, size_t(dom->D.nnz) * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (weights) cudaMemcpyAsync(weights, dom->w, size_t(dom->n) * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(dom->ctx, e, "domain export");
}

int mclsgpu_domain_query(mclsgpu_domain* dom, mclsgpu_domain_info* info) {
    if (!dom || !info || info->size < sizeof(mclsgpu_domain_info)) return MCLSGPU_ERR_INVALID_ARG;
    info->record_format = !dom->stencil_k ? MCLSGPU_RECORD_PACKED
                          : dom->rec_q16  ? MCLSGPU_RECORD_STENCIL16
                                          : MCLSGPU_RECORD_STENCIL;
    info->rows = dom->n;
    info->entries = dom->D.nnz;
    info->record_bytes = dom->p.precision == MCLSGPU_FP32 ? dom->slots * 8 : 0;
    info->max_row_entries = dom->max_row;
    info->stencil_offsets = dom->stencil_k;
    info->operator_dia = dom->op->dia_k;
    info->histories_per_lane = dom->walk_ilp;
    info->block_size = dom->walk_block;
    info->record_cache_l1 = dom->walk_l1;
    info->reserved0 = 0;
    return MCLSGPU_OK;
}

int mclsgpu_domain_walk_agreement(mclsgpu_domain* dom, int64_t histories, uint64_t seed,
                                  int64_t* histories_differing, int64_t* transitions_differing) {
    if (!dom || !histories_differing || !transitions_differing) return MCLSGPU_ERR_INVALID_ARG;
    long long h = 0, t = 0;
    int rc = walk_agreement(dom, histories, seed, &h, &t);
    if (rc) return rc;
    *histories_differing = h;
    *transitions_differing = t;
    return MCLSGPU_OK;
}

int mclsgpu_domain_reseed(mclsgpu_domain* dom, uint64_t seed) {
    if (!dom) return MCLSGPU_ERR_INVALID_ARG;
    dom->seed = seed;
    cudaMemsetAsync(dom->d_pos, 0, sizeof(unsigned long long), dom->ctx->stream);
    cudaMemsetAsync(dom->d_epoch, 0, sizeof(unsigned long long), dom->ctx->stream);
    // The seed is baked into the walk launches of every captured loop.
    if (dom->graph) {
        cudaGraphExecDestroy(dom->graph);
        dom->graph = nullptr;
    }
    if (dom->set_graph) {
        cudaGraphExecDestroy(dom->set_graph);
        dom->set_graph = nullptr;
    }
    anderson_drop_graph(dom);
    cudaError_t e = cudaStreamSynchronize(dom->ctx->stream);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(dom->ctx, e, "reseed");
}

int mclsgpu_domain_convergence_criteria(mclsgpu_domain* dom, int max_iters, double tol,
                                        uint64_t seed, mclsgpu_criteria* out) {
    if (!dom || !out || out->size < sizeof(mclsgpu_criteria)) return MCLSGPU_ERR_INVALID_ARG;
    double rho[3];
    for (int which = 0; which < 3; ++which) {
        int rc = mclsgpu_domain_spectral_radius(dom, which, max_iters, tol, seed, &rho[which]);
        if (rc) return rc;
    }
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    const int n = dom->n;
    std::vector<double> w(n), rmax(n);
    std::vector<unsigned long long> cmax(n);
    unsigned long long* d_cmax = nullptr;
    cudaError_t e = dmalloc(&d_cmax, size_t(n));
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    cudaMemsetAsync(d_cmax, 0, size_t(n) * sizeof(unsigned long long), s);
    k_row_col_max<<<grid_for(n), 256, 0, s>>>(dom->D.rp, dom->D.v, dom->D.ci, n, dom->tmp, d_cmax);
    cudaMemcpyAsync(w.data(), dom->w, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(rmax.data(), dom->tmp, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(cmax.data(), d_cmax, size_t(n) * sizeof(unsigned long long),
                    cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    dfree(d_cmax);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "convergence criteria");
    out->rho_h = rho[0];
    out->rho_abs = rho[1];
    out->rho_star = rho[2];
    out->row_sum_max = 0.0;
    out->row_sum_min = std::numeric_limits<double>::max();
    double bmin = std::numeric_limits<double>::max(), bmax = 0.0, bsum = 0.0;
    long long rows = 0;
    for (int i = 0; i < n; ++i) {
        out->row_sum_max = std::max(out->row_sum_max, w[i]);
        out->row_sum_min = std::min(out->row_sum_min, w[i]);
        double c;
        std::memcpy(&c, &cmax[i], sizeof(c));
        if (c > 0.0) {  // a state no row transitions into has no column norm
            const double r = rmax[i] / c;
            bmin = std::min(bmin, r);
            bmax = std::max(bmax, r);
            bsum += r;
            ++rows;
        }
    }
    out->balance_min = rows ? bmin : 0.0;
    out->balance_max = bmax;
    out->balance_ave = rows ? bsum / double(rows) : 0.0;
    return MCLSGPU_OK;
}

int mclsgpu_domain_spectral_radius(mclsgpu_domain* dom, int which, int max_iters, double tol,
                                   uint64_t seed, double* rho) {
    if (!dom || !rho || which < 0 || which > 2 || max_iters < 2) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    const int n = dom->n;
    double* v = dom->tmp;
    double* w = dom->tmp2;
    double* sq = dom->d_scalars + 8;
    k_fill_random<<<grid_for(n), 256, 0, s>>>(v, n, seed);
    sum_sq(s, v, n, dom->part, sq);
    k_scale<<<grid_for(n), 256, 0, s>>>(v, n, sq);
    // Two-step power iteration: rho ~ sqrt(|M^2 v| / |v|) is robust to the
    // +-lambda pairs of bipartite iteration matrices.
    double prev = -1.0, est = 0.0;
    for (int it = 0; it < max_iters; it += 2) {
        k_domain_spmv<<<grid_for(n), 256, 0, s>>>(dom->D.rp, dom->D.ci, dom->D.v, dom->w, n, which,
                                                  v, w);
        k_domain_spmv<<<grid_for(n), 256, 0, s>>>(dom->D.rp, dom->D.ci, dom->D.v, dom->w, n, which,
                                                  w, v);
        sum_sq(s, v, n, dom->part, sq);
        double h = 0.0;
        cudaMemcpyAsync(&h, sq, sizeof(double), cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "power iteration");
        est = std::sqrt(std::sqrt(h));
        if (!(h > 0.0) || !std::isfinite(h)) {
            est = h > 0.0 ? est : 0.0;
            break;
        }
        k_scale<<<grid_for(n), 256, 0, s>>>(v, n, sq);
        if (prev > 0.0 && std::fabs(est - prev) <= tol * est) break;
        prev = est;
    }
    *rho = est;
    return MCLSGPU_OK;
}

}  // extern "C"
