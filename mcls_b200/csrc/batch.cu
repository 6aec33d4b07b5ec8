// batch.cu -- many systems and many right-hand sides in one MCSA loop.
//
// m systems A_s (uneven sizes) with R_s right-hand sides each are solved
// together: the block-diagonal operator S = diag(A_1..A_m) carries one
// point-Jacobi domain H = I - D^-1 S (walks never leave a block), and the
// right-hand sides are the columns of an [rows][R] row-major matrix, R the
// largest R_s rounded up to a power of two (columns r >= R_s of system s are
// zero and ignored).  Forward walks do not depend on the source, so one set
// of histories per iteration serves every right-hand side of every system:
// each history carries R tallies (walk32_multi).  Every (system, rhs) pair has
// its own convergence test |rp_{s,r}|_2 <= tol |D^-1 b_{s,r}|_2 (the
// MCSASolverManager criterion, src/MCLS_MCSASolverManager_impl.hpp:299-318);
// the loop ends when every pair has met it or at the iteration limit.  One
// iteration is six kernels (Richardson + residual, tally source, the shared
// walk, correction, residual + per-pair norms, convergence test) captured in a
// CUDA graph whose WHILE node the last kernel controls.
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"

namespace mclsgpu {

int launch_walk_multi(mclsgpu_domain* dom, int R, const float* cR, double* Y, const int* rsys,
                      const int* sys_done);

namespace {

struct BatchState {
    int iter;
    int done;
    int max_iters;
    int check_freq;
    double tol;
    int converged;  // pairs converged
    int pairs;      // pairs in the batch
};

constexpr int kThreads = 256;

inline int grid_for(long long work, int threads = kThreads, int cap = 148 * 8) {
    long long g = (work + threads - 1) / threads;
    if (g < 1) g = 1;
    return int(g > cap ? cap : g);
}

struct BatchArgs {
    int n;
    int nsys;
    const int* rp;      // S (CSR)
    const int* ci;
    const double* v;
    const double* dinv;  // D^-1
    const int* rsys;     // row -> system
    const int* hrp;      // H rows (forward domain, FP64)
    const int* hci;
    const double* hv;
    const double* B;
    double* X;
    double* X2;
    double* RP;
    double* RP2;
    double* Y;
    float* cR;
    double* norm2;       // [nsys][R]
    double* bnorm2;
    int* conv_iter;      // [nsys][R]
    const int* nrhs;
    int* sys_done;       // per system: every right-hand side converged
    int skip;            // skip the rows of finished systems
    BatchState* st;
    double omega;        // Richardson relaxation
    double nomega;       // Neumann relaxation (1 when absent)
    double inv_per;      // 1 / histories per state
    int ev;              // expected-value estimator
    unsigned long long* d_epoch;
    int* d_counter;
    unsigned long long* d_tim;
    int* status;
};

// All per-row kernels below run one thread per (row, column) element: with
// the [rows][R] row-major layout a warp then reads whole 8R-byte rows of X,
// RP and B at every matrix entry, so every load and store is coalesced.
template <int R>
__device__ __forceinline__ void elem_rc(long long t, int& i, int& r) {
    i = int(t / R);
    r = int(t % R);
}

// x2 = x + w rp;  rp2 = D^-1 (b - S x2), with x2 at the neighbours formed on
// the fly (RichardsonIteration::doOneIteration then updatePrecResidual,
// src/MCLS_RichardsonIteration_impl.hpp:134-147).
template <int R>
__global__ void __launch_bounds__(kThreads) k_b_richardson_residual(BatchArgs a) {
    const long long total = (long long)a.n * R;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int i, r;
        elem_rc<R>(t, i, r);
        if (a.skip && a.sys_done[a.rsys[i]]) continue;
        double acc = 0.0;
        for (int p = a.rp[i]; p < a.rp[i + 1]; ++p) {
            const size_t k = size_t(a.ci[p]) * R + r;
            acc = fma(a.v[p], __dadd_rn(a.X[k], __dmul_rn(a.omega, a.RP[k])), acc);
        }
        a.X2[t] = __dadd_rn(a.X[t], __dmul_rn(a.omega, a.RP[t]));
        a.RP2[t] = a.dinv[i] * (a.B[t] - acc);
    }
}

// Tally source of every right-hand side: expected value c = H (w rp2),
// collision c = w rp2 (FP32).
template <int R>
__global__ void __launch_bounds__(kThreads) k_b_source(BatchArgs a) {
    const long long total = (long long)a.n * R;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int i, r;
        elem_rc<R>(t, i, r);
        if (a.skip && a.sys_done[a.rsys[i]]) continue;  // walks skip these rows too
        double v;
        if (a.ev) {
            v = 0.0;
            for (int p = a.hrp[i]; p < a.hrp[i + 1]; ++p)
                v = fma(a.hv[p], a.RP2[size_t(a.hci[p]) * R + r], v);
        } else {
            v = a.RP2[t];
        }
        a.cR[t] = __double2float_rn(a.nomega * v);
    }
}

// x = x2 + delta: delta = Y / per (+ w rp2 for the expected value, the
// estimator's source term); Y cleared for the next iteration
// (ForwardTally::finalize, src/MCLS_ForwardTally_impl.hpp:180-209).
template <int R>
__global__ void __launch_bounds__(kThreads) k_b_correction(BatchArgs a) {
    const long long total = (long long)a.n * R;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        if (a.skip && a.sys_done[a.rsys[int(t / R)]]) continue;
        double d = a.Y[t] * a.inv_per;
        if (a.ev) d += a.nomega * a.RP2[t];
        a.X[t] = a.X2[t] + d;
        a.Y[t] = 0.0;
    }
}

// rp = D^-1 (b - S x) and the per-(system, rhs) sums of squares.  A warp
// covers 32/R rows: when they all belong to one system the lanes of each
// column reduce with shuffles and one lane per column adds the sum,
// otherwise every lane adds its own square.
template <int R>
__global__ void __launch_bounds__(kThreads) k_b_residual_norm(BatchArgs a, const double* Xin) {
    const unsigned full = 0xffffffffu;
    const long long total = (long long)a.n * R;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < total;
         base += (long long)gridDim.x * blockDim.x) {
        const long long t = base + threadIdx.x;
        const bool live = t < total;
        double sq = 0.0;
        int sys = -1, r = 0;
        if (live) {
            int i;
            elem_rc<R>(t, i, r);
            sys = a.rsys[i];
            if (!(a.skip && a.sys_done[sys])) {
                double acc = 0.0;
                for (int p = a.rp[i]; p < a.rp[i + 1]; ++p)
                    acc = fma(a.v[p], Xin[size_t(a.ci[p]) * R + r], acc);
                const double rv = a.dinv[i] * (a.B[t] - acc);
                a.RP[t] = rv;
                sq = rv * rv;
            }
        }
        const int s0 = __shfl_sync(full, sys, 0);
        const bool uniform = __all_sync(full, sys == s0) && s0 >= 0;
        if (uniform) {
            double v = sq;
#pragma unroll
            for (int d = 16; d >= R; d >>= 1) v += __shfl_xor_sync(full, v, d);
            if ((threadIdx.x & 31) < R && v != 0.0) atomicAdd(&a.norm2[size_t(s0) * R + r], v);
        } else if (live && sq != 0.0) {
            atomicAdd(&a.norm2[size_t(sys) * R + r], sq);
        }
    }
}

// Per-pair convergence, loop control and the per-iteration bookkeeping (new
// stream epoch, work-queue reset, walk timing, norms cleared).
__global__ void k_b_check(BatchArgs a, int R, int use_cond, cudaGraphConditionalHandle handle) {
    __shared__ int s_conv;
    if (threadIdx.x == 0) s_conv = 0;
    __syncthreads();
    BatchState st = *a.st;
    const int it = st.iter + 1;
    const bool check = (it % st.check_freq) == 0 || it >= st.max_iters;
    int conv = 0;
    for (int q = threadIdx.x; q < a.nsys * R; q += blockDim.x) {
        const int s = q / R, r = q % R;
        if (r >= a.nrhs[s]) continue;
        const double nr = a.norm2[q];
        if (!isfinite(nr)) atomicOr(a.status, DEV_ERR_NONFINITE);
        if (a.conv_iter[q] < 0 && check && sqrt(nr) <= st.tol * sqrt(a.bnorm2[q]))
            a.conv_iter[q] = it;
        if (a.conv_iter[q] >= 0) ++conv;
        a.norm2[q] = 0.0;
    }
    atomicAdd(&s_conv, conv);
    __syncthreads();
    // Systems whose every right-hand side has converged stop iterating.
    for (int s = threadIdx.x; s < a.nsys; s += blockDim.x) {
        int all = 1;
        for (int r = 0; r < a.nrhs[s]; ++r) all &= a.conv_iter[size_t(s) * R + r] >= 0;
        a.sys_done[s] = all;
    }
    if (threadIdx.x == 0) {
        st.iter = it;
        st.converged = s_conv;
        const int keep = (s_conv < st.pairs) && (it < st.max_iters) && (*a.status == 0);
        st.done = !keep;
        *a.st = st;
        *a.d_epoch += 1;
        *a.d_counter = 0;
        unsigned long long* t = a.d_tim;
        if (t[1] > t[0]) t[2] += t[1] - t[0];
        t[3] += 1;
        t[0] = ~0ULL;
        t[1] = 0;
        if (use_cond) cudaGraphSetConditional(handle, keep ? 1u : 0u);
    }
}

// Before the loop: sums of squares of D^-1 b per pair.
template <int R>
__global__ void k_b_init_norms(BatchArgs a) {
    const long long total = (long long)a.n * R;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int i, r;
        elem_rc<R>(t, i, r);
        const double v = a.dinv[i] * a.B[t];
        if (v != 0.0) atomicAdd(&a.bnorm2[size_t(a.rsys[i]) * R + r], v * v);
    }
}

__global__ void k_b_state_init(BatchState* st, int max_iters, int check_freq, double tol, int pairs,
                               int* conv_iter, int count, double* norm2, int* sys_done,
                               int nsys) {
    for (int q = threadIdx.x; q < count; q += blockDim.x) {
        conv_iter[q] = -1;
        norm2[q] = 0.0;
    }
    for (int q = threadIdx.x; q < nsys; q += blockDim.x) sys_done[q] = 0;
    if (threadIdx.x == 0) {
        BatchState s{};
        s.max_iters = max_iters;
        s.check_freq = check_freq;
        s.tol = tol;
        s.pairs = pairs;
        *st = s;
    }
}

__global__ void k_b_forward_nh(int* d_nh, int nh) { *d_nh = nh; }

}  // namespace
}  // namespace mclsgpu

struct mclsgpu_batch {
    mclsgpu_context* ctx = nullptr;
    int nsys = 0;
    int R = 1;
    int n = 0;
    std::vector<int64_t> off;
    std::vector<int> nrhs;
    mclsgpu_operator* op = nullptr;
    mclsgpu_precond* pc = nullptr;
    mclsgpu_domain* dom = nullptr;
    int* d_rsys = nullptr;
    int* d_nrhs = nullptr;
    double *X = nullptr, *X2 = nullptr, *RP = nullptr, *RP2 = nullptr, *B = nullptr, *Y = nullptr;
    float* cR = nullptr;
    double* norm2 = nullptr;
    double* bnorm2 = nullptr;
    int* conv_iter = nullptr;
    int* sys_done = nullptr;
    mclsgpu::BatchState* d_state = nullptr;
    mclsgpu::BatchState* h_state = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_key = -1;
    int body_kernels = 0;
    int per = 1;
};

namespace mclsgpu {
namespace {

void batch_release(mclsgpu_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->dom) mclsgpu_domain_destroy(b->dom);
    if (b->pc) mclsgpu_precond_destroy(b->pc);
    if (b->op) mclsgpu_operator_destroy(b->op);
    dfree(b->d_rsys);
    dfree(b->d_nrhs);
    dfree(b->X);
    dfree(b->X2);
    dfree(b->RP);
    dfree(b->RP2);
    dfree(b->B);
    dfree(b->Y);
    dfree(b->cR);
    dfree(b->norm2);
    dfree(b->bnorm2);
    dfree(b->conv_iter);
    dfree(b->sys_done);
    dfree(b->d_state);
    if (b->h_state) cudaFreeHost(b->h_state);
    delete b;
}

BatchArgs batch_args(mclsgpu_batch* b, const mclsgpu_mcsa_params* mp) {
    const mclsgpu_mc_params& p = b->dom->p;
    BatchArgs a{};
    a.n = b->n;
    a.nsys = b->nsys;
    a.rp = b->op->A.rp;
    a.ci = b->op->A.ci;
    a.v = b->op->A.v;
    a.dinv = b->pc->diag;
    a.rsys = b->d_rsys;
    a.hrp = b->dom->D.rp;
    a.hci = b->dom->D.ci;
    a.hv = b->dom->D.v;
    a.B = b->B;
    a.X = b->X;
    a.X2 = b->X2;
    a.RP = b->RP;
    a.RP2 = b->RP2;
    a.Y = b->Y;
    a.cR = b->cR;
    a.norm2 = b->norm2;
    a.bnorm2 = b->bnorm2;
    a.conv_iter = b->conv_iter;
    a.nrhs = b->d_nrhs;
    a.sys_done = b->sys_done;
    a.skip = 1;
    a.st = b->d_state;
    a.omega = mp ? mp->richardson_omega : 1.0;
    a.nomega = p.neumann_relaxation > 0.0 ? p.neumann_relaxation : 1.0;
    a.inv_per = 1.0 / double(b->per);
    a.ev = p.estimator == MCLSGPU_EXPECTED_VALUE;
    a.d_epoch = b->dom->d_epoch;
    a.d_counter = b->dom->d_counter;
    a.d_tim = b->dom->d_tim;
    a.status = b->ctx->d_status;
    return a;
}

#define MCLSGPU_BATCH_R(R, CALL) \
    switch (R) {                 \
        case 1: CALL(1); break;  \
        case 2: CALL(2); break;  \
        case 4: CALL(4); break;  \
        case 8: CALL(8); break;  \
        default: CALL(16); break; \
    }

// One batched MCSA iteration (6 kernels).
int enqueue_batch_iteration(mclsgpu_batch* b, const mclsgpu_mcsa_params* mp, int use_cond,
                            cudaGraphConditionalHandle handle) {
    cudaStream_t s = b->ctx->stream;
    BatchArgs a = batch_args(b, mp);
    const int grid = grid_for((long long)b->n * b->R);
#define K1(R) k_b_richardson_residual<R><<<grid, kThreads, 0, s>>>(a)
    MCLSGPU_BATCH_R(b->R, K1)
#undef K1
#define K2(R) k_b_source<R><<<grid, kThreads, 0, s>>>(a)
    MCLSGPU_BATCH_R(b->R, K2)
#undef K2
    int rc = launch_walk_multi(b->dom, b->R, b->cR, b->Y, b->d_rsys, b->sys_done);
    if (rc) return rc;
#define K3(R) k_b_correction<R><<<grid, kThreads, 0, s>>>(a)
    MCLSGPU_BATCH_R(b->R, K3)
#undef K3
#define K4(R) k_b_residual_norm<R><<<grid, kThreads, 0, s>>>(a, b->X)
    MCLSGPU_BATCH_R(b->R, K4)
#undef K4
    k_b_check<<<1, 1024, 0, s>>>(a, b->R, use_cond, handle);
    return MCLSGPU_OK;
}

int build_batch_graph(mclsgpu_batch* b, const mclsgpu_mcsa_params* mp) {
    mclsgpu_context* ctx = b->ctx;
    cudaStream_t s = ctx->stream;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t g;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphCreate");
    cudaGraphConditionalHandle handle;
    e = cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(ctx, e, "cudaGraphConditionalHandleCreate");
    }
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(ctx, e, "cudaGraphAddNode(conditional)");
    }
    cudaGraph_t body = np.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(ctx, e, "cudaStreamBeginCaptureToGraph");
    }
    int rc = enqueue_batch_iteration(b, mp, 1, handle);
    cudaGraph_t captured = body;
    e = cudaStreamEndCapture(s, &captured);
    if (rc || e != cudaSuccess) {
        cudaGraphDestroy(g);
        return rc ? rc : cuda_fail(ctx, e, "cudaStreamEndCapture");
    }
    size_t nn = 0;
    cudaGraphGetNodes(body, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn) cudaGraphGetNodes(body, nodes.data(), &nn);
    b->body_kernels = 0;
    for (size_t k = 0; k < nn; ++k) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[k], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
            ++b->body_kernels;
    }
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        b->graph = nullptr;
        return cuda_fail(ctx, e, "cudaGraphInstantiate");
    }
    return MCLSGPU_OK;
}

}  // namespace
}  // namespace mclsgpu

using namespace mclsgpu;

extern "C" {

int mclsgpu_batch_build(mclsgpu_context* ctx, int nsys, const int64_t* n,
                        const int64_t* const* rowptr, const int64_t* const* colind,
                        const double* const* values, const int32_t* nrhs,
                        const mclsgpu_mc_params* params, mclsgpu_batch** out) {
    if (!ctx || nsys < 1 || !n || !rowptr || !colind || !values || !nrhs || !params || !out)
        return MCLSGPU_ERR_INVALID_ARG;
    *out = nullptr;
    if (params->size < sizeof(mclsgpu_mc_params))
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "mc params: size mismatch");
    if (params->direction != MCLSGPU_FORWARD || params->precision != MCLSGPU_FP32 ||
        params->weight_cutoff > 0.0)
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED,
                         "batched MCSA runs forward FP32 walks of fixed length");
    // Concatenate the systems into the block-diagonal operator.
    std::vector<int64_t> off(nsys + 1, 0);
    int maxr = 1;
    for (int s = 0; s < nsys; ++s) {
        if (n[s] < 1 || !rowptr[s] || !colind[s] || !values[s] || nrhs[s] < 1 || nrhs[s] > 16)
            return set_error(ctx, MCLSGPU_ERR_INVALID_ARG,
                             "batch system %d: empty, missing arrays or 1..16 right-hand sides", s);
        off[s + 1] = off[s] + n[s];
        if (nrhs[s] > maxr) maxr = nrhs[s];
    }
    const int64_t N = off[nsys];
    if (N >= (int64_t(1) << 30))
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "batch too large (%lld rows)", (long long)N);
    int64_t nnz = 0;
    for (int s = 0; s < nsys; ++s) nnz += rowptr[s][n[s]] - rowptr[s][0];
    if (nnz >= (int64_t(1) << 31) - 1)
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "batch too large (%lld entries)", (long long)nnz);
    std::vector<int64_t> rp(N + 1), ci(nnz);
    std::vector<double> v(nnz);
    std::vector<int> rsys(N);
    int64_t pos = 0;
    for (int s = 0; s < nsys; ++s) {
        for (int64_t i = 0; i < n[s]; ++i) {
            rp[off[s] + i] = pos;
            rsys[off[s] + i] = s;
            for (int64_t p = rowptr[s][i]; p < rowptr[s][i + 1]; ++p, ++pos) {
                if (colind[s][p] < 0 || colind[s][p] >= n[s])
                    return set_error(ctx, MCLSGPU_ERR_INVALID_ARG,
                                     "batch system %d: column index out of range", s);
                ci[pos] = colind[s][p] + off[s];
                v[pos] = values[s][p];
            }
        }
    }
    rp[N] = pos;
    int R = 1;
    while (R < maxr) R <<= 1;
    mclsgpu_batch* b = new mclsgpu_batch;
    b->ctx = ctx;
    b->nsys = nsys;
    b->R = R;
    b->n = int(N);
    b->off = off;
    b->nrhs.assign(nrhs, nrhs + nsys);
    b->per = params->sample_ratio > 0.0 ? int(std::ceil(params->sample_ratio)) : 1;
    int rc = mclsgpu_operator_upload(ctx, N, rp.data(), ci.data(), v.data(), &b->op);
    mclsgpu_precond_params pp{};
    pp.size = sizeof(pp);
    pp.kind = MCLSGPU_PREC_POINT_JACOBI;
    if (!rc) rc = mclsgpu_precond_build(ctx, b->op, &pp, &b->pc);
    if (!rc) rc = mclsgpu_domain_build(ctx, b->op, b->pc, nullptr, params, &b->dom);
    if (!rc && b->dom->stencil_k && b->dom->slots > 8) {
        // The shared walk takes stencil records of at most 64 bytes.
        mclsgpu_domain_destroy(b->dom);
        b->dom = nullptr;
        mclsgpu_mc_params pk = *params;
        pk.record_format = MCLSGPU_RECORD_PACKED;
        rc = mclsgpu_domain_build(ctx, b->op, b->pc, nullptr, &pk, &b->dom);
    }
    if (!rc && b->dom->slots > 16)
        rc = set_error(ctx, MCLSGPU_ERR_UNSUPPORTED,
                       "batched walks: rows of at most 15 retained entries");
    const size_t NR = size_t(N) * R, PR = size_t(nsys) * R;
    cudaError_t e = cudaSuccess;
    if (!rc &&
        ((e = dmalloc(&b->d_rsys, N)) != cudaSuccess || (e = dmalloc(&b->d_nrhs, nsys)) != cudaSuccess ||
         (e = dmalloc(&b->X, NR)) != cudaSuccess || (e = dmalloc(&b->X2, NR)) != cudaSuccess ||
         (e = dmalloc(&b->RP, NR)) != cudaSuccess || (e = dmalloc(&b->RP2, NR)) != cudaSuccess ||
         (e = dmalloc(&b->B, NR)) != cudaSuccess || (e = dmalloc(&b->Y, NR)) != cudaSuccess ||
         (e = dmalloc(&b->cR, NR)) != cudaSuccess || (e = dmalloc(&b->norm2, PR)) != cudaSuccess ||
         (e = dmalloc(&b->bnorm2, PR)) != cudaSuccess ||
         (e = dmalloc(&b->conv_iter, PR)) != cudaSuccess || (e = dmalloc(&b->sys_done, nsys)) != cudaSuccess ||
         (e = dmalloc(&b->d_state, 1)) != cudaSuccess ||
         (e = cudaMallocHost(reinterpret_cast<void**>(&b->h_state), sizeof(BatchState))) != cudaSuccess))
        rc = cuda_fail(ctx, e, "cudaMalloc batch");
    if (!rc) {
        cudaStream_t s = ctx->stream;
        cudaMemcpyAsync(b->d_rsys, rsys.data(), sizeof(int) * N, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(b->d_nrhs, b->nrhs.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, s);
        cudaMemsetAsync(b->Y, 0, sizeof(double) * NR, s);
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "batch build");
    }
    if (rc) {
        batch_release(b);
        return rc;
    }
    *out = b;
    return MCLSGPU_OK;
}

int mclsgpu_batch_destroy(mclsgpu_batch* b) {
    if (!b) return MCLSGPU_OK;
    batch_release(b);
    return MCLSGPU_OK;
}

int mclsgpu_batch_layout(mclsgpu_batch* b, int64_t* row_offsets, int32_t* width) {
    if (!b) return MCLSGPU_ERR_INVALID_ARG;
    if (row_offsets)
        for (int s = 0; s <= b->nsys; ++s) row_offsets[s] = b->off[s];
    if (width) *width = b->R;
    return MCLSGPU_OK;
}

int mclsgpu_batch_domain(mclsgpu_batch* b, mclsgpu_domain** dom) {
    if (!b || !dom) return MCLSGPU_ERR_INVALID_ARG;
    *dom = b->dom;
    return MCLSGPU_OK;
}

int mclsgpu_batch_set_launch(mclsgpu_batch* b, int block_size) {
    if (!b || (block_size != 128 && block_size != 256)) return MCLSGPU_ERR_INVALID_ARG;
    b->dom->walk_block = block_size;
    b->graph_key = -1;  // the captured loop bakes the launch shape in
    return MCLSGPU_OK;
}

int mclsgpu_batch_autotune(mclsgpu_batch* b, const double* b_dev, double* x_dev, int reps,
                           int* block_size, double* walk_ms) {
    if (!b || !b_dev || !x_dev || reps < 1) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_mcsa_params p{};
    p.size = sizeof(p);
    p.max_iters = reps;
    p.tolerance = 0.0;
    p.check_freq = 1;
    p.smoother_steps = 1;
    p.richardson_omega = 1.0;
    p.host_loop = 1;
    const int shapes[2] = {256, 128};
    int best = 256;
    double best_ms = 1e300;
    for (int blk : shapes) {
        b->dom->walk_block = blk;
        cudaMemsetAsync(x_dev, 0, sizeof(double) * size_t(b->n) * b->R, b->ctx->stream);
        mclsgpu_stats st{};
        st.size = sizeof(st);
        int rc = mclsgpu_batch_mcsa_solve_dev(b, b_dev, x_dev, &p, nullptr, nullptr, &st);
        if (rc) return rc;
        const double per = st.walk_launches ? st.walk_ms / double(st.walk_launches) : 1e300;
        if (per < best_ms) {
            best_ms = per;
            best = blk;
        }
    }
    b->dom->walk_block = best;
    b->graph_key = -1;
    if (block_size) *block_size = best;
    if (walk_ms) *walk_ms = best_ms;
    return MCLSGPU_OK;
}

int mclsgpu_batch_mcsa_solve_dev(mclsgpu_batch* b, const double* b_dev, double* x_dev,
                                 const mclsgpu_mcsa_params* params, int32_t* conv_iters,
                                 double* rel_resid, mclsgpu_stats* stats) {
    if (!b || !b_dev || !x_dev || !params) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = b->ctx;
    if (params->size < sizeof(mclsgpu_mcsa_params) || params->max_iters < 1 ||
        params->check_freq < 1 || !(params->tolerance >= 0.0) || params->smoother_steps != 1)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG,
                         "batch mcsa params out of range (one smoother step)");
    cudaStream_t s = ctx->stream;
    const size_t NR = size_t(b->n) * b->R, PR = size_t(b->nsys) * b->R;
    int pairs = 0;
    for (int q = 0; q < b->nsys; ++q) pairs += b->nrhs[q];
    const int key = int(params->richardson_omega * 1e6);
    if (!params->host_loop && (!b->graph || b->graph_key != key)) {
        int rc = build_batch_graph(b, params);
        if (rc) return rc;
        b->graph_key = key;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s);
    cudaMemsetAsync(b->dom->d_counter, 0, sizeof(int), s);
    cudaMemsetAsync(b->dom->d_steps, 0, sizeof(unsigned long long), s);
    {
        unsigned long long tim0[4] = {~0ULL, 0ULL, 0ULL, 0ULL};
        cudaMemcpyAsync(b->dom->d_tim, tim0, sizeof(tim0), cudaMemcpyHostToDevice, s);
    }
    cudaEventRecord(e0, s);
    cudaMemcpyAsync(b->B, b_dev, sizeof(double) * NR, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(b->X, x_dev, sizeof(double) * NR, cudaMemcpyDeviceToDevice, s);
    cudaMemsetAsync(b->bnorm2, 0, sizeof(double) * PR, s);
    k_b_forward_nh<<<1, 1, 0, s>>>(b->dom->d_nh, b->n * b->per);
    k_b_state_init<<<1, 1024, 0, s>>>(b->d_state, params->max_iters, params->check_freq,
                                       params->tolerance, pairs, b->conv_iter, int(PR), b->norm2,
                                       b->sys_done, b->nsys);
    BatchArgs a = batch_args(b, params);
    const int grid = grid_for((long long)b->n * b->R);
#define KI(R)                                                 \
    k_b_init_norms<R><<<grid, kThreads, 0, s>>>(a);           \
    k_b_residual_norm<R><<<grid, kThreads, 0, s>>>(a, b->X)
    MCLSGPU_BATCH_R(b->R, KI)
#undef KI
    cudaMemsetAsync(b->norm2, 0, sizeof(double) * PR, s);
    cudaError_t e = cudaSuccess;
    int rc = MCLSGPU_OK;
    if (!params->host_loop) {
        e = cudaGraphLaunch(b->graph, s);
    } else {
        for (int it = 0; it < params->max_iters && e == cudaSuccess && !rc; ++it) {
            rc = enqueue_batch_iteration(b, params, 0, cudaGraphConditionalHandle(0));
            cudaMemcpyAsync(b->h_state, b->d_state, sizeof(BatchState), cudaMemcpyDeviceToHost, s);
            e = cudaStreamSynchronize(s);
            if (e == cudaSuccess && b->h_state->done) break;
        }
    }
    cudaEventRecord(e1, s);
    if (e == cudaSuccess) {
        cudaMemcpyAsync(x_dev, b->X, sizeof(double) * NR, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(b->h_state, b->d_state, sizeof(BatchState), cudaMemcpyDeviceToHost, s);
        e = cudaStreamSynchronize(s);
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch mcsa");
    if ((rc = check_device_status(ctx))) return rc;
    const BatchState st = *b->h_state;
    if (conv_iters || rel_resid) {
        // Final per-pair residuals: one more residual pass on the result.
        std::vector<double> nr(PR), bn(PR);
        std::vector<int> ci(PR);
        cudaMemsetAsync(b->norm2, 0, sizeof(double) * PR, s);
        a.skip = 0;  // every system's final residual
#define KF(R) k_b_residual_norm<R><<<grid, kThreads, 0, s>>>(a, b->X)
        MCLSGPU_BATCH_R(b->R, KF)
#undef KF
        cudaMemcpyAsync(nr.data(), b->norm2, sizeof(double) * PR, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(bn.data(), b->bnorm2, sizeof(double) * PR, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(ci.data(), b->conv_iter, sizeof(int) * PR, cudaMemcpyDeviceToHost, s);
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "batch residuals");
        for (size_t q = 0; q < PR; ++q) {
            const bool valid = int(q % b->R) < b->nrhs[q / b->R];
            if (conv_iters) conv_iters[q] = valid ? ci[q] : -1;
            if (rel_resid)
                rel_resid[q] = valid ? (bn[q] > 0.0 ? std::sqrt(nr[q] / bn[q]) : std::sqrt(nr[q])) : 0.0;
        }
    }
    if (stats) {
        if (stats->size < sizeof(mclsgpu_stats))
            return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "stats: size mismatch");
        mclsgpu_stats out{};
        out.size = sizeof(out);
        unsigned long long steps = 0, tim[4] = {0, 0, 0, 0};
        cudaMemcpy(&steps, b->dom->d_steps, sizeof(steps), cudaMemcpyDeviceToHost);
        cudaMemcpy(tim, b->dom->d_tim, sizeof(tim), cudaMemcpyDeviceToHost);
        out.iterations = st.iter;
        out.converged = st.converged == st.pairs;
        out.walk_steps = int64_t(steps);
        out.histories = int64_t(st.iter) * int64_t(b->n) * b->per;
        out.solve_ms = ms;
        out.walk_ms = double(tim[2]) * 1e-6;
        out.walk_launches = int64_t(tim[3]);
        out.kernel_launches = int64_t(b->body_kernels ? b->body_kernels : 6) * st.iter + 4;
        out.rho = -1.0;
        *stats = out;
    }
    return MCLSGPU_OK;
}

}  // extern "C"
