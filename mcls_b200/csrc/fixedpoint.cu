// fixedpoint.cu -- the fixed-point iterations (the MCSA smoother's
// "Fixed Point Type") and the fixed-point solver that runs them alone.
//
//   Richardson        src/MCLS_RichardsonIteration_impl.hpp:134-147
//   Steepest Descent  src/MCLS_SteepestDescentIteration_impl.hpp:114-136
//   MINRES            src/MCLS_MinimalResidualIteration_impl.hpp:114-136
//   RNSD              src/MCLS_RNSDIteration_impl.hpp:118-142
//   solver            FixedPointSolverManager::solve,
//                     src/MCLS_FixedPointSolverManager_impl.hpp:208-321
//
// A step other than Richardson is three launches: the composite operator
// (twice for RNSD), one pass that forms both inner products and -- in the
// block that finishes last -- the step length, and one pass that updates x
// and rp.  The solver loop is a captured CUDA graph with a WHILE node whose
// condition the infinity-norm check sets.
#include <cmath>
#include <cstdio>
#include <functional>
#include <vector>

#include "internal.h"

namespace mclsgpu {
namespace {

constexpr int kThreads = 256;

inline int grid_for(long long work, int cap) {
    long long g = (work + kThreads - 1) / kThreads;
    if (g < 1) g = 1;
    return int(g > cap ? cap : g);
}

// x = x + w r, rounded as two operations (no contraction), as the reference's
// vector update.
__global__ void k_axpy(double* x, const double* r, int n, double w) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = __dadd_rn(x[i], __dmul_rn(w, r[i]));
}

// y = d .* x (a diagonal preconditioner or its transpose).
__global__ void k_diag_scale(const double* d, const double* x, double* y, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        y[i] = d[i] * x[i];
}

// Sum of the block's values in thread 0 (fixed order for a fixed launch).
__device__ __forceinline__ double block_sum(double v, double* sh) {
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kThreads / 32; ++w) t += sh[w];
    return t;
}

// NaN-propagating maximum (fmax would drop a NaN residual entry).
__device__ __forceinline__ double max_nan(double a, double b) {
    return (b > a || b != b) ? b : a;
}

__device__ __forceinline__ double block_max(double v, double* sh) {
    for (int d = 16; d > 0; d >>= 1) v = max_nan(v, __shfl_down_sync(0xffffffffu, v, d));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kThreads / 32; ++w) t = max_nan(t, sh[w]);
    return t;
}

// alpha = <a,b> / <c,d> (0 when <c,d> = 0).  Each block writes its two
// partial sums; the block that finishes last adds them in block order.
__global__ void __launch_bounds__(kThreads) k_step_length(const double* a, const double* b,
                                                          const double* c, const double* d, int n,
                                                          double* part, unsigned int* ticket,
                                                          double* alpha) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool last;
    double s0 = 0.0, s1 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        s0 = fma(a[i], b[i], s0);
        s1 = fma(c[i], d[i], s1);
    }
    const double t0 = block_sum(s0, sh);
    const double t1 = block_sum(s1, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = t0;
        part[2 * blockIdx.x + 1] = t1;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double u0 = 0.0, u1 = 0.0;
    for (int k = threadIdx.x; k < int(gridDim.x); k += blockDim.x) {
        u0 += part[2 * k];
        u1 += part[2 * k + 1];
    }
    const double num = block_sum(u0, sh);
    const double den = block_sum(u1, sh);
    if (threadIdx.x == 0) {
        *alpha = den != 0.0 ? num / den : 0.0;
        *ticket = 0u;
    }
}

// x += alpha s; rp -= alpha p
__global__ void k_fp_update(double* x, const double* s, double* r, const double* p,
                            const double* alpha, int n) {
    const double a = *alpha;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = __dadd_rn(x[i], __dmul_rn(a, s[i]));
        r[i] = __dadd_rn(r[i], __dmul_rn(-a, p[i]));
    }
}

// |v|_inf into *out (mode 0), or the fixed-point convergence check on
// |rp|_inf (mode 1; src/MCLS_FixedPointSolverManager_impl.hpp:276-287):
// one more iteration, continue while |rp|_inf > criterion and below the
// iteration limit (checked every check_freq iterations).
__global__ void __launch_bounds__(kThreads) k_inf_norm(const double* v, int n, double* part,
                                                       unsigned int* ticket, double* out,
                                                       int mode, McsaState* st, double* hist,
                                                       int hist_cap, int* status,
                                                       cudaGraphConditionalHandle handle,
                                                       int use_cond) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool last;
    double m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = max_nan(m, fabs(v[i]));
    const double t = block_max(m, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = t;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double u = 0.0;
    for (int k = threadIdx.x; k < int(gridDim.x); k += blockDim.x) u = max_nan(u, part[k]);
    const double norm = block_max(u, sh);
    if (threadIdx.x != 0) return;
    *ticket = 0u;
    if (mode == 0) {
        *out = norm;
        return;
    }
    McsaState s = *st;
    s.iter += 1;
    s.rnorm = norm;
    if (hist && s.iter <= hist_cap) hist[s.iter - 1] = norm;
    int keep = 1;
    if (s.iter % s.check_freq == 0) keep = (s.rnorm > s.crit) && (s.iter < s.max_iters);
    if (!isfinite(s.rnorm)) atomicOr(status, DEV_ERR_NONFINITE);
    if (*status) keep = 0;
    s.done = !keep;
    s.converged = s.rnorm <= s.crit;
    *st = s;
    if (use_cond) cudaGraphSetConditional(handle, keep ? 1u : 0u);
}

// Criterion tolerance * |PL b|_inf, 1 in place of a zero source norm
// (src/MCLS_FixedPointSolverManager_impl.hpp:226-245).
__global__ void k_fp_init(McsaState* st, const double* src_inf, const double* r_inf, double tol,
                          int check_freq, int max_iters) {
    McsaState s{};
    const double sn = *src_inf;
    s.crit = tol * (fabs(sn) < 10.0 * 2.220446049250313e-16 ? 1.0 : sn);
    s.check_freq = check_freq > 0 ? check_freq : 1;
    s.max_iters = max_iters;
    s.rnorm = *r_inf;
    *st = s;
}

// y = PR^T A^T PL^T x  (LinearProblem::applyTranspose, :286-315)
void composite_apply_transpose(mclsgpu_domain* dom, const double* x, double* y) {
    cudaStream_t s = dom->ctx->stream;
    const int n = dom->n;
    const int grid = grid_for(n, 148 * 8);
    const double* t = x;
    if (mclsgpu_precond* L = dom->left) {
        if (L->diag)
            k_diag_scale<<<grid, kThreads, 0, s>>>(L->diag, x, dom->tmp, n);
        else
            spmv(s, L->PT, x, dom->tmp);
        t = dom->tmp;
    }
    mclsgpu_precond* R = dom->right;
    if (!R) {
        spmv(s, dom->op->AT, t, y);
        return;
    }
    spmv(s, dom->op->AT, t, dom->tmp2);
    if (R->diag)
        k_diag_scale<<<grid, kThreads, 0, s>>>(R->diag, dom->tmp2, y, n);
    else
        spmv(s, R->PT, dom->tmp2, y);
}

int fp_params(mclsgpu_context* ctx, const mclsgpu_mcsa_params* p, mclsgpu_mcsa_params* out) {
    mclsgpu_mcsa_params d{};
    d.size = sizeof(d);
    d.max_iters = 1000;
    d.tolerance = 1.0;
    d.check_freq = 1;
    d.smoother_steps = 1;
    d.richardson_omega = 1.0;
    d.print_freq = 10;
    if (p) {
        if (p->size < sizeof(mclsgpu_mcsa_params))
            return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "fixed-point params: size mismatch");
        d = *p;
    }
    if (d.max_iters < 1 || d.check_freq < 1 || !(d.tolerance >= 0.0))
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "fixed-point params out of range");
    if (d.fixed_point_type < MCLSGPU_FIXED_POINT_RICHARDSON ||
        d.fixed_point_type > MCLSGPU_FIXED_POINT_RNSD)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "Iteration type not supported!");
    *out = d;
    return MCLSGPU_OK;
}

// The vectors and scalars a fixed-point solve needs, in the fields of a
// domain that has no Monte Carlo data.
struct Scratch {
    mclsgpu_domain d;
    ~Scratch() {
        dfree(d.x);
        dfree(d.b);
        dfree(d.rp);
        dfree(d.tmp);
        dfree(d.tmp2);
        dfree(d.x2);
        dfree(d.rp2);
        dfree(d.part);
        dfree(d.d_ticket);
        dfree(d.d_scalars);
        dfree(d.d_state);
        dfree(d.d_resid);
        if (d.h_state) cudaFreeHost(d.h_state);
    }
    cudaError_t alloc(int n, int parts, int hist) {
        cudaError_t e;
        if ((e = dmalloc(&d.x, n)) != cudaSuccess || (e = dmalloc(&d.b, n)) != cudaSuccess ||
            (e = dmalloc(&d.rp, n)) != cudaSuccess || (e = dmalloc(&d.tmp, n)) != cudaSuccess ||
            (e = dmalloc(&d.tmp2, n)) != cudaSuccess || (e = dmalloc(&d.x2, n)) != cudaSuccess ||
            (e = dmalloc(&d.rp2, n)) != cudaSuccess || (e = dmalloc(&d.part, parts)) != cudaSuccess ||
            (e = dmalloc(&d.d_ticket, 1)) != cudaSuccess ||
            (e = dmalloc(&d.d_scalars, 16)) != cudaSuccess ||
            (e = dmalloc(&d.d_state, 1)) != cudaSuccess ||
            (e = dmalloc(&d.d_resid, size_t(hist))) != cudaSuccess)
            return e;
        d.resid_cap = hist;
        return cudaMallocHost(reinterpret_cast<void**>(&d.h_state), sizeof(McsaState));
    }
};

int fixed_point_solve(mclsgpu_context* ctx, mclsgpu_operator* op, mclsgpu_precond* left,
                      mclsgpu_precond* right, const double* b_dev, double* x_dev,
                      const mclsgpu_mcsa_params* mp, mclsgpu_stats* stats) {
    cudaStream_t s = ctx->stream;
    const int n = op->A.n;
    Scratch sc;
    mclsgpu_domain& d = sc.d;
    d.ctx = ctx;
    d.op = op;
    d.left = left;
    d.right = right;
    d.n = n;
    const int parts = 2 * ctx->num_sms * 8 + 8;
    d.part_cap = parts;
    cudaError_t e = sc.alloc(n, parts, mp->max_iters);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc fixed-point buffers");
    int rc = prepare_fixed_point(&d, mp->fixed_point_type);
    if (rc) return rc;
    const int grid = grid_for(n, ctx->num_sms * 8);
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s);
    cudaMemsetAsync(d.d_ticket, 0, sizeof(unsigned int), s);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    cudaMemcpyAsync(d.b, b_dev, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(d.x, x_dev, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
    // |PL b|_inf and the initial residual's norm.
    const double* pb = d.b;
    if (left) {
        spmv(s, left->P, d.b, d.tmp);
        pb = d.tmp;
    }
    k_inf_norm<<<grid, kThreads, 0, s>>>(pb, n, d.part, d.d_ticket, d.d_scalars + 9, 0, nullptr,
                                         nullptr, 0, nullptr, cudaGraphConditionalHandle(0), 0);
    prec_residual(&d, d.x, d.b, d.rp);
    k_inf_norm<<<grid, kThreads, 0, s>>>(d.rp, n, d.part, d.d_ticket, d.d_scalars + 10, 0,
                                         nullptr, nullptr, 0, nullptr,
                                         cudaGraphConditionalHandle(0), 0);
    k_fp_init<<<1, 1, 0, s>>>(d.d_state, d.d_scalars + 9, d.d_scalars + 10, mp->tolerance,
                              mp->check_freq, mp->max_iters);
    auto body = [&](cudaGraphConditionalHandle h, int use_cond) {
        enqueue_fixed_point_step(&d, mp->fixed_point_type, mp->richardson_omega);
        k_inf_norm<<<grid, kThreads, 0, s>>>(d.rp, n, d.part, d.d_ticket, nullptr, 1, d.d_state,
                                             d.d_resid, d.resid_cap, ctx->d_status, h, use_cond);
    };
    int body_kernels = 0;
    if (!mp->host_loop) {
        cudaGraphExec_t exec = nullptr;
        rc = build_while_graph(ctx, [&](cudaGraphConditionalHandle h) { body(h, 1); }, &exec,
                               &body_kernels);
        if (rc) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return rc;
        }
        e = cudaGraphLaunch(exec, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaGraphExecDestroy(exec);
    } else {
        for (int it = 0; it < mp->max_iters && e == cudaSuccess; ++it) {
            body(cudaGraphConditionalHandle(0), 0);
            cudaMemcpyAsync(d.h_state, d.d_state, sizeof(McsaState), cudaMemcpyDeviceToHost, s);
            e = cudaStreamSynchronize(s);
            if (e == cudaSuccess && d.h_state->done) break;
        }
    }
    // Right-preconditioner recovery (:298-307).
    if (e == cudaSuccess) {
        if (right)
            spmv(s, right->P, d.x, x_dev);
        else
            cudaMemcpyAsync(x_dev, d.x, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
        cudaEventRecord(e1, s);
        cudaMemcpyAsync(d.h_state, d.d_state, sizeof(McsaState), cudaMemcpyDeviceToHost, s);
        e = cudaStreamSynchronize(s);
    }
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "fixed-point solve");
    if ((rc = check_device_status(ctx))) return rc;
    double src_inf = 0.0;
    cudaMemcpy(&src_inf, d.d_scalars + 9, sizeof(double), cudaMemcpyDeviceToHost);
    const McsaState st = *d.h_state;
    if (mp->verbose) {
        // "<name> Iteration k: Residual = |rp|_inf / |PL b|_inf" every
        // print_freq iterations and at the last (:292-300).
        static const char* names[] = {"Richardson", "Steepest Descent", "MINRES", "RNSD"};
        std::vector<double> hist(st.iter < d.resid_cap ? st.iter : d.resid_cap);
        if (!hist.empty())
            cudaMemcpy(hist.data(), d.d_resid, hist.size() * sizeof(double),
                       cudaMemcpyDeviceToHost);
        const double sn = std::fabs(src_inf) < 10.0 * 2.220446049250313e-16 ? 1.0 : src_inf;
        const int pf = mp->print_freq > 0 ? mp->print_freq : 10;
        for (int i = 0; i < int(hist.size()); ++i)
            if ((i + 1) % pf == 0 || i + 1 == st.iter)
                std::printf("%s Iteration %d: Residual = %g\n", names[mp->fixed_point_type], i + 1,
                            hist[i] / sn);
    }
    if (stats) {
        stats->iterations = st.iter;
        stats->converged = st.converged;
        stats->residual_norm = st.rnorm;
        // FixedPointSolverManager::achievedTol (:133-160)
        stats->achieved_tol = src_inf > 0.0 ? st.rnorm / src_inf : st.rnorm;
        stats->solve_ms = ms;
        stats->histories = 0;
        stats->walk_steps = 0;
        stats->walk_ms = 0.0;
        stats->walk_launches = 0;
        stats->fallback_taken = left ? left->fallback : 0;
        stats->rho = left ? left->rho : -1.0;
        stats->kernel_launches = int64_t(body_kernels) * st.iter + 4;
    }
    return MCLSGPU_OK;
}

}  // namespace

int prepare_fixed_point(mclsgpu_domain* dom, int type) {
    if (type != MCLSGPU_FIXED_POINT_RNSD) return MCLSGPU_OK;
    mclsgpu_context* ctx = dom->ctx;
    int rc = MCLSGPU_OK;
    if (!dom->op->AT.rp) rc = csr_transpose(ctx, dom->op->A, dom->op->AT);
    if (!rc && dom->left && !dom->left->diag && !dom->left->PT.rp)
        rc = csr_transpose(ctx, dom->left->P, dom->left->PT);
    if (!rc && dom->right && !dom->right->diag && !dom->right->PT.rp)
        rc = csr_transpose(ctx, dom->right->P, dom->right->PT);
    return rc;
}

void enqueue_fixed_point_step(mclsgpu_domain* dom, int type, double omega) {
    cudaStream_t s = dom->ctx->stream;
    const int n = dom->n;
    const int grid = grid_for(n, dom->ctx->num_sms * 8);
    // Two partial sums per block: at most part_cap / 2 blocks.
    const int dgrid = grid_for(n, (dom->part_cap - 8) / 2);
    double* alpha = dom->d_scalars + 7;
    switch (type) {
        case MCLSGPU_FIXED_POINT_STEEPEST_DESCENT:
            // p = Op r; a = <r,r> / <p,r>
            composite_apply(dom, dom->rp, dom->x2);
            k_step_length<<<dgrid, kThreads, 0, s>>>(dom->rp, dom->rp, dom->x2, dom->rp, n,
                                                      dom->part, dom->d_ticket, alpha);
            k_fp_update<<<grid, kThreads, 0, s>>>(dom->x, dom->rp, dom->rp, dom->x2, alpha, n);
            break;
        case MCLSGPU_FIXED_POINT_MINRES:
            // p = Op r; a = <p,r> / <p,p>
            composite_apply(dom, dom->rp, dom->x2);
            k_step_length<<<dgrid, kThreads, 0, s>>>(dom->x2, dom->rp, dom->x2, dom->x2, n,
                                                      dom->part, dom->d_ticket, alpha);
            k_fp_update<<<grid, kThreads, 0, s>>>(dom->x, dom->rp, dom->rp, dom->x2, alpha, n);
            break;
        case MCLSGPU_FIXED_POINT_RNSD:
            // v = Op^T r; w = Op v; a = <v,v> / <w,w>
            composite_apply_transpose(dom, dom->rp, dom->rp2);
            composite_apply(dom, dom->rp2, dom->x2);
            k_step_length<<<dgrid, kThreads, 0, s>>>(dom->rp2, dom->rp2, dom->x2, dom->x2, n,
                                                      dom->part, dom->d_ticket, alpha);
            k_fp_update<<<grid, kThreads, 0, s>>>(dom->x, dom->rp2, dom->rp, dom->x2, alpha, n);
            break;
        default:
            // x += w rp; rp = PL (b - A PR x)
            k_axpy<<<grid_for(n, 148 * 8), kThreads, 0, s>>>(dom->x, dom->rp, n, omega);
            prec_residual(dom, dom->x, dom->b, dom->rp);
    }
}

// A graph whose only node is a WHILE loop around the captured `body`.
int build_while_graph(mclsgpu_context* ctx,
                      const std::function<void(cudaGraphConditionalHandle)>& body,
                      cudaGraphExec_t* exec, int* body_kernels) {
    cudaStream_t s = ctx->stream;
    *exec = nullptr;
    cudaGraph_t g;
    cudaError_t e = cudaGraphCreate(&g, 0);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphCreate");
    cudaGraphConditionalHandle handle;
    e = cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
    if (e == cudaSuccess)
        e = cudaStreamBeginCaptureToGraph(s, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(ctx, e, "while graph");
    }
    body(handle);
    cudaGraph_t captured = np.conditional.phGraph_out[0];
    e = cudaStreamEndCapture(s, &captured);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(ctx, e, "cudaStreamEndCapture");
    }
    if (body_kernels) {
        size_t nn = 0;
        cudaGraphGetNodes(np.conditional.phGraph_out[0], nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        if (nn) cudaGraphGetNodes(np.conditional.phGraph_out[0], nodes.data(), &nn);
        int k = 0;
        for (size_t i = 0; i < nn; ++i) {
            cudaGraphNodeType t;
            if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
                ++k;
        }
        *body_kernels = k;
    }
    e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        *exec = nullptr;
        return cuda_fail(ctx, e, "cudaGraphInstantiate");
    }
    return MCLSGPU_OK;
}

}  // namespace mclsgpu

using namespace mclsgpu;

extern "C" {

int mclsgpu_fixed_point_solve_dev(mclsgpu_context* ctx, mclsgpu_operator* op,
                                  mclsgpu_precond* left, mclsgpu_precond* right,
                                  const double* b_dev, double* x_dev,
                                  const mclsgpu_mcsa_params* params, mclsgpu_stats* stats) {
    if (!ctx || !op || !b_dev || !x_dev) return MCLSGPU_ERR_INVALID_ARG;
    if ((left && left->P.n != op->A.n) || (right && right->P.n != op->A.n))
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "preconditioner size mismatch");
    if (left && left->kind == MCLSGPU_PREC_NONE) left = nullptr;
    if (right && right->kind == MCLSGPU_PREC_NONE) right = nullptr;
    mclsgpu_mcsa_params p;
    int rc = fp_params(ctx, params, &p);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    return fixed_point_solve(ctx, op, left, right, b_dev, x_dev, &p, stats);
}

int mclsgpu_fixed_point_solve(mclsgpu_context* ctx, mclsgpu_operator* op,
                              mclsgpu_precond* left, mclsgpu_precond* right, const double* b,
                              double* x, const mclsgpu_mcsa_params* params,
                              mclsgpu_stats* stats) {
    if (!ctx || !op || !b || !x) return MCLSGPU_ERR_INVALID_ARG;
    const int n = op->A.n;
    cudaSetDevice(ctx->device);
    double *db = nullptr, *dx = nullptr;
    cudaError_t e;
    if ((e = dmalloc(&db, n)) != cudaSuccess || (e = dmalloc(&dx, n)) != cudaSuccess) {
        dfree(db);
        dfree(dx);
        return cuda_fail(ctx, e, "cudaMalloc");
    }
    const size_t bytes = size_t(n) * sizeof(double);
    cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(dx, x, bytes, cudaMemcpyHostToDevice, ctx->stream);
    int rc = mclsgpu_fixed_point_solve_dev(ctx, op, left, right, db, dx, params, stats);
    if (!rc) {
        cudaMemcpyAsync(x, dx, bytes, cudaMemcpyDeviceToHost, ctx->stream);
        e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "copy x");
    }
    dfree(db);
    dfree(dx);
    return rc;
}

}  // extern "C"
