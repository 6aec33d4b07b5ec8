// mcsa.cu -- Monte Carlo solve and the MCSA Richardson/correction loop.
//
// MC solve (MonteCarloSolverManager::solve + MCSolver::solve,
// src/MCLS_MonteCarloSolverManager_impl.hpp:199-235, 346-380,
// src/MCLS_MCSolver_impl.hpp:82-112): source from the (left preconditioned
// unless internal, Neumann-relaxed) right-hand side, transport, normalise by
// the number of histories, right-preconditioner recovery unless internal.
//
// Estimators.  Collision: x = y / Nh with y the collision tally.
// Expected value (no counterpart in this reference snapshot): every step adds
// w * h_{s,j} to x_j for all j of the current row; summed over a history
// this equals H applied to the history's collision tally, so the kernel
// computes x = b_src + (D^T y) / Nh with one gather over the transposed
// domain instead of k scattered updates per step (forward: the tally source
// is H b_src instead of b_src).
//
// MCSA (MCSASolverManager::solve, src/MCLS_MCSASolverManager_impl.hpp:
// 278-432): each iteration runs Richardson smoothing (x += w rp, then
// rp = PL(b - A PR x)), zeroes the correction, solves the residual problem by
// MC (internal), adds the correction and recomputes the residual; the loop
// stops when |rp|_2 <= tol * |PL b|_2 or the iteration limit is reached,
// checked every "Iteration Check Frequency" iterations.  The whole loop is one
// CUDA graph: a WHILE conditional node whose body is one iteration and whose
// condition is set on the device by the convergence check, so a solve makes
// no host round trip per iteration.
#include <cmath>
#include <cstdio>
#include <vector>

#include "internal.h"
#include "rng.cuh"

namespace mclsgpu {

void launch_adjoint_source(mclsgpu_domain* dom, const double* v, double omega, int has_omega);
void launch_forward_source(mclsgpu_domain* dom, const double* v, double omega, int has_omega,
                           bool fused);
void launch_forward_setup(mclsgpu_domain* dom);
void launch_advance_walk_pos(mclsgpu_domain* dom);
void prepare_walk(mclsgpu_domain* dom);
void launch_walk(mclsgpu_domain* dom, long long max_trace, long long* tr_states, double* tr_w,
                 int* tr_ev, long long* tr_start, bool fused);

namespace {

inline int grid_for(long long work, int threads = 256, int cap = 148 * 16) {
    long long g = (work + threads - 1) / threads;
    if (g < 1) g = 1;
    return int(g > cap ? cap : g);
}

// Row dot products A(r,:) . f(col) over the two operator layouts.  Both visit
// a row's entries in ascending column order with FMA accumulation, and their
// padding entries contribute a product with 0 (which adds exactly nothing),
// so both return the CSR sum bit for bit.
struct SellView {  // SELL-32
    const int* off;
    const int* col;
    const double* val;
    int n;
    template <class F>
    __device__ __forceinline__ double dot(int r, F f) const {
        const int a = off[r >> 5];
        const int o = a + (r & 31), w = (off[(r >> 5) + 1] - a) >> 5;
        double s = 0.0;
        for (int k = 0; k < w; ++k) s = fma(val[o + 32 * k], f(col[o + 32 * k]), s);
        return s;
    }
};

// Stencil operator stored by diagonal offset (no indices).  KK > 0 fixes the
// number of offsets at compile time so the row loop unrolls and every load of
// the row is issued before the first product.
template <int KK>
struct DiaViewT {
    const double* val;
    int n;
    int k;
    int off[16];
    template <class F>
    __device__ __forceinline__ double dot(int r, F f) const {
        constexpr int kmax = KK > 0 ? KK : 16;
        const int kk = KK > 0 ? KK : k;
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < kmax; ++j) {
            if (j >= kk) break;
            const int c = r + off[j];
            if (unsigned(c) < unsigned(n)) s = fma(val[size_t(j) * n + r], f(c), s);
        }
        return s;
    }
};
using DiaView = DiaViewT<0>;

// Symmetric stencil operator (A(r, r - o) == A(r - o, r)): only the diagonal
// and the H positive-offset diagonals are read; A(r, r - o_h) is taken as
// A(r - o_h, r).  The products are the same as DiaViewT's, in the same
// (ascending column) order, so the sums are bit for bit the same with
// (1 + H) / (1 + 2H) of the matrix bytes.
template <int H>
struct DiaSymView {
    const double* val;  // [(1 + H) * n]: diagonal, then positive offsets ascending
    int n;
    int off[H];
    template <class F>
    __device__ __forceinline__ double dot(int r, F f) const {
        double s = 0.0;
#pragma unroll
        for (int h = H - 1; h >= 0; --h) {
            const int c = r - off[h];
            if (c >= 0) s = fma(val[size_t(1 + h) * n + c], f(c), s);
        }
        s = fma(val[r], f(r), s);
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const int c = r + off[h];
            if (c < n) s = fma(val[size_t(1 + h) * n + r], f(c), s);
        }
        return s;
    }
};

// rp = (b - A x) [* dinv]   (LinearProblem::updatePrecResidual, :410-442)
template <class Op>
__global__ void __launch_bounds__(256) k_residual(Op A, const double* x, const double* b,
                                                  const double* dinv, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
        const double s = A.dot(i, [&](int j) { return x[j]; });
        double r = b[i] - s;
        out[i] = dinv ? dinv[i] * r : r;
    }
}

// out = [dinv *] A x   (the A and PL factors of LinearProblem::apply, :251-279)
template <class Op>
__global__ void __launch_bounds__(256) k_matvec(Op A, const double* x, const double* dinv,
                                                double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
        const double s = A.dot(i, [&](int j) { return x[j]; });
        out[i] = dinv ? dinv[i] * s : s;
    }
}

// x += w * r  (RichardsonIteration::doOneIteration, :134-147)
__global__ void k_richardson(double* x, const double* r, int n, double w) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = __dadd_rn(x[i], __dmul_rn(w, r[i]));
}

struct FinalizeArgs {
    int n;
    int mode;            // 0 adjoint collision, 1 adjoint EV, 2 forward
    int ev;
    int accumulate;      // 1: out += delta (MCSA), 0: out = delta
    int fp32;
    double per;          // forward histories per state
    const double* sc;    // [2] = 1/nh
    const double* src;   // MC source vector before scaling
    double omega;
    int has_omega;
    const double* y64;
    const int* dtrp;
    const int* dtci;
    const float* dth32;
    const double* dth64;
    double* out;
    const int* d_nh;
    unsigned long long* d_hist;
};

__global__ void __launch_bounds__(256) k_finalize(FinalizeArgs a) {
    const double inv = a.sc[2];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        double d;
        const double srci = a.has_omega ? a.src[i] * a.omega : a.src[i];
        if (a.mode == 0) {
            // AdjointTally::normalize: x *= 1/nh  (src/MCLS_AdjointTally_impl.hpp:68-72)
            d = __dmul_rn(a.y64[i], inv);
        } else if (a.mode == 1) {
            double t = 0.0;
            if (a.fp32) {
                for (int k = a.dtrp[i]; k < a.dtrp[i + 1]; ++k)
                    t = fma(double(a.dth32[k]), a.y64[a.dtci[k]], t);
            } else {
                for (int k = a.dtrp[i]; k < a.dtrp[i + 1]; ++k)
                    t = fma(a.dth64[k], a.y64[a.dtci[k]], t);
            }
            d = __dadd_rn(__dmul_rn(t, inv), srci);
        } else {
            // ForwardTally::finalize: sum / count  (src/MCLS_ForwardTally_impl.hpp:194-208)
            d = __ddiv_rn(a.y64[i], a.per);
            if (a.ev) d = __dadd_rn(d, srci);
        }
        a.out[i] = a.accumulate ? __dadd_rn(a.out[i], d) : d;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && a.d_hist) *a.d_hist += (unsigned long long)(*a.d_nh);
}

__global__ void k_epoch_inc(unsigned long long* e) { *e += 1ULL; }

// Convergence check of one MCSA iteration (src/MCLS_MCSASolverManager_impl.hpp:380-394).
__device__ __forceinline__ int mcsa_check(McsaState* st, const double* sumsq, double* hist,
                                          int hist_cap, int* status) {
    McsaState s = *st;
    s.iter += 1;
    s.rnorm = sqrt(*sumsq);
    if (hist && s.iter <= hist_cap) hist[s.iter - 1] = s.rnorm;
    int keep = 1;
    if (s.iter % s.check_freq == 0) keep = (s.rnorm > s.crit) && (s.iter < s.max_iters);
    // A non-finite residual norm ends the loop as a divergence.
    if (!isfinite(s.rnorm)) atomicOr(status, DEV_ERR_NONFINITE);
    if (*status) keep = 0;
    s.done = !keep;
    s.converged = s.rnorm <= s.crit;
    *st = s;
    return keep;
}

__global__ void k_mcsa_check(McsaState* st, const double* sumsq, double* hist, int hist_cap,
                             int* status, cudaGraphConditionalHandle handle) {
    const int keep = mcsa_check(st, sumsq, hist, hist_cap, status);
    cudaGraphSetConditional(handle, keep ? 1u : 0u);
}

__global__ void k_mcsa_check_host(McsaState* st, const double* sumsq, double* hist, int hist_cap,
                                  int* status) {
    mcsa_check(st, sumsq, hist, hist_cap, status);
}

// ---- fused iteration kernels (smoother_steps == 1, PL in {I, point Jacobi}) ----
constexpr int kFusedThreads = 256;

// Richardson smoothing fused with the residual: x2 = x + w rp (rounded as the
// separate update would be) and rp2 = PL (b - A x2), reading x + w rp at the
// neighbours on the fly.
template <class Op>
__global__ void __launch_bounds__(kFusedThreads) k_richardson_residual(
    Op A, const double* b, const double* dinv, const double* x, const double* r, double w,
    double* x2, double* r2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
        const double s = A.dot(i, [&](int j) { return __dadd_rn(x[j], __dmul_rn(w, r[j])); });
        const double res = b[i] - s;
        r2[i] = dinv ? dinv[i] * res : res;
        x2[i] = __dadd_rn(x[i], __dmul_rn(w, r[i]));
    }
}

struct ResidArgs {
    int n;
    const double* b;
    const double* dinv;       // null: no left preconditioner
    const double* xin;        // x after smoothing
    const double* rin;        // residual after smoothing (the MC source)
    const double* y;          // tallies
    const double* sc;         // [2] = 1/nh
    double omega;
    int has_omega;
    double per;
    double inv_per;
    int per_pow2;
    int ev;
    int mode;                 // 0 adjoint collision, 1 forward, 2 x already corrected
    double* xout;
    double* rout;
    double* part;
    unsigned int* ticket;
    McsaState* st;
    double* hist;
    int hist_cap;
    int* status;
    unsigned long long* d_epoch;
    unsigned long long* d_tim;
    int* d_counter;
    unsigned long long* d_hist;
    const int* d_nh;
    cudaGraphConditionalHandle handle;
    int use_cond;
};

// x + delta at state j: the MC correction of the estimator, rounded exactly
// as the separate normalise-and-add kernel rounds it.
__device__ __forceinline__ double corrected(const ResidArgs& a, int j, double inv) {
    const double xj = a.xin[j];
    if (a.mode == 0) return __dadd_rn(xj, __dmul_rn(a.y[j], inv));
    if (a.mode == 1) {
        // sum / count (ForwardTally::finalize); for a power-of-two count the
        // product with its reciprocal is the same number and much cheaper.
        double d = a.per_pow2 ? a.y[j] * a.inv_per : __ddiv_rn(a.y[j], a.per);
        if (a.ev) d = __dadd_rn(d, a.has_omega ? a.rin[j] * a.omega : a.rin[j]);
        return __dadd_rn(xj, d);
    }
    return xj;
}

// x = x2 + delta (the MC correction applied state by state).
__global__ void __launch_bounds__(kFusedThreads) k_apply_correction(ResidArgs a) {
    const double inv = a.sc[2];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x)
        a.xout[i] = corrected(a, i, inv);
}

// rp = PL (b - A x), |rp|^2, then (last block) the MCSA convergence check,
// the stream epoch, the walk timing, the work-queue reset and the loop
// condition.
// Block sum of the threads' acc, then (last block to finish) the MCSA
// convergence check, the stream epoch, the walk timing, the work-queue reset
// and the loop condition.
__device__ __forceinline__ void norm_and_check(const ResidArgs& a, double acc) {
    __shared__ double warp_sum[kFusedThreads / 32];
    __shared__ bool last;
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, d);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kFusedThreads / 32; ++w) t += warp_sum[w];
        a.part[blockIdx.x] = t;
        __threadfence();
        last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t = 0.0;
    for (int i = threadIdx.x; i < gridDim.x; i += blockDim.x) t += a.part[i];
    for (int d = 16; d > 0; d >>= 1) t += __shfl_down_sync(0xffffffffu, t, d);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double sumsq = 0.0;
        for (int w = 0; w < kFusedThreads / 32; ++w) sumsq += warp_sum[w];
        *a.ticket = 0u;
        const int keep = mcsa_check(a.st, &sumsq, a.hist, a.hist_cap, a.status);
        *a.d_epoch += 1ULL;
        *a.d_hist += (unsigned long long)(*a.d_nh);
        unsigned long long* tm = a.d_tim;
        if (tm[1] > tm[0]) {
            tm[2] += tm[1] - tm[0];
            tm[3] += 1;
        }
        tm[0] = ~0ULL;
        tm[1] = 0;
        *a.d_counter = 0;
        if (a.use_cond) cudaGraphSetConditional(a.handle, keep ? 1u : 0u);
    }
}

template <class Op>
__global__ void __launch_bounds__(kFusedThreads) k_residual_norm(Op A, ResidArgs a) {
    const double* x = a.xout;
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const double s = A.dot(i, [&](int j) { return x[j]; });
        const double res = a.b[i] - s;
        const double r = a.dinv ? a.dinv[i] * res : res;
        a.rout[i] = r;
        acc = fma(r, r, acc);
    }
    norm_and_check(a, acc);
}

// A left preconditioner M stored on A's diagonals (learned SPAI): out = M v.
template <class Op>
__global__ void __launch_bounds__(kFusedThreads) k_dia_apply(Op M, const double* v, double* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M.n; i += gridDim.x * blockDim.x)
        out[i] = M.dot(i, [&](int j) { return v[j]; });
}

// rp = M (b - A x) from the raw residual, its norm and the convergence check.
template <class Op>
__global__ void __launch_bounds__(kFusedThreads) k_precond_norm(Op M, ResidArgs a,
                                                               const double* raw) {
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const double r = M.dot(i, [&](int j) { return raw[j]; });
        a.rout[i] = r;
        acc = fma(r, r, acc);
    }
    norm_and_check(a, acc);
}

__global__ void k_mcsa_init(McsaState* st, const double* src_sumsq, double tol, int check_freq,
                            int max_iters, const double* r_sumsq) {
    McsaState s{};
    double sn = sqrt(*src_sumsq);
    s.pad = 0;
    // Homogeneous case (:312-316)
    double crit_norm = fabs(sn) < 10.0 * 2.220446049250313e-16 ? 1.0 : sn;
    s.crit = tol * crit_norm;
    s.check_freq = check_freq > 0 ? check_freq : 1;
    s.max_iters = max_iters;
    s.iter = 0;
    s.done = 0;
    s.rnorm = sqrt(*r_sumsq);
    s.converged = 0;
    *st = s;
}

}  // namespace

// ---------------------------------------------------------------------------
static SellView sell_view(const mclsgpu_operator* op) {
    return SellView{op->S.off, op->S.col, op->S.val, op->S.n};
}

template <int H>
static DiaSymView<H> sym_view(const mclsgpu_operator* op) {
    DiaSymView<H> v{};
    v.val = op->sym_val;
    v.n = op->A.n;
    for (int h = 0; h < H; ++h) v.off[h] = op->sym_off[h];
    return v;
}

template <int KK>
static DiaViewT<KK> dia_view(const mclsgpu_operator* op) {
    DiaViewT<KK> v{};
    v.val = op->dia_val;
    v.n = op->A.n;
    v.k = op->dia_k;
    for (int j = 0; j < 16; ++j) v.off[j] = op->dia_off[j];
    return v;
}

// The diagonal-offset view of another matrix on the operator's offsets.
template <int KK>
static DiaViewT<KK> dia_view_vals(const mclsgpu_operator* op, const double* vals) {
    DiaViewT<KK> v = dia_view<KK>(op);
    v.val = vals;
    return v;
}

#define MCLSGPU_LAUNCH_M(op, vals, grid, threads, stream, kern, ...)                         \
    do {                                                                                     \
        switch ((op)->dia_k) {                                                               \
            case 5:                                                                          \
                kern<DiaViewT<5>><<<grid, threads, 0, stream>>>(dia_view_vals<5>(op, vals),  \
                                                                __VA_ARGS__);                \
                break;                                                                       \
            case 7:                                                                          \
                kern<DiaViewT<7>><<<grid, threads, 0, stream>>>(dia_view_vals<7>(op, vals),  \
                                                                __VA_ARGS__);                \
                break;                                                                       \
            case 9:                                                                          \
                kern<DiaViewT<9>><<<grid, threads, 0, stream>>>(dia_view_vals<9>(op, vals),  \
                                                                __VA_ARGS__);                \
                break;                                                                       \
            default:                                                                         \
                kern<DiaView><<<grid, threads, 0, stream>>>(dia_view_vals<0>(op, vals),      \
                                                            __VA_ARGS__);                    \
        }                                                                                    \
    } while (0)

// Launch `kern<Op>` on the operator's fastest layout: diagonal-offset values
// for stencil operators (unrolled for the 5-, 7- and 9-point stencils; only
// the diagonal and upper diagonals when the values are symmetric), SELL-32
// otherwise.
#define MCLSGPU_LAUNCH_OP(op, grid, threads, stream, kern, ...)                              \
    do {                                                                                     \
        switch ((op)->dia_k) {                                                               \
            case 0:                                                                          \
                kern<SellView><<<grid, threads, 0, stream>>>(sell_view(op), __VA_ARGS__);    \
                break;                                                                       \
            case 5:                                                                          \
                if ((op)->sym_h == 2)                                                        \
                    kern<DiaSymView<2>><<<grid, threads, 0, stream>>>(sym_view<2>(op),        \
                                                                      __VA_ARGS__);          \
                else                                                                         \
                    kern<DiaViewT<5>><<<grid, threads, 0, stream>>>(dia_view<5>(op),          \
                                                                    __VA_ARGS__);            \
                break;                                                                       \
            case 7:                                                                          \
                if ((op)->sym_h == 3)                                                        \
                    kern<DiaSymView<3>><<<grid, threads, 0, stream>>>(sym_view<3>(op),        \
                                                                      __VA_ARGS__);          \
                else                                                                         \
                    kern<DiaViewT<7>><<<grid, threads, 0, stream>>>(dia_view<7>(op),          \
                                                                    __VA_ARGS__);            \
                break;                                                                       \
            case 9:                                                                          \
                if ((op)->sym_h == 4)                                                        \
                    kern<DiaSymView<4>><<<grid, threads, 0, stream>>>(sym_view<4>(op),        \
                                                                      __VA_ARGS__);          \
                else                                                                         \
                    kern<DiaViewT<9>><<<grid, threads, 0, stream>>>(dia_view<9>(op),          \
                                                                    __VA_ARGS__);            \
                break;                                                                       \
            default:                                                                         \
                kern<DiaView><<<grid, threads, 0, stream>>>(dia_view<0>(op), __VA_ARGS__);   \
        }                                                                                    \
    } while (0)

// rp = PL (b - A PR x)
static void update_prec_residual(mclsgpu_domain* dom, const double* x, const double* b,
                                 double* rp_out) {
    cudaStream_t s = dom->ctx->stream;
    const mclsgpu_operator* op = dom->op;
    const int grid = grid_for(op->A.n, 256, 148 * 8);
    const double* xin = x;
    if (dom->right) {
        spmv(s, dom->right->P, x, dom->tmp2);
        xin = dom->tmp2;
    }
    mclsgpu_precond* L = dom->left;
    if (!L) {
        MCLSGPU_LAUNCH_OP(op, grid, 256, s, k_residual, xin, b, nullptr, rp_out);
    } else if (L->kind == MCLSGPU_PREC_POINT_JACOBI) {
        MCLSGPU_LAUNCH_OP(op, grid, 256, s, k_residual, xin, b, L->diag, rp_out);
    } else {
        MCLSGPU_LAUNCH_OP(op, grid, 256, s, k_residual, xin, b, nullptr, dom->tmp);
        spmv(s, L->P, dom->tmp, rp_out);
    }
}

void prec_residual(mclsgpu_domain* dom, const double* x, const double* b, double* rp_out) {
    update_prec_residual(dom, x, b, rp_out);
}

// y = PL A PR x  (LinearProblem::apply, src/MCLS_LinearProblem_impl.hpp:251-279)
void composite_apply(mclsgpu_domain* dom, const double* x, double* y) {
    cudaStream_t s = dom->ctx->stream;
    const mclsgpu_operator* op = dom->op;
    const int grid = grid_for(op->A.n, 256, 148 * 8);
    const double* xin = x;
    if (dom->right) {
        spmv(s, dom->right->P, x, dom->tmp2);
        xin = dom->tmp2;
    }
    mclsgpu_precond* L = dom->left;
    if (!L) {
        MCLSGPU_LAUNCH_OP(op, grid, 256, s, k_matvec, xin, nullptr, y);
    } else if (L->kind == MCLSGPU_PREC_POINT_JACOBI) {
        MCLSGPU_LAUNCH_OP(op, grid, 256, s, k_matvec, xin, L->diag, y);
    } else {
        MCLSGPU_LAUNCH_OP(op, grid, 256, s, k_matvec, xin, nullptr, dom->tmp);
        spmv(s, L->P, dom->tmp, y);
    }
}

// One MC solve of the source vector `v` (device, already left preconditioned
// when required) into out (accumulate: out += delta).  `fused`: inside the
// fused MCSA iteration the normalise-and-add of the collision and forward
// estimators, the epoch increment and the walk bookkeeping are done by
// k_update_residual; only the adjoint expected-value gather runs here.
static void enqueue_mc(mclsgpu_domain* dom, const double* v, double* out, int accumulate,
                       long long max_trace, long long* tr_states, double* tr_w, int* tr_ev,
                       long long* tr_start, bool fused = false) {
    const mclsgpu_mc_params& p = dom->p;
    const double omega = p.neumann_relaxation;
    const int has_omega = p.neumann_relaxation > 0.0;
    if (p.direction == MCLSGPU_ADJOINT)
        launch_adjoint_source(dom, v, omega, has_omega);
    else
        launch_forward_source(dom, v, omega, has_omega, fused);
    launch_walk(dom, max_trace, tr_states, tr_w, tr_ev, tr_start, fused);
    launch_advance_walk_pos(dom);
    if (fused && !(p.direction == MCLSGPU_ADJOINT && p.estimator == MCLSGPU_EXPECTED_VALUE))
        return;
    FinalizeArgs f{};
    f.n = dom->n;
    f.mode = p.direction == MCLSGPU_FORWARD ? 2 : (p.estimator == MCLSGPU_EXPECTED_VALUE ? 1 : 0);
    f.ev = p.estimator == MCLSGPU_EXPECTED_VALUE;
    f.accumulate = accumulate;
    f.fp32 = p.precision == MCLSGPU_FP32;
    f.per = p.sample_ratio > 0.0 ? std::ceil(p.sample_ratio) : 1.0;
    f.sc = dom->d_scalars;
    f.src = v;
    f.omega = omega;
    f.has_omega = has_omega;
    f.y64 = dom->y64;
    f.dtrp = dom->DT.rp;
    f.dtci = dom->DT.ci;
    f.dth32 = dom->dt_h32;
    f.dth64 = dom->DT.v;
    f.out = out;
    f.d_nh = dom->d_nh;
    f.d_hist = fused ? nullptr : dom->d_hist;
    k_finalize<<<grid_for(dom->n, 256, 148 * 8), 256, 0, dom->ctx->stream>>>(f);
    if (!fused) k_epoch_inc<<<1, 1, 0, dom->ctx->stream>>>(dom->d_epoch);
}

static int read_stats(mclsgpu_domain* dom, mclsgpu_stats* st) {
    if (!st) return MCLSGPU_OK;
    unsigned long long steps = 0, hist = 0, tim[4] = {0, 0, 0, 0};
    cudaMemcpyAsync(&steps, dom->d_steps, sizeof(steps), cudaMemcpyDeviceToHost, dom->ctx->stream);
    cudaMemcpyAsync(&hist, dom->d_hist, sizeof(hist), cudaMemcpyDeviceToHost, dom->ctx->stream);
    cudaMemcpyAsync(tim, dom->d_tim, sizeof(tim), cudaMemcpyDeviceToHost, dom->ctx->stream);
    cudaError_t e = cudaStreamSynchronize(dom->ctx->stream);
    if (e != cudaSuccess) return cuda_fail(dom->ctx, e, "stats");
    st->walk_steps = (int64_t)steps;
    st->histories = (int64_t)hist;
    st->walk_ms = double(tim[2]) * 1e-6;
    st->walk_launches = (int64_t)tim[3];
    return MCLSGPU_OK;
}

static void reset_counters(mclsgpu_domain* dom) {
    cudaStream_t s = dom->ctx->stream;
    cudaMemsetAsync(dom->d_steps, 0, sizeof(unsigned long long), s);
    cudaMemsetAsync(dom->d_hist, 0, sizeof(unsigned long long), s);
    cudaMemsetAsync(dom->d_tim + 2, 0, 2 * sizeof(unsigned long long), s);
}

// MC solve with device vectors.
static int mc_solve_device(mclsgpu_domain* dom, const double* rhs_dev, double* x_dev, int internal,
                           long long max_trace, long long* tr_states, double* tr_w, int* tr_ev,
                           long long* tr_start, mclsgpu_stats* stats) {
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s);
    reset_counters(dom);
    const double* v = rhs_dev;
    if (dom->left && !internal) {
        spmv(s, dom->left->P, rhs_dev, dom->tmp);
        v = dom->tmp;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    if (dom->right && !internal) {
        // v is rhs_dev or tmp, so tmp2 is free for the unrecovered result.
        enqueue_mc(dom, v, dom->tmp2, 0, max_trace, tr_states, tr_w, tr_ev, tr_start);
        spmv(s, dom->right->P, dom->tmp2, x_dev);
    } else {
        enqueue_mc(dom, v, x_dev, 0, max_trace, tr_states, tr_w, tr_ev, tr_start);
    }
    cudaEventRecord(e1, s);
    cudaError_t e = cudaStreamSynchronize(s);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "mc solve");
    int rc = check_device_status(ctx);
    if (rc) return rc;
    if (stats) {
        if ((rc = read_stats(dom, stats))) return rc;
        stats->solve_ms = ms;
        stats->iterations = 0;
        stats->converged = 1;
    }
    return MCLSGPU_OK;
}

// x2 = x + w r (rounded as the reference's vector update)
__global__ void k_axpy_to(const double* x, const double* r, double w, double* x2, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x2[i] = __dadd_rn(x[i], __dmul_rn(w, r[i]));
}

int mcsa_read_stats(mclsgpu_domain* dom, mclsgpu_stats* st) { return read_stats(dom, st); }
void mcsa_reset_counters(mclsgpu_domain* dom) { reset_counters(dom); }

void mc_correction(mclsgpu_domain* dom, const double* v, double* out) {
    enqueue_mc(dom, v, out, 0, 0, nullptr, nullptr, nullptr, nullptr);
}

// The fused iteration covers one smoothing step, no right preconditioner and
// a left preconditioner that is the identity or point Jacobi.
static bool fused_iteration(const mclsgpu_domain* dom, const mclsgpu_mcsa_params* mp) {
    return mp->smoother_steps == 1 && mp->fixed_point_type == MCLSGPU_FIXED_POINT_RICHARDSON &&
           !dom->right &&
           (!dom->left || dom->left->kind == MCLSGPU_PREC_POINT_JACOBI ||
            (dom->left->mdia && dom->op->dia_k > 0));
}

// At most 8 blocks per SM: the per-block partial sums of k_apply_correction
// and k_residual_norm go to dom->part, sized for that many blocks.
static int fused_grid(const mclsgpu_domain* dom) {
    return grid_for(dom->n, kFusedThreads, dom->ctx->num_sms * 8);
}

void richardson_residual(mclsgpu_domain* dom, const double* x, const double* r, double w,
                         double* x2, double* r2) {
    cudaStream_t s = dom->ctx->stream;
    const mclsgpu_operator* op = dom->op;
    const int grid = fused_grid(dom);
    const mclsgpu_precond* L = dom->left;
    if (!dom->right && (!L || L->kind == MCLSGPU_PREC_POINT_JACOBI)) {
        MCLSGPU_LAUNCH_OP(op, grid, kFusedThreads, s, k_richardson_residual, dom->b,
                          L ? L->diag : nullptr, x, r, w, x2, r2);
    } else if (!dom->right && L->mdia && op->dia_k > 0) {
        MCLSGPU_LAUNCH_OP(op, grid, kFusedThreads, s, k_richardson_residual, dom->b, nullptr, x,
                          r, w, x2, dom->tmp);
        MCLSGPU_LAUNCH_M(op, L->mdia, grid, kFusedThreads, s, k_dia_apply, dom->tmp, r2);
    } else {
        k_axpy_to<<<grid, kFusedThreads, 0, s>>>(x, r, w, x2, dom->n);
        update_prec_residual(dom, x2, dom->b, r2);
    }
}

// One MCSA iteration including its convergence check.  The fused form is
// three kernels around the walk: Richardson + residual, the source build
// (forward: tally sources into the records), the walk, and correction +
// residual + norm + check.
static void enqueue_iteration(mclsgpu_domain* dom, const mclsgpu_mcsa_params* mp,
                              cudaGraphConditionalHandle handle, int use_cond) {
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    const int n = dom->n;
    if (!fused_iteration(dom, mp)) {
        for (int l = 0; l < mp->smoother_steps; ++l)
            enqueue_fixed_point_step(dom, mp->fixed_point_type, mp->richardson_omega);
        enqueue_mc(dom, dom->rp, dom->x, 1, 0, nullptr, nullptr, nullptr, nullptr);
        update_prec_residual(dom, dom->x, dom->b, dom->rp);
        sum_sq(s, dom->rp, n, dom->part, dom->d_scalars + 5);
        if (use_cond)
            k_mcsa_check<<<1, 1, 0, s>>>(dom->d_state, dom->d_scalars + 5, dom->d_resid,
                                         dom->resid_cap, ctx->d_status, handle);
        else
            k_mcsa_check_host<<<1, 1, 0, s>>>(dom->d_state, dom->d_scalars + 5, dom->d_resid,
                                               dom->resid_cap, ctx->d_status);
        return;
    }
    const mclsgpu_operator* op = dom->op;
    const double* dinv = dom->left ? dom->left->diag : nullptr;
    // A left preconditioner on A's diagonals (learned SPAI): the raw residual
    // goes to tmp and a second pass applies M.
    const double* mdia = dom->left ? dom->left->mdia : nullptr;
    const int grid = fused_grid(dom);
    if (mdia) {
        MCLSGPU_LAUNCH_OP(op, grid, kFusedThreads, s, k_richardson_residual, dom->b, nullptr,
                          dom->x, dom->rp, mp->richardson_omega, dom->x2, dom->tmp);
        MCLSGPU_LAUNCH_M(op, mdia, grid, kFusedThreads, s, k_dia_apply, dom->tmp, dom->rp2);
    } else {
        MCLSGPU_LAUNCH_OP(op, grid, kFusedThreads, s, k_richardson_residual, dom->b, dinv, dom->x,
                          dom->rp, mp->richardson_omega, dom->x2, dom->rp2);
    }
    const mclsgpu_mc_params& p = dom->p;
    const bool adj_ev = p.direction == MCLSGPU_ADJOINT && p.estimator == MCLSGPU_EXPECTED_VALUE;
    enqueue_mc(dom, dom->rp2, dom->x2, 1, 0, nullptr, nullptr, nullptr, nullptr, true);
    ResidArgs a{};
    a.n = n;
    a.b = dom->b;
    a.dinv = dinv;
    a.xin = dom->x2;
    a.rin = dom->rp2;
    a.y = dom->y64;
    a.sc = dom->d_scalars;
    a.omega = p.neumann_relaxation;
    a.has_omega = p.neumann_relaxation > 0.0;
    a.per = p.sample_ratio > 0.0 ? std::ceil(p.sample_ratio) : 1.0;
    {
        int ex = 0;
        a.per_pow2 = std::frexp(a.per, &ex) == 0.5;  // per = 2^(ex-1)
        a.inv_per = 1.0 / a.per;
    }
    a.ev = p.estimator == MCLSGPU_EXPECTED_VALUE;
    a.mode = p.direction == MCLSGPU_FORWARD ? 1 : (adj_ev ? 2 : 0);
    a.xout = dom->x;
    a.rout = dom->rp;
    a.part = dom->part;
    a.ticket = dom->d_ticket;
    a.st = dom->d_state;
    a.hist = dom->d_resid;
    a.hist_cap = dom->resid_cap;
    a.status = ctx->d_status;
    a.d_epoch = dom->d_epoch;
    a.d_tim = dom->d_tim;
    a.d_counter = dom->d_counter;
    a.d_hist = dom->d_hist;
    a.d_nh = dom->d_nh;
    a.handle = handle;
    a.use_cond = use_cond;
    k_apply_correction<<<grid, kFusedThreads, 0, s>>>(a);
    if (mdia) {
        MCLSGPU_LAUNCH_OP(op, grid, kFusedThreads, s, k_residual, dom->x, dom->b, nullptr,
                          dom->tmp);
        MCLSGPU_LAUNCH_M(op, mdia, grid, kFusedThreads, s, k_precond_norm, a, dom->tmp);
    } else {
        MCLSGPU_LAUNCH_OP(op, grid, kFusedThreads, s, k_residual_norm, a);
    }
}

// Build the CUDA graph of the MCSA loop (WHILE node, one iteration per body).
static int build_mcsa_graph(mclsgpu_domain* dom, const mclsgpu_mcsa_params* mp) {
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    if (dom->graph) {
        cudaGraphExecDestroy(dom->graph);
        dom->graph = nullptr;
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
    e = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(ctx, e, "cudaStreamBeginCaptureToGraph");
    }
    enqueue_iteration(dom, mp, handle, 1);
    cudaGraph_t captured = body;
    e = cudaStreamEndCapture(s, &captured);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(ctx, e, "cudaStreamEndCapture");
    }
    size_t nn = 0;
    cudaGraphGetNodes(body, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn) cudaGraphGetNodes(body, nodes.data(), &nn);
    dom->body_kernels = 0;
    for (size_t k = 0; k < nn; ++k) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[k], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
            ++dom->body_kernels;
    }
    e = cudaGraphInstantiate(&dom->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        dom->graph = nullptr;
        return cuda_fail(ctx, e, "cudaGraphInstantiate");
    }
    return MCLSGPU_OK;
}

static int mcsa_solve_device(mclsgpu_domain* dom, const double* b_dev, double* x_dev,
                             const mclsgpu_mcsa_params* mp, mclsgpu_stats* stats) {
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    const int n = dom->n;
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s);
    reset_counters(dom);
    // The fused iteration expects a zero work-queue counter and ticket on
    // entry (it resets both itself at the end of every iteration).
    cudaMemsetAsync(dom->d_counter, 0, sizeof(int), s);
    cudaMemsetAsync(dom->d_ticket, 0, sizeof(unsigned int), s);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    if (mp->max_iters > dom->resid_cap) {
        dfree(dom->d_resid);
        cudaError_t e = dmalloc(&dom->d_resid, size_t(mp->max_iters));
        if (e != cudaSuccess) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return cuda_fail(ctx, e, "cudaMalloc");
        }
        dom->resid_cap = mp->max_iters;
        if (dom->graph) {
            cudaGraphExecDestroy(dom->graph);
            dom->graph = nullptr;
        }
    }
    // Graph key: everything baked into the captured iteration.
    const int key = (mp->smoother_steps * 1000003 ^ int(mp->richardson_omega * 1e6)) * 4 +
                    mp->fixed_point_type;
    if (int rc = prepare_fixed_point(dom, mp->fixed_point_type)) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return rc;
    }
    // Variable-length reference-stream walks synchronise with the host.
    const bool host_loop = mp->host_loop || walk_needs_rounds(dom);
    if (!host_loop && (!dom->graph || dom->graph_key != key)) {
        int rc = build_mcsa_graph(dom, mp);
        if (rc) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return rc;
        }
        dom->graph_key = key;
    }
    cudaEventRecord(e0, s);
    if (b_dev != dom->b)
        cudaMemcpyAsync(dom->b, b_dev, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (x_dev != dom->x)
        cudaMemcpyAsync(dom->x, x_dev, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
    // Source norm |PL b|_2 (:299-318) and the initial preconditioned residual.
    const double* pb = dom->b;
    if (dom->left) {
        spmv(s, dom->left->P, dom->b, dom->tmp);
        pb = dom->tmp;
    }
    sum_sq(s, pb, n, dom->part, dom->d_scalars + 6);
    update_prec_residual(dom, dom->x, dom->b, dom->rp);
    sum_sq(s, dom->rp, n, dom->part, dom->d_scalars + 5);
    k_mcsa_init<<<1, 1, 0, s>>>(dom->d_state, dom->d_scalars + 6, mp->tolerance, mp->check_freq,
                                mp->max_iters, dom->d_scalars + 5);
    if (fused_iteration(dom, mp) && dom->p.direction == MCLSGPU_FORWARD) launch_forward_setup(dom);
    cudaError_t e = cudaSuccess;
    if (!host_loop) {
        e = cudaGraphLaunch(dom->graph, s);
    } else {
        // Host-driven loop: the same iteration, one state read-back each.
        for (int it = 0; it < mp->max_iters && e == cudaSuccess; ++it) {
            enqueue_iteration(dom, mp, cudaGraphConditionalHandle(0), 0);
            cudaMemcpyAsync(dom->h_state, dom->d_state, sizeof(McsaState), cudaMemcpyDeviceToHost, s);
            e = cudaStreamSynchronize(s);
            if (e == cudaSuccess && dom->h_state->done) break;
        }
    }
    cudaEventRecord(e1, s);
    if (e == cudaSuccess) {
        // Right preconditioner recovery (:410-418).
        if (dom->right) {
            spmv(s, dom->right->P, dom->x, dom->tmp);
            cudaMemcpyAsync(x_dev, dom->tmp, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
        } else if (x_dev != dom->x) {
            cudaMemcpyAsync(x_dev, dom->x, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
        }
        cudaMemcpyAsync(dom->h_state, dom->d_state, sizeof(McsaState), cudaMemcpyDeviceToHost, s);
        e = cudaStreamSynchronize(s);
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "mcsa graph");
    int rc = check_device_status(ctx);
    if (rc) return rc;
    double src_sumsq = 0.0;
    cudaMemcpy(&src_sumsq, dom->d_scalars + 6, sizeof(double), cudaMemcpyDeviceToHost);
    const McsaState st = *dom->h_state;
    if (mp->verbose) {
        std::vector<double> hist(st.iter < dom->resid_cap ? st.iter : dom->resid_cap);
        if (!hist.empty())
            cudaMemcpy(hist.data(), dom->d_resid, hist.size() * sizeof(double), cudaMemcpyDeviceToHost);
        const double sn = std::sqrt(src_sumsq) > 0.0 ? std::sqrt(src_sumsq) : 1.0;
        std::printf("\n**************************************************\n");
        std::printf("*       MCLS: Monte Carlo Linear Solvers         *\n");
        std::printf("**************************************************\n\n");
        std::printf("                     MCSA                         \n\n");
        std::printf("%18s%18s\n", "Iteration", "|r|_2 / |b|_2");
        const int pf = mp->print_freq > 0 ? mp->print_freq : 10;
        for (int i = 0; i < (int)hist.size(); ++i)
            if ((i + 1) % pf == 0 || i + 1 == st.iter)
                std::printf("%18d%18.4e\n", i + 1, hist[i] / sn);
        std::printf("\n**************************************************\n\n");
    }
    if (stats) {
        if ((rc = read_stats(dom, stats))) return rc;
        stats->iterations = st.iter;
        stats->converged = st.converged;
        stats->residual_norm = st.rnorm;
        const double sn = std::sqrt(src_sumsq);
        stats->achieved_tol = sn > 0.0 ? st.rnorm / sn : st.rnorm;  // achievedTol (:142-173)
        stats->solve_ms = ms;
        stats->fallback_taken = dom->left ? dom->left->fallback : 0;
        // kernels of the captured iterations plus the set-up launches
        // (source norm, initial residual and norm, state init)
        stats->kernel_launches = int64_t(dom->body_kernels) * st.iter + 9;
        stats->rho = dom->left ? dom->left->rho : -1.0;
    }
    return MCLSGPU_OK;
}

// ---- multi-set loop pieces (multiset.cu) ------------------------------------
// Start of an MCSA loop on dom->x and dom->b: |PL b|_2, the initial
// preconditioned residual and its norm, the loop state.
void mcsa_loop_begin(mclsgpu_domain* dom, const double* b_dev, const double* x_dev,
                     const mclsgpu_mcsa_params* mp) {
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    const int n = dom->n;
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s);
    reset_counters(dom);
    if (b_dev != dom->b)
        cudaMemcpyAsync(dom->b, b_dev, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (x_dev != dom->x)
        cudaMemcpyAsync(dom->x, x_dev, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
    const double* pb = dom->b;
    if (dom->left) {
        spmv(s, dom->left->P, dom->b, dom->tmp);
        pb = dom->tmp;
    }
    sum_sq(s, pb, n, dom->part, dom->d_scalars + 6);
    update_prec_residual(dom, dom->x, dom->b, dom->rp);
    sum_sq(s, dom->rp, n, dom->part, dom->d_scalars + 5);
    k_mcsa_init<<<1, 1, 0, s>>>(dom->d_state, dom->d_scalars + 6, mp->tolerance, mp->check_freq,
                                mp->max_iters, dom->d_scalars + 5);
}

// The convergence check on |rp|_2 (d_scalars[5]), ending a device-side loop
// through `handle` when use_cond.
void mcsa_loop_check(mclsgpu_domain* dom, cudaGraphConditionalHandle handle, int use_cond) {
    cudaStream_t s = dom->ctx->stream;
    if (use_cond)
        k_mcsa_check<<<1, 1, 0, s>>>(dom->d_state, dom->d_scalars + 5, dom->d_resid,
                                     dom->resid_cap, dom->ctx->d_status, handle);
    else
        k_mcsa_check_host<<<1, 1, 0, s>>>(dom->d_state, dom->d_scalars + 5, dom->d_resid,
                                           dom->resid_cap, dom->ctx->d_status);
}

// End of the loop: x_dev = PR x, the loop state and the statistics.
int mcsa_loop_finish(mclsgpu_domain* dom, double* x_dev, float ms, int kernels_per_iter,
                     mclsgpu_stats* stats) {
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    const size_t bytes = size_t(dom->n) * sizeof(double);
    if (dom->right) {
        spmv(s, dom->right->P, dom->x, dom->tmp);
        cudaMemcpyAsync(x_dev, dom->tmp, bytes, cudaMemcpyDeviceToDevice, s);
    } else if (x_dev != dom->x) {
        cudaMemcpyAsync(x_dev, dom->x, bytes, cudaMemcpyDeviceToDevice, s);
    }
    cudaMemcpyAsync(dom->h_state, dom->d_state, sizeof(McsaState), cudaMemcpyDeviceToHost, s);
    double src_sumsq = 0.0;
    cudaMemcpyAsync(&src_sumsq, dom->d_scalars + 6, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "mcsa loop");
    int rc = check_device_status(ctx);
    if (rc) return rc;
    const McsaState st = *dom->h_state;
    if (stats) {
        if ((rc = read_stats(dom, stats))) return rc;
        stats->iterations = st.iter;
        stats->converged = st.converged;
        stats->residual_norm = st.rnorm;
        const double sn = std::sqrt(src_sumsq);
        stats->achieved_tol = sn > 0.0 ? st.rnorm / sn : st.rnorm;
        stats->solve_ms = ms;
        stats->fallback_taken = dom->left ? dom->left->fallback : 0;
        stats->kernel_launches = int64_t(kernels_per_iter) * st.iter;
        stats->rho = dom->left ? dom->left->rho : -1.0;
    }
    return MCLSGPU_OK;
}

}  // namespace mclsgpu

using namespace mclsgpu;

static int check_mcsa_params(mclsgpu_domain* dom, const mclsgpu_mcsa_params* p,
                             mclsgpu_mcsa_params* out);

namespace mclsgpu {
int mcsa_check_params(mclsgpu_domain* dom, const mclsgpu_mcsa_params* p,
                      mclsgpu_mcsa_params* out) {
    return check_mcsa_params(dom, p, out);
}
}  // namespace mclsgpu

static int check_mcsa_params(mclsgpu_domain* dom, const mclsgpu_mcsa_params* p,
                             mclsgpu_mcsa_params* out) {
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
            return set_error(dom->ctx, MCLSGPU_ERR_INVALID_ARG, "mcsa params: size mismatch");
        d = *p;
    }
    if (d.max_iters < 1 || d.check_freq < 1 || d.smoother_steps < 0 || !(d.tolerance >= 0.0))
        return set_error(dom->ctx, MCLSGPU_ERR_INVALID_ARG, "mcsa params out of range");
    if (d.fixed_point_type < MCLSGPU_FIXED_POINT_RICHARDSON ||
        d.fixed_point_type > MCLSGPU_FIXED_POINT_RNSD)
        return set_error(dom->ctx, MCLSGPU_ERR_INVALID_ARG, "Iteration type not supported!");
    *out = d;
    return MCLSGPU_OK;
}

extern "C" {

int mclsgpu_mc_solve_dev(mclsgpu_domain* dom, const double* rhs_dev, double* x_dev, int internal,
                         mclsgpu_stats* stats) {
    if (!dom || !rhs_dev || !x_dev) return MCLSGPU_ERR_INVALID_ARG;
    return mc_solve_device(dom, rhs_dev, x_dev, internal, 0, nullptr, nullptr, nullptr, nullptr,
                           stats);
}

int mclsgpu_mc_solve(mclsgpu_domain* dom, const double* rhs, double* x, int internal,
                     mclsgpu_stats* stats) {
    if (!dom || !rhs || !x) return MCLSGPU_ERR_INVALID_ARG;
    cudaStream_t s = dom->ctx->stream;
    const size_t bytes = size_t(dom->n) * sizeof(double);
    cudaMemcpyAsync(dom->b, rhs, bytes, cudaMemcpyHostToDevice, s);
    int rc = mc_solve_device(dom, dom->b, dom->x, internal, 0, nullptr, nullptr, nullptr, nullptr,
                             stats);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyAsync(x, dom->x, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(dom->ctx, e, "mc_solve copy-out");
}

int mclsgpu_mc_trace(mclsgpu_domain* dom, const double* rhs, double* x, int internal,
                     int64_t max_trace, int64_t* states, double* final_weight, int32_t* events,
                     int64_t* start_state, int64_t* num_histories) {
    if (!dom || !rhs || !x || max_trace < 0) return MCLSGPU_ERR_INVALID_ARG;
    if (dom->p.precision != MCLSGPU_FP64)
        return set_error(dom->ctx, MCLSGPU_ERR_UNSUPPORTED, "trace needs the FP64 walk");
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    const int L = dom->p.history_length;
    const size_t bytes = size_t(dom->n) * sizeof(double);
    long long *d_states = nullptr, *d_start = nullptr;
    double* d_w = nullptr;
    int* d_ev = nullptr;
    cudaError_t e;
    if (max_trace > 0) {
        if ((e = dmalloc(&d_states, size_t(max_trace) * (L + 1))) != cudaSuccess ||
            (e = dmalloc(&d_start, size_t(max_trace))) != cudaSuccess ||
            (e = dmalloc(&d_w, size_t(max_trace))) != cudaSuccess ||
            (e = dmalloc(&d_ev, size_t(max_trace))) != cudaSuccess) {
            dfree(d_states); dfree(d_start); dfree(d_w); dfree(d_ev);
            return cuda_fail(ctx, e, "cudaMalloc trace");
        }
    }
    cudaMemcpyAsync(dom->b, rhs, bytes, cudaMemcpyHostToDevice, s);
    int rc = mc_solve_device(dom, dom->b, dom->x, internal, max_trace, d_states, d_w, d_ev, d_start,
                             nullptr);
    if (!rc) {
        int nh = 0;
        cudaMemcpyAsync(&nh, dom->d_nh, sizeof(int), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(x, dom->x, bytes, cudaMemcpyDeviceToHost, s);
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "trace copy-out");
        if (!rc) {
            long long k = nh < max_trace ? nh : max_trace;
            if (num_histories) *num_histories = nh;
            if (k > 0) {
                if (states)
                    cudaMemcpy(states, d_states, size_t(k) * (L + 1) * sizeof(long long),
                               cudaMemcpyDeviceToHost);
                if (start_state)
                    cudaMemcpy(start_state, d_start, size_t(k) * sizeof(long long),
                               cudaMemcpyDeviceToHost);
                if (final_weight)
                    cudaMemcpy(final_weight, d_w, size_t(k) * sizeof(double), cudaMemcpyDeviceToHost);
                if (events) cudaMemcpy(events, d_ev, size_t(k) * sizeof(int), cudaMemcpyDeviceToHost);
            }
        }
    }
    dfree(d_states); dfree(d_start); dfree(d_w); dfree(d_ev);
    return rc;
}

int mclsgpu_mcsa_solve_dev(mclsgpu_domain* dom, const double* b_dev, double* x_dev,
                           const mclsgpu_mcsa_params* params, mclsgpu_stats* stats) {
    if (!dom || !b_dev || !x_dev) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_mcsa_params p;
    int rc = check_mcsa_params(dom, params, &p);
    if (rc) return rc;
    return mcsa_solve_device(dom, b_dev, x_dev, &p, stats);
}

int mclsgpu_mcsa_begin(mclsgpu_domain* dom, const double* b_dev, const double* x0_dev,
                       const mclsgpu_mcsa_params* params, double* rnorm, double* bnorm) {
    if (!dom || !b_dev || !x0_dev) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_mcsa_params p;
    int rc = check_mcsa_params(dom, params, &p);
    if (rc) return rc;
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    const int n = dom->n;
    if ((rc = prepare_fixed_point(dom, p.fixed_point_type))) return rc;
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s);
    cudaMemsetAsync(dom->d_ticket, 0, sizeof(unsigned int), s);
    reset_counters(dom);
    if (b_dev != dom->b) cudaMemcpyAsync(dom->b, b_dev, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (x0_dev != dom->x) cudaMemcpyAsync(dom->x, x0_dev, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
    // |PL b|_2 and the initial preconditioned residual
    // (src/MCLS_MCSASolverManager_impl.hpp:299-346).
    const double* pb = dom->b;
    if (dom->left) {
        spmv(s, dom->left->P, dom->b, dom->tmp);
        pb = dom->tmp;
    }
    sum_sq(s, pb, n, dom->part, dom->d_scalars + 6);
    update_prec_residual(dom, dom->x, dom->b, dom->rp);
    sum_sq(s, dom->rp, n, dom->part, dom->d_scalars + 5);
    double h[2] = {0.0, 0.0};
    cudaMemcpyAsync(h, dom->d_scalars + 5, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "mcsa begin");
    if ((rc = check_device_status(ctx))) return rc;
    if (rnorm) *rnorm = std::sqrt(h[0]);
    if (bnorm) *bnorm = std::sqrt(h[1]);
    dom->step_p = p;
    dom->step_ready = 1;
    return MCLSGPU_OK;
}

int mclsgpu_mcsa_correction(mclsgpu_domain* dom, double* delta_dev) {
    if (!dom || !delta_dev) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = dom->ctx;
    if (!dom->step_ready)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "mclsgpu_mcsa_begin first");
    cudaStream_t s = ctx->stream;
    const mclsgpu_mcsa_params& p = dom->step_p;
    for (int l = 0; l < p.smoother_steps; ++l)
        enqueue_fixed_point_step(dom, p.fixed_point_type, p.richardson_omega);
    // The residual problem's source is already left preconditioned.
    enqueue_mc(dom, dom->rp, delta_dev, 0, 0, nullptr, nullptr, nullptr, nullptr);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "mcsa correction");
    return check_device_status(ctx);
}

int mclsgpu_mcsa_apply(mclsgpu_domain* dom, const double* delta_dev, double scale,
                       double* rnorm) {
    if (!dom || !delta_dev) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = dom->ctx;
    if (!dom->step_ready)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "mclsgpu_mcsa_begin first");
    cudaStream_t s = ctx->stream;
    const int n = dom->n;
    k_richardson<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(dom->x, delta_dev, n, scale);
    update_prec_residual(dom, dom->x, dom->b, dom->rp);
    sum_sq(s, dom->rp, n, dom->part, dom->d_scalars + 5);
    double h = 0.0;
    cudaMemcpyAsync(&h, dom->d_scalars + 5, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "mcsa apply");
    int rc = check_device_status(ctx);
    if (rc) return rc;
    if (!std::isfinite(h)) return set_error(ctx, MCLSGPU_ERR_DIVERGED, "non-finite residual");
    if (rnorm) *rnorm = std::sqrt(h);
    return MCLSGPU_OK;
}

int mclsgpu_mcsa_finish(mclsgpu_domain* dom, double* x_dev, mclsgpu_stats* stats) {
    if (!dom || !x_dev) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = dom->ctx;
    if (!dom->step_ready)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "mclsgpu_mcsa_begin first");
    cudaStream_t s = ctx->stream;
    const size_t bytes = size_t(dom->n) * sizeof(double);
    if (dom->right) {
        spmv(s, dom->right->P, dom->x, dom->tmp);  // right-preconditioner recovery
        cudaMemcpyAsync(x_dev, dom->tmp, bytes, cudaMemcpyDeviceToDevice, s);
    } else if (x_dev != dom->x) {
        cudaMemcpyAsync(x_dev, dom->x, bytes, cudaMemcpyDeviceToDevice, s);
    }
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "mcsa finish");
    dom->step_ready = 0;
    return stats ? read_stats(dom, stats) : MCLSGPU_OK;
}

int mclsgpu_domain_residual(mclsgpu_domain* dom, double* rp_dev) {
    if (!dom || !rp_dev || !dom->rp) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = dom->ctx;
    cudaError_t e = cudaMemcpyAsync(rp_dev, dom->rp, size_t(dom->n) * sizeof(double),
                                    cudaMemcpyDeviceToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(ctx, e, "domain residual");
}

int mclsgpu_domain_set_launch(mclsgpu_domain* dom, int histories_per_lane, int block_size) {
    if (!dom ||
        (histories_per_lane != 1 && histories_per_lane != 2 && histories_per_lane != 4 &&
         histories_per_lane != 8) ||
        (block_size != 128 && block_size != 256))
        return MCLSGPU_ERR_INVALID_ARG;
    dom->walk_ilp = histories_per_lane;
    dom->walk_block = block_size;
    prepare_walk(dom);
    dom->graph_key = -1;  // the launch shape is baked into the captured loop
    return MCLSGPU_OK;
}

int mclsgpu_domain_set_record_cache(mclsgpu_domain* dom, int allocate_l1) {
    if (!dom || (allocate_l1 != 0 && allocate_l1 != 1)) return MCLSGPU_ERR_INVALID_ARG;
    dom->walk_l1 = allocate_l1;
    dom->graph_key = -1;  // baked into the captured loop
    if (dom->set_graph) {
        cudaGraphExecDestroy(dom->set_graph);
        dom->set_graph = nullptr;
    }
    return MCLSGPU_OK;
}

int mclsgpu_domain_autotune(mclsgpu_domain* dom, const double* rhs_dev, int reps,
                            int* histories_per_lane, int* block_size, double* walk_ms) {
    if (!dom || !rhs_dev || reps < 1) return MCLSGPU_ERR_INVALID_ARG;
    if (dom->p.precision != MCLSGPU_FP32)
        return set_error(dom->ctx, MCLSGPU_ERR_UNSUPPORTED, "autotune applies to FP32 walks");
    cudaStream_t s = dom->ctx->stream;
    unsigned long long saved[2] = {0, 0};
    cudaMemcpyAsync(&saved[0], dom->d_epoch, sizeof(saved[0]), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&saved[1], dom->d_pos, sizeof(saved[1]), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(dom->ctx, e, "autotune");
    // Four or eight histories per lane apply to fixed-length histories on
    // 32-byte records only.
    const bool four = dom->slots == 4 && !(dom->p.weight_cutoff > 0.0);
    // Each shape with the record loads bypassing L1 and allocated in it.
    const int shapes[16][3] = {{1, 256, 0}, {2, 256, 0}, {1, 128, 0}, {2, 128, 0},
                               {4, 256, 0}, {4, 128, 0}, {8, 256, 0}, {8, 128, 0},
                               {1, 256, 1}, {2, 256, 1}, {1, 128, 1}, {2, 128, 1},
                               {4, 256, 1}, {4, 128, 1}, {8, 256, 1}, {8, 128, 1}};
    double best = 1e300;
    int bh = 1, bb = 256, bl = 0;
    for (const auto& sh : shapes) {
        if (sh[0] >= 4 && !four) continue;
        int rc = mclsgpu_domain_set_launch(dom, sh[0], sh[1]);
        if (!rc) rc = mclsgpu_domain_set_record_cache(dom, sh[2]);
        if (rc) return rc;
        mclsgpu_stats st{};
        st.size = sizeof(st);
        rc = mc_solve_device(dom, rhs_dev, dom->tmp2, 1, 0, nullptr, nullptr, nullptr, nullptr,
                             &st);  // warm-up
        double tot = 0.0;
        for (int r = 0; r < reps && !rc; ++r) {
            rc = mc_solve_device(dom, rhs_dev, dom->tmp2, 1, 0, nullptr, nullptr, nullptr,
                                 nullptr, &st);
            tot += st.walk_ms;
        }
        if (rc) return rc;
        if (tot / reps < best) {
            best = tot / reps;
            bh = sh[0];
            bb = sh[1];
            bl = sh[2];
        }
    }
    int rc = mclsgpu_domain_set_launch(dom, bh, bb);
    if (!rc) rc = mclsgpu_domain_set_record_cache(dom, bl);
    cudaMemcpyAsync(dom->d_epoch, &saved[0], sizeof(saved[0]), cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dom->d_pos, &saved[1], sizeof(saved[1]), cudaMemcpyHostToDevice, s);
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(dom->ctx, e, "autotune");
    if (histories_per_lane) *histories_per_lane = bh;
    if (block_size) *block_size = bb;
    if (walk_ms) *walk_ms = best;
    return rc;
}

int mclsgpu_mcsa_solve(mclsgpu_domain* dom, const double* b, double* x,
                       const mclsgpu_mcsa_params* params, mclsgpu_stats* stats) {
    if (!dom || !b || !x) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_mcsa_params p;
    int rc = check_mcsa_params(dom, params, &p);
    if (rc) return rc;
    cudaStream_t s = dom->ctx->stream;
    const size_t bytes = size_t(dom->n) * sizeof(double);
    cudaMemcpyAsync(dom->b, b, bytes, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dom->x, x, bytes, cudaMemcpyHostToDevice, s);
    rc = mcsa_solve_device(dom, dom->b, dom->x, &p, stats);
    if (rc) return rc;
    cudaError_t e = cudaMemcpyAsync(x, dom->x, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(dom->ctx, e, "mcsa copy-out");
}

}  // extern "C"
