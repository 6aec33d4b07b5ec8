// anderson.cu -- Anderson-accelerated MCSA on the device.
//
// AndersonSolverManager (src/MCLS_AndersonSolverManager_impl.hpp:65-284)
// hands the MCSAModelEvaluator fixed-point map
// (src/MCLS_MCSAModelEvaluator_impl.hpp:306-350) to NOX's Anderson solver.
// NOX is not part of the reference tree; the acceleration follows Walker &
// Ni, "Anderson acceleration for fixed-point iterations", SIAM J. Numer.
// Anal. 49 (2011): x_{k+1} = x_k + beta F_k - (dX + beta dF) gamma with
// gamma the least-squares fit of F_k by the stored differences dF, solved
// through a QR factorisation of dF that is updated as columns are added
// (modified Gram-Schmidt) and dropped (Givens rotations).
//
// One step on the device, all inside a captured graph with a WHILE node:
//   smoothing + residual (one fused pass), the Monte Carlo correction,
//   first pass     F = f + delta - x and |F|^2; when a column is added also
//                  the drop's rotations on Q, v = F - F_old, dX = x - x_old
//                  and r = <q_0, v> (|v|^2 for an empty store)
//   MGS passes     one per further stored column: v -= r q_{j-1},
//                  r = <q_j, v> (|v|^2 after the last)
//   control        R's new diagonal; optional drops for the condition number
//   RHS pass       q_new = v / |v|, post-add rotations, <F, q_j>; the last
//                  block back-solves R gamma = Q^T F
//   update pass    x = x + beta F - sum (gamma_j dX_j + beta (R gamma)_j q_j)
//   residual       rp = PL (b - A x), |rp|_2, the status test, and (one
//                  thread) the plan of the next step: whether it adds a
//                  column and which one it drops first.
// The passes move two elements per thread access (16 bytes).  Q and dX hold
// storage_depth columns each at a stride rounded up to 32 elements; dX is a
// ring indexed from the device state, so the captured graph never changes.
#include <cmath>
#include <type_traits>
#include <vector>

#include "internal.h"

namespace mclsgpu {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxDepth = 16;
constexpr int kMaxRot = kMaxDepth * kMaxDepth;

struct AaState {
    int k;            // steps taken (NOX's iteration count)
    int nstore;       // stored columns
    int add;          // this step adds a column
    int newcol;       // its index
    int ok;           // the new column was kept (nonzero norm)
    int nrot;         // Givens rotations waiting for the next Q pass
    int dx_head;      // ring slot of the oldest dX column
    int done;
    int converged;
    int max_iters;
    int m;            // storage depth
    int start;        // acceleration start iteration
    int adjust;       // drop columns for the condition number
    int pad;
    double beta;
    double droptol;
    double crit;      // tolerance * |b|_2
    double bnorm;
    double rnorm;     // |PL (b - A x)|_2 at the current iterate
    double fnorm2;    // |F|^2 of this step
    double vnorm2;    // |v|^2 after Gram-Schmidt
    double inv_rnn;   // 1 / R(new, new)
    double R[kMaxDepth][kMaxDepth];
    double rc[kMaxRot], rs[kMaxRot];
    int ri[kMaxRot];
    double gamma[kMaxDepth];
    double rgamma[kMaxDepth];
};

struct Args {
    int n;
    size_t ld;             // column stride of Q and dX (n rounded up to 32)
    const double* f;       // smoothed iterate
    const double* delta;   // Monte Carlo correction (summed over the sets)
    double dscale;         // 1 / number of sets
    double* x;
    double* F;
    double* Fold;
    double* xold;
    double* V;
    double* Q;             // [m][ld]
    double* DX;            // [m][ld] ring
    const double* rp;      // residual at the updated iterate
    double* part;
    unsigned int* ticket;
    AaState* st;
    double* hist;
    int hist_cap;
    int* status;
    cudaGraphConditionalHandle handle;
    int use_cond;
};

inline int grid_for(long long work, int cap) {
    long long g = (work + kThreads - 1) / kThreads;
    if (g < 1) g = 1;
    return int(g > cap ? cap : g);
}

// W consecutive elements (W = 2: one 16-byte access; W = 1: the odd tail).
template <int W>
struct Vec {
    double v[W];
};
template <int W>
__device__ __forceinline__ Vec<W> ldv(const double* p, int i) {
    Vec<W> r;
    if constexpr (W == 2) {
        const double2 t = *reinterpret_cast<const double2*>(p + i);
        r.v[0] = t.x;
        r.v[1] = t.y;
    } else {
        r.v[0] = p[i];
    }
    return r;
}
template <int W>
__device__ __forceinline__ void stv(double* p, int i, const Vec<W>& r) {
    if constexpr (W == 2)
        *reinterpret_cast<double2*>(p + i) = make_double2(r.v[0], r.v[1]);
    else
        p[i] = r.v[0];
}

// body(integral_constant<int, W>, i) over the elements: pairs grid-stride,
// then the odd last element in the last thread of the grid.
template <class Body>
__device__ __forceinline__ void for_elements(int n, Body body) {
    const int np = n >> 1;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < np; p += gridDim.x * blockDim.x)
        body(std::integral_constant<int, 2>{}, 2 * p);
    if ((n & 1) && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1)
        body(std::integral_constant<int, 1>{}, n - 1);
}

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

// Publish this block's sums of v0 and v1; true in the block that finishes
// last, whose thread 0 then holds the grid totals (block order, fixed for a
// fixed launch).
__device__ __forceinline__ bool grid_sum2(double v0, double v1, const Args& a, double* t0,
                                          double* t1) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool last;
    const double s0 = block_sum(v0, sh);
    const double s1 = block_sum(v1, sh);
    if (threadIdx.x == 0) {
        a.part[2 * blockIdx.x] = s0;
        a.part[2 * blockIdx.x + 1] = s1;
        __threadfence();
        last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double u0 = 0.0, u1 = 0.0;
    for (int k = threadIdx.x; k < int(gridDim.x); k += blockDim.x) {
        u0 += a.part[2 * k];
        u1 += a.part[2 * k + 1];
    }
    const double r0 = block_sum(u0, sh);
    const double r1 = block_sum(u1, sh);
    if (threadIdx.x == 0) {
        *t0 = r0;
        *t1 = r1;
        *a.ticket = 0u;
    }
    return true;
}

// Drop the oldest column (one thread): rotations that restore R's triangle
// after its first column is removed, recorded for the next Q pass.
__device__ void qr_delete(AaState* st) {
    const int N = st->nstore;
    for (int i = 0; i + 1 < N; ++i) {
        const double a = st->R[i][i + 1], b = st->R[i + 1][i + 1];
        const double t = sqrt(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)));
        const double c = a / t, s = b / t;
        st->R[i][i + 1] = t;
        st->R[i + 1][i + 1] = 0.0;
        for (int j = i + 2; j < N; ++j) {
            const double u = __dadd_rn(__dmul_rn(c, st->R[i][j]), __dmul_rn(s, st->R[i + 1][j]));
            st->R[i + 1][j] =
                __dadd_rn(__dmul_rn(-s, st->R[i][j]), __dmul_rn(c, st->R[i + 1][j]));
            st->R[i][j] = u;
        }
        const int r = st->nrot++;
        st->ri[r] = i;
        st->rc[r] = c;
        st->rs[r] = s;
    }
    for (int i = 0; i < N; ++i)
        for (int j = 0; j + 1 < N; ++j) st->R[i][j] = st->R[i][j + 1];
    for (int i = 0; i < N; ++i) st->R[i][N - 1] = 0.0;
    st->nstore = N - 1;
    st->dx_head = (st->dx_head + 1) % st->m;
}

// Reciprocal 1-norm condition number of the stored R (one thread).
__device__ double rcond(const AaState* st) {
    const int N = st->nstore;
    double Ri[kMaxDepth][kMaxDepth];
    for (int j = 0; j < N; ++j)
        for (int i = j; i >= 0; --i) {
            double s = i == j ? 1.0 : 0.0;
            for (int k = i + 1; k <= j; ++k) s = __dadd_rn(s, -__dmul_rn(st->R[i][k], Ri[k][j]));
            Ri[i][j] = s / st->R[i][i];
        }
    double n1 = 0.0, ni = 0.0;
    for (int j = 0; j < N; ++j) {
        double x = 0.0, y = 0.0;
        for (int i = 0; i <= j; ++i) {
            x += fabs(st->R[i][j]);
            y += fabs(Ri[i][j]);
        }
        n1 = fmax(n1, x);
        ni = fmax(ni, y);
    }
    return 1.0 / (n1 * ni);
}

// What step k does with the store (one thread): from the start iteration on
// it adds a column, first dropping the oldest when the store is full.
__device__ void plan(AaState* st) {
    st->nrot = 0;
    st->add = 0;
    st->ok = 0;
    if (st->m > 0 && st->k >= st->start) {
        if (st->k == st->start) {
            st->nstore = 0;
            st->dx_head = 0;
        } else if (st->nstore == st->m) {
            qr_delete(st);
        }
        st->add = 1;
        st->newcol = st->nstore;
    }
}

// Apply the recorded rotations to elements i..i+W-1 of the Q columns.
template <int W>
__device__ __forceinline__ void rotate_q(const Args& a, const AaState* st, int nrot, int i) {
    for (int r = 0; r < nrot; ++r) {
        const int c0 = st->ri[r];
        const double c = st->rc[r], s = st->rs[r];
        double* qa = a.Q + size_t(c0) * a.ld;
        double* qb = qa + a.ld;
        const Vec<W> u = ldv<W>(qa, i), v = ldv<W>(qb, i);
        Vec<W> ua, vb;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            ua.v[w] = __dadd_rn(__dmul_rn(c, u.v[w]), __dmul_rn(s, v.v[w]));
            vb.v[w] = __dadd_rn(__dmul_rn(-s, u.v[w]), __dmul_rn(c, v.v[w]));
        }
        stv<W>(qa, i, ua);
        stv<W>(qb, i, vb);
    }
}

__global__ void k_aa_init(AaState* st, int max_iters, int m, int start, int adjust, double beta,
                          double droptol, double tol, const double* b_sumsq,
                          const double* r_sumsq, int* status) {
    AaState s;
    memset(&s, 0, sizeof(s));
    s.max_iters = max_iters;
    s.m = m;
    s.start = start;
    s.adjust = adjust;
    s.beta = beta;
    s.droptol = droptol;
    s.bnorm = sqrt(*b_sumsq);
    s.crit = tol * s.bnorm;
    s.rnorm = sqrt(*r_sumsq);
    s.converged = s.rnorm < s.crit;
    if (!isfinite(s.rnorm)) atomicOr(status, DEV_ERR_NONFINITE);
    s.done = s.converged || !isfinite(s.rnorm);
    plan(&s);
    *st = s;
}

// First pass of a step: F = (f + delta) - x and |F|^2; when the step adds a
// column also the drop's rotations on Q, v = F - F_old, dX = x - x_old and
// the first Gram-Schmidt product <q_0, v> (|v|^2 for an empty store).
__global__ void __launch_bounds__(kThreads) k_aa_first(Args a) {
    const AaState* st = a.st;
    const int add = st->add, nc = st->newcol, nrot = st->nrot;
    double* dxn = add ? a.DX + size_t((st->dx_head + nc) % st->m) * a.ld : nullptr;
    const double* __restrict__ f = a.f;
    const double* __restrict__ dl = a.delta;
    double accF = 0.0, accV = 0.0;
    for_elements(a.n, [&](auto wt, int i) {
        constexpr int W = decltype(wt)::value;
        const Vec<W> fv = ldv<W>(f, i), dv = ldv<W>(dl, i), xv = ldv<W>(a.x, i);
        Vec<W> Fv;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            Fv.v[w] = __dadd_rn(__dadd_rn(fv.v[w], __dmul_rn(a.dscale, dv.v[w])), -xv.v[w]);
            accF = fma(Fv.v[w], Fv.v[w], accF);
        }
        stv<W>(a.F, i, Fv);
        if (!add) return;
        if (nrot) rotate_q<W>(a, st, nrot, i);
        const Vec<W> Fo = ldv<W>(a.Fold, i), xo = ldv<W>(a.xold, i);
        Vec<W> v, dx;
#pragma unroll
        for (int w = 0; w < W; ++w) {
            v.v[w] = __dadd_rn(Fv.v[w], -Fo.v[w]);
            dx.v[w] = __dadd_rn(xv.v[w], -xo.v[w]);
        }
        stv<W>(a.V, i, v);
        stv<W>(dxn, i, dx);
        if (nc > 0) {
            const Vec<W> q = ldv<W>(a.Q, i);
#pragma unroll
            for (int w = 0; w < W; ++w) accV = fma(q.v[w], v.v[w], accV);
        } else {
#pragma unroll
            for (int w = 0; w < W; ++w) accV = fma(v.v[w], v.v[w], accV);
        }
    });
    double tF, tV;
    if (!grid_sum2(accF, accV, a, &tF, &tV) || threadIdx.x != 0) return;
    AaState* sw = a.st;
    sw->fnorm2 = tF;
    if (add) {
        if (nc > 0)
            sw->R[0][nc] = tV;
        else
            sw->vnorm2 = tV;
    }
}

// Gram-Schmidt pass j >= 1 of the new column (modified Gram-Schmidt: one
// stored column per pass): v -= R(j-1, new) q_{j-1}; R(j, new) = <q_j, v>,
// or |v|^2 after the last stored column.
__global__ void __launch_bounds__(kThreads) k_aa_mgs(Args a, int j) {
    const AaState* st = a.st;
    const int add = st->add, nc = st->newcol;
    if (!add || j > nc) return;  // the same in every block
    const double r_prev = st->R[j - 1][nc];
    const double* __restrict__ qprev = a.Q + size_t(j - 1) * a.ld;
    const double* __restrict__ qj = j < nc ? a.Q + size_t(j) * a.ld : nullptr;
    double* __restrict__ V = a.V;
    double acc = 0.0;
    for_elements(a.n, [&](auto wt, int i) {
        constexpr int W = decltype(wt)::value;
        const Vec<W> vo = ldv<W>(V, i), qp = ldv<W>(qprev, i);
        Vec<W> v;
#pragma unroll
        for (int w = 0; w < W; ++w) v.v[w] = __dadd_rn(vo.v[w], __dmul_rn(-r_prev, qp.v[w]));
        stv<W>(V, i, v);
        if (qj) {
            const Vec<W> q = ldv<W>(qj, i);
#pragma unroll
            for (int w = 0; w < W; ++w) acc = fma(q.v[w], v.v[w], acc);
        } else {
#pragma unroll
            for (int w = 0; w < W; ++w) acc = fma(v.v[w], v.v[w], acc);
        }
    });
    double t, unused;
    if (!grid_sum2(acc, 0.0, a, &t, &unused) || threadIdx.x != 0) return;
    if (j < nc)
        a.st->R[j][nc] = t;
    else
        a.st->vnorm2 = t;
}

// New diagonal entry of R, then the drops for the condition number.
__global__ void k_aa_ctrl(AaState* st) {
    st->nrot = 0;
    st->ok = 0;
    if (st->add) {
        const int nc = st->newcol;
        const double rn = sqrt(st->vnorm2);
        if (rn > 0.0 && isfinite(rn)) {
            st->R[nc][nc] = rn;
            st->inv_rnn = 1.0 / rn;
            st->nstore = nc + 1;
            st->ok = 1;
        } else {
            for (int j = 0; j < nc; ++j) st->R[j][nc] = 0.0;
        }
    }
    if (st->adjust)
        while (st->nstore > 1 && rcond(st) < st->droptol) qr_delete(st);
}

// q_new = v / |v|, the post-add rotations, <F, q_j>; the last block solves
// R gamma = Q^T F and forms beta R gamma.  MD >= the storage depth bounds the
// per-thread accumulators (registers, hence occupancy).
template <int MD>
__global__ void __launch_bounds__(kThreads) k_aa_rhs(Args a) {
    __shared__ double sh[kThreads / 32];
    __shared__ bool last;
    __shared__ double rhs[kMaxDepth];
    AaState* st = a.st;
    const int N = st->nstore, ok = st->ok, nc = st->newcol, nrot = st->nrot;
    const double inv = st->inv_rnn;
    double acc[MD];
#pragma unroll
    for (int j = 0; j < MD; ++j) acc[j] = 0.0;
    double* qn = a.Q + size_t(nc) * a.ld;
    for_elements(a.n, [&](auto wt, int i) {
        constexpr int W = decltype(wt)::value;
        if (ok) {
            const Vec<W> v = ldv<W>(a.V, i);
            Vec<W> q;
#pragma unroll
            for (int w = 0; w < W; ++w) q.v[w] = __dmul_rn(inv, v.v[w]);
            stv<W>(qn, i, q);
        }
        if (nrot) rotate_q<W>(a, st, nrot, i);
        const Vec<W> F = ldv<W>(a.F, i);
#pragma unroll
        for (int j = 0; j < MD; ++j)
            if (j < N) {
                const Vec<W> q = ldv<W>(a.Q + size_t(j) * a.ld, i);
#pragma unroll
                for (int w = 0; w < W; ++w) acc[j] = fma(F.v[w], q.v[w], acc[j]);
            }
    });
#pragma unroll
    for (int j = 0; j < MD; ++j) {
        if (j < N) {  // N is the same in every thread of the block
            const double t = block_sum(acc[j], sh);
            if (threadIdx.x == 0) a.part[size_t(blockIdx.x) * kMaxDepth + j] = t;
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int j = 0; j < N; ++j) {
        double u = 0.0;
        for (int k = threadIdx.x; k < int(gridDim.x); k += blockDim.x)
            u += a.part[size_t(k) * kMaxDepth + j];
        const double t = block_sum(u, sh);
        if (threadIdx.x == 0) rhs[j] = t;
    }
    if (threadIdx.x != 0) return;
    *a.ticket = 0u;
    for (int j = N - 1; j >= 0; --j) {
        double g = rhs[j];
        for (int i = j + 1; i < N; ++i) g = __dadd_rn(g, -__dmul_rn(st->R[j][i], st->gamma[i]));
        st->gamma[j] = g / st->R[j][j];
    }
    for (int i = 0; i < N; ++i) {
        double s = 0.0;
        for (int j = i; j < N; ++j) s = __dadd_rn(s, __dmul_rn(st->R[i][j], st->gamma[j]));
        st->rgamma[i] = __dmul_rn(st->beta, s);
    }
    st->nrot = 0;
}

// x_{k+1} = x_k + beta F - sum_j (gamma_j dX_j + (beta R gamma)_j q_j);
// x_old = x_k, F_old = F.  The coefficients and the ring slots of dX sit in
// shared memory, so the thread keeps only its loads in flight.
__global__ void __launch_bounds__(kThreads) k_aa_update(Args a) {
    __shared__ double sg[kMaxDepth], srg[kMaxDepth];
    __shared__ const double* sdx[kMaxDepth];
    const AaState* st = a.st;
    const int N = st->nstore;
    const double beta = st->beta;
    if (threadIdx.x < N) {
        const int j = threadIdx.x;
        sg[j] = st->gamma[j];
        srg[j] = st->rgamma[j];
        sdx[j] = a.DX + size_t((st->dx_head + j) % st->m) * a.ld;
    }
    __syncthreads();
    for_elements(a.n, [&](auto wt, int i) {
        constexpr int W = decltype(wt)::value;
        const Vec<W> xv = ldv<W>(a.x, i), F = ldv<W>(a.F, i);
        Vec<W> w;
#pragma unroll
        for (int e = 0; e < W; ++e) w.v[e] = __dmul_rn(beta, F.v[e]);
#pragma unroll 4
        for (int j = 0; j < N; ++j) {
            const Vec<W> d = ldv<W>(sdx[j], i), q = ldv<W>(a.Q + size_t(j) * a.ld, i);
            const double g = sg[j], rg = srg[j];
#pragma unroll
            for (int e = 0; e < W; ++e)
                w.v[e] = __dadd_rn(__dadd_rn(w.v[e], __dmul_rn(-g, d.v[e])),
                                   __dmul_rn(-rg, q.v[e]));
        }
        Vec<W> xn;
#pragma unroll
        for (int e = 0; e < W; ++e) xn.v[e] = __dadd_rn(xv.v[e], w.v[e]);
        stv<W>(a.xold, i, xv);
        stv<W>(a.Fold, i, F);
        stv<W>(a.x, i, xn);
    });
}

// |rp|_2 and the status tests (MCSAStatusTest, MaxIters, FiniteValue); the
// last block also plans the next step.
__global__ void __launch_bounds__(kThreads) k_aa_check(Args a) {
    double acc = 0.0;
    const double* __restrict__ rp = a.rp;
    for_elements(a.n, [&](auto wt, int i) {
        constexpr int W = decltype(wt)::value;
        const Vec<W> r = ldv<W>(rp, i);
#pragma unroll
        for (int w = 0; w < W; ++w) acc = fma(r.v[w], r.v[w], acc);
    });
    double total, unused;
    if (!grid_sum2(acc, 0.0, a, &total, &unused) || threadIdx.x != 0) return;
    AaState* st = a.st;
    st->k += 1;
    st->rnorm = sqrt(total);
    if (a.hist && st->k <= a.hist_cap) a.hist[st->k - 1] = st->rnorm;
    st->converged = st->rnorm < st->crit;
    if (!isfinite(st->rnorm) || !isfinite(st->fnorm2)) atomicOr(a.status, DEV_ERR_NONFINITE);
    const int keep = !st->converged && st->k < st->max_iters && !*a.status;
    st->done = !keep;
    plan(st);
    if (a.use_cond) cudaGraphSetConditional(a.handle, keep ? 1u : 0u);
}

__global__ void k_axpy1(double* x, const double* r, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = __dadd_rn(x[i], r[i]);
}

int check_params(mclsgpu_context* ctx, const mclsgpu_anderson_params* p,
                 mclsgpu_anderson_params* out) {
    mclsgpu_anderson_params d{};
    d.size = sizeof(d);
    d.max_iters = 1000;
    d.tolerance = 1.0e-8;
    d.smoother_steps = 1;
    d.storage_depth = 2;
    d.mixing = 1.0;
    d.start_iteration = 1;
    d.drop_tolerance = 1.0e-12;
    if (p) {
        if (p->size < sizeof(mclsgpu_anderson_params))
            return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "anderson params: size mismatch");
        d = *p;
    }
    if (d.max_iters < 1 || d.smoother_steps < 0 || !(d.tolerance >= 0.0) ||
        d.storage_depth < 0 || d.storage_depth > kMaxDepth || d.start_iteration < 1 ||
        !std::isfinite(d.mixing))
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "anderson params out of range");
    *out = d;
    return MCLSGPU_OK;
}

}  // namespace

struct AndersonWork {
    int n = 0;
    int m = 0;
    int grid = 1;
    size_t ld = 0;
    double* F = nullptr;
    double* Fold = nullptr;
    double* xold = nullptr;
    double* V = nullptr;
    double* delta = nullptr;
    double* Q = nullptr;
    double* DX = nullptr;
    double* part = nullptr;
    unsigned int* ticket = nullptr;
    AaState* st = nullptr;
    AaState* h_st = nullptr;
    cudaGraphExec_t graph = nullptr;
    long long graph_key = -1;
    const double* graph_hist = nullptr;  // residual history the graph writes
    int body_kernels = 0;
    // Step-wise solves (mclsgpu_anderson_begin .. _finish).
    mclsgpu_anderson_params step_p{};
    const double* step_f = nullptr;      // smoothed iterate of the pending step
    ~AndersonWork() {
        dfree(F);
        dfree(Fold);
        dfree(xold);
        dfree(V);
        dfree(delta);
        dfree(Q);
        dfree(DX);
        dfree(part);
        dfree(ticket);
        dfree(st);
        if (h_st) cudaFreeHost(h_st);
        if (graph) cudaGraphExecDestroy(graph);
    }
};

void release_anderson(mclsgpu_domain* dom) {
    delete dom->aa;
    dom->aa = nullptr;
}

namespace {

int ensure_work(mclsgpu_domain* dom, int m) {
    mclsgpu_context* ctx = dom->ctx;
    const int mm = m > 0 ? m : 1;
    if (dom->aa && dom->aa->m >= mm) return MCLSGPU_OK;
    release_anderson(dom);
    AndersonWork* w = new AndersonWork;
    w->n = dom->n;
    w->m = mm;
    w->grid = grid_for((dom->n + 1) / 2, ctx->num_sms * 8);
    w->ld = (size_t(dom->n) + 31) & ~size_t(31);
    const size_t n = size_t(dom->n);
    cudaError_t e;
    if ((e = dmalloc(&w->F, n)) != cudaSuccess || (e = dmalloc(&w->Fold, n)) != cudaSuccess ||
        (e = dmalloc(&w->xold, n)) != cudaSuccess || (e = dmalloc(&w->V, n)) != cudaSuccess ||
        (e = dmalloc(&w->delta, n)) != cudaSuccess || (e = dmalloc(&w->Q, w->ld * mm)) != cudaSuccess ||
        (e = dmalloc(&w->DX, w->ld * mm)) != cudaSuccess ||
        (e = dmalloc(&w->part, size_t(w->grid) * kMaxDepth)) != cudaSuccess ||
        (e = dmalloc(&w->ticket, 1)) != cudaSuccess || (e = dmalloc(&w->st, 1)) != cudaSuccess ||
        (e = cudaMallocHost(reinterpret_cast<void**>(&w->h_st), sizeof(AaState))) != cudaSuccess) {
        delete w;
        return cuda_fail(ctx, e, "cudaMalloc anderson work space");
    }
    cudaMemsetAsync(w->ticket, 0, sizeof(unsigned int), ctx->stream);
    dom->aa = w;
    return MCLSGPU_OK;
}

// The map's evaluation (MCSAModelEvaluator::evalModelImpl, :318-345):
// f = x, "Smoother Steps" steps f += r, r = PL (b - A f), then this set's
// Monte Carlo correction of the residual problem into delta.  Returns f.
const double* enqueue_eval(mclsgpu_domain* dom, const mclsgpu_anderson_params* p,
                           double* delta) {
    cudaStream_t s = dom->ctx->stream;
    AndersonWork* w = dom->aa;
    const int n = dom->n;
    const double* f = dom->x;
    const double* r = dom->rp;
    if (p->smoother_steps == 1) {
        richardson_residual(dom, dom->x, dom->rp, 1.0, dom->x2, dom->rp2);
        f = dom->x2;
        r = dom->rp2;
    } else if (p->smoother_steps > 1) {
        cudaMemcpyAsync(dom->x2, dom->x, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(dom->rp2, dom->rp, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice,
                        s);
        for (int l = 0; l < p->smoother_steps; ++l) {
            k_axpy1<<<w->grid, kThreads, 0, s>>>(dom->x2, dom->rp2, n);
            prec_residual(dom, dom->x2, dom->b, dom->rp2);
        }
        f = dom->x2;
        r = dom->rp2;
    }
    mc_correction(dom, r, delta);
    return f;
}

// The accelerated update from F = f + dscale * delta - x, the new residual
// and the status test.
void enqueue_accel(mclsgpu_domain* dom, const mclsgpu_anderson_params* p, const double* f,
                   const double* delta, double dscale, cudaGraphConditionalHandle h,
                   int use_cond) {
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    AndersonWork* w = dom->aa;
    Args a{};
    a.n = dom->n;
    a.ld = w->ld;
    a.f = f;
    a.delta = delta;
    a.dscale = dscale;
    a.x = dom->x;
    a.F = w->F;
    a.Fold = w->Fold;
    a.xold = w->xold;
    a.V = w->V;
    a.Q = w->Q;
    a.DX = w->DX;
    a.rp = dom->rp;
    a.part = w->part;
    a.ticket = w->ticket;
    a.st = w->st;
    a.hist = dom->d_resid;
    a.hist_cap = dom->resid_cap;
    a.status = ctx->d_status;
    a.handle = h;
    a.use_cond = use_cond;
    k_aa_first<<<w->grid, kThreads, 0, s>>>(a);
    if (p->storage_depth > 0) {
        for (int j = 1; j < p->storage_depth; ++j) k_aa_mgs<<<w->grid, kThreads, 0, s>>>(a, j);
        k_aa_ctrl<<<1, 1, 0, s>>>(w->st);
        if (p->storage_depth <= 4)
            k_aa_rhs<4><<<w->grid, kThreads, 0, s>>>(a);
        else if (p->storage_depth <= 8)
            k_aa_rhs<8><<<w->grid, kThreads, 0, s>>>(a);
        else
            k_aa_rhs<kMaxDepth><<<w->grid, kThreads, 0, s>>>(a);
    }
    k_aa_update<<<w->grid, kThreads, 0, s>>>(a);
    prec_residual(dom, dom->x, dom->b, dom->rp);
    k_aa_check<<<w->grid, kThreads, 0, s>>>(a);
}

// One Anderson step and its status test (captured into the graph body).
void enqueue_step(mclsgpu_domain* dom, const mclsgpu_anderson_params* p,
                  cudaGraphConditionalHandle h, int use_cond) {
    const double* f = enqueue_eval(dom, p, dom->aa->delta);
    enqueue_accel(dom, p, f, dom->aa->delta, 1.0, h, use_cond);
}

// Work space and residual history buffer for a solve with these parameters.
int anderson_prepare(mclsgpu_domain* dom, const mclsgpu_anderson_params* p) {
    mclsgpu_context* ctx = dom->ctx;
    if (dom->right)
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED,
                         "the Anderson solver applies the left preconditioner only");
    int rc = ensure_work(dom, p->storage_depth);
    if (rc) return rc;
    if (p->max_iters > dom->resid_cap) {
        cudaStreamSynchronize(ctx->stream);
        dfree(dom->d_resid);
        cudaError_t e = dmalloc(&dom->d_resid, size_t(p->max_iters));
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
        dom->resid_cap = p->max_iters;
        // The captured MCSA graph holds the old history pointer.
        if (dom->graph) cudaGraphExecDestroy(dom->graph);
        dom->graph = nullptr;
    }
    return MCLSGPU_OK;
}

// Counters, b and x0, the initial residual and state (the status test on
// x0).  Leaves the state copying to the host, not synced.
void anderson_begin(mclsgpu_domain* dom, const double* b_dev, const double* x_dev,
                    const mclsgpu_anderson_params* p) {
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    const int n = dom->n;
    AndersonWork* w = dom->aa;
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s);
    cudaMemsetAsync(w->ticket, 0, sizeof(unsigned int), s);
    mcsa_reset_counters(dom);
    if (b_dev != dom->b)
        cudaMemcpyAsync(dom->b, b_dev, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (x_dev != dom->x)
        cudaMemcpyAsync(dom->x, x_dev, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
    // |b|_2 (MCSAStatusTest uses the unpreconditioned right-hand side) and
    // the residual of the initial guess, tested before the first step.
    sum_sq(s, dom->b, n, dom->part, dom->d_scalars + 6);
    prec_residual(dom, dom->x, dom->b, dom->rp);
    sum_sq(s, dom->rp, n, dom->part, dom->d_scalars + 5);
    k_aa_init<<<1, 1, 0, s>>>(w->st, p->max_iters, p->storage_depth, p->start_iteration,
                              p->adjust_condition, p->mixing, p->drop_tolerance, p->tolerance,
                              dom->d_scalars + 6, dom->d_scalars + 5, ctx->d_status);
    cudaMemcpyAsync(w->h_st, w->st, sizeof(AaState), cudaMemcpyDeviceToHost, s);
}

void fill_stats(mclsgpu_domain* dom, const AaState& st, double ms, mclsgpu_stats* stats) {
    AndersonWork* w = dom->aa;
    stats->iterations = st.k;
    stats->converged = st.converged;
    stats->residual_norm = st.rnorm;
    stats->achieved_tol = st.bnorm > 0.0 ? st.rnorm / st.bnorm : st.rnorm;
    stats->solve_ms = ms;
    stats->fallback_taken = dom->left ? dom->left->fallback : 0;
    stats->rho = dom->left ? dom->left->rho : -1.0;
    stats->kernel_launches = int64_t(w->body_kernels) * st.k + 4;
}

int anderson_solve(mclsgpu_domain* dom, const double* b_dev, double* x_dev,
                   const mclsgpu_anderson_params* p, mclsgpu_stats* stats) {
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    const int n = dom->n;
    int rc = anderson_prepare(dom, p);
    if (rc) return rc;
    AndersonWork* w = dom->aa;
    const long long key = (long long)p->smoother_steps * 64 + p->storage_depth;
    // Variable-length reference-stream walks synchronise with the host.
    const bool host_loop = p->host_loop || walk_needs_rounds(dom);
    if (!host_loop && (!w->graph || w->graph_key != key || w->graph_hist != dom->d_resid)) {
        if (w->graph) cudaGraphExecDestroy(w->graph);
        w->graph = nullptr;
        rc = build_while_graph(
            ctx, [&](cudaGraphConditionalHandle h) { enqueue_step(dom, p, h, 1); }, &w->graph,
            &w->body_kernels);
        if (rc) return rc;
        w->graph_key = key;
        w->graph_hist = dom->d_resid;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    anderson_begin(dom, b_dev, x_dev, p);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && !w->h_st->done) {
        if (!host_loop) {
            e = cudaGraphLaunch(w->graph, s);
        } else {
            for (int it = 0; it < p->max_iters && e == cudaSuccess; ++it) {
                enqueue_step(dom, p, cudaGraphConditionalHandle(0), 0);
                cudaMemcpyAsync(w->h_st, w->st, sizeof(AaState), cudaMemcpyDeviceToHost, s);
                e = cudaStreamSynchronize(s);
                if (e == cudaSuccess && w->h_st->done) break;
            }
        }
    }
    if (e == cudaSuccess) {
        if (x_dev != dom->x)
            cudaMemcpyAsync(x_dev, dom->x, size_t(n) * sizeof(double), cudaMemcpyDeviceToDevice, s);
        cudaEventRecord(e1, s);
        cudaMemcpyAsync(w->h_st, w->st, sizeof(AaState), cudaMemcpyDeviceToHost, s);
        e = cudaStreamSynchronize(s);
    }
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "anderson solve");
    if ((rc = check_device_status(ctx))) return rc;
    if (stats) {
        if ((rc = mcsa_read_stats(dom, stats))) return rc;
        fill_stats(dom, *w->h_st, ms, stats);
    }
    return MCLSGPU_OK;
}

}  // namespace

void anderson_drop_graph(mclsgpu_domain* dom) {
    if (dom->aa && dom->aa->graph) {
        cudaGraphExecDestroy(dom->aa->graph);
        dom->aa->graph = nullptr;
    }
}

}  // namespace mclsgpu

using namespace mclsgpu;

extern "C" {

int mclsgpu_anderson_solve_dev(mclsgpu_domain* dom, const double* b_dev, double* x_dev,
                               const mclsgpu_anderson_params* params, mclsgpu_stats* stats) {
    if (!dom || !b_dev || !x_dev) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_anderson_params p;
    int rc = check_params(dom->ctx, params, &p);
    if (rc) return rc;
    cudaSetDevice(dom->ctx->device);
    return anderson_solve(dom, b_dev, x_dev, &p, stats);
}

int mclsgpu_anderson_begin(mclsgpu_domain* dom, const double* b_dev, const double* x0_dev,
                           const mclsgpu_anderson_params* params, double* rnorm, double* bnorm,
                           int32_t* done) {
    if (!dom || !b_dev || !x0_dev) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_anderson_params p;
    int rc = check_params(dom->ctx, params, &p);
    if (rc) return rc;
    cudaSetDevice(dom->ctx->device);
    dom->aa_step_ready = 0;
    if ((rc = anderson_prepare(dom, &p))) return rc;
    anderson_begin(dom, b_dev, x0_dev, &p);
    cudaError_t e = cudaStreamSynchronize(dom->ctx->stream);
    if (e != cudaSuccess) return cuda_fail(dom->ctx, e, "anderson begin");
    if ((rc = check_device_status(dom->ctx))) return rc;
    const AaState& st = *dom->aa->h_st;
    if (rnorm) *rnorm = st.rnorm;
    if (bnorm) *bnorm = st.bnorm;
    if (done) *done = st.done;
    dom->aa->step_p = p;
    dom->aa_step_ready = 1;
    return MCLSGPU_OK;
}

int mclsgpu_anderson_correction(mclsgpu_domain* dom, double* delta_dev) {
    if (!dom || !delta_dev) return MCLSGPU_ERR_INVALID_ARG;
    if (!dom->aa_step_ready)
        return set_error(dom->ctx, MCLSGPU_ERR_INVALID_ARG, "mclsgpu_anderson_begin first");
    AndersonWork* w = dom->aa;
    w->step_f = enqueue_eval(dom, &w->step_p, delta_dev);
    cudaError_t e = cudaStreamSynchronize(dom->ctx->stream);
    if (e != cudaSuccess) return cuda_fail(dom->ctx, e, "anderson correction");
    return check_device_status(dom->ctx);
}

int mclsgpu_anderson_apply(mclsgpu_domain* dom, const double* delta_dev, double scale,
                           double* rnorm, int32_t* done) {
    if (!dom || !delta_dev) return MCLSGPU_ERR_INVALID_ARG;
    if (!dom->aa_step_ready || !dom->aa->step_f)
        return set_error(dom->ctx, MCLSGPU_ERR_INVALID_ARG,
                         "mclsgpu_anderson_correction first");
    AndersonWork* w = dom->aa;
    cudaStream_t s = dom->ctx->stream;
    enqueue_accel(dom, &w->step_p, w->step_f, delta_dev, scale, cudaGraphConditionalHandle(0), 0);
    w->step_f = nullptr;
    cudaMemcpyAsync(w->h_st, w->st, sizeof(AaState), cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(dom->ctx, e, "anderson apply");
    int rc = check_device_status(dom->ctx);
    if (rc) return rc;
    if (rnorm) *rnorm = w->h_st->rnorm;
    if (done) *done = w->h_st->done;
    return MCLSGPU_OK;
}

int mclsgpu_anderson_finish(mclsgpu_domain* dom, double* x_dev, mclsgpu_stats* stats) {
    if (!dom || !x_dev) return MCLSGPU_ERR_INVALID_ARG;
    if (!dom->aa_step_ready)
        return set_error(dom->ctx, MCLSGPU_ERR_INVALID_ARG, "mclsgpu_anderson_begin first");
    cudaStream_t s = dom->ctx->stream;
    if (x_dev != dom->x)
        cudaMemcpyAsync(x_dev, dom->x, size_t(dom->n) * sizeof(double), cudaMemcpyDeviceToDevice,
                        s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(dom->ctx, e, "anderson finish");
    dom->aa_step_ready = 0;
    if (!stats) return MCLSGPU_OK;
    int rc = mcsa_read_stats(dom, stats);
    if (!rc) fill_stats(dom, *dom->aa->h_st, 0.0, stats);
    return rc;
}

int mclsgpu_anderson_solve(mclsgpu_domain* dom, const double* b, double* x,
                           const mclsgpu_anderson_params* params, mclsgpu_stats* stats) {
    if (!dom || !b || !x) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = dom->ctx;
    cudaSetDevice(ctx->device);
    const size_t bytes = size_t(dom->n) * sizeof(double);
    // The domain's own vectors hold b and x for the solve.
    cudaMemcpyAsync(dom->b, b, bytes, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(dom->x, x, bytes, cudaMemcpyHostToDevice, ctx->stream);
    int rc = mclsgpu_anderson_solve_dev(dom, dom->b, dom->x, params, stats);
    if (!rc) {
        cudaMemcpyAsync(x, dom->x, bytes, cudaMemcpyDeviceToHost, ctx->stream);
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "copy x");
    }
    return rc;
}

}  // extern "C"
