// batch.cu -- many systems and many right-hand sides in one MCSA loop.
//
// m systems A_s (uneven sizes) with R_s right-hand sides each are solved
// together: the block-diagonal operator S = diag(A_1..A_m) carries one
// point-Jacobi domain H = I - D^-1 S (walks never leave a block).  System s
// gets W_s = R_s rounded up to a power of two columns; the systems are
// grouped by W_s into five width classes (1, 2, 4, 8, 16 columns), each a
// contiguous range of rows whose vectors are row-major [rows][W] blocks of
// the element arrays (BatchClasses), so a system with one right-hand side
// costs one column, not the widest system's sixteen.  Forward walks do not
// depend on the source, so one set of histories per iteration serves every
// right-hand side of every system: each history carries one tally per column
// of its row's class (walk32_batch).  Every (system, rhs) pair has its own
// convergence test |rp_{s,r}|_2 <= tol |D^-1 b_{s,r}|_2 (the
// MCSASolverManager criterion, src/MCLS_MCSASolverManager_impl.hpp:299-318);
// a system whose pairs have all met it stops (its rows and walks are
// skipped), and the loop ends when every pair has met it or at the iteration
// limit.  One iteration is four kernels in a CUDA graph whose WHILE node the
// last one controls: Richardson step + residual, tally source, the shared
// walk, and correction + residual + per-pair norms, whose last block to
// finish runs the convergence test.
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "internal.h"

namespace mclsgpu {
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

struct BatchArgs {
    int nsys;
    int pw;              // per-pair row width: pair (s, r) is s * pw + r
    int per;             // histories per row
    const int* rp;       // S (CSR)
    const int* ci;
    const double* v;
    const double* dinv;  // D^-1
    const int* hrp;      // H rows (forward domain, FP64)
    const int* hci;
    const double* hv;
    // Per system: first row, first element, log2 of its width, rows.
    const int* srow0;
    const long long* seoff;
    const int* slog;
    const int* sn;
    const int* sorder;   // the systems in placement order
    // The systems this launch works on: lsys[k] for k < *lcount, their
    // elements at [lecum[k], lecum[k+1]) of the launch's element space.
    const int* lsys;
    const long long* lecum;
    const int* lcount;
    // The active list the convergence test rebuilds (the iteration's list).
    int* act_sys;
    long long* act_ecum;
    int* act_hcum;
    int* act_count;
    const double* B;
    double* X;
    double* X2;
    double* RP;
    double* RP2;
    double* Y;
    float* cR;
    double* norm2;       // [nsys][pw]
    double* bnorm2;
    int* conv_iter;      // [nsys][pw]
    const int* nrhs;
    int* sys_done;       // per system: every right-hand side converged
    BatchState* st;
    unsigned* blocks_done;
    double omega;        // Richardson relaxation
    double nomega;       // Neumann relaxation (1 when absent)
    double inv_per;      // 1 / histories per state
    int ev;              // expected-value estimator
    unsigned long long* d_epoch;
    int* d_counter;
    unsigned long long* d_tim;
    int* status;
};

// One element of a launch's element space: system s, row i, column r, log2
// width c, its index e in the element arrays and the element index of its
// row's column 0 minus the row times the width (so that the element of row j,
// column r of the same system is base + (j << c) + r).
struct Elem {
    int s, i, r, c;
    size_t e;
    long long base;
};

// The list entry k with lecum[k] <= t < lecum[k+1] (count >= 1 entries).
__device__ __forceinline__ int elem_entry(const long long* lecum, int count, long long t) {
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (lecum[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// A thread's position in the launch's list: entry k and its system's fields,
// reloaded only when the thread's element crosses into the next entry (the
// elements a thread visits only increase).
struct Cursor {
    int k, s, c, row0;
    long long lo, hi, eoff;
    __device__ __forceinline__ void load(const BatchArgs& a, int kk) {
        k = kk;
        s = a.lsys[k];
        c = a.slog[s];
        row0 = a.srow0[s];
        eoff = a.seoff[s];
        lo = a.lecum[k];
        hi = a.lecum[k + 1];
    }
    // Element t (lo <= t after the first call; t < lecum[count]).
    __device__ __forceinline__ Elem at(const BatchArgs& a, long long t) {
        while (t >= hi) load(a, k + 1);
        Elem q;
        q.s = s;
        q.c = c;
        const long long local = t - lo;
        q.i = row0 + int(local >> c);
        q.r = int(local & ((1 << c) - 1));
        q.e = size_t(eoff + local);
        q.base = eoff - ((long long)row0 << c);
        return q;
    }
};

// Loop over the launch's elements: each block takes one contiguous range in
// tiles of blockDim elements; the block's first thread finds the list entry
// of the range's first element, and every thread steps its own cursor
// forward from there.  body(live, q) runs on every thread of the block for
// every tile (block-uniform trip count, so body may use warp collectives).
template <class Body>
__device__ __forceinline__ void for_elements(const BatchArgs& a, Body body) {
    __shared__ int s_k0;
    const int count = *a.lcount;
    const long long total = count > 0 ? a.lecum[count] : 0;
    const long long T = blockDim.x;
    const long long span = ((total + gridDim.x - 1) / gridDim.x + T - 1) / T * T;
    const long long beg = (long long)blockIdx.x * span;
    const long long end = beg + span < total ? beg + span : total;
    if (beg >= end) return;  // the whole block
    if (threadIdx.x == 0) s_k0 = elem_entry(a.lecum, count, beg);
    __syncthreads();
    Cursor cur;
    cur.load(a, s_k0);
    for (long long base = beg; base < end; base += T) {
        const long long t = base + threadIdx.x;
        const bool live = t < end;
        Elem q{};
        if (live) q = cur.at(a, t);
        body(live, q);
    }
}

// x2 = x + w rp;  rp2 = D^-1 (b - S x2), with x2 at the neighbours formed on
// the fly (RichardsonIteration::doOneIteration then updatePrecResidual,
// src/MCLS_RichardsonIteration_impl.hpp:134-147); the walk tallies Y are
// cleared for this iteration's walk.
__global__ void __launch_bounds__(kThreads, 8) k_b_richardson_residual(BatchArgs a) {
    for_elements(a, [&](bool live, const Elem& q) {
        if (!live) return;
        double acc = 0.0;
        for (int p = a.rp[q.i]; p < a.rp[q.i + 1]; ++p) {
            const size_t k = size_t(q.base + ((long long)a.ci[p] << q.c) + q.r);
            acc = fma(a.v[p], __dadd_rn(a.X[k], __dmul_rn(a.omega, a.RP[k])), acc);
        }
        a.X2[q.e] = __dadd_rn(a.X[q.e], __dmul_rn(a.omega, a.RP[q.e]));
        a.RP2[q.e] = a.dinv[q.i] * (a.B[q.e] - acc);
        a.Y[q.e] = 0.0;
    });
}

// Tally source of every right-hand side: expected value c = H (w rp2),
// collision c = w rp2 (FP32).
__global__ void __launch_bounds__(kThreads, 8) k_b_source(BatchArgs a) {
    for_elements(a, [&](bool live, const Elem& q) {
        if (!live) return;
        double v;
        if (a.ev) {
            v = 0.0;
            for (int p = a.hrp[q.i]; p < a.hrp[q.i + 1]; ++p)
                v = fma(a.hv[p], a.RP2[size_t(q.base + ((long long)a.hci[p] << q.c) + q.r)], v);
        } else {
            v = a.RP2[q.e];
        }
        a.cR[q.e] = __double2float_rn(a.nomega * v);
    });
}

// The corrected iterate at element k: x2 + Y / per (+ w rp2 for the expected
// value, the estimator's source term; ForwardTally::finalize,
// src/MCLS_ForwardTally_impl.hpp:180-209).
__device__ __forceinline__ double corrected(const BatchArgs& a, size_t k) {
    double d = a.Y[k] * a.inv_per;
    if (a.ev) d += a.nomega * a.RP2[k];
    return a.X2[k] + d;
}

// The active list from sys_done, in placement order, by one block: each
// thread counts a contiguous run of systems, a block scan places the runs.
__device__ void build_active(const BatchArgs& a) {
    __shared__ int s_cnt[1024];
    __shared__ long long s_el[1024];
    __shared__ int s_h[1024];
    const int T = blockDim.x, tid = threadIdx.x;
    const int seg = (a.nsys + T - 1) / T;
    const int j0 = min(tid * seg, a.nsys), j1 = min(j0 + seg, a.nsys);
    int cnt = 0, hs = 0;
    long long el = 0;
    for (int j = j0; j < j1; ++j) {
        const int s = a.sorder[j];
        if (a.sys_done[s]) continue;
        ++cnt;
        el += (long long)a.sn[s] << a.slog[s];
        hs += a.sn[s] * a.per;
    }
    s_cnt[tid] = cnt;
    s_el[tid] = el;
    s_h[tid] = hs;
    __syncthreads();
    for (int d = 1; d < T; d <<= 1) {  // inclusive scan (Hillis-Steele)
        int c2 = 0, h2 = 0;
        long long e2 = 0;
        if (tid >= d) {
            c2 = s_cnt[tid - d];
            e2 = s_el[tid - d];
            h2 = s_h[tid - d];
        }
        __syncthreads();
        s_cnt[tid] += c2;
        s_el[tid] += e2;
        s_h[tid] += h2;
        __syncthreads();
    }
    int k = s_cnt[tid] - cnt;
    long long eo = s_el[tid] - el;
    int ho = s_h[tid] - hs;
    for (int j = j0; j < j1; ++j) {
        const int s = a.sorder[j];
        if (a.sys_done[s]) continue;
        a.act_sys[k] = s;
        a.act_ecum[k] = eo;
        a.act_hcum[k] = ho;
        eo += (long long)a.sn[s] << a.slog[s];
        ho += a.sn[s] * a.per;
        ++k;
    }
    if (tid == T - 1) {
        *a.act_count = s_cnt[tid];
        a.act_ecum[s_cnt[tid]] = s_el[tid];
        a.act_hcum[s_cnt[tid]] = s_h[tid];
    }
}

// Per-pair convergence, loop control and the per-iteration bookkeeping (new
// stream epoch, work-queue reset, walk timing, norms cleared, the active
// list rebuilt), run by one block.
__device__ void batch_check(const BatchArgs& a, int use_cond, cudaGraphConditionalHandle handle) {
    __shared__ int s_conv;
    if (threadIdx.x == 0) s_conv = 0;
    __syncthreads();
    BatchState st = *a.st;
    const int it = st.iter + 1;
    const bool check = (it % st.check_freq) == 0 || it >= st.max_iters;
    int conv = 0;
    for (int q = threadIdx.x; q < a.nsys * a.pw; q += blockDim.x) {
        const int s = q / a.pw, r = q % a.pw;
        if (r >= a.nrhs[s]) continue;
        const double nr = __ldcg(&a.norm2[q]);
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
        for (int r = 0; r < a.nrhs[s]; ++r) all &= a.conv_iter[size_t(s) * a.pw + r] >= 0;
        a.sys_done[s] = all;
    }
    __syncthreads();
    build_active(a);
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

// Per-(system, column) sums of squares of one tile: a warp whose 32
// elements all belong to one system reduces the lanes of each column with
// shuffles and its lanes r < W keep the column sums in registers (a lane's
// column stays the same from tile to tile while its system does), adding
// them into the global sums only when the lane's system changes or the loop
// ends; a warp that straddles systems adds each lane's square directly.
struct PairSums {
    double* sums;   // [nsys][pw]
    int pw;
    int s = -1, r = 0;
    double v = 0.0;
    __device__ __forceinline__ void flush() {
        if (s >= 0 && v != 0.0) atomicAdd(&sums[size_t(s) * pw + r], v);
        s = -1;
        v = 0.0;
    }
    __device__ __forceinline__ void add(int sys, int c, int rr, double sq) {
        const unsigned full = 0xffffffffu;
        const int s0 = __shfl_sync(full, sys, 0);
        const int c0 = __shfl_sync(full, c, 0);
        if (__all_sync(full, sys == s0) && s0 >= 0) {
            double x = sq;
            for (int d = 16; d >= (1 << c0); d >>= 1) x += __shfl_xor_sync(full, x, d);
            if ((threadIdx.x & 31) < (1 << c0)) {
                if (s != s0 || r != rr) {
                    flush();
                    s = s0;
                    r = rr;
                }
                v += x;
            }
        } else if (sys >= 0 && sq != 0.0) {
            atomicAdd(&sums[size_t(sys) * pw + rr], sq);
        }
    }
};

// rp = D^-1 (b - S x) and the per-(system, rhs) sums of squares.  CORR: x is
// this iteration's corrected iterate (formed on the fly at the neighbours
// and written to X), otherwise Xin.  CHECK: the last block to finish runs
// the convergence test (the other blocks' sums are complete and visible by
// then).
template <bool CORR, bool CHECK>
__global__ void __launch_bounds__(kThreads, 6) k_b_update(BatchArgs a, const double* Xin, int use_cond,
                                                       cudaGraphConditionalHandle handle) {
    PairSums ps{a.norm2, a.pw};
    for_elements(a, [&](bool live, const Elem& q) {
        double sq = 0.0;
        if (live) {
            double acc = 0.0;
            for (int p = a.rp[q.i]; p < a.rp[q.i + 1]; ++p) {
                const size_t k = size_t(q.base + ((long long)a.ci[p] << q.c) + q.r);
                acc = fma(a.v[p], CORR ? corrected(a, k) : Xin[k], acc);
            }
            if (CORR) a.X[q.e] = corrected(a, q.e);
            const double rv = a.dinv[q.i] * (a.B[q.e] - acc);
            a.RP[q.e] = rv;
            sq = rv * rv;
        }
        ps.add(live ? q.s : -1, q.c, q.r, sq);
    });
    ps.flush();
    if (CHECK) {
        __shared__ bool s_last;
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) s_last = atomicAdd(a.blocks_done, 1u) == gridDim.x - 1;
        __syncthreads();
        if (s_last) {
            __threadfence();
            batch_check(a, use_cond, handle);
            if (threadIdx.x == 0) *a.blocks_done = 0u;
        }
    }
}

// Before the loop: sums of squares of D^-1 b per pair (every system).
__global__ void k_b_init_norms(BatchArgs a) {
    PairSums ps{a.bnorm2, a.pw};
    for_elements(a, [&](bool live, const Elem& q) {
        const double v = live ? a.dinv[q.i] * a.B[q.e] : 0.0;
        ps.add(live ? q.s : -1, q.c, q.r, v * v);
    });
    ps.flush();
}

// Loop state, per-pair bookkeeping and the active list (every system), by
// one block.
__global__ void k_b_state_init(BatchArgs a, int max_iters, int check_freq, double tol,
                               int pairs) {
    const int count = a.nsys * a.pw;
    for (int q = threadIdx.x; q < count; q += blockDim.x) {
        a.conv_iter[q] = -1;
        a.norm2[q] = 0.0;
    }
    for (int q = threadIdx.x; q < a.nsys; q += blockDim.x) a.sys_done[q] = 0;
    __syncthreads();
    build_active(a);
    if (threadIdx.x == 0) {
        BatchState s{};
        s.max_iters = max_iters;
        s.check_freq = check_freq;
        s.tol = tol;
        s.pairs = pairs;
        *a.st = s;
    }
}

}  // namespace
}  // namespace mclsgpu


struct mclsgpu_batch {
    mclsgpu_context* ctx = nullptr;
    int nsys = 0;
    int pw = 1;                    // widest system's width (per-pair arrays)
    int n = 0;                     // rows
    long long ne = 0;              // elements (padding included)
    mclsgpu::BatchClasses cls{};
    std::vector<int64_t> row0;     // system -> its first row (placement order)
    std::vector<int64_t> eoff;     // system -> its first element
    std::vector<int> width;        // system -> its width (power of two)
    std::vector<int> nrhs;
    mclsgpu_operator* op = nullptr;
    mclsgpu_precond* pc = nullptr;
    mclsgpu_domain* dom = nullptr;
    int* d_nrhs = nullptr;
    // Per system (device): first row, first element, log2 width, rows, and
    // the systems in placement order.
    int* d_srow0 = nullptr;
    long long* d_seoff = nullptr;
    int* d_slog = nullptr;
    int* d_sn = nullptr;
    int* d_sorder = nullptr;
    // The active list (rebuilt every iteration) and the list of every system.
    int* act_sys = nullptr;
    long long* act_ecum = nullptr;
    int* act_hcum = nullptr;
    int* act_count = nullptr;
    int* all_sys = nullptr;
    long long* all_ecum = nullptr;
    int* all_count = nullptr;
    double *X = nullptr, *X2 = nullptr, *RP = nullptr, *RP2 = nullptr, *B = nullptr, *Y = nullptr;
    float* cR = nullptr;
    double* norm2 = nullptr;
    double* bnorm2 = nullptr;
    int* conv_iter = nullptr;
    int* sys_done = nullptr;
    unsigned* blocks_done = nullptr;
    mclsgpu::BatchState* d_state = nullptr;
    mclsgpu::BatchState* h_state = nullptr;
    cudaGraphExec_t graph = nullptr;
    long long graph_key = -1;
    uint64_t graph_seed = 0;       // the domain seed the captured walks carry
    int body_kernels = 0;
    int per = 1;
    int grab = 1;                  // walk work-queue grab, in 32-history chunks
    // Grids of the element kernels: every block resident at once (each block
    // takes one contiguous range, so a second wave would double the time).
    int g_rich = 1, g_src = 1, g_upd = 1, g_upd0 = 1, g_init = 1;
};

namespace mclsgpu {
namespace {

void batch_release(mclsgpu_batch* b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->dom) mclsgpu_domain_destroy(b->dom);
    if (b->pc) mclsgpu_precond_destroy(b->pc);
    if (b->op) mclsgpu_operator_destroy(b->op);
    dfree(b->d_nrhs);
    dfree(b->d_srow0);
    dfree(b->d_seoff);
    dfree(b->d_slog);
    dfree(b->d_sn);
    dfree(b->d_sorder);
    dfree(b->act_sys);
    dfree(b->act_ecum);
    dfree(b->act_hcum);
    dfree(b->act_count);
    dfree(b->all_sys);
    dfree(b->all_ecum);
    dfree(b->all_count);
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
    dfree(b->blocks_done);
    dfree(b->d_state);
    if (b->h_state) cudaFreeHost(b->h_state);
    delete b;
}

// Kernel arguments over the active list (all = false) or every system.
BatchArgs batch_args(mclsgpu_batch* b, const mclsgpu_mcsa_params* mp, bool all) {
    const mclsgpu_mc_params& p = b->dom->p;
    BatchArgs a{};
    a.nsys = b->nsys;
    a.pw = b->pw;
    a.per = b->per;
    a.rp = b->op->A.rp;
    a.ci = b->op->A.ci;
    a.v = b->op->A.v;
    a.dinv = b->pc->diag;
    a.hrp = b->dom->D.rp;
    a.hci = b->dom->D.ci;
    a.hv = b->dom->D.v;
    a.srow0 = b->d_srow0;
    a.seoff = b->d_seoff;
    a.slog = b->d_slog;
    a.sn = b->d_sn;
    a.sorder = b->d_sorder;
    a.lsys = all ? b->all_sys : b->act_sys;
    a.lecum = all ? b->all_ecum : b->act_ecum;
    a.lcount = all ? b->all_count : b->act_count;
    a.act_sys = b->act_sys;
    a.act_ecum = b->act_ecum;
    a.act_hcum = b->act_hcum;
    a.act_count = b->act_count;
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
    a.st = b->d_state;
    a.blocks_done = b->blocks_done;
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

template <class K>
int resident_grid(K kernel, int sms) {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kThreads, 0);
    return sms * (b > 0 ? b : 1);
}

// One batched MCSA iteration (4 kernels) over the active systems.
int enqueue_batch_iteration(mclsgpu_batch* b, const mclsgpu_mcsa_params* mp, int use_cond,
                            cudaGraphConditionalHandle handle) {
    cudaStream_t s = b->ctx->stream;
    BatchArgs a = batch_args(b, mp, false);
    k_b_richardson_residual<<<b->g_rich, kThreads, 0, s>>>(a);
    k_b_source<<<b->g_src, kThreads, 0, s>>>(a);
    const BatchList list{b->act_sys, b->act_hcum, b->act_count, b->d_srow0};
    int rc = launch_walk_batch(b->dom, b->cls, list, b->cR, b->Y, b->grab);
    if (rc) return rc;
    k_b_update<true, true><<<b->g_upd, kThreads, 0, s>>>(a, nullptr, use_cond, handle);
    return MCLSGPU_OK;
}

int build_batch_graph(mclsgpu_batch* b, const mclsgpu_mcsa_params* mp) {
    mclsgpu_context* ctx = b->ctx;
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    int red = MCLSGPU_OK;
    const int rc = build_while_graph(
        ctx, [&](cudaGraphConditionalHandle h) { red = enqueue_batch_iteration(b, mp, 1, h); },
        &b->graph, &b->body_kernels);
    return rc ? rc : red;
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
    // Width classes: system s gets W_s = nrhs_s rounded up to a power of two;
    // the systems are placed class by class (in argument order within a class).
    std::vector<int> width(nsys), cls_of(nsys);
    int pw = 1;
    for (int s = 0; s < nsys; ++s) {
        if (n[s] < 1 || !rowptr[s] || !colind[s] || !values[s] || nrhs[s] < 1 || nrhs[s] > 16)
            return set_error(ctx, MCLSGPU_ERR_INVALID_ARG,
                             "batch system %d: empty, missing arrays or 1..16 right-hand sides", s);
        int c = 0;
        while ((1 << c) < nrhs[s]) ++c;
        cls_of[s] = c;
        width[s] = 1 << c;
        if (width[s] > pw) pw = width[s];
    }
    std::vector<int> order;
    for (int c = 0; c < 5; ++c)
        for (int s = 0; s < nsys; ++s)
            if (cls_of[s] == c) order.push_back(s);
    BatchClasses cls{};
    std::vector<int64_t> row0(nsys), eoff(nsys);
    int64_t N = 0, NE = 0;
    size_t k = 0;
    for (int c = 0; c < 5; ++c) {
        cls.crow[c] = int(std::min<int64_t>(N, int64_t(1) << 30));
        NE = (NE + 15) / 16 * 16;  // class blocks start on 16-element boundaries
        cls.cel[c] = NE;
        for (; k < order.size() && cls_of[order[k]] == c; ++k) {
            const int s = order[k];
            row0[s] = N;
            eoff[s] = NE;
            N += n[s];
            NE += n[s] << c;
        }
    }
    cls.crow[5] = int(std::min<int64_t>(N, int64_t(1) << 30));
    NE = (NE + 15) / 16 * 16;
    cls.cel[5] = NE;
    if (N >= (int64_t(1) << 30))
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "batch too large (%lld rows)", (long long)N);
    int64_t nnz = 0;
    for (int s = 0; s < nsys; ++s) nnz += rowptr[s][n[s]] - rowptr[s][0];
    if (nnz >= (int64_t(1) << 31) - 1)
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "batch too large (%lld entries)", (long long)nnz);
    // The block-diagonal operator in placement order.
    std::vector<int64_t> rp(N + 1), ci(nnz);
    std::vector<double> v(nnz);
    int64_t pos = 0;
    for (int s : order) {
        const int64_t o = row0[s];
        for (int64_t i = 0; i < n[s]; ++i) {
            rp[o + i] = pos;
            for (int64_t p = rowptr[s][i]; p < rowptr[s][i + 1]; ++p, ++pos) {
                if (colind[s][p] < 0 || colind[s][p] >= n[s])
                    return set_error(ctx, MCLSGPU_ERR_INVALID_ARG,
                                     "batch system %d: column index out of range", s);
                ci[pos] = colind[s][p] + o;
                v[pos] = values[s][p];
            }
        }
    }
    rp[N] = pos;
    mclsgpu_batch* b = new mclsgpu_batch;
    b->ctx = ctx;
    b->nsys = nsys;
    b->pw = pw;
    b->n = int(N);
    b->ne = NE;
    b->cls = cls;
    b->row0 = row0;
    b->eoff = eoff;
    b->width = width;
    b->nrhs.assign(nrhs, nrhs + nsys);
    b->per = params->sample_ratio > 0.0 ? int(std::ceil(params->sample_ratio)) : 1;
    if (double(N) * b->per >= double(int64_t(1) << 31)) {
        delete b;
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "batch too large (histories per iteration)");
    }
    // Per-system tables and the list of every system (placement order).
    std::vector<int> srow0(nsys), sn(nsys), all_count(1, nsys);
    std::vector<long long> seoff(nsys), all_ecum(nsys + 1, 0);
    for (int s = 0; s < nsys; ++s) {
        srow0[s] = int(row0[s]);
        seoff[s] = eoff[s];
        sn[s] = int(n[s]);
    }
    for (int k = 0; k < nsys; ++k) {
        const int s = order[k];
        all_ecum[k + 1] = all_ecum[k] + ((long long)n[s] << cls_of[s]);
    }
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
    if (!rc && (b->dom->slots > 16 || b->dom->rec_q16))
        rc = set_error(ctx, MCLSGPU_ERR_UNSUPPORTED,
                       "batched walks: rows of at most 15 retained entries");
    const size_t PR = size_t(nsys) * pw;
    cudaError_t e = cudaSuccess;
    if (!rc &&
        ((e = dmalloc(&b->d_nrhs, nsys)) != cudaSuccess ||
         (e = dmalloc(&b->d_srow0, nsys)) != cudaSuccess ||
         (e = dmalloc(&b->d_seoff, nsys)) != cudaSuccess ||
         (e = dmalloc(&b->d_slog, nsys)) != cudaSuccess || (e = dmalloc(&b->d_sn, nsys)) != cudaSuccess ||
         (e = dmalloc(&b->d_sorder, nsys)) != cudaSuccess ||
         (e = dmalloc(&b->act_sys, nsys)) != cudaSuccess ||
         (e = dmalloc(&b->act_ecum, nsys + 1)) != cudaSuccess ||
         (e = dmalloc(&b->act_hcum, nsys + 1)) != cudaSuccess ||
         (e = dmalloc(&b->act_count, 1)) != cudaSuccess ||
         (e = dmalloc(&b->all_sys, nsys)) != cudaSuccess ||
         (e = dmalloc(&b->all_ecum, nsys + 1)) != cudaSuccess ||
         (e = dmalloc(&b->all_count, 1)) != cudaSuccess ||
         (e = dmalloc(&b->X, NE)) != cudaSuccess || (e = dmalloc(&b->X2, NE)) != cudaSuccess ||
         (e = dmalloc(&b->RP, NE)) != cudaSuccess || (e = dmalloc(&b->RP2, NE)) != cudaSuccess ||
         (e = dmalloc(&b->B, NE)) != cudaSuccess || (e = dmalloc(&b->Y, NE)) != cudaSuccess ||
         (e = dmalloc(&b->cR, NE)) != cudaSuccess || (e = dmalloc(&b->norm2, PR)) != cudaSuccess ||
         (e = dmalloc(&b->bnorm2, PR)) != cudaSuccess ||
         (e = dmalloc(&b->conv_iter, PR)) != cudaSuccess || (e = dmalloc(&b->sys_done, nsys)) != cudaSuccess ||
         (e = dmalloc(&b->blocks_done, 1)) != cudaSuccess || (e = dmalloc(&b->d_state, 1)) != cudaSuccess ||
         (e = cudaMallocHost(reinterpret_cast<void**>(&b->h_state), sizeof(BatchState))) != cudaSuccess))
        rc = cuda_fail(ctx, e, "cudaMalloc batch");
    if (!rc) {
        const int sms = ctx->num_sms;
        b->g_rich = resident_grid(k_b_richardson_residual, sms);
        b->g_src = resident_grid(k_b_source, sms);
        b->g_upd = resident_grid(k_b_update<true, true>, sms);
        b->g_upd0 = resident_grid(k_b_update<false, false>, sms);
        b->g_init = resident_grid(k_b_init_norms, sms);
        cudaStream_t s = ctx->stream;
        cudaMemcpyAsync(b->d_nrhs, b->nrhs.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(b->d_srow0, srow0.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(b->d_seoff, seoff.data(), sizeof(long long) * nsys, cudaMemcpyHostToDevice,
                        s);
        cudaMemcpyAsync(b->d_slog, cls_of.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(b->d_sn, sn.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(b->d_sorder, order.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(b->all_sys, order.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(b->all_ecum, all_ecum.data(), sizeof(long long) * (nsys + 1),
                        cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(b->all_count, all_count.data(), sizeof(int), cudaMemcpyHostToDevice, s);
        // Padding elements are never written by the loop: zero every array once.
        cudaMemsetAsync(b->X, 0, sizeof(double) * NE, s);
        cudaMemsetAsync(b->X2, 0, sizeof(double) * NE, s);
        cudaMemsetAsync(b->RP, 0, sizeof(double) * NE, s);
        cudaMemsetAsync(b->RP2, 0, sizeof(double) * NE, s);
        cudaMemsetAsync(b->Y, 0, sizeof(double) * NE, s);
        cudaMemsetAsync(b->cR, 0, sizeof(float) * NE, s);
        cudaMemsetAsync(b->blocks_done, 0, sizeof(unsigned), s);
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

int mclsgpu_batch_layout(mclsgpu_batch* b, int64_t* elem_offsets, int32_t* widths,
                         int64_t* elements, int32_t* max_width) {
    if (!b) return MCLSGPU_ERR_INVALID_ARG;
    for (int s = 0; s < b->nsys; ++s) {
        if (elem_offsets) elem_offsets[s] = b->eoff[s];
        if (widths) widths[s] = b->width[s];
    }
    if (elements) *elements = b->ne;
    if (max_width) *max_width = b->pw;
    return MCLSGPU_OK;
}

int mclsgpu_batch_domain(mclsgpu_batch* b, mclsgpu_domain** dom) {
    if (!b || !dom) return MCLSGPU_ERR_INVALID_ARG;
    *dom = b->dom;
    return MCLSGPU_OK;
}

int mclsgpu_batch_set_launch(mclsgpu_batch* b, int block_size, int grab) {
    if (!b || (block_size != 128 && block_size != 256) || grab < 1 || grab > 8)
        return MCLSGPU_ERR_INVALID_ARG;
    b->dom->walk_block = block_size;
    b->grab = grab;
    b->graph_key = -1;  // the captured loop bakes the launch shape in
    return MCLSGPU_OK;
}

int mclsgpu_batch_autotune(mclsgpu_batch* b, const double* b_dev, double* x_dev, int reps,
                           int* block_size, int* grab, double* walk_ms) {
    if (!b || !b_dev || !x_dev || reps < 1) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_mcsa_params p{};
    p.size = sizeof(p);
    p.max_iters = reps;
    p.tolerance = 0.0;
    p.check_freq = 1;
    p.smoother_steps = 1;
    p.richardson_omega = 1.0;
    p.host_loop = 1;
    const int blocks[2] = {256, 128};
    const int grabs[3] = {1, 2, 4};
    int best_b = 256, best_g = 1;
    double best_ms = 1e300;
    for (int blk : blocks)
        for (int g : grabs) {
            b->dom->walk_block = blk;
            b->grab = g;
            cudaMemsetAsync(x_dev, 0, sizeof(double) * size_t(b->ne), b->ctx->stream);
            mclsgpu_stats st{};
            st.size = sizeof(st);
            int rc = mclsgpu_batch_mcsa_solve_dev(b, b_dev, x_dev, &p, nullptr, nullptr, &st);
            if (rc) return rc;
            const double per = st.walk_launches ? st.walk_ms / double(st.walk_launches) : 1e300;
            if (per < best_ms) {
                best_ms = per;
                best_b = blk;
                best_g = g;
            }
        }
    b->dom->walk_block = best_b;
    b->grab = best_g;
    b->graph_key = -1;
    if (block_size) *block_size = best_b;
    if (grab) *grab = best_g;
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
    const size_t NE = size_t(b->ne), PR = size_t(b->nsys) * b->pw;
    int pairs = 0;
    for (int q = 0; q < b->nsys; ++q) pairs += b->nrhs[q];
    const long long key = (long long)(params->richardson_omega * 1e6) * 64 +
                          (long long)b->grab * 2 + (b->dom->walk_block == 128 ? 1 : 0);
    if (!params->host_loop && (!b->graph || b->graph_key != key || b->graph_seed != b->dom->seed)) {
        int rc = build_batch_graph(b, params);
        if (rc) return rc;
        b->graph_key = key;
        b->graph_seed = b->dom->seed;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s);
    cudaMemsetAsync(b->dom->d_counter, 0, sizeof(int), s);
    cudaMemsetAsync(b->dom->d_steps, 0, sizeof(unsigned long long), s);
    cudaMemsetAsync(b->blocks_done, 0, sizeof(unsigned), s);
    {
        unsigned long long tim0[4] = {~0ULL, 0ULL, 0ULL, 0ULL};
        cudaMemcpyAsync(b->dom->d_tim, tim0, sizeof(tim0), cudaMemcpyHostToDevice, s);
    }
    cudaEventRecord(e0, s);
    cudaMemcpyAsync(b->B, b_dev, sizeof(double) * NE, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(b->X, x_dev, sizeof(double) * NE, cudaMemcpyDeviceToDevice, s);
    cudaMemsetAsync(b->bnorm2, 0, sizeof(double) * PR, s);
    BatchArgs a = batch_args(b, params, true);  // every system
    k_b_state_init<<<1, 1024, 0, s>>>(a, params->max_iters, params->check_freq,
                                       params->tolerance, pairs);
    k_b_init_norms<<<b->g_init, kThreads, 0, s>>>(a);
    k_b_update<false, false><<<b->g_upd0, kThreads, 0, s>>>(a, b->X, 0,
                                                          cudaGraphConditionalHandle(0));
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
        cudaMemcpyAsync(x_dev, b->X, sizeof(double) * NE, cudaMemcpyDeviceToDevice, s);
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
        k_b_update<false, false><<<b->g_upd0, kThreads, 0, s>>>(a, b->X, 0,
                                                              cudaGraphConditionalHandle(0));
        cudaMemcpyAsync(nr.data(), b->norm2, sizeof(double) * PR, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(bn.data(), b->bnorm2, sizeof(double) * PR, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(ci.data(), b->conv_iter, sizeof(int) * PR, cudaMemcpyDeviceToHost, s);
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "batch residuals");
        for (size_t q = 0; q < PR; ++q) {
            const bool valid = int(q % b->pw) < b->nrhs[q / b->pw];
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
        out.kernel_launches = int64_t(b->body_kernels ? b->body_kernels : 4) * st.iter + 3;
        out.rho = -1.0;
        *stats = out;
    }
    return MCLSGPU_OK;
}

}  // extern "C"
