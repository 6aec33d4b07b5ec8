// internal.h -- shared types of the mclsgpu translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <functional>
#include <string>

#include "../../include/mclsgpu.h"

namespace mclsgpu {

// Device status word bits (set by kernels, read and cleared by the host).
enum : int {
    DEV_ERR_DEGENERATE = 1,   // empty / zero-weight domain row
    DEV_ERR_NONFINITE = 2,    // non-finite weight, residual or tally
    DEV_ERR_TIMEOUT = 4,      // a bounded wait gave up
    DEV_ERR_BOUNDS = 8,       // an index failed a bounds check
    DEV_ERR_CAPACITY = 16     // more histories than the buffers were sized for
};

struct Status {
    int code = MCLSGPU_OK;
    std::string msg;
};

}  // namespace mclsgpu

struct mclsgpu_context {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    int* d_status = nullptr;      // device error word
    int* h_status = nullptr;      // pinned mirror
    std::string err;
};

namespace mclsgpu {

// Device CSR with int32 indices (n, nnz < 2^31).
struct DevCsr {
    int n = 0;
    int nnz = 0;
    int* rp = nullptr;
    int* ci = nullptr;
    double* v = nullptr;
    void release();
};

// Sliced ELL with slices of 32 rows (SELL-32): slice s holds rows 32s..32s+31
// column-major, width w_s = the longest row of the slice, at off[s]; entry k
// of row r sits at off[r/32] + 32k + r%32.  Padding entries repeat the row's
// own index with value 0.  A warp that owns one slice reads each entry column
// with one coalesced access.
struct DevSell {
    int n = 0;
    int nslices = 0;
    int* off = nullptr;      // nslices + 1 entry offsets
    int* col = nullptr;
    double* val = nullptr;
    void release();
};

}  // namespace mclsgpu

struct mclsgpu_operator {
    mclsgpu_context* ctx = nullptr;
    mclsgpu::DevCsr A;
    mclsgpu::DevSell S;           // the same matrix as SELL-32 (residual kernels)
    // Stencil operators (every column is row + dia_off[j], at most 16 offsets):
    // values by diagonal, dia_val[j * n + r] = A(r, r + dia_off[j]) or 0.
    int dia_k = 0;
    int dia_off[16] = {0};
    double* dia_val = nullptr;
    // Symmetric stencil operators (A(r, r - o) == A(r - o, r) for every offset)
    // also keep the diagonal and the positive-offset diagonals only:
    // sym_val[0 * n + r] = A(r, r), sym_val[(1 + h) * n + r] = A(r, r + sym_off[h]).
    int sym_h = 0;
    int sym_off[8] = {0};
    double* sym_val = nullptr;
    double* dinv = nullptr;       // reciprocal diagonal (built on demand)
    mclsgpu::DevCsr AT;           // A^T (built on demand: RNSD iterations)
    uint64_t serial = 0;          // identity for "operator changed" checks
};

struct mclsgpu_precond {
    mclsgpu_context* ctx = nullptr;
    int kind = MCLSGPU_PREC_NONE;
    int block_size = 1;
    mclsgpu::DevCsr P;            // left preconditioner as CSR
    mclsgpu::DevCsr PT;           // P^T (built on demand: RNSD iterations)
    double* diag = nullptr;       // POINT_JACOBI: the reciprocal diagonal
    double* mdia = nullptr;       // LEARNED_SPAI kept: M by A's diagonal offsets
    double rho = -1.0;            // LEARNED_SPAI: rho(H) estimate
    int fallback = 0;             // LEARNED_SPAI replaced by Jacobi
};

namespace mclsgpu {

struct AndersonWork;

struct McsaState {
    int iter;            // iterations completed
    int done;            // 1 once the loop must stop
    int check_freq;
    int max_iters;
    double crit;         // tolerance * |PL b|
    double rnorm;        // last |rp|_2
    int converged;
    int pad;
};

}  // namespace mclsgpu

struct mclsgpu_domain {
    mclsgpu_context* ctx = nullptr;
    mclsgpu_operator* op = nullptr;
    mclsgpu_precond* left = nullptr;
    mclsgpu_precond* right = nullptr;
    mclsgpu_mc_params p{};
    int n = 0;
    // FP64 domain (AlmostOptimalDomain data): row r lists (col, h, cdf).
    mclsgpu::DevCsr D;            // D.v holds h
    double* cdf = nullptr;
    double* w = nullptr;
    mclsgpu::DevSell DS;          // the domain as SELL-32 (forward tally source)
    // Transposed domain for the expected-value estimator: DT(j,s) = h_sj.
    mclsgpu::DevCsr DT;
    float* dt_h32 = nullptr;
    // Packed FP32 walk records: row r at rec + r*slots, slot 0 = {W, len},
    // slots 1..slots-1 = {cdf (float bits), col | sign<<31}.
    uint2* rec = nullptr;
    int slots = 0;
    int max_row = 0;
    // FP32 walk launch shape (autotuned): histories per lane and block size.
    int walk_ilp = 1;
    int walk_block = 256;
    int walk_l1 = 0;               // record loads allocated in L1
    // Stencil records (stencil_k > 0): row r's slot j is column r + stencil_off[j].
    int stencil_k = 0;
    int rec_q16 = 0;               // stencil records with 16-bit CDF thresholds
    int stencil_off[32] = {0};
    // Random stream.
    uint64_t seed = 1;
    unsigned long long* d_epoch = nullptr;  // counter mode: MC solves so far
    uint64_t* d_jump = nullptr;    // reference mode: 64x64 jump tables
    unsigned long long* d_pos = nullptr;  // reference mode: draws consumed
    // Source / tally work buffers.
    int64_t nh_cap = 0;
    double* src = nullptr;         // scaled source vector (n)
    double* scdf = nullptr;        // source CDF (n)
    int* guide = nullptr;          // guide table (n)
    int* counts = nullptr;         // histories per state (n)
    int* offs = nullptr;           // emission offsets (n)
    int* start = nullptr;          // start state | sign<<31 per history
    double* y64 = nullptr;         // tallies, reduced in FP64 (n)
    float* c32 = nullptr;          // forward: FP32 tally source (n)
    double* c64 = nullptr;         // forward: FP64 tally source (n)
    int* d_nh = nullptr;           // histories of the current solve
    int* d_counter = nullptr;      // walk work-queue counter
    double* d_scalars = nullptr;   // [0] |src|_1, [1] cdf total, [2] 1/nh ...
    unsigned long long* d_steps = nullptr;  // walk steps (running total)
    unsigned long long* d_tim = nullptr;    // FP32 walk timing (see walk.cu)
    double* part = nullptr;        // reduction / scan partials
    int* ipart = nullptr;
    int part_cap = 0;
    // MCSA buffers.
    double* x = nullptr;
    double* b = nullptr;
    double* rp = nullptr;
    double* tmp = nullptr;
    double* tmp2 = nullptr;
    double* x2 = nullptr;          // fused iteration: x after smoothing
    double* rp2 = nullptr;         // fused iteration: residual after smoothing
    unsigned int* d_ticket = nullptr;  // last-block ticket of the fused residual
    mclsgpu::McsaState* d_state = nullptr;
    mclsgpu::McsaState* h_state = nullptr;  // pinned
    cudaGraphExec_t graph = nullptr;
    int graph_key = -1;
    int body_kernels = 0;          // kernel nodes in one MCSA iteration
    unsigned long long* d_hist = nullptr;   // histories transported (total)
    double* d_resid = nullptr;     // per-iteration |rp|_2 history
    int resid_cap = 0;
    // Step-wise MCSA (mclsgpu_mcsa_begin .. _finish).
    mclsgpu_mcsa_params step_p{};
    int step_ready = 0;
    // Reference stream with a weight cutoff (variable-length histories): each
    // history's first draw is the sum of the earlier histories' lengths,
    // found by rounds of FP64 walks (walk.cu).
    int* hoff = nullptr;           // per-history stream offsets (nh_cap)
    int* hlen = nullptr;           // per-history lengths of the last round
    int* hoff2 = nullptr;          // offsets recomputed from hlen (nh_cap + 1)
    double* y_save = nullptr;      // tallies before the first round (n)
    int walk_rounds = 0;           // rounds the last Monte Carlo solve took
    // Multi-set MCSA (multiset.cu): this set's correction and the device-side
    // loop captured for one reducer.
    double* delta = nullptr;
    cudaGraphExec_t set_graph = nullptr;
    void* set_graph_reduce = nullptr;
    void* set_graph_user = nullptr;
    int set_graph_sets = 0;
    long long set_graph_key = -1;
    int set_body_kernels = 0;
    // Anderson-accelerated MCSA work space (anderson.cu), built on first use.
    mclsgpu::AndersonWork* aa = nullptr;
    int aa_step_ready = 0;
};

namespace mclsgpu {

// ---- helpers (context.cu) --------------------------------------------------
int set_error(mclsgpu_context* ctx, int code, const char* fmt, ...);
int cuda_fail(mclsgpu_context* ctx, cudaError_t e, const char* what);
int check_device_status(mclsgpu_context* ctx);
// Every device allocation and release of the library goes through dmalloc and
// dfree; the counters behind mclsgpu_debug_device_allocations count them.
extern std::atomic<long long> g_device_allocs;
extern std::atomic<long long> g_device_frees;
template <class T>
inline cudaError_t dmalloc(T** p, size_t count) {
    g_device_allocs.fetch_add(1, std::memory_order_relaxed);
    return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T) + 16);
}
template <class T>
inline void dfree(T*& p) {
    if (p) {
        g_device_frees.fetch_add(1, std::memory_order_relaxed);
        cudaFree(p);
    }
    p = nullptr;
}

// ---- sparse (sparse.cu) ----------------------------------------------------
// Upload a host CSR (int64 indices) to a DevCsr (int32).  Validates.
// ncols < 0: square (ncols = n).
int upload_csr(mclsgpu_context* ctx, int64_t n, const int64_t* rp,
               const int64_t* ci, const double* v, DevCsr& out, int64_t ncols = -1);
int csr_transpose(mclsgpu_context* ctx, const DevCsr& A, DevCsr& T);
// C = A*B (accumulated over A's row entries in column order) then filtered
// by `threshold` relative to the signed row max.
int csr_multiply(mclsgpu_context* ctx, const DevCsr& A, const DevCsr& B,
                 double threshold, DevCsr& C);
int csr_copy(mclsgpu_context* ctx, const DevCsr& A, DevCsr& B);
// Column scaling: T.v[k] *= s[T.ci[k]] (composite with a diagonal factor).
void csr_scale_cols(mclsgpu_context* ctx, DevCsr& T, const double* s);
// ncols: A's column count (< 0: square).
int csr_filter(mclsgpu_context* ctx, const DevCsr& A, double threshold,
               DevCsr& out, int ncols = -1);
void spmv(cudaStream_t s, const DevCsr& A, const double* x, double* y);
int reciprocal_diagonal(mclsgpu_context* ctx, const DevCsr& A, double* dinv);
int block_jacobi(mclsgpu_context* ctx, const DevCsr& A, int bs, DevCsr& P);
int point_jacobi_csr(mclsgpu_context* ctx, int n, const double* dinv,
                     DevCsr& P);
// SELL-32 copy of a CSR matrix (set-up).
int csr_to_sell(mclsgpu_context* ctx, const DevCsr& A, DevSell& S);
// Sorted distinct column offsets (col - row) of A, at most max_k <= 32
// (*K = 0 if more).
// row0: global index of A's first row (column offsets are col - global row).
int collect_offsets(mclsgpu_context* ctx, const DevCsr& A, int max_k, int* offsets, int* K,
                    int row0 = 0);
// Diagonal-offset values of a stencil matrix (K offsets): val[j*n + r].
int csr_to_dia(mclsgpu_context* ctx, const DevCsr& A, int K, const int* offsets,
               double** val);
// The diagonal and positive-offset diagonals of a DIA matrix whose K offsets
// are symmetric about 0 and whose values are (bit for bit) symmetric; *kh = 0
// and no allocation otherwise.
int dia_symmetric(mclsgpu_context* ctx, int n, int K, const int* offsets, const double* val,
                  double** sym, int* kh, int* sym_off);
// y = A x over a SELL-32 matrix.
void sell_spmv(cudaStream_t s, const DevSell& A, const double* x, double* y);
// Exclusive scan of set-up counts into rp[0..n]; *total = sum.
int exclusive_scan_counts_dev(mclsgpu_context* ctx, const int* d_cnt, int n, int* d_rp,
                              long long* total);
// Domain arrays and FP32 records from the composite operator (domain.cu).
// row0: global index of M's first row (rows of one part of a row-partitioned
// domain; its columns are global).
int build_domain_arrays(mclsgpu_context* ctx, const DevCsr& M, double relax,
                        mclsgpu_domain* dom, int row0 = 0);

// Releases the domain's captured Anderson loop (rebuilt on the next solve).
void anderson_drop_graph(mclsgpu_domain* dom);

// FP32 forward walks: the tally source of v into the domain's records (H v
// for the expected-value estimator, v for collision, with the Neumann
// relaxation when has_omega) and the tallies y cleared.  row0: the global
// index of the domain's first row (v is the whole vector, nv entries).
void launch_forward_records(mclsgpu_domain* dom, const double* v, int nv, double omega,
                            int has_omega, int row0, double* y);

// ---- batched walks (walk.cu, batch.cu) -------------------------------------------
// Width classes of a batch: the rows [crow[c], crow[c+1]) belong to systems
// with 2^c right-hand-side columns, and their elements occupy
// [cel[c], cel[c] + (crow[c+1] - crow[c]) * 2^c) of every element array,
// row-major [rows][2^c]; cel[c] is a multiple of 16 (aligned vector loads),
// cel[5] the element count (padding included).
struct BatchClasses {
    int crow[6];
    long long cel[6];
};
// The systems a batched iteration works on: lsys[k] for k < *lcount, whose
// histories occupy [hcum[k], hcum[k+1]) of the iteration's history space
// (n_s * per each, hcum[*lcount] in all).
struct BatchList {
    const int* lsys;
    const int* hcum;
    const int* lcount;
    const int* srow0;   // system -> its first row
};
// Forward walks shared by the right-hand sides of a batch: every history
// carries one Kahan-compensated FP32 tally per column of its start row's
// class, reading the tally source cR at each state's elements and adding into
// Y at the start row's elements.  Only the listed systems' histories run;
// history h of system s is history srow0[s] * per + (h - hcum[k]) of the
// whole batch, on that history's own random stream, whatever the list.
// Each warp takes 32 * grab histories per work-queue grab.  The work-queue
// counter must be zero on entry; the caller resets it afterwards.
int launch_walk_batch(mclsgpu_domain* dom, const BatchClasses& cls, const BatchList& list,
                      const float* cR, double* Y, int grab);

// ---- MCSA helpers (mcsa.cu) ----------------------------------------------------
// rp_out = PL (b - A PR x)   (LinearProblem::updatePrecResidual)
void prec_residual(mclsgpu_domain* dom, const double* x, const double* b, double* rp_out);
// y = PL A PR x   (LinearProblem::apply); uses dom->tmp and dom->tmp2.
void composite_apply(mclsgpu_domain* dom, const double* x, double* y);
// x2 = x + w r; r2 = PL (b - A PR x2): one fused pass when PL is I, point
// Jacobi or held on A's diagonals and there is no PR (x2 != x, r2 != r).
void richardson_residual(mclsgpu_domain* dom, const double* x, const double* r, double w,
                         double* x2, double* r2);
// out = the Monte Carlo estimate for the source v (already left
// preconditioned): one MC solve, advancing the domain's random stream.
void mc_correction(mclsgpu_domain* dom, const double* v, double* out);
// True when the domain walks variable-length histories on the reference
// stream: those walks synchronise with the host (rounds), so the MCSA and
// Anderson loops run from the host instead of a captured graph.
inline bool walk_needs_rounds(const mclsgpu_domain* dom) {
    return dom->p.rng_mode == MCLSGPU_RNG_REFERENCE && dom->p.weight_cutoff > 0.0;
}
// Walk statistics since the last reset (steps, histories, walk time).
int mcsa_read_stats(mclsgpu_domain* dom, mclsgpu_stats* st);
void mcsa_reset_counters(mclsgpu_domain* dom);

// ---- Anderson-accelerated MCSA (anderson.cu) ------------------------------------
void release_anderson(mclsgpu_domain* dom);

// ---- fixed-point iterations (fixedpoint.cu) ------------------------------------
// Transposes the RNSD iteration needs (set-up: never inside a stream capture).
int prepare_fixed_point(mclsgpu_domain* dom, int type);
// One fixed-point step of `type` on dom->x and dom->rp (dom->x2, rp2, tmp and
// tmp2 as scratch; dom->part, d_ticket and d_scalars[7] for the step length).
void enqueue_fixed_point_step(mclsgpu_domain* dom, int type, double omega);
// Instantiate a graph whose only node is a WHILE loop around the launches
// `body` enqueues on ctx->stream (captured); body_kernels = its kernel nodes.
int build_while_graph(mclsgpu_context* ctx,
                      const std::function<void(cudaGraphConditionalHandle)>& body,
                      cudaGraphExec_t* exec, int* body_kernels);

// ---- row-partitioned domains (walk.cu, subdomain.cu) ---------------------------
constexpr int kMaxParts = 64;

// One history crossing between parts (24 bytes, the C ABI's
// mclsgpu_history_wire).
struct HistoryWire {
    uint64_t rng;     // Xorshift state after the last draw
    int32_t state;    // the global state it moved to; -1: a forward tally return
    int32_t step;     // transitions taken
    float weight;
    int32_t id;       // its index in the global source
    float acc;        // forward: the history's Kahan-compensated sum so far
    float comp;       //          and its compensation
};
static_assert(sizeof(HistoryWire) == 32, "history wire format");

struct PartWalk {
    const uint2* rec;       // FP32 records of rows [row0, row0 + n)
    int slots;
    int row0;
    int n;
    int L;
    int dir;                // MCLSGPU_ADJOINT or MCLSGPU_FORWARD
    int kind;               // records: 0 packed, 1 stencil, 2 stencil16
    int stoff[32];          // stencil records: column offset of each slot
    int per;                // forward: histories per start row
    float cutoff;           // relative weight cutoff (0: fixed length)
    // first round: the histories e_begin <= e < e_end of the global source
    // (adjoint: its start list; forward: history e starts at row e / per)
    const int* start;
    long long e_begin, e_end;
    const double* sc;       // [0] = adjoint starting weight |b|_1
    uint64_t seed;
    const unsigned long long* d_epoch;
    // later rounds: histories handed over by other parts
    const HistoryWire* in;
    long long n_in;
    // departures: out[q * cap + slot] for the owner q of the new state
    HistoryWire* out;
    long long cap;
    unsigned long long* out_cnt;
    int nparts;
    const int* bounds;      // nparts + 1 global row bounds (device)
    double* y;              // tallies of the part's rows
    unsigned long long* d_steps;
    int* status;
};
void launch_walk_part(const PartWalk& p, mclsgpu_context* ctx);

// ---- scans and reductions (scan.cu) ------------------------------------------
int scan_partials_needed(int n);
// Deterministic FP64 sum of |v[i]*scale| (scale applied when has_scale).
void abs_sum(cudaStream_t s, const double* v, int n, double scale,
             int has_scale, double* part, double* out);
// Source CDF: c[0] = v[0]*sc, c[i] = c[i-1] + |v[i]*sc|, then c /= c[n-1];
// writes total to *total.  sequential != 0 reproduces the reference's
// left-to-right order in one thread.
void source_cdf(cudaStream_t s, const double* v, int n, double scale,
                int has_scale, int sequential, double* part, double* cdf,
                double* total);
// Exclusive suffix sum: out[i] = sum_{j>i} in[j]; *total = sum.
void suffix_scan_int(cudaStream_t s, const int* in, int n, int* part,
                     int* out, int* total);
// Inclusive max-scan in place (guide table).
void max_scan_int(cudaStream_t s, int* a, int n, int* part);
// Sum of squares (deterministic).
void sum_sq(cudaStream_t s, const double* v, int n, double* part,
            double* out);

}  // namespace mclsgpu
