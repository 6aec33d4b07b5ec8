// subdomain.cu -- one part of a row-partitioned Monte Carlo domain
// (domain-decomposed transport).
//
// The reference splits the domain over MPI ranks: each rank holds its rows of
// the iteration matrix, walks histories until they leave its rows (a
// BOUNDARY event) and hands them to the owning rank through buffered
// history messages (src/MCLS_DomainTransporter_impl.hpp:70-119,
// src/MCLS_DomainCommunicator_impl.hpp, src/MCLS_SourceTransporter_impl.hpp,
// src/MCLS_History_impl.hpp:56-89 for the packed history).
//
// Here a part is one GPU's rows [row0, row0 + n): their FP32 records, FP64
// domain and tallies.  A solve is
//   begin      the global adjoint source of the (replicated) residual, built
//              exactly as the whole-domain solve builds it; the part keeps
//              the histories that start in its rows (a contiguous range of
//              the LIFO emission order) and its rows' step-0 tallies
//   transport  rounds: walk the part's starting histories, then the
//              histories other parts handed over; departures are written to
//              per-destination outboxes (HistoryWire: the Xorshift state
//              travels with the history, so it continues on its own stream)
//   finish     tallies / histories for the part's rows.
// The rounds and the exchange between parts are the caller's (NCCL
// all-to-all between GPUs, device copies between parts of one GPU); no
// kernel waits on another part.  Every transition and tally is the one the
// whole-domain walk makes, so the parts' results equal the whole-domain
// solve's up to the order of the FP64 tally additions.
#include <cmath>
#include <vector>

#include "internal.h"

namespace mclsgpu {

void launch_adjoint_source(mclsgpu_domain* dom, const double* v, double omega, int has_omega);
void prepare_source(mclsgpu_domain* dom);

namespace {

inline int grid_for(long long work, int cap = 148 * 8) {
    long long g = (work + 255) / 256;
    if (g < 1) g = 1;
    return int(g > cap ? cap : g);
}

// Histories are emitted state by state from the last state down, so the
// states along the start list never increase: the part's histories are
// those from the first with state < hi to the first with state < lo.
__device__ long long first_below(const int* start, long long nh, int bound) {
    long long lo = 0, hi = nh;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if ((start[mid] & 0x7fffffff) >= bound) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__global__ void k_part_range(const int* start, const int* d_nh, int lo, int hi,
                             long long* range) {
    const long long nh = *d_nh;
    range[0] = first_below(start, nh, hi);
    range[1] = first_below(start, nh, lo);
    range[2] = nh;
}

__global__ void k_part_finish(const double* y, const double* sc, int n, double* x) {
    const double inv = sc[2];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = __dmul_rn(y[i], inv);  // AdjointTally::normalize
}

// ForwardTally::finalize (src/MCLS_ForwardTally_impl.hpp:194-208): sum /
// count, plus the source term for the expected-value estimator.
__global__ void k_part_finish_forward(const double* y, const double* srcp, int n, int per,
                                      int ev, double omega, int has, double* x) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = __ddiv_rn(y[i], per);
        if (ev) d = __dadd_rn(d, has ? srcp[i] * omega : srcp[i]);
        x[i] = d;
    }
}

__global__ void k_epoch_next(unsigned long long* e) { *e += 1ULL; }

void release_source(mclsgpu_domain* d) {
    dfree(d->src);
    dfree(d->scdf);
    dfree(d->guide);
    dfree(d->counts);
    dfree(d->offs);
    dfree(d->start);
    dfree(d->y64);
    dfree(d->d_nh);
    dfree(d->d_scalars);
    dfree(d->part);
    dfree(d->ipart);
    dfree(d->d_epoch);
    dfree(d->d_pos);
}

void release_records(mclsgpu_domain* d) {
    d->D.release();
    dfree(d->cdf);
    dfree(d->w);
    dfree(d->rec);
}

}  // namespace
}  // namespace mclsgpu

using namespace mclsgpu;

struct mclsgpu_subdomain {
    mclsgpu_context* ctx = nullptr;
    mclsgpu_mc_params p{};
    int64_t N = 0;
    int nparts = 0;
    int part = 0;
    int row0 = 0;
    int n = 0;
    int* d_bounds = nullptr;
    mclsgpu_domain src;    // the global source: N states, no records
    mclsgpu_domain recs;   // the part's rows: records and FP64 domain
    double* y = nullptr;   // tallies of the part's rows
    double* srcp = nullptr;  // forward: the part's slice of the source
    int per = 1;             // forward: histories per start row
    unsigned long long* d_out_cnt = nullptr;
    unsigned long long* d_steps = nullptr;
    long long* d_range = nullptr;
    long long range[3] = {0, 0, 0};
    int ready = 0;
    ~mclsgpu_subdomain() {
        release_source(&src);
        release_records(&recs);
        dfree(d_bounds);
        dfree(y);
        dfree(srcp);
        dfree(d_out_cnt);
        dfree(d_steps);
        dfree(d_range);
    }
};

extern "C" {

int mclsgpu_subdomain_build(mclsgpu_context* ctx, int64_t n_global, int32_t nparts,
                            const int64_t* bounds, int32_t part, const int64_t* rowptr,
                            const int64_t* colind, const double* values,
                            const mclsgpu_mc_params* p, mclsgpu_subdomain** out) {
    if (!ctx || !bounds || !rowptr || !colind || !values || !p || !out)
        return MCLSGPU_ERR_INVALID_ARG;
    *out = nullptr;
    if (p->size < sizeof(mclsgpu_mc_params))
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "mc params: size mismatch");
    if (nparts < 1 || nparts > kMaxParts || part < 0 || part >= nparts)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "parts: 1..%d parts, 0 <= part < parts",
                         kMaxParts);
    if (n_global <= 0 || n_global >= (int64_t(1) << 31) || bounds[0] != 0 ||
        bounds[nparts] != n_global)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "parts: bounds must run from 0 to n");
    for (int q = 0; q < nparts; ++q)
        if (bounds[q + 1] <= bounds[q])
            return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "parts: empty or decreasing part %d",
                             q);
    const bool adjoint = p->direction == MCLSGPU_ADJOINT;
    if ((adjoint && p->estimator != MCLSGPU_COLLISION) ||
        (!adjoint && p->direction != MCLSGPU_FORWARD) || p->precision != MCLSGPU_FP32 ||
        p->rng_mode != MCLSGPU_RNG_COUNTER || p->weight_cutoff < 0.0 || p->history_length < 1)
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED,
                         "partitioned domains take FP32 walks on the counter-based stream: "
                         "adjoint collision or forward (collision or expected value)");
    cudaSetDevice(ctx->device);
    mclsgpu_subdomain* sd = new mclsgpu_subdomain;
    sd->ctx = ctx;
    sd->p = *p;
    sd->N = n_global;
    sd->nparts = nparts;
    sd->part = part;
    sd->row0 = int(bounds[part]);
    sd->n = int(bounds[part + 1] - bounds[part]);
    sd->per = p->sample_ratio > 0.0 ? int(std::ceil(p->sample_ratio)) : 1;
    if (!adjoint && double(n_global) * sd->per >= double(int64_t(1) << 31)) {
        delete sd;
        return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "too many histories per solve");
    }
    cudaStream_t s = ctx->stream;
    const int N = int(n_global);
    int rc = MCLSGPU_OK;
    cudaError_t e = cudaSuccess;
    // Records of the part's rows: h = delta_ij - w m_ij over the given rows
    // of the transposed composite operator, filtered as the whole domain is.
    {
        DevCsr M, F;
        rc = upload_csr(ctx, sd->n, rowptr, colind, values, M, n_global);
        if (!rc) rc = csr_filter(ctx, M, p->composite_threshold, F, N);
        M.release();
        mclsgpu_domain& r = sd->recs;
        r.ctx = ctx;
        r.p = sd->p;
        r.n = sd->n;
        const double relax = p->neumann_relaxation > 0.0 ? p->neumann_relaxation : 1.0;
        if (!rc) rc = build_domain_arrays(ctx, F, relax, &r, sd->row0);
        F.release();
        if (!rc && r.slots == 0)
            rc = set_error(ctx, MCLSGPU_ERR_UNSUPPORTED,
                           "domain rows longer than 31 entries need the FP64 walk");
    }
    // The global source (as mclsgpu_domain_build sizes it) and the part's
    // tallies and exchange counters.
    if (!rc) {
        mclsgpu_domain& g = sd->src;
        g.ctx = ctx;
        g.p = sd->p;
        g.n = N;
        g.seed = p->seed;
        const int64_t nh_req =
            p->sample_ratio > 0.0 ? int64_t(double(N) * p->sample_ratio) : int64_t(N);
        g.nh_cap = nh_req + (p->source_sampling == MCLSGPU_SOURCE_STRATIFIED ? N : 0);
        if (g.nh_cap >= (int64_t(1) << 31) - (int64_t(1) << 24))
            rc = set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "too many histories per solve");
        const int parts = scan_partials_needed(N) + ctx->num_sms * 8 + 8;
        if (!rc &&
            ((e = dmalloc(&g.src, N)) != cudaSuccess || (e = dmalloc(&g.scdf, N)) != cudaSuccess ||
             (e = dmalloc(&g.guide, N)) != cudaSuccess ||
             (e = dmalloc(&g.counts, N)) != cudaSuccess ||
             (e = dmalloc(&g.offs, N)) != cudaSuccess ||
             (e = dmalloc(&g.start, size_t(g.nh_cap) + 1)) != cudaSuccess ||
             (e = dmalloc(&g.y64, N)) != cudaSuccess || (e = dmalloc(&g.d_nh, 1)) != cudaSuccess ||
             (e = dmalloc(&g.d_scalars, 16)) != cudaSuccess ||
             (e = dmalloc(&g.part, parts)) != cudaSuccess ||
             (e = dmalloc(&g.ipart, parts)) != cudaSuccess ||
             (e = dmalloc(&g.d_epoch, 1)) != cudaSuccess || (e = dmalloc(&g.d_pos, 1)) != cudaSuccess ||
             (e = dmalloc(&sd->y, sd->n)) != cudaSuccess ||
             (e = dmalloc(&sd->srcp, sd->n)) != cudaSuccess ||
             (e = dmalloc(&sd->d_bounds, nparts + 1)) != cudaSuccess ||
             (e = dmalloc(&sd->d_out_cnt, nparts)) != cudaSuccess ||
             (e = dmalloc(&sd->d_steps, 1)) != cudaSuccess ||
             (e = dmalloc(&sd->d_range, 3)) != cudaSuccess))
            rc = cuda_fail(ctx, e, "cudaMalloc subdomain");
        if (!rc) {
            g.part_cap = parts;
            cudaMemsetAsync(g.d_epoch, 0, sizeof(unsigned long long), s);
            cudaMemsetAsync(g.d_pos, 0, sizeof(unsigned long long), s);
            cudaMemsetAsync(g.d_scalars, 0, 16 * sizeof(double), s);
            cudaMemsetAsync(sd->d_steps, 0, sizeof(unsigned long long), s);
            std::vector<int> hb(nparts + 1);
            for (int q = 0; q <= nparts; ++q) hb[q] = int(bounds[q]);
            cudaMemcpyAsync(sd->d_bounds, hb.data(), hb.size() * sizeof(int),
                            cudaMemcpyHostToDevice, s);
            prepare_source(&g);
            e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) rc = cuda_fail(ctx, e, "subdomain build");
        }
    }
    if (rc) {
        delete sd;
        return rc;
    }
    *out = sd;
    return MCLSGPU_OK;
}

int mclsgpu_subdomain_destroy(mclsgpu_subdomain* sd) {
    delete sd;
    return MCLSGPU_OK;
}

int mclsgpu_subdomain_info(const mclsgpu_subdomain* sd, int64_t* row_begin, int64_t* rows,
                           int32_t* record_bytes) {
    if (!sd) return MCLSGPU_ERR_INVALID_ARG;
    if (row_begin) *row_begin = sd->row0;
    if (rows) *rows = sd->n;
    if (record_bytes) *record_bytes = sd->recs.slots * 8;
    return MCLSGPU_OK;
}

int mclsgpu_subdomain_begin(mclsgpu_subdomain* sd, const double* rhs_dev, int64_t* n_start,
                            int64_t* n_total) {
    if (!sd || !rhs_dev) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = sd->ctx;
    cudaStream_t s = ctx->stream;
    cudaSetDevice(ctx->device);
    cudaMemsetAsync(ctx->d_status, 0, sizeof(int), s);
    const double omega = sd->p.neumann_relaxation;
    if (sd->p.direction == MCLSGPU_FORWARD) {
        // History e starts at row e / per: the part's are a contiguous range.
        // The part's rows' tally source into their records (the whole-domain
        // build's kernels, over the part's rows), the tallies cleared, and the
        // part's slice of the source kept for the finalisation.
        launch_forward_records(&sd->recs, rhs_dev, int(sd->N), omega, omega > 0.0, sd->row0,
                               sd->y);
        cudaMemcpyAsync(sd->srcp, rhs_dev + sd->row0, size_t(sd->n) * sizeof(double),
                        cudaMemcpyDeviceToDevice, s);
        sd->range[0] = (long long)sd->row0 * sd->per;
        sd->range[1] = (long long)(sd->row0 + sd->n) * sd->per;
        sd->range[2] = (long long)sd->N * sd->per;
    } else {
        launch_adjoint_source(&sd->src, rhs_dev, omega, omega > 0.0);
        k_part_range<<<1, 1, 0, s>>>(sd->src.start, sd->src.d_nh, sd->row0, sd->row0 + sd->n,
                                     sd->d_range);
        // Step-0 tallies of the part's rows (counts x starting weight).
        cudaMemcpyAsync(sd->y, sd->src.y64 + sd->row0, size_t(sd->n) * sizeof(double),
                        cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(sd->range, sd->d_range, sizeof(sd->range), cudaMemcpyDeviceToHost, s);
    }
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "subdomain begin");
    int rc = check_device_status(ctx);
    if (rc) return rc;
    if (n_start) *n_start = sd->range[1] - sd->range[0];
    if (n_total) *n_total = sd->range[2];
    sd->ready = 1;
    return MCLSGPU_OK;
}

int mclsgpu_subdomain_transport(mclsgpu_subdomain* sd, const mclsgpu_history_wire* inbox_dev,
                                int64_t n_in, mclsgpu_history_wire* outbox_dev,
                                int64_t capacity, int64_t* out_counts) {
    if (!sd || !outbox_dev || !out_counts || capacity < 1 || n_in < 0 ||
        (n_in > 0 && !inbox_dev))
        return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = sd->ctx;
    if (!sd->ready) return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "mclsgpu_subdomain_begin first");
    cudaStream_t s = ctx->stream;
    cudaSetDevice(ctx->device);
    cudaMemsetAsync(sd->d_out_cnt, 0, sd->nparts * sizeof(unsigned long long), s);
    PartWalk w{};
    w.rec = sd->recs.rec;
    w.slots = sd->recs.slots;
    w.kind = !sd->recs.stencil_k ? 0 : (sd->recs.rec_q16 ? 2 : 1);
    for (int j = 0; j < 32; ++j) w.stoff[j] = sd->recs.stencil_off[j];
    w.row0 = sd->row0;
    w.n = sd->n;
    w.L = sd->p.history_length;
    w.dir = sd->p.direction;
    w.per = sd->per;
    w.cutoff = float(sd->p.weight_cutoff);
    w.start = sd->src.start;
    w.e_begin = sd->range[0];
    w.e_end = sd->range[1];
    w.sc = sd->src.d_scalars;
    w.seed = sd->p.seed;
    w.d_epoch = sd->src.d_epoch;
    w.in = reinterpret_cast<const HistoryWire*>(inbox_dev);
    w.n_in = inbox_dev ? n_in : 0;
    w.out = reinterpret_cast<HistoryWire*>(outbox_dev);
    w.cap = capacity;
    w.out_cnt = sd->d_out_cnt;
    w.nparts = sd->nparts;
    w.bounds = sd->d_bounds;
    w.y = sd->y;
    w.d_steps = sd->d_steps;
    w.status = ctx->d_status;
    launch_walk_part(w, ctx);
    std::vector<unsigned long long> cnt(sd->nparts);
    cudaMemcpyAsync(cnt.data(), sd->d_out_cnt, cnt.size() * sizeof(unsigned long long),
                    cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "subdomain transport");
    for (int q = 0; q < sd->nparts; ++q) out_counts[q] = int64_t(cnt[q]);
    for (int q = 0; q < sd->nparts; ++q)
        if (out_counts[q] > capacity)
            return set_error(ctx, MCLSGPU_ERR_INVALID_ARG,
                             "outbox capacity %lld too small: %lld histories for part %d",
                             (long long)capacity, (long long)out_counts[q], q);
    return check_device_status(ctx);
}

int mclsgpu_subdomain_finish(mclsgpu_subdomain* sd, double* x_part_dev, mclsgpu_stats* stats) {
    if (!sd || !x_part_dev) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = sd->ctx;
    if (!sd->ready) return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "mclsgpu_subdomain_begin first");
    cudaStream_t s = ctx->stream;
    cudaSetDevice(ctx->device);
    if (sd->p.direction == MCLSGPU_FORWARD) {
        const double omega = sd->p.neumann_relaxation;
        k_part_finish_forward<<<grid_for(sd->n), 256, 0, s>>>(
            sd->y, sd->srcp, sd->n, sd->per, sd->p.estimator == MCLSGPU_EXPECTED_VALUE, omega,
            omega > 0.0, x_part_dev);
    } else {
        k_part_finish<<<grid_for(sd->n), 256, 0, s>>>(sd->y, sd->src.d_scalars, sd->n,
                                                      x_part_dev);
    }
    k_epoch_next<<<1, 1, 0, s>>>(sd->src.d_epoch);
    unsigned long long steps = 0;
    cudaMemcpyAsync(&steps, sd->d_steps, sizeof(steps), cudaMemcpyDeviceToHost, s);
    cudaMemsetAsync(sd->d_steps, 0, sizeof(unsigned long long), s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "subdomain finish");
    sd->ready = 0;
    if (stats) {
        stats->walk_steps = int64_t(steps);
        stats->histories = sd->range[1] - sd->range[0];
        stats->iterations = 0;
        stats->converged = 1;
    }
    return check_device_status(ctx);
}

int32_t mclsgpu_history_wire_size(void) { return int32_t(sizeof(HistoryWire)); }

}  // extern "C"
