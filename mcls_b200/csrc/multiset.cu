// multiset.cu -- multi-set MCSA: several sets (one per GPU, or per process)
// each transport their own histories and sum their Monte Carlo corrections
// every iteration (MultiSetLinearProblem::blockConstantVectorSum,
// src/MCLS_MultiSetLinearProblem_impl.hpp:102-120, called by
// MCSASolverManager::solve, src/MCLS_MCSASolverManager_impl.hpp:374-377).
//
// One iteration on every set: the smoothing steps, this set's Monte Carlo
// correction delta, the caller's sum of delta over the sets (in place, the
// same order on every set), x += delta / num_sets, the preconditioned
// residual and its norm.  Every set starts from the same x and b and applies
// the same summed delta, so x, the residual and the stopping decision are
// identical on all sets without a second exchange.
//
// The sum is a callback, so any transport serves: the library's NCCL
// communicator (below), which is captured with the rest of the iteration
// into the device-side WHILE loop, or a host reduction (MPI, gloo), which
// runs the loop from the host.
#include <dlfcn.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "internal.h"

namespace mclsgpu {

void mcsa_loop_begin(mclsgpu_domain* dom, const double* b_dev, const double* x_dev,
                     const mclsgpu_mcsa_params* mp);
void mcsa_loop_check(mclsgpu_domain* dom, cudaGraphConditionalHandle handle, int use_cond);
int mcsa_loop_finish(mclsgpu_domain* dom, double* x_dev, float ms, int kernels_per_iter,
                     mclsgpu_stats* stats);
int mcsa_check_params(mclsgpu_domain* dom, const mclsgpu_mcsa_params* in,
                      mclsgpu_mcsa_params* out);

namespace {

__global__ void k_add_scaled(double* x, const double* d, int n, double scale) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        x[i] = __dadd_rn(x[i], __dmul_rn(scale, d[i]));
}

inline int grid_for(long long work, int threads = 256, int cap = 148 * 8) {
    long long g = (work + threads - 1) / threads;
    if (g < 1) g = 1;
    return int(g > cap ? cap : g);
}

// One multi-set iteration (see the file comment); returns the reducer's
// status.
int enqueue_set_iteration(mclsgpu_domain* dom, const mclsgpu_mcsa_params* mp,
                          const mclsgpu_set_params* sp, cudaGraphConditionalHandle handle,
                          int use_cond) {
    cudaStream_t s = dom->ctx->stream;
    const int n = dom->n;
    for (int l = 0; l < mp->smoother_steps; ++l)
        enqueue_fixed_point_step(dom, mp->fixed_point_type, mp->richardson_omega);
    mc_correction(dom, dom->rp, dom->delta);
    const int rc = sp->reduce(sp->user, dom->delta, int64_t(n), s);
    k_add_scaled<<<grid_for(n), 256, 0, s>>>(dom->x, dom->delta, n, 1.0 / double(sp->num_sets));
    prec_residual(dom, dom->x, dom->b, dom->rp);
    sum_sq(s, dom->rp, n, dom->part, dom->d_scalars + 5);
    mcsa_loop_check(dom, handle, use_cond);
    return rc;
}

// ---- NCCL, loaded at run time ----------------------------------------------
// The library does not link NCCL: the first communicator loads libnccl.so.2
// (whichever the process finds) and resolves the five calls it uses.
struct NcclUniqueId {
    char internal[128];
};
typedef void* NcclComm;
enum { kNcclDouble = 8, kNcclSum = 0 };
struct NcclApi {
    int (*get_unique_id)(NcclUniqueId*) = nullptr;
    int (*comm_init_rank)(NcclComm*, int, NcclUniqueId, int) = nullptr;
    int (*all_reduce)(const void*, void*, size_t, int, int, NcclComm, cudaStream_t) = nullptr;
    int (*comm_destroy)(NcclComm) = nullptr;
    const char* (*error_string)(int) = nullptr;
    bool ok = false;
};
std::mutex g_nccl_mutex;
NcclApi g_nccl;

const NcclApi* nccl_api(std::string* why) {
    std::lock_guard<std::mutex> lock(g_nccl_mutex);
    if (g_nccl.ok) return &g_nccl;
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_LOCAL);
    if (!h) {
        *why = "libnccl.so.2 not found";
        return nullptr;
    }
    g_nccl.get_unique_id = reinterpret_cast<int (*)(NcclUniqueId*)>(dlsym(h, "ncclGetUniqueId"));
    g_nccl.comm_init_rank =
        reinterpret_cast<int (*)(NcclComm*, int, NcclUniqueId, int)>(dlsym(h, "ncclCommInitRank"));
    g_nccl.all_reduce = reinterpret_cast<int (*)(const void*, void*, size_t, int, int, NcclComm,
                                                 cudaStream_t)>(dlsym(h, "ncclAllReduce"));
    g_nccl.comm_destroy = reinterpret_cast<int (*)(NcclComm)>(dlsym(h, "ncclCommDestroy"));
    g_nccl.error_string = reinterpret_cast<const char* (*)(int)>(dlsym(h, "ncclGetErrorString"));
    if (!g_nccl.get_unique_id || !g_nccl.comm_init_rank || !g_nccl.all_reduce ||
        !g_nccl.comm_destroy || !g_nccl.error_string) {
        *why = "libnccl.so.2 lacks a required symbol";
        return nullptr;
    }
    g_nccl.ok = true;
    return &g_nccl;
}

}  // namespace
}  // namespace mclsgpu

struct mclsgpu_comm {
    mclsgpu_context* ctx = nullptr;
    mclsgpu::NcclComm nccl = nullptr;
    int nranks = 0;
    int rank = 0;
};

using namespace mclsgpu;

namespace {

// The library's reducer: an in-place NCCL sum on the set's stream.
int nccl_reduce(void* user, double* data, int64_t n, void* stream) {
    mclsgpu_comm* c = static_cast<mclsgpu_comm*>(user);
    const int r = g_nccl.all_reduce(data, data, size_t(n), kNcclDouble, kNcclSum, c->nccl,
                                    static_cast<cudaStream_t>(stream));
    return r == 0 ? MCLSGPU_OK : MCLSGPU_ERR_CUDA;
}

int solve_sets(mclsgpu_domain* dom, const mclsgpu_set_params* sp, const double* b_dev,
               double* x_dev, const mclsgpu_mcsa_params* params, mclsgpu_stats* stats,
               int32_t* device_loop) {
    mclsgpu_context* ctx = dom->ctx;
    if (!sp || sp->size < sizeof(mclsgpu_set_params) || sp->num_sets < 1 || !sp->reduce)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "set params: num_sets >= 1 and a reducer");
    mclsgpu_mcsa_params mp;
    int rc = mcsa_check_params(dom, params, &mp);
    if (rc) return rc;
    if ((rc = prepare_fixed_point(dom, mp.fixed_point_type))) return rc;
    const int n = dom->n;
    cudaStream_t s = ctx->stream;
    if (!dom->delta) {
        cudaError_t e = dmalloc(&dom->delta, size_t(n));
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    }
    if (mp.max_iters > dom->resid_cap) {
        dfree(dom->d_resid);
        cudaError_t e = dmalloc(&dom->d_resid, size_t(mp.max_iters));
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
        dom->resid_cap = mp.max_iters;
        if (dom->graph) {  // the single-set loop recorded the old history buffer
            cudaGraphExecDestroy(dom->graph);
            dom->graph = nullptr;
        }
        if (dom->set_graph) {
            cudaGraphExecDestroy(dom->set_graph);
            dom->set_graph = nullptr;
        }
    }
    // The device-side loop when the reducer can be captured; the graph is kept
    // for the next solve with the same reducer, set count and smoother.
    bool graph = sp->capturable && !mp.host_loop && !walk_needs_rounds(dom);
    if (graph) {
        const long long key = (long long)mp.smoother_steps * 1000003LL + mp.fixed_point_type * 7 +
                              (long long)(mp.richardson_omega * 1e6);
        if (!dom->set_graph || dom->set_graph_reduce != reinterpret_cast<void*>(sp->reduce) ||
            dom->set_graph_user != sp->user || dom->set_graph_sets != sp->num_sets ||
            dom->set_graph_key != key) {
            if (dom->set_graph) cudaGraphExecDestroy(dom->set_graph);
            dom->set_graph = nullptr;
            int red = MCLSGPU_OK;
            rc = build_while_graph(
                ctx,
                [&](cudaGraphConditionalHandle h) {
                    red = enqueue_set_iteration(dom, &mp, sp, h, 1);
                },
                &dom->set_graph, &dom->set_body_kernels);
            if (rc || red) {
                // Not capturable after all: clear the error, loop from the host.
                cudaGetLastError();
                if (dom->set_graph) cudaGraphExecDestroy(dom->set_graph);
                dom->set_graph = nullptr;
                graph = false;
            } else {
                dom->set_graph_reduce = reinterpret_cast<void*>(sp->reduce);
                dom->set_graph_user = sp->user;
                dom->set_graph_sets = sp->num_sets;
                dom->set_graph_key = key;
            }
        }
    }
    if (device_loop) *device_loop = graph ? 1 : 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    mcsa_loop_begin(dom, b_dev, x_dev, &mp);
    cudaError_t e = cudaSuccess;
    int red = MCLSGPU_OK;
    int kernels = dom->set_body_kernels;
    if (graph) {
        e = cudaGraphLaunch(dom->set_graph, s);
    } else {
        kernels = 0;
        for (int it = 0; it < mp.max_iters && e == cudaSuccess && !red; ++it) {
            red = enqueue_set_iteration(dom, &mp, sp, cudaGraphConditionalHandle(0), 0);
            cudaMemcpyAsync(dom->h_state, dom->d_state, sizeof(McsaState), cudaMemcpyDeviceToHost,
                            s);
            e = cudaStreamSynchronize(s);
            if (e == cudaSuccess && dom->h_state->done) break;
        }
    }
    cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "multi-set mcsa");
    if (red) return set_error(ctx, red, "multi-set reducer failed (status %d)", red);
    return mcsa_loop_finish(dom, x_dev, ms, kernels, stats);
}

}  // namespace

extern "C" {

int mclsgpu_mcsa_solve_sets_dev(mclsgpu_domain* dom, const mclsgpu_set_params* sets,
                                const double* b_dev, double* x_dev,
                                const mclsgpu_mcsa_params* params, mclsgpu_stats* stats,
                                int32_t* device_loop) {
    if (!dom || !b_dev || !x_dev) return MCLSGPU_ERR_INVALID_ARG;
    return solve_sets(dom, sets, b_dev, x_dev, params, stats, device_loop);
}

int mclsgpu_mcsa_solve_sets(mclsgpu_domain* dom, const mclsgpu_set_params* sets, const double* b,
                            double* x, const mclsgpu_mcsa_params* params, mclsgpu_stats* stats,
                            int32_t* device_loop) {
    if (!dom || !b || !x) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = dom->ctx;
    const size_t bytes = size_t(dom->n) * sizeof(double);
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(dom->b, b, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dom->x, x, bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy b, x");
    int rc = solve_sets(dom, sets, dom->b, dom->x, params, stats, device_loop);
    if (rc) return rc;
    e = cudaMemcpyAsync(x, dom->x, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(ctx, e, "copy x");
}

int mclsgpu_anderson_solve_sets(mclsgpu_domain* dom, const mclsgpu_set_params* sets,
                                const double* b, double* x,
                                const mclsgpu_anderson_params* params, mclsgpu_stats* stats) {
    if (!dom || !b || !x) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = dom->ctx;
    if (!sets || sets->size < sizeof(mclsgpu_set_params) || sets->num_sets < 1 || !sets->reduce)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "set params: num_sets >= 1 and a reducer");
    const int n = dom->n;
    cudaStream_t s = ctx->stream;
    if (!dom->delta) {
        cudaError_t e = dmalloc(&dom->delta, size_t(n));
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc");
    }
    // b and x0 go straight into the solver's own vectors.
    const size_t bytes = size_t(n) * sizeof(double);
    cudaError_t e = cudaMemcpyAsync(dom->b, b, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dom->x, x, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy b, x");
    double rnorm = 0.0, bnorm = 0.0;
    int32_t done = 0;
    int rc = mclsgpu_anderson_begin(dom, dom->b, dom->x, params, &rnorm, &bnorm, &done);
    const double scale = 1.0 / double(sets->num_sets);
    while (!rc && !done) {
        rc = mclsgpu_anderson_correction(dom, dom->delta);
        if (!rc) {
            rc = sets->reduce(sets->user, dom->delta, int64_t(n), s);
            if (rc) set_error(ctx, rc, "multi-set reducer failed (status %d)", rc);
        }
        if (!rc) rc = mclsgpu_anderson_apply(dom, dom->delta, scale, &rnorm, &done);
    }
    if (rc) return rc;
    rc = mclsgpu_anderson_finish(dom, dom->x, stats);
    if (rc) return rc;
    e = cudaMemcpyAsync(x, dom->x, bytes, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(ctx, e, "copy x");
}

int mclsgpu_comm_unique_id(uint8_t* id) {
    if (!id) return MCLSGPU_ERR_INVALID_ARG;
    std::string why;
    const NcclApi* api = nccl_api(&why);
    if (!api) return MCLSGPU_ERR_UNSUPPORTED;
    NcclUniqueId u;
    if (api->get_unique_id(&u) != 0) return MCLSGPU_ERR_CUDA;
    std::memcpy(id, u.internal, 128);
    return MCLSGPU_OK;
}

int mclsgpu_comm_create(mclsgpu_context* ctx, int nranks, int rank, const uint8_t* id,
                        mclsgpu_comm** out) {
    if (!ctx || !id || !out || nranks < 1 || rank < 0 || rank >= nranks)
        return MCLSGPU_ERR_INVALID_ARG;
    *out = nullptr;
    std::string why;
    const NcclApi* api = nccl_api(&why);
    if (!api) return set_error(ctx, MCLSGPU_ERR_UNSUPPORTED, "NCCL: %s", why.c_str());
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
    NcclUniqueId u;
    std::memcpy(u.internal, id, 128);
    mclsgpu_comm* c = new mclsgpu_comm;
    c->ctx = ctx;
    c->nranks = nranks;
    c->rank = rank;
    const int r = api->comm_init_rank(&c->nccl, nranks, u, rank);
    if (r != 0) {
        delete c;
        return set_error(ctx, MCLSGPU_ERR_CUDA, "ncclCommInitRank: %s", api->error_string(r));
    }
    *out = c;
    return MCLSGPU_OK;
}

int mclsgpu_comm_destroy(mclsgpu_comm* comm) {
    if (!comm) return MCLSGPU_OK;
    if (comm->nccl && g_nccl.ok) g_nccl.comm_destroy(comm->nccl);
    delete comm;
    return MCLSGPU_OK;
}

int mclsgpu_comm_set_params(mclsgpu_comm* comm, mclsgpu_set_params* out) {
    if (!comm || !out) return MCLSGPU_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    out->size = sizeof(mclsgpu_set_params);
    out->num_sets = comm->nranks;
    out->reduce = &nccl_reduce;
    out->user = comm;
    out->capturable = 1;
    return MCLSGPU_OK;
}

}  // extern "C"
