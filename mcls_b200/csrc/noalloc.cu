// noalloc.cu -- y = A x with host vectors and no device allocation.
//
// mclsgpu_operator_apply stages the host vectors through device buffers it
// allocates and frees on every call.  Some callers cannot let a library call
// cudaMalloc/cudaFree: a host thread that runs under a real-time budget
// (cudaMalloc and cudaFree can synchronise the device and take milliseconds),
// an application whose memory pool owns every byte of device memory, or code
// that must not change the device's allocation state while other work runs.
// mclsgpu_operator_apply_static serves them: the same SpMV kernel, staged
// through one file-scope device array instead of per-call buffers.
//
// Limits and sharing rules:
//   * The staging array holds x and y for at most kStaticApplyMaxRows rows
//     (2 x 8 MiB); larger operators are rejected with MCLSGPU_ERR_INVALID_ARG.
//   * Every GPU that loads this library holds the array until the process
//     exits.
//   * All calls on a device share the one array and it keeps the last call's
//     contents.  Calls that overlap on the GPU (another host thread, another
//     context or stream on the same device) race on it; serialise them.
//   * The first call on a device looks up the array's device address (once
//     per device, with that device current).  Make that first call before
//     any stream capture begins.  The address is cached together with the
//     device's current CUDA context; after cudaDeviceReset (or any other
//     teardown of the primary context) the module is loaded again, the
//     context handle changes and the next call looks the address up anew.
#include <cuda.h>

#include <mutex>

#include "internal.h"

namespace mclsgpu {
namespace {

constexpr int kStaticApplyMaxRows = 1 << 20;
constexpr int kMaxDevices = 64;

// Staging for x (first half) and y (second half).  In host code this name is
// only a stand-in for the symbol; the kernel gets the device address.
static __device__ __align__(256) double g_apply_stage[2 * kStaticApplyMaxRows];

std::mutex g_addr_mutex;
double* g_addr[kMaxDevices] = {nullptr};
CUcontext g_addr_ctx[kMaxDevices] = {nullptr};

typedef CUresult (*CtxGetCurrentFn)(CUcontext*);

// cuCtxGetCurrent through the runtime's driver entry point table, so the
// library needs no link against libcuda.  Called with g_addr_mutex held.
int current_context(mclsgpu_context* ctx, CUcontext* out) {
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000,
                                                         cudaEnableDefault, &q);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "driver entry point cuCtxGetCurrent");
        if (q != cudaDriverEntryPointSuccess || !f)
            return set_error(ctx, MCLSGPU_ERR_CUDA, "driver entry point cuCtxGetCurrent not found");
        fn = reinterpret_cast<CtxGetCurrentFn>(f);
    }
    if (fn(out) != CUDA_SUCCESS || !*out)
        return set_error(ctx, MCLSGPU_ERR_CUDA, "no current CUDA context");
    return MCLSGPU_OK;
}

// Device address of the staging array on `device` (the current device), looked
// up once per device and again whenever the device's context has changed.
int stage_address(mclsgpu_context* ctx, double** out) {
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (ctx->device < 0 || ctx->device >= kMaxDevices)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG, "device ordinal out of range");
    CUcontext cur = nullptr;
    int rc = current_context(ctx, &cur);
    if (rc) return rc;
    if (!g_addr[ctx->device] || g_addr_ctx[ctx->device] != cur) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_apply_stage);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGetSymbolAddress(staging array)");
        g_addr[ctx->device] = static_cast<double*>(p);
        g_addr_ctx[ctx->device] = cur;
    }
    *out = g_addr[ctx->device];
    return MCLSGPU_OK;
}

}  // namespace
}  // namespace mclsgpu

using namespace mclsgpu;

extern "C" int mclsgpu_operator_apply_static(mclsgpu_operator* op, const double* x, double* y) {
    if (!op || !x || !y) return MCLSGPU_ERR_INVALID_ARG;
    mclsgpu_context* ctx = op->ctx;
    if (op->A.n > kStaticApplyMaxRows)
        return set_error(ctx, MCLSGPU_ERR_INVALID_ARG,
                         "operator has %d rows; the static staging array holds at most %d",
                         op->A.n, kStaticApplyMaxRows);
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
    double* stage = nullptr;
    int rc = stage_address(ctx, &stage);
    if (rc) return rc;
    double* dx = stage;
    double* dy = stage + kStaticApplyMaxRows;
    const size_t bytes = size_t(op->A.n) * sizeof(double);
    // Every y row is written by the kernel, so nothing needs clearing.
    e = cudaMemcpyAsync(dx, x, bytes, cudaMemcpyHostToDevice, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy x");
    spmv(ctx->stream, op->A, dx, dy);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "static apply: spmv launch");
    e = cudaMemcpyAsync(y, dy, bytes, cudaMemcpyDeviceToHost, ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy y");
    e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? MCLSGPU_OK : cuda_fail(ctx, e, "static apply");
}
