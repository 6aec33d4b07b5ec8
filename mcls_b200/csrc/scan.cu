// scan.cu -- deterministic scans and reductions used by the source build and
// the residual norms.  Reduce-then-scan over tiles of 2048 elements staged
// through shared memory (coalesced loads), a single-block scan of the tile
// partials, and a rescan that adds each tile's carry.  The association order
// is fixed, so results are reproducible run to run.
#include <cfloat>
#include <climits>

#include "internal.h"

namespace mclsgpu {
namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;
constexpr unsigned kFull = 0xffffffffu;

struct AddOp {
    template <class T>
    __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
};
struct MaxOp {
    __device__ __forceinline__ int operator()(int a, int b) const { return a > b ? a : b; }
};

// Inclusive block scan of one value per thread (256 threads).  On return
// *excl holds the exclusive value of this thread.
template <class T, class Op>
__device__ __forceinline__ T block_scan(T v, Op op, T identity, T* warp_tot, T* excl) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T o = __shfl_up_sync(kFull, v, d);
        if (lane >= d) v = op(o, v);
    }
    if (lane == 31) warp_tot[wid] = v;
    __syncthreads();
    if (wid == 0) {
        T t = lane < kThreads / 32 ? warp_tot[lane] : identity;
#pragma unroll
        for (int d = 1; d < 8; d <<= 1) {
            T o = __shfl_up_sync(kFull, t, d);
            if (lane >= d) t = op(o, t);
        }
        if (lane < kThreads / 32) warp_tot[lane] = t;
    }
    __syncthreads();
    if (wid > 0) v = op(warp_tot[wid - 1], v);
    T prev = __shfl_up_sync(kFull, v, 1);
    if (lane == 0) prev = wid > 0 ? warp_tot[wid - 1] : identity;
    *excl = prev;
    __syncthreads();
    return v;
}

// Loaders ---------------------------------------------------------------------
struct CdfLoad {  // source CDF input: signed first element, |.| after
    const double* v;
    double scale;
    int has_scale;
    __device__ __forceinline__ double operator()(int i) const {
        double x = has_scale ? v[i] * scale : v[i];
        return i == 0 ? x : fabs(x);
    }
};
struct AbsLoad {
    const double* v;
    double scale;
    int has_scale;
    __device__ __forceinline__ double operator()(int i) const {
        double x = has_scale ? v[i] * scale : v[i];
        return fabs(x);
    }
};
struct SqLoad {
    const double* v;
    __device__ __forceinline__ double operator()(int i) const { return v[i] * v[i]; }
};
struct RevIntLoad {  // reversed index for suffix sums
    const int* v;
    int n;
    __device__ __forceinline__ int operator()(int r) const { return v[n - 1 - r]; }
};
struct IntLoad {
    const int* v;
    __device__ __forceinline__ int operator()(int i) const { return v[i]; }
};

template <class T, class Load>
__device__ __forceinline__ void stage_tile(Load ld, int n, T identity, T* stage) {
    const int base = blockIdx.x * kTile;
    for (int k = threadIdx.x; k < kTile; k += kThreads) {
        int i = base + k;
        stage[k] = i < n ? ld(i) : identity;
    }
    __syncthreads();
}

template <class T, class Op, class Load>
__global__ void __launch_bounds__(kThreads) tile_reduce(Load ld, int n, Op op, T identity,
                                                        T* part) {
    __shared__ T stage[kTile];
    __shared__ T warp_tot[32];
    stage_tile(ld, n, identity, stage);
    T acc = stage[threadIdx.x * kItems];
#pragma unroll
    for (int k = 1; k < kItems; ++k) acc = op(acc, stage[threadIdx.x * kItems + k]);
    T excl;
    T incl = block_scan(acc, op, identity, warp_tot, &excl);
    if (threadIdx.x == kThreads - 1) part[blockIdx.x] = incl;
}

// Exclusive scan of the tile partials in one block; part[nb] = total.
template <class T, class Op>
__global__ void __launch_bounds__(kThreads) partial_scan(T* part, int nb, Op op, T identity) {
    __shared__ T warp_tot[32];
    __shared__ T carry_s;
    if (threadIdx.x == 0) carry_s = identity;
    __syncthreads();
    for (int base = 0; base < nb; base += kThreads) {
        int i = base + threadIdx.x;
        T v = i < nb ? part[i] : identity;
        T excl;
        T incl = block_scan(v, op, identity, warp_tot, &excl);
        T carry = carry_s;
        if (i < nb) part[i] = op(carry, excl);
        __syncthreads();
        if (threadIdx.x == kThreads - 1) carry_s = op(carry, incl);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[nb] = carry_s;
}

template <class T, class Op, class Load, class Store>
__global__ void __launch_bounds__(kThreads) tile_rescan(Load ld, int n, Op op, T identity,
                                                        const T* part, Store st) {
    __shared__ T stage[kTile];
    __shared__ T warp_tot[32];
    stage_tile(ld, n, identity, stage);
    T loc[kItems];
    loc[0] = stage[threadIdx.x * kItems];
#pragma unroll
    for (int k = 1; k < kItems; ++k) loc[k] = op(loc[k - 1], stage[threadIdx.x * kItems + k]);
    T excl;
    block_scan(loc[kItems - 1], op, identity, warp_tot, &excl);
    const T carry = part[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kItems; ++k)
        stage[threadIdx.x * kItems + k] = op(carry, op(excl, loc[k]));
    __syncthreads();
    const int base = blockIdx.x * kTile;
    for (int k = threadIdx.x; k < kTile; k += kThreads) {
        int i = base + k;
        if (i < n) st(i, stage[k]);
    }
}

struct RawCdfStore {  // unnormalised CDF
    double* cdf;
    __device__ __forceinline__ void operator()(int i, double v) const { cdf[i] = v; }
};
struct RevExclStore {  // inclusive over reversed index -> exclusive suffix
    int* out;
    const int* in;
    int n;
    __device__ __forceinline__ void operator()(int r, int v) const {
        int i = n - 1 - r;
        out[i] = v - in[i];
    }
};
struct PlainStore {
    int* out;
    __device__ __forceinline__ void operator()(int i, int v) const { out[i] = v; }
};

// cdf[i] /= cdf.back()  (src/MCLS_UniformAdjointSource_impl.hpp:201-205).  The
// total is the reduce-then-scan total, which uses the same association as the
// |b|_1 reduction, so total == |b|_1 bit for bit whenever b[0] > 0 (as in the
// reference's sequential sums); the last element is set to exactly 1.
__global__ void normalize_cdf(double* cdf, int n, const double* total) {
    const double t = *total;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        cdf[i] = i == n - 1 ? 1.0 : cdf[i] / t;
}

__global__ void seq_source_cdf(CdfLoad ld, int n, double* cdf, double* total) {
    // buildRandomSource left-to-right order (src/MCLS_UniformAdjointSource_impl.hpp:184-204)
    double c = ld(0);
    cdf[0] = c;
    for (int i = 1; i < n; ++i) {
        c = c + ld(i);
        cdf[i] = c;
    }
    const double back = c;
    for (int i = 0; i < n; ++i) cdf[i] = cdf[i] / back;
    *total = back;
}

__global__ void seq_abs_sum(AbsLoad ld, int n, double* out) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s = s + ld(i);
    *out = s;
}

template <class T>
__global__ void copy_total(const T* part, int nb, T* out) {
    *out = part[nb];
}

inline int tiles(int n) { return (n + kTile - 1) / kTile; }

}  // namespace

int scan_partials_needed(int n) { return tiles(n) + 2; }

void abs_sum(cudaStream_t s, const double* v, int n, double scale, int has_scale,
             double* part, double* out) {
    AbsLoad ld{v, scale, has_scale};
    if (part == nullptr) {
        seq_abs_sum<<<1, 1, 0, s>>>(ld, n, out);
        return;
    }
    int nb = tiles(n);
    tile_reduce<double><<<nb, kThreads, 0, s>>>(ld, n, AddOp(), 0.0, part);
    partial_scan<double><<<1, kThreads, 0, s>>>(part, nb, AddOp(), 0.0);
    copy_total<double><<<1, 1, 0, s>>>(part, nb, out);
}

void sum_sq(cudaStream_t s, const double* v, int n, double* part, double* out) {
    SqLoad ld{v};
    int nb = tiles(n);
    tile_reduce<double><<<nb, kThreads, 0, s>>>(ld, n, AddOp(), 0.0, part);
    partial_scan<double><<<1, kThreads, 0, s>>>(part, nb, AddOp(), 0.0);
    copy_total<double><<<1, 1, 0, s>>>(part, nb, out);
}

void source_cdf(cudaStream_t s, const double* v, int n, double scale, int has_scale,
                int sequential, double* part, double* cdf, double* total) {
    CdfLoad ld{v, scale, has_scale};
    if (sequential) {
        seq_source_cdf<<<1, 1, 0, s>>>(ld, n, cdf, total);
        return;
    }
    int nb = tiles(n);
    tile_reduce<double><<<nb, kThreads, 0, s>>>(ld, n, AddOp(), 0.0, part);
    partial_scan<double><<<1, kThreads, 0, s>>>(part, nb, AddOp(), 0.0);
    copy_total<double><<<1, 1, 0, s>>>(part, nb, total);
    tile_rescan<double><<<nb, kThreads, 0, s>>>(ld, n, AddOp(), 0.0, part, RawCdfStore{cdf});
    normalize_cdf<<<(n + 1023) / 1024 < 1184 ? (n + 1023) / 1024 : 1184, 1024, 0, s>>>(cdf, n, total);
}

void suffix_scan_int(cudaStream_t s, const int* in, int n, int* part, int* out, int* total) {
    RevIntLoad ld{in, n};
    int nb = tiles(n);
    tile_reduce<int><<<nb, kThreads, 0, s>>>(ld, n, AddOp(), 0, part);
    partial_scan<int><<<1, kThreads, 0, s>>>(part, nb, AddOp(), 0);
    if (total) copy_total<int><<<1, 1, 0, s>>>(part, nb, total);
    tile_rescan<int><<<nb, kThreads, 0, s>>>(ld, n, AddOp(), 0, part, RevExclStore{out, in, n});
}

void max_scan_int(cudaStream_t s, int* a, int n, int* part) {
    IntLoad ld{a};
    int nb = tiles(n);
    tile_reduce<int><<<nb, kThreads, 0, s>>>(ld, n, MaxOp(), INT_MIN, part);
    partial_scan<int><<<1, kThreads, 0, s>>>(part, nb, MaxOp(), INT_MIN);
    tile_rescan<int><<<nb, kThreads, 0, s>>>(ld, n, MaxOp(), INT_MIN, part, PlainStore{a});
}

}  // namespace mclsgpu
