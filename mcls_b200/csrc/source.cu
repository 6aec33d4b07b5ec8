// source.cu -- device build of the Monte Carlo source.
//
// Adjoint (UniformAdjointSource, src/MCLS_UniformAdjointSource_impl.hpp:58-263):
//   weight = |b|_1; random sampling draws nh = int(Nh * cdf.back() / |b|_1)
//   starting states from the CDF of |b| (whose first element is the signed
//   b[0], :185) with lower_bound; stratified sampling takes
//   ceil(|b_i| * nh_local / sum|b|) histories per state.  Histories are
//   emitted from the highest state down (the LIFO stack of :157-175); the
//   emission order fixes which uniforms each history consumes in the
//   reference stream.
// Forward (UniformForwardSource, src/MCLS_UniformForwardSource_impl.hpp:60-148):
//   ceil(Sample Ratio) histories per state in state order, weight 1.
//
// Sampling uses a guide table over the FP64 CDF: guide[t] is the first state
// whose floor(cdf*G) reaches t, so the lower_bound of u lies in
// [guide[t], guide[t+1]] with t = floor(u*G); a short binary search in that
// window returns exactly std::lower_bound's answer.
#include <cfloat>
#include <climits>

#include <mutex>

#include "internal.h"
#include "rng.cuh"

namespace mclsgpu {
namespace {

inline int grid_for(long long work, int threads = 256, int cap = 148 * 16) {
    long long g = (work + threads - 1) / threads;
    if (g < 1) g = 1;
    return int(g > cap ? cap : g);
}

__device__ __forceinline__ double load_src(const double* v, int i, double omega, int has) {
    return has ? v[i] * omega : v[i];
}

// nh = int(Nh_total * cdf.back() / norm1)  (:198); weight = norm1 (:67)
__global__ void k_random_count(int nh_req, double* sc, int* d_nh, int cap, int* status) {
    const double norm1 = sc[0], total = sc[1];
    const double r = __ddiv_rn(__dmul_rn(double(nh_req), total), norm1);
    int nh = (r >= 0.0 && r < 2147483647.0) ? int(r) : (r >= 2147483647.0 ? INT_MAX : 0);
    if (!isfinite(norm1) || !isfinite(total)) {
        nh = 0;
        atomicOr(status, DEV_ERR_NONFINITE);
    } else if (!(norm1 > 0.0)) {
        nh = 0;  // zero source (an exact iterate): no histories, zero correction
    }
    if (nh > cap) {
        // total <= norm1 in exact arithmetic, so nh <= nh_req <= cap; more
        // means the source sums lost all precision (a diverging iteration).
        atomicOr(status, DEV_ERR_NONFINITE);
        nh = cap;
    }
    *d_nh = nh;
    sc[2] = nh > 0 ? 1.0 / double(nh) : 0.0;
}

__global__ void k_guide_marks(const double* cdf, int n, int* marks) {
    // marks[t] = max j whose window starts at t = floor(cdf[j-1]*G)+1.
    const double G = double(n);
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        long long t0 = 0;
        if (j > 0) {
            double f = floor(cdf[j - 1] * G);
            t0 = f < -1.0 ? 0 : (long long)f + 1;
        }
        if (t0 < 0) t0 = 0;
        if (t0 <= n - 1) atomicMax(&marks[t0], j);
    }
}

__device__ __forceinline__ int guided_lower_bound(const double* cdf, const int* guide, int n,
                                                  double u) {
    long long t = (long long)floor(u * double(n));
    if (t < 0) t = 0;
    if (t > n - 1) t = n - 1;
    int lo = guide[t];
    int hi = t + 1 < n ? guide[t + 1] : n - 1;
    if (lo < 0) lo = 0;
    if (hi < lo) hi = lo;
    // first j in [lo, hi] with cdf[j] >= u (cdf[hi] >= u by construction)
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (cdf[mid] < u) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Random sampling: draw k in [0, nh) -> counts[lower_bound(cdf, u_k)]++.
// Reference stream: each thread owns a contiguous run of draws and jumps once.
__global__ void k_sample(const double* cdf, const int* guide, int n, const int* d_nh,
                         int rng_mode, uint64_t seed, const unsigned long long* d_epoch,
                         const uint64_t* jump, const unsigned long long* d_pos, int* counts) {
    const int nh = *d_nh;
    const uint64_t ekey = epoch_key(seed, *d_epoch);
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthreads = gridDim.x * blockDim.x;
    if (rng_mode == MCLSGPU_RNG_COUNTER) {
        for (int k = tid; k < nh; k += nthreads) {
            uint64_t x = xs_step(counter_state(ekey, 1, uint64_t(k)));
            int j = guided_lower_bound(cdf, guide, n, canonical64(x));
            atomicAdd(&counts[j], 1);
        }
    } else {
        const int per = (nh + nthreads - 1) / nthreads;
        const long long k0 = (long long)tid * per;
        if (k0 >= nh) return;
        const long long k1 = k0 + per < nh ? k0 + per : nh;
        uint64_t x = xs_jump(jump, seed, *d_pos + uint64_t(k0));
        for (long long k = k0; k < k1; ++k) {
            x = xs_step(x);
            int j = guided_lower_bound(cdf, guide, n, canonical64(x));
            atomicAdd(&counts[j], 1);
        }
    }
}

__global__ void k_advance_pos(unsigned long long* d_pos, const int* d_nh, int mult) {
    *d_pos += (unsigned long long)(*d_nh) * (unsigned long long)mult;
}

// Stratified: nh_local = ceil(Nh * local_sum / weight) (:241);
// counts_i = ceil(|b_i| * (nh_local / local_sum)) (:246-262).
__global__ void k_strat_prep(int nh_req, double* sc) {
    const double s = sc[0];
    if (!(s > 0.0)) {  // zero source: no histories (non-finite sums are flagged elsewhere)
        sc[3] = 0.0;
        return;
    }
    const double nh_local = ceil(__ddiv_rn(__dmul_rn(double(nh_req), s), s));
    sc[3] = __ddiv_rn(double(int(nh_local)), s);
}

__global__ void k_strat_counts(const double* v, int n, double omega, int has, const double* sc,
                               int* counts) {
    const double num_over_sum = sc[3];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double c = ceil(__dmul_rn(fabs(load_src(v, i, omega, has)), num_over_sum));
        counts[i] = c > 0.0 ? int(c) : 0;
    }
}

__global__ void k_strat_total(int* d_nh, double* sc, int cap, int* status) {
    int nh = *d_nh;
    if (nh > cap) {
        atomicOr(status, DEV_ERR_CAPACITY);
        nh = cap;
        *d_nh = nh;
    }
    sc[2] = nh > 0 ? 1.0 / double(nh) : 0.0;
}

// Emission order and step-0 collision tally: start[offs_i + t] = i | sign,
// y_i = counts_i * w0_i (the tally every history makes at its first state).
template <class TY>
__global__ void k_expand(const double* v, int n, double omega, int has, const int* counts,
                         const int* offs, const double* sc, int cap, int* start, TY* y,
                         int* status) {
    const double weight = sc[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = counts[i];
        const double b = load_src(v, i, omega, has);
        const unsigned sign = b > 0.0 ? 0u : 0x80000000u;  // weight_sign (:169)
        if (c > 0) {
            const int base = offs[i];
            if (base + c > cap) {
                atomicOr(status, DEV_ERR_CAPACITY);
            } else {
                for (int t = 0; t < c; ++t) start[base + t] = int(unsigned(i) | sign);
            }
            const double w0 = sign ? -weight : weight;
            y[i] = TY(double(c) * w0);
        } else {
            y[i] = TY(0);
        }
    }
}

// Forward tally source: c = src (collision) or H src (expected value).
template <class TC>
__global__ void k_forward_c(const double* v, int n, double omega, int has, int ev, const int* rp,
                            const int* ci, const double* h, TC* c) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s;
        if (!ev) {
            s = load_src(v, i, omega, has);
        } else {
            s = 0.0;
            for (int k = rp[i]; k < rp[i + 1]; ++k)
                s = fma(h[k], load_src(v, ci[k], omega, has), s);
        }
        c[i] = TC(s);
    }
}

// FP32 forward walk: the tally source of each state goes into its record's
// header word (slot 0, second word) so that a step reads one record only;
// the history-sum tallies are cleared in the same pass.
__global__ void __launch_bounds__(256) k_forward_rec(const double* v, int n, int row0,
                                                     double omega, int has, int ev,
                                                     const int* off, const int* col,
                                                     const double* h, int slots, uint2* rec,
                                                     double* y) {
    // H over SELL-32: a warp owns one slice, every entry column is one
    // coalesced access.
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double c;
        if (!ev) {
            c = load_src(v, row0 + i, omega, has);
        } else {
            c = 0.0;
            const int o = off[i >> 5] + (i & 31), w = (off[(i >> 5) + 1] - off[i >> 5]) >> 5;
            for (int k = 0; k < w; ++k)
                c = fma(h[o + 32 * k], load_src(v, col[o + 32 * k], omega, has), c);
        }
        rec[size_t(i) * slots].y = __float_as_uint(__double2float_rn(c));
        y[i] = 0.0;
    }
}

struct StencilOffsets {
    int off[32];
};

// Stencil records: the tally source H b is rebuilt from the record itself,
// |h_j| = W * (cdf_j - cdf_prev), so the pass reads 32 bytes per row instead
// of the FP64 domain.
// Tally source of one stencil record of WORDS 32-bit words: c = sum_j h_j
// v[i + off_j] with |h_j| = W (|cdf_j| - |cdf_prev|) and the sign of slot j.
// The record is read with 256-bit loads and its first 32 bytes (W, c and the
// first CDF slots) written back with one 256-bit store.
// The source at the stencil neighbours of state i, loaded before the record
// so that both round trips overlap (an index outside [0, n) -- a neighbour
// the row does not have -- is clamped and its value never used).
template <int SLOTS>
__device__ __forceinline__ void prefetch_neighbours(const double* v, int i, int n, double omega,
                                                    int has, int K, const StencilOffsets& so,
                                                    double (&vs)[SLOTS]) {
    // Every slot is loaded (a slot past K has offset 0: the state itself), so
    // the loop unrolls and vs stays in registers.
#pragma unroll
    for (int j = 0; j < SLOTS; ++j) {
        int g = i + so.off[j];
        g = g < 0 ? 0 : (g >= n ? n - 1 : g);
        vs[j] = load_src(v, g, omega, has);
    }
}

template <int WORDS>
__device__ __forceinline__ void rec_stencil_source(uint32_t* r, int i, int n, const double* v,
                                                   double omega, int has, int K,
                                                   const StencilOffsets& so) {
    // 32-byte records: the neighbours' source loaded before the record; larger
    // records load it slot by slot after the record (their slot counts would
    // cost the registers of several resident blocks).
    constexpr bool kPre = WORDS == 8;
    double vs[kPre ? WORDS - 2 : 1];
    if constexpr (kPre) prefetch_neighbours<WORDS - 2>(v, i, n, omega, has, K, so, vs);
    uint32_t q[WORDS];
#pragma unroll
    for (int t = 0; t < WORDS / 8; ++t)
        asm volatile("ld.global.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(q[8 * t]), "=r"(q[8 * t + 1]), "=r"(q[8 * t + 2]), "=r"(q[8 * t + 3]),
                       "=r"(q[8 * t + 4]), "=r"(q[8 * t + 5]), "=r"(q[8 * t + 6]),
                       "=r"(q[8 * t + 7])
                     : "l"(r + 8 * t));
    const float W = __uint_as_float(q[0]);
    float prev = 0.f;
    double c = 0.0;
#pragma unroll
    for (int j = 0; j < WORDS - 2; ++j) {
        if (j >= K) break;
        const float qv = __uint_as_float(q[2 + j]);
        if (isnan(qv)) continue;
        const float a = fabsf(qv);
        const float h = W * (a - prev);
        prev = a;
        double src;
        if constexpr (kPre) src = vs[j];
        else src = load_src(v, i + so.off[j], omega, has);
        c = fma(double(qv < 0.f ? -h : h), src, c);
    }
    q[1] = __float_as_uint(__double2float_rn(c));
    asm volatile("st.global.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(r), "r"(q[0]),
                 "r"(q[1]), "r"(q[2]), "r"(q[3]), "r"(q[4]), "r"(q[5]), "r"(q[6]), "r"(q[7])
                 : "memory");
}

// The same for a stencil16 record: slot j carries |h_j| = W (t_j - t_prev) /
// 65536 (the last entry's 65535 standing for 65536), the transition
// probabilities the walk samples, and the sign in bit j of word 2.
template <int WORDS>
__device__ __forceinline__ void rec_stencil16_source(uint32_t* r, int i, int n, const double* v,
                                                     double omega, int has, int K,
                                                     const StencilOffsets& so) {
    constexpr bool kPre = WORDS == 8;
    double vs[kPre ? 2 * (WORDS - 3) : 1];
    if constexpr (kPre) prefetch_neighbours<2 * (WORDS - 3)>(v, i, n, omega, has, K, so, vs);
    uint32_t q[WORDS];
#pragma unroll
    for (int t = 0; t < WORDS / 8; ++t)
        asm volatile("ld.global.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(q[8 * t]), "=r"(q[8 * t + 1]), "=r"(q[8 * t + 2]), "=r"(q[8 * t + 3]),
                       "=r"(q[8 * t + 4]), "=r"(q[8 * t + 5]), "=r"(q[8 * t + 6]),
                       "=r"(q[8 * t + 7])
                     : "l"(r + 8 * t));
    const float W = __uint_as_float(q[0]);
    unsigned prev = 0u;
    double c = 0.0;
#pragma unroll
    for (int j = 0; j < 2 * (WORDS - 3); ++j) {
        if (j >= K) break;
        unsigned t = (q[3 + j / 2] >> (16 * (j & 1))) & 0xffffu;
        if (t == 0u) continue;
        if (t == 65535u) t = 65536u;
        const float h = W * (float(t - prev) * 0x1p-16f);
        prev = t;
        double src;
        if constexpr (kPre) src = vs[j];
        else src = load_src(v, i + so.off[j], omega, has);
        c = fma(double(((q[2] >> j) & 1u) ? -h : h), src, c);
    }
    q[1] = __float_as_uint(__double2float_rn(c));
    asm volatile("st.global.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(r), "r"(q[0]),
                 "r"(q[1]), "r"(q[2]), "r"(q[3]), "r"(q[4]), "r"(q[5]), "r"(q[6]), "r"(q[7])
                 : "memory");
}

// One kernel per record layout (WORDS 32-bit words, Q16: 16-bit
// thresholds), so that each keeps only its own slots' prefetched source in
// registers.
template <int WORDS, bool Q16>
__global__ void __launch_bounds__(256) k_forward_rec_stencil(const double* v, int nv, int n,
                                                             int row0, double omega, int has,
                                                             int ev, int K, StencilOffsets so,
                                                             uint32_t* rec, double* y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t* r = rec + size_t(i) * WORDS;
        const int g = row0 + i;  // the state's index in v
        if (!ev)
            r[1] = __float_as_uint(__double2float_rn(load_src(v, g, omega, has)));
        else if constexpr (Q16)
            rec_stencil16_source<WORDS>(r, g, nv, v, omega, has, K, so);
        else
            rec_stencil_source<WORDS>(r, g, nv, v, omega, has, K, so);
        y[i] = 0.0;
    }
}

__global__ void k_forward_nh(int* d_nh, int nh, double* sc) {
    *d_nh = nh;
    sc[0] = 1.0;
    sc[2] = 1.0 / double(nh);
}

// ---- small systems: the whole adjoint source in one CTA ------------------
// For a few thousand states the multi-kernel source build (reductions,
// scans, guide table, sampling, expansion: about 19 launches) is all launch
// latency.  One block of 1024 threads does the same steps in shared memory
// and registers: |v|_1 and the CDF with the reference's signed first element
// (both sums with one association, so that they agree when v[0] >= 0), the
// history count, the normalised CDF, the counter-stream draws with
// lower_bound (the guide table only narrows that search), the counts' suffix
// scan (LIFO emission order) and the expansion into starting states.
constexpr int kSmallThreads = 1024;
constexpr int kSmallSourceMax = 16384;

// Inclusive block scan of one value per thread (all 1024 threads call it).
__device__ __forceinline__ double block_scan_incl(double x, double* warp_tot) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        double t = warp_tot[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, t, d);
            if (lane >= d) t += y;
        }
        warp_tot[lane] = t;
    }
    __syncthreads();
    const double r = w > 0 ? x + warp_tot[w - 1] : x;
    __syncthreads();
    return r;
}

__device__ __forceinline__ int block_scan_incl_int(int x, int* warp_tot) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = warp_tot[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, d);
            if (lane >= d) t += y;
        }
        warp_tot[lane] = t;
    }
    __syncthreads();
    const int r = w > 0 ? x + warp_tot[w - 1] : x;
    __syncthreads();
    return r;
}

// Shared memory: the CDF (n doubles) and the per-state counts (n ints).
constexpr int kSmallSmem = kSmallSourceMax * (sizeof(double) + sizeof(int));

__global__ void __launch_bounds__(kSmallThreads) k_small_adjoint_source(
    const double* v, int n, double omega, int has, int nh_req, int cap, uint64_t seed,
    const unsigned long long* d_epoch, int* start, double* y, double* sc, int* d_nh,
    int* status) {
    extern __shared__ __align__(16) unsigned char smem_src[];
    double* cdf = reinterpret_cast<double*>(smem_src);
    int* counts = reinterpret_cast<int*>(smem_src + sizeof(double) * kSmallSourceMax);
    __shared__ double wtot[32];
    __shared__ int wtoti[32];
    __shared__ double s_carry[2];
    __shared__ int s_carry_i;
    __shared__ int s_nh;
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_carry[0] = 0.0;
        s_carry[1] = 0.0;
        s_carry_i = 0;
    }
    __syncthreads();
    // 1. Raw CDF (signed first element) and |v|_1 with the same association.
    for (int base = 0; base < n; base += kSmallThreads) {
        const int i = base + tid;
        double a = 0.0, sgn = 0.0;
        if (i < n) {
            const double b = load_src(v, i, omega, has);
            a = fabs(b);
            sgn = i == 0 ? b : a;
        }
        const double cs = block_scan_incl(sgn, wtot) + s_carry[0];
        const double ca = block_scan_incl(a, wtot) + s_carry[1];
        if (i < n) cdf[i] = cs;
        __syncthreads();
        if (tid == kSmallThreads - 1) {
            s_carry[0] = cs;
            s_carry[1] = ca;
        }
        __syncthreads();
    }
    // 2. History count nh = int(Nh * cdf.back() / |v|_1) (:198), weights.
    if (tid == 0) {
        const double norm1 = s_carry[1], total = s_carry[0];
        const double r = __ddiv_rn(__dmul_rn(double(nh_req), total), norm1);
        int nh = (r >= 0.0 && r < 2147483647.0) ? int(r) : (r >= 2147483647.0 ? INT_MAX : 0);
        if (!isfinite(norm1) || !isfinite(total)) {
            nh = 0;
            atomicOr(status, DEV_ERR_NONFINITE);
        } else if (!(norm1 > 0.0)) {
            nh = 0;
        }
        if (nh > cap) {
            atomicOr(status, DEV_ERR_NONFINITE);
            nh = cap;
        }
        sc[0] = norm1;
        sc[1] = total;
        sc[2] = nh > 0 ? 1.0 / double(nh) : 0.0;
        *d_nh = nh;
        s_nh = nh;
    }
    __syncthreads();
    const int nh = s_nh;
    // 3. Normalise (cdf[n-1] = 1 exactly) and clear the counts.
    const double total = s_carry[0];
    for (int i = tid; i < n; i += kSmallThreads) {
        cdf[i] = i == n - 1 ? 1.0 : cdf[i] / total;
        counts[i] = 0;
    }
    __syncthreads();
    // 4. Draw the starting states (counter stream, kind 1).
    const uint64_t ekey = epoch_key(seed, *d_epoch);
    for (int k = tid; k < nh; k += kSmallThreads) {
        const double u = canonical64(xs_step(counter_state(ekey, 1, uint64_t(k))));
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (cdf[mid] < u) lo = mid + 1; else hi = mid;
        }
        atomicAdd(&counts[lo], 1);
    }
    __syncthreads();
    // 5. Exclusive suffix sum of the counts (LIFO emission: highest state
    //    first) and, chunk by chunk, the expansion into starting states and
    //    step-0 tallies.
    const double weight = sc[0];
    for (int base = 0; base < n; base += kSmallThreads) {
        const int k = base + tid;      // position in reversed order
        const int i = n - 1 - k;       // state
        const int c = k < n ? counts[i] : 0;
        const int incl = block_scan_incl_int(c, wtoti) + s_carry_i;
        if (k < n) {
            const int o = incl - c;
            const double b = load_src(v, i, omega, has);
            const unsigned sign = b > 0.0 ? 0u : 0x80000000u;
            if (c > 0) {
                if (o + c > cap) {
                    atomicOr(status, DEV_ERR_CAPACITY);
                } else {
                    for (int t = 0; t < c; ++t) start[o + t] = int(unsigned(i) | sign);
                }
                y[i] = double(c) * (sign ? -weight : weight);
            } else {
                y[i] = 0.0;
            }
        }
        __syncthreads();
        if (tid == kSmallThreads - 1) s_carry_i = incl;
        __syncthreads();
    }
}

// Dynamic shared memory opt-in for k_small_adjoint_source, once per device.
std::mutex g_small_mutex;
bool g_small_set[64] = {false};

bool small_source_ready(mclsgpu_context* ctx) {
    std::lock_guard<std::mutex> lock(g_small_mutex);
    const int d = ctx->device;
    if (d >= 0 && d < 64 && g_small_set[d]) return true;
    if (cudaFuncSetAttribute(k_small_adjoint_source, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kSmallSmem) != cudaSuccess) {
        cudaGetLastError();
        return false;  // keep the multi-kernel path
    }
    if (d >= 0 && d < 64) g_small_set[d] = true;
    return true;
}

}  // namespace

// Set-up time (outside any stream capture): the small-system source kernel's
// shared-memory opt-in.
void prepare_source(mclsgpu_domain* dom) {
    if (dom->n <= kSmallSourceMax && dom->p.direction == MCLSGPU_ADJOINT)
        small_source_ready(dom->ctx);
}

// Build the adjoint source from v*omega (omega applied when has_omega).
void launch_adjoint_source(mclsgpu_domain* dom, const double* v, double omega, int has_omega) {
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    const int n = dom->n;
    const mclsgpu_mc_params& p = dom->p;
    // The reproducible mode (FP64 walks on the reference stream) is the parity
    // template: |b|_1 and the source CDF follow the reference's left-to-right
    // summation order (one thread).  Every other mode uses the parallel tree
    // order, which can differ in the last bits of |b|_1 and the CDF.
    const bool parity = p.precision == MCLSGPU_FP64 && p.rng_mode == MCLSGPU_RNG_REFERENCE;
    const int nh_req = p.sample_ratio > 0.0 ? int(double(n) * p.sample_ratio) : n;
    const int cap = int(dom->nh_cap);
    if (!parity && p.rng_mode == MCLSGPU_RNG_COUNTER &&
        p.source_sampling == MCLSGPU_SOURCE_RANDOM && n <= kSmallSourceMax &&
        small_source_ready(ctx)) {
        k_small_adjoint_source<<<1, kSmallThreads, kSmallSmem, s>>>(
            v, n, omega, has_omega, nh_req, cap, dom->seed, dom->d_epoch, dom->start, dom->y64,
            dom->d_scalars, dom->d_nh, ctx->d_status);
        return;
    }
    // weight = |b|_1
    abs_sum(s, v, n, omega, has_omega, parity ? nullptr : dom->part, dom->d_scalars + 0);
    cudaMemsetAsync(dom->counts, 0, size_t(n) * sizeof(int), s);
    if (p.source_sampling == MCLSGPU_SOURCE_RANDOM) {
        source_cdf(s, v, n, omega, has_omega, parity ? 1 : 0, dom->part, dom->scdf,
                   dom->d_scalars + 1);
        k_random_count<<<1, 1, 0, s>>>(nh_req, dom->d_scalars, dom->d_nh, cap, ctx->d_status);
        cudaMemsetAsync(dom->guide, 0xFF, size_t(n) * sizeof(int), s);
        k_guide_marks<<<grid_for(n), 256, 0, s>>>(dom->scdf, n, dom->guide);
        max_scan_int(s, dom->guide, n, dom->ipart);
        const int sample_grid = p.rng_mode == MCLSGPU_RNG_COUNTER ? ctx->num_sms * 8 : 64;
        k_sample<<<sample_grid, 256, 0, s>>>(dom->scdf, dom->guide, n, dom->d_nh, p.rng_mode,
                                             dom->seed, dom->d_epoch, dom->d_jump, dom->d_pos,
                                             dom->counts);
        if (p.rng_mode == MCLSGPU_RNG_REFERENCE) k_advance_pos<<<1, 1, 0, s>>>(dom->d_pos, dom->d_nh, 1);
        suffix_scan_int(s, dom->counts, n, dom->ipart, dom->offs, nullptr);
    } else {
        k_strat_prep<<<1, 1, 0, s>>>(nh_req, dom->d_scalars);
        k_strat_counts<<<grid_for(n), 256, 0, s>>>(v, n, omega, has_omega, dom->d_scalars,
                                                   dom->counts);
        suffix_scan_int(s, dom->counts, n, dom->ipart, dom->offs, dom->d_nh);
        k_strat_total<<<1, 1, 0, s>>>(dom->d_nh, dom->d_scalars, cap, ctx->d_status);
    }
    k_expand<double><<<grid_for(n), 256, 0, s>>>(v, n, omega, has_omega, dom->counts, dom->offs,
                                                 dom->d_scalars, cap, dom->start, dom->y64,
                                                 ctx->d_status);
}

void launch_forward_setup(mclsgpu_domain* dom) {
    const mclsgpu_mc_params& p = dom->p;
    const int per = p.sample_ratio > 0.0 ? int(ceil(p.sample_ratio)) : 1;
    k_forward_nh<<<1, 1, 0, dom->ctx->stream>>>(dom->d_nh, dom->n * per, dom->d_scalars);
}

void launch_forward_records(mclsgpu_domain* dom, const double* v, int nv, double omega,
                            int has_omega, int row0, double* y) {
    cudaStream_t s = dom->ctx->stream;
    const int n = dom->n;
    const int ev = dom->p.estimator == MCLSGPU_EXPECTED_VALUE;
    if (dom->stencil_k) {
        StencilOffsets so{};
        for (int j = 0; j < 32; ++j) so.off[j] = dom->stencil_off[j];
        const int grid = grid_for(n, 256, 148 * 8);
        uint32_t* rec = reinterpret_cast<uint32_t*>(dom->rec);
        const int K = dom->stencil_k, words = 2 * dom->slots;
#define MCLSGPU_SRC(W, Q)                                                                 \
    k_forward_rec_stencil<W, Q><<<grid, 256, 0, s>>>(v, nv, n, row0, omega, has_omega, ev, K, \
                                                     so, rec, y)
        if (dom->rec_q16) {
            if (words == 8) MCLSGPU_SRC(8, true);
            else MCLSGPU_SRC(16, true);
        } else if (words == 8) {
            MCLSGPU_SRC(8, false);
        } else if (words == 16) {
            MCLSGPU_SRC(16, false);
        } else {
            MCLSGPU_SRC(32, false);
        }
#undef MCLSGPU_SRC
    } else {
        k_forward_rec<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(v, n, row0, omega, has_omega, ev,
                                                               dom->DS.off, dom->DS.col,
                                                               dom->DS.val, dom->slots, dom->rec,
                                                               y);
    }
}

// `fused`: the history count was set once by launch_forward_setup.
void launch_forward_source(mclsgpu_domain* dom, const double* v, double omega, int has_omega,
                           bool fused) {
    mclsgpu_context* ctx = dom->ctx;
    cudaStream_t s = ctx->stream;
    const int n = dom->n;
    const mclsgpu_mc_params& p = dom->p;
    const int per = p.sample_ratio > 0.0 ? int(ceil(p.sample_ratio)) : 1;
    const int ev = p.estimator == MCLSGPU_EXPECTED_VALUE;
    if (!fused) k_forward_nh<<<1, 1, 0, s>>>(dom->d_nh, n * per, dom->d_scalars);
    if (p.precision == MCLSGPU_FP32) {
        launch_forward_records(dom, v, n, omega, has_omega, 0, dom->y64);
    } else {
        k_forward_c<double><<<grid_for(n), 256, 0, s>>>(v, n, omega, has_omega, ev, dom->D.rp,
                                                        dom->D.ci, dom->D.v, dom->c64);
        cudaMemsetAsync(dom->y64, 0, size_t(n) * sizeof(double), s);
    }
}

void launch_advance_walk_pos(mclsgpu_domain* dom) {
    // Variable-length histories advance the stream by their summed lengths
    // in the walk itself.
    if (dom->p.rng_mode == MCLSGPU_RNG_REFERENCE && !walk_needs_rounds(dom))
        k_advance_pos<<<1, 1, 0, dom->ctx->stream>>>(dom->d_pos, dom->d_nh, dom->p.history_length);
}

}  // namespace mclsgpu
