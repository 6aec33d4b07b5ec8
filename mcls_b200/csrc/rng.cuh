// rng.cuh -- random streams of the walk and source kernels (host + device).
//
// Two streams are provided.
//
// REFERENCE: the reference's single Xorshift<uint_fast64_t,13,7,17> stream
// (src/MCLS_Xorshift.hpp:100-108) consumed in the reference's order, mapped
// to [0,1) as libstdc++'s uniform_real_distribution<double> does for a
// 2^64-range engine (one draw, (double)r * 2^-64, clamped below 1).  Xorshift
// is linear over GF(2), so the state after d draws is T^d(seed) with T a
// 64x64 bit matrix; the tables J_p = T^(2^p) let every history jump straight
// to its first draw, which makes the reference stream counter-addressable.
//
// COUNTER: per-history streams keyed by (seed, epoch, kind, index): two
// splitmix64 finalisations of the key give the initial state, then Xorshift
// steps with the same mappings.  kind 1 = source samples, kind 2 = histories.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define MCLS_HD __host__ __device__ __forceinline__
#else
#define MCLS_HD inline
#endif

namespace mclsgpu {

MCLS_HD uint64_t xs_step(uint64_t x) {
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    return x;
}

MCLS_HD uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

MCLS_HD uint64_t epoch_key(uint64_t seed, uint64_t epoch) {
    return splitmix64(seed ^ splitmix64(epoch));
}

MCLS_HD uint64_t counter_state(uint64_t ekey, int kind, uint64_t idx) {
    uint64_t s = splitmix64(ekey ^ splitmix64((uint64_t(kind) << 56) ^ idx));
    return s ? s : 0x9E3779B97F4A7C15ULL;
}

// libstdc++ generate_canonical<double,53> for a 2^64-range engine.
MCLS_HD double canonical64(uint64_t r) {
#if defined(__CUDA_ARCH__)
    double d = __ull2double_rn(r) * 0x1p-64;
#else
    double d = double(r) * 0x1p-64;
#endif
    return d >= 1.0 ? 0x1.fffffffffffffp-1 : d;
}

// 24-bit uniform in [0, 1 - 2^-24] for the FP32 walk.
MCLS_HD float canonical32(uint64_t r) {
#if defined(__CUDA_ARCH__)
    return __uint2float_rn(uint32_t(r >> 40)) * 0x1p-24f;
#else
    return float(uint32_t(r >> 40)) * 0x1p-24f;
#endif
}

// Apply the bit matrix whose columns are `col[0..63]` to v.
MCLS_HD uint64_t gf2_apply(const uint64_t* col, uint64_t v) {
    uint64_t r = 0;
#if defined(__CUDA_ARCH__)
#pragma unroll 8
#endif
    for (int k = 0; k < 64; ++k)
        if ((v >> k) & 1ULL) r ^= col[k];
    return r;
}

// State after `n` further draws: T^n(v), with tab = 64 tables of 64 columns.
MCLS_HD uint64_t xs_jump(const uint64_t* tab, uint64_t v, uint64_t n) {
    for (int p = 0; n; ++p, n >>= 1)
        if (n & 1ULL) v = gf2_apply(tab + 64 * p, v);
    return v;
}

// Host: fill the 64 x 64 jump tables (J_p = T^(2^p)).
inline void xs_jump_tables(uint64_t* tab) {
    for (int k = 0; k < 64; ++k) tab[k] = xs_step(1ULL << k);
    for (int p = 1; p < 64; ++p) {
        const uint64_t* prev = tab + 64 * (p - 1);
        uint64_t* cur = tab + 64 * p;
        for (int k = 0; k < 64; ++k) cur[k] = gf2_apply(prev, prev[k]);
    }
}

}  // namespace mclsgpu
