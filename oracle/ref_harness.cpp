// ref_harness.cpp -- exposes the reference's own RNG and CDF sampler.
//
// TEST INFRASTRUCTURE.  Compiled (by oracle/Makefile, target `ref`) against
// the unmodified reference headers src/MCLS_Xorshift.hpp,
// src/MCLS_RNGTraits.hpp, src/MCLS_SamplingTools.hpp and src/MCLS_DBC.cpp
// where they lie in the MCLS source tree, with three stub headers standing in
// for Trilinos (oracle/ref_stub).  The output library lives in oracle/_ref and
// is used only to generate and check golden vectors for the oracle.
#include <climits>
#include <cstdint>
#include <limits>
#include <random>

#include "MCLS_SamplingTools.hpp"
#include "MCLS_Xorshift.hpp"

typedef MCLS::Xorshift<> RefRNG;
typedef MCLS::RNGTraits<RefRNG> RNGT;
typedef RNGT::uniform_real_distribution_type RealDist;
typedef MCLS::RandomDistributionTraits<RealDist> RDT;

extern "C" {

// Uniform draws exactly as AlmostOptimalDomain / UniformAdjointSource take
// them: d_rng->random(*d_rng_dist) with a [0,1) real distribution.
void ref_xorshift_uniforms(uint64_t seed, int64_t n, double* out) {
    Teuchos::RCP<RefRNG> rng = RNGT::create(seed);
    Teuchos::RCP<RealDist> dist = RDT::create(0.0, 1.0);
    for (int64_t i = 0; i < n; ++i) out[i] = RNGT::random(*rng, *dist);
}

// Raw engine output (the Xorshift state after each step).
void ref_xorshift_raw(uint64_t seed, int64_t n, uint64_t* out) {
    RefRNG rng(seed);
    for (int64_t i = 0; i < n; ++i) out[i] = rng();
}

// PRNG<RNG>::PRNG(comm_rank) seeding (src/MCLS_PRNG_impl.hpp:56-75) is not
// exposed: with libstdc++ 13, uniform_int_distribution<int> requires static
// min()/max() on the engine and MCLS::Xorshift<> declares them as non-static
// members, so the reference's per-rank seed derivation does not compile with
// this toolchain.  The oracle's rank-seed restatement is therefore unpinned.

int ref_sample_discrete_cdf(const double* cdf, int size, double u) {
    return MCLS::SamplingTools::sampleDiscreteCDF(cdf, size, u);
}

}  // extern "C"
