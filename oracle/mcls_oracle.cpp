// mcls_oracle.cpp -- CPU oracle for the MCSA hot path (TEST INFRASTRUCTURE).
//
// A plain FP64 C++ restatement of the reference MCLS algorithm, used only as
// the checker of the CUDA product path (tests, smoke check, CPU baseline).
// Each function cites the reference file:line it follows; paths are
// relative to the MCLS source tree.  Stated assumptions (Tpetra/Kokkos code
// that is not in the reference tree):
//   * one MPI rank: column order inside a row is ascending global column
//     (Tpetra's 1-rank column map equals the domain map; fillComplete sorts);
//   * Tpetra SpGEMM accumulates C(i,j) over A's row entries in column order;
//   * Tpetra norm1/norm2 sum in index order (Kokkos Serial execution space);
//   * no floating-point contraction (built with -ffp-contract=off).
#include "mcls_oracle.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <random>
#include <stack>
#include <thread>
#include <utility>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// RNG
// ---------------------------------------------------------------------------
// Xorshift<uint_fast64_t,13,7,17>: src/MCLS_Xorshift.hpp:57-109.
struct Xorshift64 {
    typedef uint_fast64_t result_type;
    result_type x;
    explicit Xorshift64(result_type s) : x(s) {}
    static constexpr result_type min() { return 0; }
    static constexpr result_type max() { return ~result_type(0); }
    result_type operator()() {
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        return x;
    }
};

// libstdc++ generate_canonical<double,53> for a 2^64-range engine, as used by
// uniform_real_distribution<double>(0,1) (src/MCLS_RNGTraits.hpp:147-160):
// one draw, (double)r / 2^64, clamped below 1.
inline double canonical(uint64_t r) {
    double d = static_cast<double>(r) / 18446744073709551616.0;
    if (d >= 1.0) d = std::nextafter(1.0, 0.0);
    return d;
}

// Counter-based generator (no reference counterpart).  A stream is keyed by
// (seed, epoch, kind, index); its state is two splitmix64 finalisations of
// the key, then Xorshift(13,7,17) steps with the same canonical mapping.
inline uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
inline uint64_t counter_state(uint64_t seed, uint64_t epoch, int kind,
                              uint64_t idx) {
    uint64_t ekey = splitmix64(seed ^ splitmix64(epoch));
    uint64_t s = splitmix64(ekey ^ splitmix64((uint64_t(kind) << 56) ^ idx));
    return s ? s : 0x9E3779B97F4A7C15ULL;
}
inline uint64_t xs_step(uint64_t x) {
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    return x;
}

// Stream of uniforms for the MC kernels.  Reference mode consumes one
// Xorshift in the reference's order; counter mode derives each history's
// stream from its emission index.
struct Stream {
    int mode;
    uint64_t seed;
    Xorshift64 xs;
    uint64_t position;  // draws consumed so far (reference mode)
    uint64_t epoch;     // MC solves so far (counter mode)
    explicit Stream(int m = 0, uint64_t s = 1)
        : mode(m), seed(s), xs(s), position(0), epoch(0) {}
};

// src/MCLS_SamplingTools.hpp:67-80
inline int sample_cdf(const double* cdf, int size, double u) {
    return int(std::lower_bound(cdf, cdf + size, u) - cdf);
}

// ---------------------------------------------------------------------------
// CSR
// ---------------------------------------------------------------------------
struct Csr {
    int64_t n = 0;
    std::vector<int64_t> rp, ci;
    std::vector<double> v;
    int64_t nnz() const { return int64_t(ci.size()); }
};

// Tpetra::RowMatrixTransposer (tpetra/src/MCLS_TpetraCrsMatrixAdapter.hpp:
// 415-422): rows of the transpose list columns in ascending order.
Csr transpose(const Csr& A) {
    Csr T;
    T.n = A.n;
    T.rp.assign(A.n + 1, 0);
    for (int64_t k = 0; k < A.nnz(); ++k) T.rp[A.ci[k] + 1]++;
    for (int64_t i = 0; i < A.n; ++i) T.rp[i + 1] += T.rp[i];
    T.ci.resize(A.nnz());
    T.v.resize(A.nnz());
    std::vector<int64_t> pos(T.rp.begin(), T.rp.end() - 1);
    for (int64_t i = 0; i < A.n; ++i)
        for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
            int64_t p = pos[A.ci[k]]++;
            T.ci[p] = i;
            T.v[p] = A.v[k];
        }
    return T;
}

// TpetraMatrixHelpers::filter (tpetra/src/MCLS_TpetraHelpers.hpp:196-259):
// row threshold is the SIGNED row max times `threshold`; entries with
// |v| <= row threshold are zeroed, then zeros are removed from the values and
// -1 markers from the indices.
void filter_row(std::vector<int64_t>& cols, std::vector<double>& vals,
                double threshold) {
    if (vals.empty()) return;
    double row_thr = *std::max_element(vals.begin(), vals.end()) * threshold;
    for (size_t j = 0; j < vals.size(); ++j) {
        if (std::abs(vals[j]) <= row_thr) {
            vals[j] = 0.0;
            cols[j] = -1;
        }
    }
    auto vend = std::remove(vals.begin(), vals.end(), 0.0);
    auto cend = std::remove(cols.begin(), cols.end(), int64_t(-1));
    size_t nv = size_t(vend - vals.begin());
    vals.resize(nv);
    cols.resize(std::min(nv, size_t(cend - cols.begin())));
    cols.resize(nv, -1);
}

// MatrixTraits::multiply (tpetra/src/MCLS_TpetraCrsMatrixAdapter.hpp:
// 388-400): C = A*B accumulated over A's row entries in column order, then
// filtered.
Csr multiply(const Csr& A, const Csr& B, double threshold) {
    Csr C;
    C.n = A.n;
    C.rp.assign(1, 0);
    std::map<int64_t, double> acc;
    std::vector<int64_t> cols;
    std::vector<double> vals;
    for (int64_t i = 0; i < A.n; ++i) {
        acc.clear();
        for (int64_t ka = A.rp[i]; ka < A.rp[i + 1]; ++ka) {
            int64_t k = A.ci[ka];
            double a = A.v[ka];
            for (int64_t kb = B.rp[k]; kb < B.rp[k + 1]; ++kb) {
                double prod = a * B.v[kb];
                auto it = acc.find(B.ci[kb]);
                if (it == acc.end())
                    acc.emplace(B.ci[kb], prod);
                else
                    it->second = it->second + prod;
            }
        }
        cols.clear();
        vals.clear();
        for (auto& kv : acc) {
            cols.push_back(kv.first);
            vals.push_back(kv.second);
        }
        filter_row(cols, vals, threshold);
        C.ci.insert(C.ci.end(), cols.begin(), cols.end());
        C.v.insert(C.v.end(), vals.begin(), vals.end());
        C.rp.push_back(int64_t(C.ci.size()));
    }
    return C;
}

// LinearProblem::getCompositeOperator / getTransposeCompositeOperator
// (src/MCLS_LinearProblem_impl.hpp:143-221).
Csr composite(const Csr& A, const Csr* PL, const Csr* PR, bool trans,
              double thr) {
    if (!trans) {
        if (PL && PR) return multiply(*PL, multiply(A, *PR, thr), thr);
        if (PL) return multiply(*PL, A, thr);
        if (PR) return multiply(A, *PR, thr);
        return A;
    }
    if (PL && PR) {
        Csr temp = multiply(transpose(A), transpose(*PL), thr);
        return multiply(transpose(*PR), temp, thr);
    }
    if (PR) return multiply(transpose(*PR), transpose(A), thr);
    if (PL) return multiply(transpose(A), transpose(*PL), thr);
    return transpose(A);
}

// Host threads for the oracle's long row loops (orc_set_threads; 1 = one
// thread, as one reference rank runs).  Every row is computed exactly as the
// one-thread loop computes it, so results do not depend on the count.
int g_threads = 1;

// f(lo, hi) over contiguous row ranges [lo, hi) of [0, n), one per thread.
template <class F>
void parallel_ranges(int64_t n, const F& f) {
    const int T = g_threads;
    if (T <= 1 || n < (1 << 16)) {
        f(int64_t(0), n);
        return;
    }
    std::vector<std::thread> pool;
    for (int t = 1; t < T; ++t) pool.emplace_back(f, n * t / T, n * (t + 1) / T);
    f(int64_t(0), n / T);
    for (auto& th : pool) th.join();
}

// Sum over threads of g(lo, hi) on the ranges parallel_ranges uses, added in
// range order (deterministic for a given thread count).
template <class G>
double parallel_sum(int64_t n, const G& g) {
    const int T = (g_threads <= 1 || n < (1 << 16)) ? 1 : g_threads;
    std::vector<double> part(T, 0.0);
    std::vector<std::thread> pool;
    for (int t = 1; t < T; ++t)
        pool.emplace_back([&, t]() { part[t] = g(n * t / T, n * (t + 1) / T); });
    part[0] = g(int64_t(0), n / T);
    for (auto& th : pool) th.join();
    double s = 0.0;
    for (double v : part) s += v;
    return s;
}

// Tpetra CrsMatrix::apply on one rank: y_i = sum_j a_ij x_j in column order.
void spmv(const Csr& A, const double* x, double* y) {
    parallel_ranges(A.n, [&](int64_t lo, int64_t hi) {
        for (int64_t i = lo; i < hi; ++i) {
            double s = 0.0;
            for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) s = s + A.v[k] * x[A.ci[k]];
            y[i] = s;
        }
    });
}

// TpetraPointJacobiPreconditioner::buildPreconditioner
// (tpetra/src/MCLS_TpetraPointJacobiPreconditioner_impl.hpp:104-139):
// diagonal copy (0 where absent), reciprocal, one entry per row.
Csr point_jacobi(const Csr& A) {
    Csr P;
    P.n = A.n;
    P.rp.resize(A.n + 1);
    P.ci.resize(A.n);
    P.v.resize(A.n);
    for (int64_t i = 0; i < A.n; ++i) {
        double d = 0.0;
        for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
            if (A.ci[k] == i) d = A.v[k];
        P.rp[i] = i;
        P.ci[i] = i;
        P.v[i] = 1.0 / d;
    }
    P.rp[A.n] = A.n;
    return P;
}

// Dense LU with partial pivoting and inverse from the factors (the algorithm
// of LAPACK GETRF/GETRI, restated unblocked).  Column-major n x n in `a`.
bool invert_dense(std::vector<double>& a, int n) {
    std::vector<int> piv(n);
    for (int j = 0; j < n; ++j) {
        int p = j;
        double mx = std::abs(a[j + j * n]);
        for (int i = j + 1; i < n; ++i)
            if (std::abs(a[i + j * n]) > mx) { mx = std::abs(a[i + j * n]); p = i; }
        piv[j] = p;
        if (a[p + j * n] == 0.0) return false;
        if (p != j)
            for (int c = 0; c < n; ++c) std::swap(a[j + c * n], a[p + c * n]);
        double r = 1.0 / a[j + j * n];
        for (int i = j + 1; i < n; ++i) a[i + j * n] *= r;
        for (int c = j + 1; c < n; ++c)
            for (int i = j + 1; i < n; ++i) a[i + c * n] -= a[i + j * n] * a[j + c * n];
    }
    // inv(U)
    for (int j = 0; j < n; ++j) {
        a[j + j * n] = 1.0 / a[j + j * n];
        double ajj = -a[j + j * n];
        for (int i = 0; i < j; ++i) {
            double s = 0.0;
            for (int k = i; k < j; ++k) s += a[i + k * n] * a[k + j * n];
            a[i + j * n] = s;
        }
        for (int i = 0; i < j; ++i) a[i + j * n] *= ajj;
    }
    // solve inv(A)*L = inv(U)
    std::vector<double> work(n);
    for (int j = n - 2; j >= 0; --j) {
        for (int i = j + 1; i < n; ++i) { work[i] = a[i + j * n]; a[i + j * n] = 0.0; }
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int k = j + 1; k < n; ++k) s += a[i + k * n] * work[k];
            a[i + j * n] -= s;
        }
    }
    for (int j = n - 2; j >= 0; --j)
        if (piv[j] != j)
            for (int i = 0; i < n; ++i) std::swap(a[i + j * n], a[i + piv[j] * n]);
    return true;
}

// TpetraBlockJacobiPreconditioner::buildPreconditioner
// (tpetra/src/MCLS_TpetraBlockJacobiPreconditioner_impl.hpp:122-223):
// contiguous blocks; the block is assembled transposed (column-major with
// block(j,i) = A(row_i, col_j)), inverted, and row i of the preconditioner is
// column i of the inverted transposed block, i.e. row i of inv(B).
bool block_jacobi(const Csr& A, int bs, Csr& P) {
    if (bs <= 0 || A.n % bs) return false;
    P.n = A.n;
    P.rp.assign(1, 0);
    std::vector<double> blk(size_t(bs) * bs);
    for (int64_t b0 = 0; b0 < A.n; b0 += bs) {
        std::fill(blk.begin(), blk.end(), 0.0);
        for (int i = 0; i < bs; ++i)
            for (int64_t k = A.rp[b0 + i]; k < A.rp[b0 + i + 1]; ++k) {
                int64_t c = A.ci[k] - b0;
                if (c >= 0 && c < bs) blk[c + size_t(i) * bs] = A.v[k];
            }
        if (!invert_dense(blk, bs)) return false;
        for (int i = 0; i < bs; ++i) {
            for (int j = 0; j < bs; ++j) {
                P.ci.push_back(b0 + j);
                P.v.push_back(blk[j + size_t(i) * bs]);
            }
            P.rp.push_back(int64_t(P.ci.size()));
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// AlmostOptimalDomain::addMatrixToDomain
// (src/MCLS_AlmostOptimalDomain_impl.hpp:257-366)
// ---------------------------------------------------------------------------
struct Domain {
    int64_t n = 0;
    std::vector<int64_t> rp, col;
    std::vector<double> h, cdf, w;
};

bool build_domain(const Csr& M, double relaxation, Domain& D) {
    D.n = M.n;
    D.rp.assign(1, 0);
    D.w.resize(M.n);
    std::vector<double> c;
    std::vector<int64_t> g;
    for (int64_t i = 0; i < M.n; ++i) {
        int64_t ne = M.rp[i + 1] - M.rp[i];
        if (ne <= 0) return false;  // MCLS_CHECK( num_entries > 0 ), :295
        c.assign(M.v.begin() + M.rp[i], M.v.begin() + M.rp[i + 1]);
        g.assign(M.ci.begin() + M.rp[i], M.ci.begin() + M.rp[i + 1]);
        for (int64_t j = 0; j < ne; ++j) {
            // :306-309 -- identity minus the relaxed operator, on the pattern
            double prod = relaxation * c[j];
            c[j] = (g[j] == i) ? 1.0 - prod : -prod;
            // :312-317 -- mark |h| < epsilon for removal
            if (std::abs(c[j]) < std::numeric_limits<double>::epsilon()) {
                c[j] = std::numeric_limits<double>::max();
                g[j] = -1;
            }
        }
        c.erase(std::remove(c.begin(), c.end(), std::numeric_limits<double>::max()),
                c.end());
        g.erase(std::remove(g.begin(), g.end(), int64_t(-1)), g.end());
        if (c.empty()) return false;
        // :336-338 -- the iteration matrix keeps the signed values
        D.h.insert(D.h.end(), c.begin(), c.end());
        D.col.insert(D.col.end(), g.begin(), g.end());
        // :342-348 -- non-normalized CDF of |h|, left to right
        c[0] = std::abs(c[0]);
        for (size_t j = 1; j < c.size(); ++j) c[j] = std::abs(c[j]) + c[j - 1];
        // :353 -- row weight is the absolute row sum
        double W = c.back();
        if (!(W > 0.0)) return false;
        D.w[i] = W;
        // :357-362 -- normalize
        for (double& v : c) v /= W;
        D.cdf.insert(D.cdf.end(), c.begin(), c.end());
        D.rp.push_back(int64_t(D.h.size()));
    }
    return true;
}

}  // namespace

// ===========================================================================
// C interface
// ===========================================================================
struct orc_csr {
    Csr m;
};

struct orc_mc {
    orc_mc_params p;
    Csr A;
    bool has_pl = false, has_pr = false;
    Csr PL, PR;
    Domain D;
    Stream rng;
    int64_t total_steps = 0;
};

extern "C" {

void orc_xorshift_uniforms(uint64_t seed, int64_t n, double* out) {
    Xorshift64 x(seed);
    for (int64_t i = 0; i < n; ++i) out[i] = canonical(x());
}

uint64_t orc_rank_seed(uint64_t master_seed, int rank) {
    // src/MCLS_PRNG_impl.hpp:61-72: master engine, then the (rank+1)-th draw
    // of uniform_int_distribution<int>(0, INT_MAX).
    Xorshift64 master(master_seed);
    std::uniform_int_distribution<int> dist(0, std::numeric_limits<int>::max());
    int seed = 0;
    for (int i = -1; i < rank; ++i) seed = dist(master);
    return uint64_t(seed);
}

void orc_counter_uniforms(uint64_t seed, uint64_t epoch, int kind, int64_t idx,
                          int64_t n, double* out) {
    uint64_t s = counter_state(seed, epoch, kind, uint64_t(idx));
    for (int64_t i = 0; i < n; ++i) {
        s = xs_step(s);
        out[i] = canonical(s);
    }
}

int orc_sample_discrete_cdf(const double* cdf, int size, double u) {
    return sample_cdf(cdf, size, u);
}

orc_csr* orc_csr_create(int64_t n, const int64_t* rowptr, const int64_t* col,
                        const double* val) {
    orc_csr* c = new orc_csr;
    c->m.n = n;
    c->m.rp.assign(rowptr, rowptr + n + 1);
    int64_t nnz = rowptr[n];
    c->m.ci.assign(col, col + nnz);
    c->m.v.assign(val, val + nnz);
    return c;
}
void orc_csr_free(orc_csr* c) { delete c; }
int64_t orc_csr_n(const orc_csr* c) { return c->m.n; }
int64_t orc_csr_nnz(const orc_csr* c) { return c->m.nnz(); }
void orc_csr_copy(const orc_csr* c, int64_t* rp, int64_t* ci, double* v) {
    if (rp) std::copy(c->m.rp.begin(), c->m.rp.end(), rp);
    if (ci) std::copy(c->m.ci.begin(), c->m.ci.end(), ci);
    if (v) std::copy(c->m.v.begin(), c->m.v.end(), v);
}
orc_csr* orc_transpose(const orc_csr* A) { return new orc_csr{transpose(A->m)}; }
orc_csr* orc_multiply(const orc_csr* A, const orc_csr* B, double thr) {
    return new orc_csr{multiply(A->m, B->m, thr)};
}
orc_csr* orc_composite(const orc_csr* A, const orc_csr* PL, const orc_csr* PR,
                       int trans, double thr) {
    return new orc_csr{composite(A->m, PL ? &PL->m : nullptr,
                                 PR ? &PR->m : nullptr, trans != 0, thr)};
}
orc_csr* orc_point_jacobi(const orc_csr* A) { return new orc_csr{point_jacobi(A->m)}; }
orc_csr* orc_block_jacobi(const orc_csr* A, int bs) {
    orc_csr* c = new orc_csr;
    if (!block_jacobi(A->m, bs, c->m)) {
        delete c;
        return nullptr;
    }
    return c;
}
void orc_spmv(const orc_csr* A, const double* x, double* y) { spmv(A->m, x, y); }

orc_mc* orc_mc_create(const orc_csr* A, const orc_csr* PL, const orc_csr* PR,
                      const orc_mc_params* p) {
    orc_mc* mc = new orc_mc;
    mc->p = *p;
    mc->A = A->m;
    if (PL) { mc->has_pl = true; mc->PL = PL->m; }
    if (PR) { mc->has_pr = true; mc->PR = PR->m; }
    // MonteCarloSolverManager::buildMonteCarloDomain
    // (src/MCLS_MonteCarloSolverManager_impl.hpp:308-340): the adjoint domain
    // is built on the transposed composite, the forward one on the composite.
    Csr M = composite(mc->A, mc->has_pl ? &mc->PL : nullptr,
                      mc->has_pr ? &mc->PR : nullptr, p->direction == 0,
                      p->composite_threshold);
    double relax = p->neumann_relaxation > 0.0 ? p->neumann_relaxation : 1.0;
    if (!build_domain(M, relax, mc->D)) {
        delete mc;
        return nullptr;
    }
    mc->rng = Stream(p->rng_mode, p->seed);
    return mc;
}
void orc_mc_free(orc_mc* mc) { delete mc; }
int64_t orc_mc_domain_nnz(const orc_mc* mc) { return int64_t(mc->D.col.size()); }
void orc_mc_domain_copy(const orc_mc* mc, int64_t* rp, int64_t* col, double* h,
                        double* cdf, double* w) {
    const Domain& D = mc->D;
    if (rp) std::copy(D.rp.begin(), D.rp.end(), rp);
    if (col) std::copy(D.col.begin(), D.col.end(), col);
    if (h) std::copy(D.h.begin(), D.h.end(), h);
    if (cdf) std::copy(D.cdf.begin(), D.cdf.end(), cdf);
    if (w) std::copy(D.w.begin(), D.w.end(), w);
}
uint64_t orc_mc_stream_position(const orc_mc* mc) { return mc->rng.position; }
int64_t orc_mc_total_steps(const orc_mc* mc) { return mc->total_steps; }

int64_t orc_mc_solve(orc_mc* mc, const double* rhs, double* x, int internal,
                     int64_t max_trace, int64_t* trace_states,
                     double* final_weight, int* events, int64_t* start_state) {
    const orc_mc_params& p = mc->p;
    const Domain& D = mc->D;
    const int64_t n = D.n;
    const int L = p.history_length;

    // MonteCarloSolverManager::buildMonteCarloSource
    // (src/MCLS_MonteCarloSolverManager_impl.hpp:346-380): copy, left
    // precondition unless internal, scale by the Neumann relaxation if set.
    std::vector<double> src(rhs, rhs + n);
    if (mc->has_pl && !internal) {
        std::vector<double> t(n);
        spmv(mc->PL, src.data(), t.data());
        src = t;
    }
    if (p.neumann_relaxation > 0.0)
        for (double& v : src) v *= p.neumann_relaxation;

    std::vector<double> tally(n, 0.0);  // MCSolver::solve zeroOut, src/MCLS_MCSolver_impl.hpp:91
    Stream& rng = mc->rng;
    auto draw_ref = [&]() {
        rng.position++;
        return canonical(rng.xs());
    };

    // Starting states in emission order and their weights.
    std::vector<int64_t> starts;
    std::vector<double> w0;
    int64_t nh_total = 0;
    // Forward histories on the counter stream are independent and walked by
    // threads over ranges of start states (below).
    const bool threaded = p.direction == 1 && rng.mode == 1 && !trace_states && !final_weight &&
                          !events && !start_state && g_threads > 1;
    const bool fwd_lazy = threaded;
    int fwd_per = 1;
    if (p.direction == 0) {
        // UniformAdjointSource (src/MCLS_UniformAdjointSource_impl.hpp:58-263)
        int nh_requested = int(double(n) * (p.sample_ratio > 0.0 ? p.sample_ratio : 1.0));
        if (!(p.sample_ratio > 0.0)) nh_requested = int(n);
        int nh_total_req = nh_requested;
        double norm1 = 0.0;
        for (int64_t i = 0; i < n; ++i) norm1 += std::abs(src[i]);
        const double weight = norm1;  // :67 d_weight( VT::norm1(*d_b) )
        std::vector<int> counts(n, 0);
        int nh_domain = 0;
        if (!p.stratified) {
            // buildRandomSource :180-224
            std::vector<double> cdf(n);
            cdf[0] = src[0];  // :185 signed first element
            for (int64_t i = 1; i < n; ++i) cdf[i] = cdf[i - 1] + std::abs(src[i]);
            nh_domain = int(double(nh_total_req) * cdf.back() / norm1);  // :198
            double back = cdf.back();
            for (int64_t i = 0; i < n; ++i) cdf[i] /= back;
            for (int k = 0; k < nh_domain; ++k) {
                double u;
                if (rng.mode == 0)
                    u = draw_ref();
                else {
                    uint64_t s = xs_step(counter_state(rng.seed, rng.epoch, 1, uint64_t(k)));
                    u = canonical(s);
                }
                counts[sample_cdf(cdf.data(), int(n), u)]++;
            }
        } else {
            // buildStratifiedSource :230-263
            double local_sum = 0.0;
            for (int64_t i = 0; i < n; ++i) local_sum += std::abs(src[i]);
            int nh_local = int(std::ceil(double(nh_total_req) * local_sum / weight));
            double num_over_sum = double(nh_local) / local_sum;
            for (int64_t i = 0; i < n; ++i) {
                int c = int(std::ceil(std::abs(src[i]) * num_over_sum));
                if (c > 0) { counts[i] = c; nh_domain += c; }
            }
        }
        nh_total = nh_domain;
        // Stack pushed in ascending state order; getHistory pops the top
        // (:157-175), so emission runs from the highest state down.
        for (int64_t i = n - 1; i >= 0; --i)
            for (int c = 0; c < counts[i]; ++c) {
                starts.push_back(i);
                w0.push_back(weight * double(src[i] > 0.0 ? 1 : -1));
            }
    } else {
        // UniformForwardSource (src/MCLS_UniformForwardSource_impl.hpp:60-148):
        // ceil(Sample Ratio) histories per state in state order, weight 1.
        // (History e starts at state e / per; the threaded walk below uses
        // that directly instead of the lists.)
        fwd_per = p.sample_ratio > 0.0 ? int(std::ceil(p.sample_ratio)) : 1;
        if (!fwd_lazy)
            for (int64_t i = 0; i < n; ++i)
                for (int c = 0; c < fwd_per; ++c) {
                    starts.push_back(i);
                    w0.push_back(1.0);
                }
        nh_total = int64_t(n) * fwd_per;
    }

    // Expected-value estimator helper for the forward walk: (H b)_s per row.
    std::vector<double> hb;
    if (p.direction == 1 && p.estimator == 1) {
        hb.assign(n, 0.0);
        parallel_ranges(n, [&](int64_t lo, int64_t hi) {
            for (int64_t i = lo; i < hi; ++i) {
                double s = 0.0;
                for (int64_t k = D.rp[i]; k < D.rp[i + 1]; ++k) s = s + D.h[k] * src[D.col[k]];
                hb[i] = s;
            }
        });
    }
    std::vector<double> fsum, fcount;
    if (p.direction == 1) { fsum.assign(n, 0.0); fcount.assign(n, 0.0); }

    // DomainTransporter::transport (src/MCLS_DomainTransporter_impl.hpp:70-119)
    const int64_t nh = fwd_lazy ? nh_total : int64_t(starts.size());
    if (threaded) {
        // Forward histories on the counter stream are independent: threads
        // take contiguous ranges of start states (all histories of a state in
        // one thread, in emission order), so every sum is the one-thread sum.
        const int per = fwd_per;
        std::atomic<int64_t> total{0};
        parallel_ranges(n, [&](int64_t lo, int64_t hi) {
            int64_t st = 0;
            for (int64_t e = lo * per; e < hi * per; ++e) {
                const int64_t s0 = e / per;
                int64_t state = s0;
                double w = 1.0;
                const double wabs0 = 1.0;
                uint64_t cs = counter_state(rng.seed, rng.epoch, 2, uint64_t(e));
                int steps = 0;
                double htally = 0.0;
                while (true) {
                    htally += w * (p.estimator == 0 ? src[state] : hb[state]);
                    cs = xs_step(cs);
                    const double u = canonical(cs);
                    int64_t r0 = D.rp[state];
                    int j = sample_cdf(&D.cdf[r0], int(D.rp[state + 1] - r0), u);
                    int sign = (D.h[r0 + j] > 0.0) ? 1 : -1;
                    w *= D.w[state] * double(sign);
                    state = D.col[r0 + j];
                    ++steps;
                    if (steps >= L ||
                        (p.weight_cutoff > 0.0 && std::abs(w) < p.weight_cutoff * wabs0))
                        break;
                }
                st += steps;
                fsum[s0] += htally;
                fcount[s0] += 1.0;
            }
            total += st;
        });
        mc->total_steps += total.load();
    }
    for (int64_t e = 0; e < nh && !threaded; ++e) {
        int64_t state = starts[e];
        double w = w0[e];
        const double wabs0 = std::abs(w0[e]);
        uint64_t cs = 0;
        if (rng.mode == 1) cs = counter_state(rng.seed, rng.epoch, 2, uint64_t(e));
        int steps = 0;
        int event = 1;
        double htally = 0.0;
        bool tr = trace_states && e < max_trace;
        if (tr) {
            for (int k = 0; k <= L; ++k) trace_states[e * (L + 1) + k] = -1;
            trace_states[e * (L + 1)] = state;
        }
        while (true) {
            // Tally at the pre-transition state.
            if (p.direction == 0) {
                if (p.estimator == 0) {
                    tally[state] += w;  // AdjointTally::tallyHistory
                } else {
                    for (int64_t k = D.rp[state]; k < D.rp[state + 1]; ++k)
                        tally[D.col[k]] += w * D.h[k];
                }
            } else {
                // ForwardTally::tallyHistory (src/MCLS_ForwardTally.hpp:123-132)
                htally += w * (p.estimator == 0 ? src[state] : hb[state]);
            }
            // AlmostOptimalDomain::processTransition
            // (src/MCLS_AlmostOptimalDomain.hpp:254-284)
            double u;
            if (rng.mode == 0)
                u = draw_ref();
            else {
                cs = xs_step(cs);
                u = canonical(cs);
            }
            int64_t r0 = D.rp[state];
            int j = sample_cdf(&D.cdf[r0], int(D.rp[state + 1] - r0), u);
            int sign = (D.h[r0 + j] > 0.0) ? 1 : -1;
            w *= D.w[state] * double(sign);
            state = D.col[r0 + j];
            ++steps;
            mc->total_steps++;
            if (tr) trace_states[e * (L + 1) + steps] = state;
            // terminateHistory (src/MCLS_AlmostOptimalDomain.hpp:135-136);
            // the relative weight cutoff is the legacy "Weight Cutoff" key.
            if (steps >= L || (p.weight_cutoff > 0.0 && std::abs(w) < p.weight_cutoff * wabs0)) {
                event = 2;  // Event::CUTOFF
                break;
            }
        }
        if (p.direction == 1) {
            // ForwardTally::postProcessHistory (src/MCLS_ForwardTally_impl.hpp:84-110)
            fsum[starts[e]] += htally;
            fcount[starts[e]] += 1.0;
        }
        if (final_weight && e < max_trace) final_weight[e] = w;
        if (events && e < max_trace) events[e] = event;
        if (start_state && e < max_trace) start_state[e] = starts[e];
    }
    if (rng.mode == 1) rng.epoch++;

    if (p.direction == 0) {
        // AdjointTally::normalize (src/MCLS_AdjointTally_impl.hpp:68-72)
        double s = 1.0 / double(nh_total);
        for (int64_t i = 0; i < n; ++i) tally[i] = tally[i] * s;
    } else {
        // ForwardTally::finalize (src/MCLS_ForwardTally_impl.hpp:135-209)
        for (int64_t i = 0; i < n; ++i)
            tally[i] = fcount[i] > 0.0 ? fsum[i] / fcount[i] : 0.0;
    }
    if (p.estimator == 1)
        for (int64_t i = 0; i < n; ++i) tally[i] += src[i];

    // Right preconditioner recovery (src/MCLS_MonteCarloSolverManager_impl.hpp:222-230)
    if (mc->has_pr && !internal) {
        std::vector<double> t(n);
        spmv(mc->PR, tally.data(), t.data());
        tally = t;
    }
    std::copy(tally.begin(), tally.end(), x);
    return nh_total;
}

}  // extern "C"

namespace {

// The linear problem's operators (src/MCLS_LinearProblem_impl.hpp) over the
// oracle's CSR matrices; transposes are formed when first needed.
struct Problem {
    const Csr& A;
    const Csr* PL;
    const Csr* PR;
    const double* b;
    int64_t n;
    std::vector<double> tmp, tmp2;
    Csr AT, PLT, PRT;
    bool have_t = false;
    Problem(const Csr& A_, const Csr* PL_, const Csr* PR_, const double* b_)
        : A(A_), PL(PL_), PR(PR_), b(b_), n(A_.n), tmp(A_.n), tmp2(A_.n) {}
    // LinearProblem::updatePrecResidual (:410-442): rp = PL (b - A PR x)
    void prec_residual(const std::vector<double>& x, std::vector<double>& rp) {
        if (PR) {
            spmv(*PR, x.data(), tmp.data());
            spmv(A, tmp.data(), rp.data());
        } else {
            spmv(A, x.data(), rp.data());
        }
        for (int64_t i = 0; i < n; ++i) rp[i] = -rp[i] + b[i];
        if (PL) {
            tmp = rp;
            spmv(*PL, tmp.data(), rp.data());
        }
    }
    // LinearProblem::apply (:251-279): y = PL A PR x
    void apply(const std::vector<double>& x, std::vector<double>& y) {
        const double* t = x.data();
        if (PR) {
            spmv(*PR, x.data(), tmp2.data());
            t = tmp2.data();
        }
        if (PL) {
            spmv(A, t, tmp.data());
            spmv(*PL, tmp.data(), y.data());
        } else {
            spmv(A, t, y.data());
        }
    }
    // LinearProblem::applyTranspose (:286-315): y = PR^T A^T PL^T x
    void apply_transpose(const std::vector<double>& x, std::vector<double>& y) {
        if (!have_t) {
            AT = transpose(A);
            if (PL) PLT = transpose(*PL);
            if (PR) PRT = transpose(*PR);
            have_t = true;
        }
        const double* t = x.data();
        if (PL) {
            spmv(PLT, x.data(), tmp.data());
            t = tmp.data();
        }
        if (PR) {
            spmv(AT, t, tmp2.data());
            spmv(PRT, tmp2.data(), y.data());
        } else {
            spmv(AT, t, y.data());
        }
    }
};

double dot(const std::vector<double>& a, const std::vector<double>& b) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s = s + a[i] * b[i];
    return s;
}

// One fixed-point iteration on (x, rp) with p, v as work vectors.  A zero
// denominator gives a step of 0 (the reference divides by it).
void fixed_point_step(Problem& P, int type, double omega, std::vector<double>& x,
                      std::vector<double>& rp, std::vector<double>& p, std::vector<double>& v) {
    const int64_t n = P.n;
    auto step = [&](double num, double den, const std::vector<double>& s) {
        const double a = den != 0.0 ? num / den : 0.0;
        for (int64_t i = 0; i < n; ++i) {
            x[i] = x[i] + a * s[i];
            rp[i] = rp[i] + (-a) * p[i];
        }
    };
    switch (type) {
        case 1:  // SteepestDescentIteration::doOneIteration (src/MCLS_SteepestDescentIteration_impl.hpp:114-136)
            P.apply(rp, p);
            step(dot(rp, rp), dot(p, rp), rp);
            break;
        case 2:  // MinimalResidualIteration::doOneIteration (src/MCLS_MinimalResidualIteration_impl.hpp:114-136)
            P.apply(rp, p);
            step(dot(p, rp), dot(p, p), rp);
            break;
        case 3:  // RNSDIteration::doOneIteration (src/MCLS_RNSDIteration_impl.hpp:118-142)
            P.apply_transpose(rp, v);
            P.apply(v, p);
            step(dot(v, v), dot(p, p), v);
            break;
        default:  // RichardsonIteration::doOneIteration (src/MCLS_RichardsonIteration_impl.hpp:134-147)
            for (int64_t i = 0; i < n; ++i) x[i] = x[i] + omega * rp[i];
            P.prec_residual(x, rp);
    }
}

// Anderson acceleration (Walker & Ni 2011, NOX's "Anderson Accelerated
// Fixed-Point" solver): the least-squares problem min |F_k - dF gamma| is
// solved through a QR factorisation of dF that is updated as columns come
// and go.  Columns are kept oldest first.
struct Anderson {
    int m, start, adjust;
    double beta, droptol;
    int64_t n;
    int nstore = 0;
    std::vector<std::vector<double>> Q, DX;
    std::vector<std::vector<double>> R;
    std::vector<double> Fold, xold;
    Anderson(const orc_anderson_params& p, int64_t n_)
        : m(p.storage_depth), start(p.start_iteration), adjust(p.adjust_condition),
          beta(p.mixing), droptol(p.drop_tolerance), n(n_),
          R(size_t(std::max(m, 1)), std::vector<double>(size_t(std::max(m, 1)), 0.0)) {}
    // Drop the oldest column: Givens rotations restore R's triangle after
    // its first column is removed; Q takes the same rotations.
    void qr_delete() {
        for (int i = 0; i + 1 < nstore; ++i) {
            const double a = R[i][i + 1], bb = R[i + 1][i + 1];
            const double t = std::sqrt(a * a + bb * bb);
            const double c = a / t, s = bb / t;
            R[i][i + 1] = t;
            R[i + 1][i + 1] = 0.0;
            for (int j = i + 2; j < nstore; ++j) {
                const double u = c * R[i][j] + s * R[i + 1][j];
                R[i + 1][j] = (-s) * R[i][j] + c * R[i + 1][j];
                R[i][j] = u;
            }
            for (int64_t e = 0; e < n; ++e) {
                const double qa = Q[i][e], qb = Q[i + 1][e];
                Q[i][e] = c * qa + s * qb;
                Q[i + 1][e] = (-s) * qa + c * qb;
            }
        }
        for (int i = 0; i < nstore; ++i)
            for (int j = 0; j + 1 < nstore; ++j) R[i][j] = R[i][j + 1];
        for (int i = 0; i < nstore; ++i) R[i][nstore - 1] = 0.0;
        Q.pop_back();
        DX.erase(DX.begin());
        --nstore;
    }
    // Modified Gram-Schmidt of the new column against Q; false (and no
    // column) when what is left of it has zero or non-finite norm.
    bool qr_add(std::vector<double> v) {
        const int N = nstore;
        for (int j = 0; j < N; ++j) {
            double r = 0.0;
            for (int64_t e = 0; e < n; ++e) r = r + Q[j][e] * v[e];
            R[j][N] = r;
            for (int64_t e = 0; e < n; ++e) v[e] = v[e] + (-r) * Q[j][e];
        }
        double vv = 0.0;
        for (int64_t e = 0; e < n; ++e) vv = vv + v[e] * v[e];
        const double rn = std::sqrt(vv);
        if (!(rn > 0.0) || !std::isfinite(rn)) {
            for (int j = 0; j < N; ++j) R[j][N] = 0.0;
            return false;
        }
        R[N][N] = rn;
        const double inv = 1.0 / rn;
        for (int64_t e = 0; e < n; ++e) v[e] = inv * v[e];
        Q.push_back(std::move(v));
        ++nstore;
        return true;
    }
    // Reciprocal 1-norm condition number of the leading nstore x nstore R.
    double rcond() const {
        const int N = nstore;
        std::vector<std::vector<double>> Ri(size_t(N), std::vector<double>(size_t(N), 0.0));
        for (int j = 0; j < N; ++j) {
            // column j of R^-1 by back substitution of e_j
            for (int i = j; i >= 0; --i) {
                double s = i == j ? 1.0 : 0.0;
                for (int k = i + 1; k <= j; ++k) s = s - R[i][k] * Ri[k][j];
                Ri[i][j] = s / R[i][i];
            }
        }
        double n1 = 0.0, ni = 0.0;
        for (int j = 0; j < N; ++j) {
            double a = 0.0, c = 0.0;
            for (int i = 0; i <= j; ++i) {
                a = a + std::abs(R[i][j]);
                c = c + std::abs(Ri[i][j]);
            }
            n1 = std::max(n1, a);
            ni = std::max(ni, c);
        }
        return 1.0 / (n1 * ni);
    }
    // One step from x_k with F_k = g(x_k) - x_k (k = steps taken so far).
    void step(int k, std::vector<double>& x, const std::vector<double>& F) {
        if (m > 0 && k >= start) {
            if (k == start) {
                nstore = 0;
                Q.clear();
                DX.clear();
            } else if (nstore == m) {
                qr_delete();
            }
            std::vector<double> v(static_cast<size_t>(n)), dx(static_cast<size_t>(n));
            for (int64_t e = 0; e < n; ++e) {
                v[e] = F[e] - Fold[e];
                dx[e] = x[e] - xold[e];
            }
            if (qr_add(std::move(v))) DX.push_back(std::move(dx));
            if (adjust)
                while (nstore > 1 && rcond() < droptol) qr_delete();
        }
        const int N = nstore;
        std::vector<double> gamma(static_cast<size_t>(N)), rg(static_cast<size_t>(N));
        for (int j = N - 1; j >= 0; --j) {
            double rhs = 0.0;
            for (int64_t e = 0; e < n; ++e) rhs = rhs + F[e] * Q[j][e];
            double g = rhs;
            for (int i = j + 1; i < N; ++i) g = g - R[j][i] * gamma[i];
            gamma[j] = g / R[j][j];
        }
        for (int i = 0; i < N; ++i) {
            double s = 0.0;
            for (int j = i; j < N; ++j) s = s + R[i][j] * gamma[j];
            rg[i] = beta * s;
        }
        Fold = F;
        xold = x;
        for (int64_t e = 0; e < n; ++e) {
            double w = beta * F[e];
            for (int j = 0; j < N; ++j) w = (w + (-gamma[j]) * DX[j][e]) + (-rg[j]) * Q[j][e];
            x[e] = x[e] + w;
        }
    }
};

}  // namespace

extern "C" {

int orc_anderson_solve(const orc_csr* A, const orc_csr* PL, const orc_mc_params* mp,
                       const orc_anderson_params* ap, const double* b, double* x, int* iters,
                       double* achieved, int max_hist, double* res_hist, int64_t* total_steps) {
    // AndersonSolverManager::solve (src/MCLS_AndersonSolverManager_impl.hpp:186-224) with
    // MCSAStatusTest (src/MCLS_MCSAStatusTest_impl.hpp:65-110): converged when
    // |PL (b - A x)|_2 < tolerance |b|_2, checked on the initial guess and after each step.
    if (ap->storage_depth < 0 || ap->start_iteration < 1) return -1;
    orc_mc* mc = orc_mc_create(A, PL, nullptr, mp);
    if (!mc) return -1;
    const int64_t n = A->m.n;
    Problem P(A->m, PL ? &PL->m : nullptr, nullptr, b);
    auto norm2 = [](const std::vector<double>& v) {
        double s = 0.0;
        for (double e : v) s += e * e;
        return std::sqrt(s);
    };
    std::vector<double> xv(x, x + n), rp(n), f(n), delta(n), F(n), bv(b, b + n);
    const double bnorm = norm2(bv);
    const double crit = ap->tolerance * bnorm;
    Anderson aa(*ap, n);
    P.prec_residual(xv, rp);
    double rnorm = norm2(rp);
    int k = 0;
    while (!(rnorm < crit) && k < ap->max_iters && std::isfinite(rnorm)) {
        // MCSAModelEvaluator::evalModelImpl (src/MCLS_MCSAModelEvaluator_impl.hpp:306-350):
        // f = x, smoothing f += r, Monte Carlo correction of the residual
        // problem, F = f + delta - x.
        f = xv;
        for (int l = 0; l < ap->smoother_steps; ++l) {
            for (int64_t i = 0; i < n; ++i) f[i] = f[i] + rp[i];
            P.prec_residual(f, rp);
        }
        std::fill(delta.begin(), delta.end(), 0.0);
        if (orc_mc_solve(mc, rp.data(), delta.data(), 1, 0, nullptr, nullptr, nullptr, nullptr) < 0) {
            orc_mc_free(mc);
            return -1;
        }
        for (int64_t i = 0; i < n; ++i) F[i] = (f[i] + delta[i]) - xv[i];
        aa.step(k, xv, F);
        ++k;
        P.prec_residual(xv, rp);
        rnorm = norm2(rp);
        if (res_hist && k <= max_hist) res_hist[k - 1] = rnorm;
    }
    std::copy(xv.begin(), xv.end(), x);
    if (iters) *iters = k;
    if (achieved) *achieved = bnorm > 0.0 ? rnorm / bnorm : rnorm;
    if (total_steps) *total_steps = mc->total_steps;
    orc_mc_free(mc);
    return rnorm < crit ? 1 : 0;
}

int orc_anderson_linear(const orc_csr* M, const double* c, const orc_anderson_params* ap,
                        double* x, int* iters, int max_hist, double* iterates) {
    const int64_t n = M->m.n;
    std::vector<double> xv(x, x + n), g(n), F(n);
    double cn = 0.0;
    for (int64_t i = 0; i < n; ++i) cn += c[i] * c[i];
    const double crit = ap->tolerance * std::sqrt(cn);
    Anderson aa(*ap, n);
    if (iterates) std::copy(xv.begin(), xv.end(), iterates);
    int k = 0;
    bool conv = false;
    while (k < ap->max_iters) {
        spmv(M->m, xv.data(), g.data());
        double fn = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            F[i] = (g[i] + c[i]) - xv[i];
            fn += F[i] * F[i];
        }
        if (std::sqrt(fn) < crit) {
            conv = true;
            break;
        }
        aa.step(k, xv, F);
        ++k;
        if (iterates && k <= max_hist) std::copy(xv.begin(), xv.end(), iterates + k * n);
    }
    std::copy(xv.begin(), xv.end(), x);
    if (iters) *iters = k;
    return conv ? 1 : 0;
}

int orc_fixed_point_solve(const orc_csr* A, const orc_csr* PL, const orc_csr* PR,
                          const orc_mcsa_params* sp, const double* b, double* x, int* iters,
                          double* achieved, int max_hist, double* res_hist) {
    // FixedPointSolverManager::solve (src/MCLS_FixedPointSolverManager_impl.hpp:208-321)
    const int64_t n = A->m.n;
    Problem P(A->m, PL ? &PL->m : nullptr, PR ? &PR->m : nullptr, b);
    auto norm_inf = [](const std::vector<double>& v) {
        double m = 0.0;
        for (double e : v) m = std::max(m, std::abs(e));
        return m;
    };
    std::vector<double> xv(x, x + n), rp(n), p(n), v(n), bv(b, b + n);
    double source_norm;
    if (PL) {
        std::vector<double> t(n);
        spmv(PL->m, b, t.data());
        source_norm = norm_inf(t);
    } else {
        source_norm = norm_inf(bv);
    }
    const double raw_source = source_norm;
    if (std::abs(source_norm) < 10.0 * std::numeric_limits<double>::epsilon()) source_norm = 1.0;
    const double criteria = sp->tolerance * source_norm;
    P.prec_residual(xv, rp);
    double rnorm = norm_inf(rp);
    int it = 0;
    bool go = true;
    while (go) {
        ++it;
        fixed_point_step(P, sp->fixed_point_type, sp->richardson_omega, xv, rp, p, v);
        rnorm = norm_inf(rp);
        if (res_hist && it <= max_hist) res_hist[it - 1] = rnorm;
        if (it % sp->check_freq == 0) go = (rnorm > criteria) && (it < sp->max_iters);
    }
    if (PR) {
        spmv(PR->m, xv.data(), p.data());
        xv = p;
    }
    std::copy(xv.begin(), xv.end(), x);
    if (iters) *iters = it;
    if (achieved) *achieved = raw_source > 0.0 ? rnorm / raw_source : rnorm;
    return rnorm <= criteria ? 1 : 0;
}

void orc_set_threads(int threads) { g_threads = threads < 1 ? 1 : threads; }

int orc_pcg(const orc_csr* A, const double* b, double* x, double tol, int max_iters,
            int* iters, double* relres) {
    // Conjugate gradients with the diagonal as preconditioner (Hestenes and
    // Stiefel; M = diag(A)), FP64, for symmetric positive definite A.  Not a
    // reference routine: the FP64 solve MCSA results are measured against.
    const Csr& M = A->m;
    const int64_t n = M.n;
    std::vector<double> dinv(n), r(n), z(n), p(n), q(n);
    for (int64_t i = 0; i < n; ++i) {
        double d = 0.0;
        for (int64_t k = M.rp[i]; k < M.rp[i + 1]; ++k)
            if (M.ci[k] == i) d = M.v[k];
        if (d <= 0.0) return -1;
        dinv[i] = 1.0 / d;
    }
    auto dot = [&](const std::vector<double>& a, const std::vector<double>& c) {
        return parallel_sum(n, [&](int64_t lo, int64_t hi) {
            double t = 0.0;
            for (int64_t i = lo; i < hi; ++i) t += a[i] * c[i];
            return t;
        });
    };
    std::vector<double> bv(b, b + n);
    const double bn = std::sqrt(dot(bv, bv));
    int it = 0;
    double rn = 0.0;
    // The recursively updated residual drifts from b - A x; CG restarts from
    // the true residual until that one meets the tolerance.
    for (int restart = 0; restart < 8; ++restart) {
        spmv(M, x, q.data());
        for (int64_t i = 0; i < n; ++i) {
            r[i] = b[i] - q[i];
            z[i] = dinv[i] * r[i];
            p[i] = z[i];
        }
        double rz = dot(r, z);
        rn = std::sqrt(dot(r, r));
        if (rn <= tol * bn || it >= max_iters) break;
        while (rn > tol * bn && it < max_iters) {
            ++it;
            spmv(M, p.data(), q.data());
            const double alpha = rz / dot(p, q);
            parallel_ranges(n, [&](int64_t lo, int64_t hi) {
                for (int64_t i = lo; i < hi; ++i) {
                    x[i] += alpha * p[i];
                    r[i] -= alpha * q[i];
                    z[i] = dinv[i] * r[i];
                }
            });
            rn = std::sqrt(dot(r, r));
            const double rz2 = dot(r, z);
            const double beta = rz2 / rz;
            rz = rz2;
            parallel_ranges(n, [&](int64_t lo, int64_t hi) {
                for (int64_t i = lo; i < hi; ++i) p[i] = z[i] + beta * p[i];
            });
        }
    }
    if (iters) *iters = it;
    if (relres) *relres = bn > 0.0 ? rn / bn : rn;
    return rn <= tol * bn ? 1 : 0;
}

namespace {
double g_mcsa_setup_s = 0.0, g_mcsa_loop_s = 0.0;
}

void orc_mcsa_last_timing(double* setup_s, double* loop_s) {
    if (setup_s) *setup_s = g_mcsa_setup_s;
    if (loop_s) *loop_s = g_mcsa_loop_s;
}

int orc_mcsa_solve(const orc_csr* A, const orc_csr* PL, const orc_csr* PR,
                   const orc_mc_params* mp, const orc_mcsa_params* sp,
                   const double* b, double* x, int* iters, double* achieved,
                   int max_hist, double* res_hist, int64_t* total_steps) {
    // MCSASolverManager::solve (src/MCLS_MCSASolverManager_impl.hpp:278-432)
    const auto t_setup = std::chrono::steady_clock::now();
    orc_mc* mc = orc_mc_create(A, PL, PR, mp);
    if (!mc) return -1;
    const Csr& Am = A->m;
    const int64_t n = Am.n;
    auto norm2 = [&](const std::vector<double>& v) {
        double s = 0.0;
        for (double e : v) s += e * e;
        return std::sqrt(s);
    };
    std::vector<double> xv(x, x + n), rp(n), tmp(n), delta(n), pw(n), vw(n);
    Problem P(Am, PL ? &PL->m : nullptr, PR ? &PR->m : nullptr, b);
    // LinearProblem::updatePrecResidual (src/MCLS_LinearProblem_impl.hpp:410-442)
    auto update_prec_residual = [&]() { P.prec_residual(xv, rp); };
    std::vector<double> bv(b, b + n);
    double source_norm;
    if (PL) {
        spmv(PL->m, b, tmp.data());
        source_norm = norm2(tmp);
    } else {
        source_norm = norm2(bv);
    }
    double achieved_norm = source_norm;
    if (std::abs(source_norm) < 10.0 * std::numeric_limits<double>::epsilon())
        source_norm = 1.0;
    const double criteria = sp->tolerance * source_norm;
    update_prec_residual();
    double rnorm = norm2(rp);
    int it = 0;
    bool go = true;
    const auto t_loop = std::chrono::steady_clock::now();
    g_mcsa_setup_s = std::chrono::duration<double>(t_loop - t_setup).count();
    while (go) {
        ++it;
        for (int l = 0; l < sp->smoother_steps; ++l)
            fixed_point_step(P, sp->fixed_point_type, sp->richardson_omega, xv, rp, pw, vw);
        std::fill(delta.begin(), delta.end(), 0.0);
        if (orc_mc_solve(mc, rp.data(), delta.data(), 1, 0, nullptr, nullptr, nullptr, nullptr) < 0) {
            orc_mc_free(mc);
            return -1;
        }
        for (int64_t i = 0; i < n; ++i) xv[i] = xv[i] + delta[i];
        update_prec_residual();
        rnorm = norm2(rp);
        if (res_hist && it <= max_hist) res_hist[it - 1] = rnorm;
        if (it % sp->check_freq == 0) go = (rnorm > criteria) && (it < sp->max_iters);
    }
    g_mcsa_loop_s =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t_loop).count();
    if (PR) {
        spmv(PR->m, xv.data(), tmp.data());
        xv = tmp;
    }
    std::copy(xv.begin(), xv.end(), x);
    if (iters) *iters = it;
    if (achieved) *achieved = achieved_norm > 0.0 ? rnorm / achieved_norm : rnorm;
    if (total_steps) *total_steps = mc->total_steps;
    orc_mc_free(mc);
    return rnorm <= criteria ? 1 : 0;
}

namespace {

// Forward histories laid out as the forward source lays them out
// (src/MCLS_UniformForwardSource_impl.hpp:60-148): history e starts at state
// e mod n with weight 1.  Each step adds w * b[s] (collision) or
// w * (H b)_s (expected value) to the history's sum
// (src/MCLS_ForwardTally.hpp:123-132), which goes to its start state
// (src/MCLS_ForwardTally_impl.hpp:84-110); x_i is the mean over the
// histories started at i, plus b_i for the expected value, as the forward
// solve finishes it.
int64_t bench_walks_forward(const orc_mc* mc, const double* rhs, int64_t nh, int threads,
                            double* x, double* secs) {
    const Domain& D = mc->D;
    const int64_t n = D.n;
    const int L = mc->p.history_length;
    const bool ev = mc->p.estimator == 1;
    std::vector<double> hb;
    if (ev) {
        hb.assign(n, 0.0);
        for (int64_t i = 0; i < n; ++i) {
            double s = 0.0;
            for (int64_t k = D.rp[i]; k < D.rp[i + 1]; ++k) s = s + D.h[k] * rhs[D.col[k]];
            hb[i] = s;
        }
    }
    const double* tsrc = ev ? hb.data() : rhs;
    if (threads < 1) threads = 1;
    std::vector<std::vector<double>> sums(threads, std::vector<double>(n, 0.0));
    std::vector<int64_t> steps(threads, 0);
    auto t0 = std::chrono::steady_clock::now();
    auto work = [&](int t) {
        Xorshift64 xs(orc_rank_seed(0x5EEDULL, t) | 1ULL);
        std::vector<double>& sm = sums[t];
        int64_t lo = nh * t / threads, hi = nh * (t + 1) / threads;
        int64_t st = 0;
        for (int64_t e = lo; e < hi; ++e) {
            const int64_t s0 = e % n;
            int64_t s = s0;
            double w = 1.0, h = 0.0;
            for (int k = 0; k < L; ++k) {
                h += w * tsrc[s];
                int64_t r0 = D.rp[s];
                int j = sample_cdf(&D.cdf[r0], int(D.rp[s + 1] - r0), canonical(xs()));
                w *= D.w[s] * (D.h[r0 + j] > 0.0 ? 1.0 : -1.0);
                s = D.col[r0 + j];
                ++st;
            }
            sm[s0] += h;
        }
        steps[t] = st;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    auto t1 = std::chrono::steady_clock::now();
    if (secs) *secs = std::chrono::duration<double>(t1 - t0).count();
    int64_t total = 0;
    for (int t = 0; t < threads; ++t) total += steps[t];
    if (x) {
        for (int64_t i = 0; i < n; ++i) {
            double s = 0.0;
            for (int t = 0; t < threads; ++t) s += sums[t][i];
            const int64_t count = nh / n + (i < nh % n ? 1 : 0);
            x[i] = (count ? s / double(count) : 0.0) + (ev ? rhs[i] : 0.0);
        }
    }
    return total;
}

}  // namespace

int64_t orc_bench_walks(const orc_mc* mc, const double* rhs, int64_t nh,
                        int threads, double* x, double* secs) {
    if (mc->p.direction == 1) return bench_walks_forward(mc, rhs, nh, threads, x, secs);
    // Independent adjoint collision histories, one Xorshift per thread, the
    // source sampled per thread from the |rhs| CDF (buildRandomSource), the
    // per-thread tallies summed at the end.
    const Domain& D = mc->D;
    const int64_t n = D.n;
    const int L = mc->p.history_length;
    std::vector<double> cdf(n);
    double norm1 = 0.0;
    for (int64_t i = 0; i < n; ++i) norm1 += std::abs(rhs[i]);
    cdf[0] = std::abs(rhs[0]);
    for (int64_t i = 1; i < n; ++i) cdf[i] = cdf[i - 1] + std::abs(rhs[i]);
    for (int64_t i = 0; i < n; ++i) cdf[i] /= norm1;
    if (threads < 1) threads = 1;
    std::vector<std::vector<double>> tallies(threads, std::vector<double>(n, 0.0));
    std::vector<int64_t> steps(threads, 0);
    auto t0 = std::chrono::steady_clock::now();
    auto work = [&](int t) {
        Xorshift64 xs(orc_rank_seed(0x5EEDULL, t) | 1ULL);
        std::vector<double>& tl = tallies[t];
        int64_t lo = nh * t / threads, hi = nh * (t + 1) / threads;
        int64_t st = 0;
        for (int64_t e = lo; e < hi; ++e) {
            int64_t s = sample_cdf(cdf.data(), int(n), canonical(xs()));
            double w = norm1 * (rhs[s] > 0.0 ? 1.0 : -1.0);
            for (int k = 0; k < L; ++k) {
                tl[s] += w;
                int64_t r0 = D.rp[s];
                int j = sample_cdf(&D.cdf[r0], int(D.rp[s + 1] - r0), canonical(xs()));
                w *= D.w[s] * (D.h[r0 + j] > 0.0 ? 1.0 : -1.0);
                s = D.col[r0 + j];
                ++st;
            }
        }
        steps[t] = st;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto& th : pool) th.join();
    auto t1 = std::chrono::steady_clock::now();
    if (secs) *secs = std::chrono::duration<double>(t1 - t0).count();
    int64_t total = 0;
    for (int t = 0; t < threads; ++t) total += steps[t];
    if (x) {
        for (int64_t i = 0; i < n; ++i) {
            double s = 0.0;
            for (int t = 0; t < threads; ++t) s += tallies[t][i];
            x[i] = s / double(nh);
        }
    }
    return total;
}

}  // extern "C"
