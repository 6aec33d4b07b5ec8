/*
 * mcls_oracle.h -- C interface of the CPU oracle for the MCSA hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: a plain C++
 * restatement of the reference MCLS algorithm (adjoint/forward Neumann-Ulam
 * transport inside MCSA's Richardson loop).  Only the tests, the smoke check
 * and the CPU-baseline leg of bench.py may load it; the product library
 * (libmclsgpu.so) never links or calls it.
 *
 * Every routine cites the reference file:line it restates (paths relative to
 * the MCLS source tree).  Parity is pinned by (i) the reference's own
 * known-answer tests restated in tests/test_oracle_*.py and (ii) golden
 * vectors produced by the reference's own Xorshift / RNGTraits /
 * SamplingTools code compiled from its sources into oracle/_ref.
 */
#ifndef MCLS_ORACLE_H
#define MCLS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- RNG ------------------------------------------------------------- */
/* Reference Xorshift<uint_fast64_t,13,7,17> draws mapped through libstdc++
 * uniform_real_distribution<double>(0,1) (src/MCLS_Xorshift.hpp:100-108,
 * src/MCLS_RNGTraits.hpp:147-160). */
void orc_xorshift_uniforms(uint64_t seed, int64_t n, double* out);
/* Seed of rank `rank` derived as in src/MCLS_PRNG_impl.hpp:56-75 with the
 * std::random_device draw replaced by `master_seed`. */
uint64_t orc_rank_seed(uint64_t master_seed, int rank);
/* Counter-based generator of the FP32 walks (no reference counterpart): the
 * Xorshift stream started from the state hashed from (seed, epoch, kind, idx),
 * n uniforms in the reference's canonical mapping. */
void orc_counter_uniforms(uint64_t seed, uint64_t epoch, int kind, int64_t idx,
                          int64_t n, double* out);
/* src/MCLS_SamplingTools.hpp:67-80 */
int orc_sample_discrete_cdf(const double* cdf, int size, double u);

/* ---- sparse matrices (opaque CSR, FP64) ------------------------------ */
typedef struct orc_csr orc_csr;
orc_csr* orc_csr_create(int64_t n, const int64_t* rowptr, const int64_t* col,
                        const double* val);
void orc_csr_free(orc_csr*);
int64_t orc_csr_n(const orc_csr*);
int64_t orc_csr_nnz(const orc_csr*);
void orc_csr_copy(const orc_csr*, int64_t* rowptr, int64_t* col, double* val);

orc_csr* orc_transpose(const orc_csr* A);
orc_csr* orc_multiply(const orc_csr* A, const orc_csr* B, double threshold);
/* (PL A PR) or its transpose, per src/MCLS_LinearProblem_impl.hpp:143-221 */
orc_csr* orc_composite(const orc_csr* A, const orc_csr* PL, const orc_csr* PR,
                       int transpose, double threshold);
orc_csr* orc_point_jacobi(const orc_csr* A);
orc_csr* orc_block_jacobi(const orc_csr* A, int block_size);
void orc_spmv(const orc_csr* A, const double* x, double* y);

/* ---- Monte Carlo parameters ----------------------------------------- */
typedef struct {
    int direction;            /* 0 adjoint, 1 forward                          */
    int estimator;            /* 0 collision, 1 expected value                 */
    int history_length;       /* "History Length" (default 10)                 */
    double weight_cutoff;     /* "Weight Cutoff" relative to |w0|; 0 = off    */
    double sample_ratio;      /* "Sample Ratio"; <= 0 means key absent        */
    int stratified;           /* "Source Sampling Type" == "Stratified"        */
    double neumann_relaxation;/* "Neumann Relaxation"; <= 0 means key absent  */
    double composite_threshold;
    int rng_mode;             /* 0 reference Xorshift stream, 1 counter-based  */
    uint64_t seed;            /* xorshift seed (mode 0) or key (mode 1)        */
} orc_mc_params;

/* Monte Carlo solver over one operator: owns the composite operator, the
 * AlmostOptimalDomain restatement and the PRNG position. */
typedef struct orc_mc orc_mc;
orc_mc* orc_mc_create(const orc_csr* A, const orc_csr* PL, const orc_csr* PR,
                      const orc_mc_params* p);
void orc_mc_free(orc_mc*);
/* Domain export: rowptr[n+1], col[], h[], cdf[], weights[n]. */
int64_t orc_mc_domain_nnz(const orc_mc*);
void orc_mc_domain_copy(const orc_mc*, int64_t* rowptr, int64_t* col,
                        double* h, double* cdf, double* weights);
/* One MC solve of (I-H) x = rhs_scaled.  `internal` follows
 * MonteCarloSolverManager(internal_solver): when 0 the RHS is left
 * preconditioned and the result right preconditioned.  Optional trace
 * buffers (may be NULL) are indexed by emission order:
 *   trace_states[e*(L+1)+k] state before step k (k<=steps), -1 after death;
 *   final_weight[e], events[e] (2 = CUTOFF), start_state[e].
 * Returns the number of histories (normalization), or -1 on error. */
int64_t orc_mc_solve(orc_mc*, const double* rhs, double* x, int internal,
                     int64_t max_trace, int64_t* trace_states,
                     double* final_weight, int* events, int64_t* start_state);
uint64_t orc_mc_stream_position(const orc_mc*);
int64_t orc_mc_total_steps(const orc_mc*);

/* ---- MCSA ------------------------------------------------------------ */
typedef struct {
    double tolerance;          /* "Convergence Tolerance" (default 1.0)     */
    int max_iters;             /* "Maximum Iterations" (default 1000)       */
    int check_freq;            /* "Iteration Check Frequency" (default 1)   */
    int smoother_steps;        /* "Smoother Steps" (default 1)              */
    double richardson_omega;   /* "Richardson Relaxation" (default 1.0)     */
    int fixed_point_type;      /* "Fixed Point Type": 0 Richardson, 1 Steepest
                                * Descent, 2 MINRES, 3 RNSD (default 0)     */
} orc_mcsa_params;

/* MCSASolverManager::solve restatement.  x is updated in place.  Writes the
 * iteration count, achieved relative residual and (optionally, up to
 * max_hist entries) the per-iteration |rp|_2 history.  Returns 1 if
 * converged, 0 if not, -1 on error. */
int orc_mcsa_solve(const orc_csr* A, const orc_csr* PL, const orc_csr* PR,
                   const orc_mc_params* mp, const orc_mcsa_params* sp,
                   const double* b, double* x, int* iters, double* achieved,
                   int max_hist, double* res_hist, int64_t* total_steps);

/* Wall seconds of the last orc_mcsa_solve: set-up (domain build, initial
 * residual) and the iteration loop. */
void orc_mcsa_last_timing(double* setup_s, double* loop_s);

/* FixedPointSolverManager::solve restatement: sp->fixed_point_type
 * iterations alone until |rp|_inf <= tolerance |PL b|_inf (or max_iters).
 * x is updated in place (x = PR x at the end).  res_hist gets |rp|_inf per
 * iteration (up to max_hist).  Returns 1 if converged, 0 if not. */
int orc_fixed_point_solve(const orc_csr* A, const orc_csr* PL, const orc_csr* PR,
                          const orc_mcsa_params* sp, const double* b, double* x,
                          int* iters, double* achieved, int max_hist, double* res_hist);

/* ---- Anderson-accelerated MCSA ----------------------------------------- */
/* AndersonSolverManager (src/MCLS_AndersonSolverManager_impl.hpp:65-284):
 * NOX's Anderson-accelerated fixed point on the MCSAModelEvaluator map
 * (src/MCLS_MCSAModelEvaluator_impl.hpp:306-350).  NOX is not in the
 * reference tree; its algorithm is restated from Walker & Ni, "Anderson
 * acceleration for fixed-point iterations", SIAM J. Numer. Anal. 49 (2011),
 * with the QR-updating least-squares solve (modified Gram-Schmidt to add a
 * column, Givens rotations to drop the oldest) and NOX's parameter names. */
typedef struct {
    double tolerance;          /* "Convergence Tolerance" (default 1e-8)        */
    int max_iters;             /* "Maximum Iterations" (default 1000)           */
    int smoother_steps;        /* "Smoother Steps" (default 1)                  */
    int storage_depth;         /* "Anderson Parameters"/"Storage Depth" (2)     */
    double mixing;             /* "Mixing Parameter" (1.0)                      */
    int start_iteration;       /* "Acceleration Start Iteration" (1)            */
    int adjust_condition;      /* "Adjust Matrix for Condition Number" (0)      */
    double drop_tolerance;     /* "Condition Number Drop Tolerance" (1e-12)     */
} orc_anderson_params;

/* Anderson-accelerated MCSA.  x holds x0 and receives the solution.  Stops
 * when |PL (b - A x)|_2 < tolerance |b|_2 (MCSAStatusTest) or after
 * max_iters steps.  res_hist gets |PL (b - A x_k)|_2 for k = 1.. (up to
 * max_hist).  Returns 1 if converged, 0 if not, -1 on error. */
int orc_anderson_solve(const orc_csr* A, const orc_csr* PL, const orc_mc_params* mp,
                       const orc_anderson_params* ap, const double* b, double* x, int* iters,
                       double* achieved, int max_hist, double* res_hist, int64_t* total_steps);

/* The same acceleration of the linear map g(x) = M x + c (no Monte Carlo):
 * stops when |g(x) - x|_2 < tolerance |c|_2 or after max_iters steps.
 * iterates (optional, (max_hist + 1) x n) receives x_0, x_1, ...  Returns 1
 * if converged. */
int orc_anderson_linear(const orc_csr* M, const double* c, const orc_anderson_params* ap,
                        double* x, int* iters, int max_hist, double* iterates);

/* Host threads for the oracle's long loops: the SpMVs, the expected-value
 * source and forward walks on the counter stream (histories partitioned by
 * start state, as ranks own rows).  Results do not depend on the count;
 * default 1 (one reference rank). */
void orc_set_threads(int threads);

/* FP64 conjugate gradients with the diagonal as preconditioner (no reference
 * counterpart): the oracle solve MCSA results are measured against, for
 * symmetric positive definite A.  x holds x0 and receives the solution;
 * stops when |b - A x|_2 <= tol |b|_2 or after max_iters.  Returns 1 if
 * converged, 0 if not, -1 for a non-positive diagonal. */
int orc_pcg(const orc_csr* A, const double* b, double* x, double tol, int max_iters,
            int* iters, double* relres);

/* CPU baseline: independent histories on `threads` threads (one Xorshift per
 * thread, as one MPI rank per core with subdomain transport), `nh` histories
 * of fixed length in the domain's direction: adjoint collision walks from
 * the |rhs| CDF, or forward walks (history e starts at state e mod n; the
 * domain's estimator, collision or expected value).  x gets the estimate.
 * Returns walk steps performed; elapsed seconds through *secs. */
int64_t orc_bench_walks(const orc_mc*, const double* rhs, int64_t nh,
                        int threads, double* x, double* secs);

#ifdef __cplusplus
}
#endif
#endif
