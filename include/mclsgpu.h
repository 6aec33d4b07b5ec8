/*
 * mclsgpu.h -- C ABI of the B200 MCSA library (libmclsgpu.so).
 *
 * This is the drop-in boundary under the MCLS solver managers: the C++
 * facade (include/MCLS_*.hpp) and any FFI binding call only these entry
 * points.  Plain pointers and sizes; no CUDA or C++ types in signatures.
 * Every entry point returns an mclsgpu_status and never throws; the message
 * of the last failure on a context is available through mclsgpu_last_error.
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the MCLS source tree).
 *
 * Threading: one context owns one CUDA stream; calls on one context must be
 * serialised by the caller (the reference is single-threaded per rank).
 * Distinct contexts may be used from distinct host threads.
 * Streams: the context's stream does not wait for the legacy default stream,
 * so device vectors given to the *_dev entry points must be complete when
 * the call is made (synchronise the stream that wrote them); every call
 * returns after its own work has finished, so its outputs are complete.
 * Ownership: host arrays are borrowed for the duration of a call and copied;
 * the *_dev variants borrow caller device memory for the duration of the
 * call.  Handles are owned by the caller and released with *_destroy.
 */
#ifndef MCLSGPU_H
#define MCLSGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MCLSGPU_ABI_VERSION 1

typedef enum {
    MCLSGPU_OK = 0,
    MCLSGPU_ERR_INVALID_ARG = 1,  /* bad argument (MCLS_REQUIRE analogue)        */
    MCLSGPU_ERR_CUDA = 2,         /* CUDA runtime error                           */
    MCLSGPU_ERR_DIVERGED = 3,     /* non-finite residual or weight                */
    MCLSGPU_ERR_TIMEOUT = 4,      /* a bounded device wait gave up                */
    MCLSGPU_ERR_NOT_CONVERGED = 5,/* informational: max iterations reached        */
    MCLSGPU_ERR_DEGENERATE = 6,   /* empty or zero-weight domain row (MCLS_CHECK) */
    MCLSGPU_ERR_NO_DEVICE = 7,    /* no usable CUDA device                        */
    MCLSGPU_ERR_UNSUPPORTED = 8   /* configuration outside the library's limits  */
} mclsgpu_status;

/* Monte Carlo direction (MonteCarloTag of the reference managers). */
enum { MCLSGPU_ADJOINT = 0, MCLSGPU_FORWARD = 1 };
/* Estimator: "Estimator Type" = "Collision" | "Expected Value". */
enum { MCLSGPU_COLLISION = 0, MCLSGPU_EXPECTED_VALUE = 1 };
/* "Source Sampling Type" = "Random" | "Stratified". */
enum { MCLSGPU_SOURCE_RANDOM = 0, MCLSGPU_SOURCE_STRATIFIED = 1 };
/* Walk precision: FP64 records/uniforms/weights/tallies (bit-exact parity
 * mode) or FP32 packed records, uniforms, weights and tallies. */
enum { MCLSGPU_FP64 = 0, MCLSGPU_FP32 = 1 };
/* Random stream: the reference's single Xorshift stream reproduced exactly
 * (GF(2) jump-ahead per history) or the counter-based per-history stream. */
enum { MCLSGPU_RNG_REFERENCE = 0, MCLSGPU_RNG_COUNTER = 1 };
/* Preconditioner kinds. */
enum {
    MCLSGPU_PREC_NONE = 0,
    MCLSGPU_PREC_POINT_JACOBI = 1,
    MCLSGPU_PREC_BLOCK_JACOBI = 2,
    MCLSGPU_PREC_LEARNED_SPAI = 3,
    MCLSGPU_PREC_USER_CSR = 4
};

typedef struct mclsgpu_context mclsgpu_context;
typedef struct mclsgpu_operator mclsgpu_operator;
typedef struct mclsgpu_precond mclsgpu_precond;
typedef struct mclsgpu_domain mclsgpu_domain;

/* Monte Carlo parameters.  Field <-> ParameterList key:
 *   history_length      "History Length" (src/MCLS_AlmostOptimalDomain_impl.hpp:88-91)
 *   weight_cutoff       "Weight Cutoff", relative to |starting weight|; 0 = off
 *   sample_ratio        "Sample Ratio"; <= 0 means the key is absent
 *                       (src/MCLS_UniformAdjointSource_impl.hpp:82-86)
 *   source_sampling     "Source Sampling Type" (:90-101)
 *   neumann_relaxation  "Neumann Relaxation"; <= 0 means absent
 *   composite_threshold "Composite Operator Threshold"
 *   rng_mode            "Reproducible MC Mode" = true selects REFERENCE
 *   seed                Xorshift seed (REFERENCE) or stream key (COUNTER)
 */
typedef struct {
    uint32_t size;            /* sizeof(mclsgpu_mc_params) */
    int32_t direction;
    int32_t estimator;
    int32_t history_length;
    double weight_cutoff;
    double sample_ratio;
    int32_t source_sampling;
    int32_t precision;
    double neumann_relaxation;
    double composite_threshold;
    int32_t rng_mode;
    int32_t record_format;    /* FP32 walk records: 0 = automatic, 1 = packed
                               * (column, CDF) pairs, 2 = stencil (CDF slots for
                               * a fixed set of column offsets), 3 = stencil
                               * with 16-bit CDF thresholds (opt-in) */
    uint64_t seed;
} mclsgpu_mc_params;

/* Record formats (mclsgpu_mc_params.record_format).  STENCIL16 keeps W and
 * the tally source in FP32 and quantises each transition's cumulative
 * probability to 16 bits (a selection differs from the FP32 one with
 * probability below 2^-16 per column), so that a row of up to 10 column
 * offsets fits 32 bytes and up to 26 fit 64 bytes; the walk then samples an
 * iteration matrix within 2^-16 W of H.  No counterpart in the reference. */
enum {
    MCLSGPU_RECORD_AUTO = 0,
    MCLSGPU_RECORD_PACKED = 1,
    MCLSGPU_RECORD_STENCIL = 2,
    MCLSGPU_RECORD_STENCIL16 = 3
};

/* MCSA parameters (src/MCLS_MCSASolverManager_impl.hpp:290-343). */
typedef struct {
    uint32_t size;            /* sizeof(mclsgpu_mcsa_params) */
    int32_t max_iters;        /* "Maximum Iterations" (1000)        */
    double tolerance;         /* "Convergence Tolerance" (1.0)      */
    int32_t check_freq;       /* "Iteration Check Frequency" (1)    */
    int32_t smoother_steps;   /* "Smoother Steps" (1)               */
    double richardson_omega;  /* "Richardson Relaxation" (1.0)      */
    int32_t print_freq;       /* "Iteration Print Frequency" (10)   */
    int32_t verbose;          /* print the reference's banner lines */
    int32_t host_loop;        /* 1: host-driven loop (one launch sequence and
                               * host check per iteration) instead of the
                               * device-side graph loop; for profilers */
    int32_t fixed_point_type; /* "Fixed Point Type": MCLSGPU_FIXED_POINT_*
                               * (Richardson) -- the smoother's iteration */
} mclsgpu_mcsa_params;

/* Fixed-point iterations (FixedPointIterationFactory names,
 * src/MCLS_FixedPointIterationFactory_impl.hpp:61-64). */
enum {
    MCLSGPU_FIXED_POINT_RICHARDSON = 0,       /* "Richardson"       */
    MCLSGPU_FIXED_POINT_STEEPEST_DESCENT = 1, /* "Steepest Descent" */
    MCLSGPU_FIXED_POINT_MINRES = 2,           /* "MINRES"           */
    MCLSGPU_FIXED_POINT_RNSD = 3              /* "RNSD"             */
};

/* Preconditioner parameters. */
typedef struct {
    uint32_t size;            /* sizeof(mclsgpu_precond_params) */
    int32_t kind;             /* MCLSGPU_PREC_*                                 */
    int32_t block_size;       /* "Jacobi Block Size" for BLOCK_JACOBI           */
    int32_t reserved0;
    /* USER_CSR: a host CSR matrix used as the left preconditioner. */
    int64_t user_n;
    const int64_t* user_rowptr;
    const int64_t* user_colind;
    const double* user_values;
    /* LEARNED_SPAI: network handle from mclsgpu_spai_* (may be NULL) and the
     * spectral-radius threshold at which Jacobi is used instead (0.95). */
    const void* spai_net;
    double rho_fallback;
} mclsgpu_precond_params;

/* Statistics of the last solve. */
typedef struct {
    uint32_t size;            /* sizeof(mclsgpu_stats) */
    int32_t iterations;
    int32_t converged;
    int32_t fallback_taken;   /* learned preconditioner replaced by Jacobi */
    double achieved_tol;      /* |rp|_2 / |PL b|_2 (MCSASolverManager::achievedTol) */
    double residual_norm;     /* final |rp|_2 */
    int64_t histories;        /* histories transported (all iterations) */
    int64_t walk_steps;       /* transitions performed (all iterations) */
    double solve_ms;          /* device time of the solve (CUDA events) */
    double walk_ms;           /* FP32 walk kernels: summed device duration */
    double rho;               /* spectral radius estimate (when computed) */
    int64_t walk_launches;    /* FP32 walk kernel launches in the solve */
    int64_t kernel_launches;  /* library kernels launched by the solve */
} mclsgpu_stats;

/* ---- version / device --------------------------------------------------- */
int mclsgpu_abi_version(void);
/* Library build information (architecture, options). */
const char* mclsgpu_build_info(void);

/* Diagnostics, no counterpart in the reference: the number of device
 * allocations (cudaMalloc) and releases (cudaFree) the library has made since
 * it was loaded, over all contexts and devices (either pointer may be NULL). */
int mclsgpu_debug_device_allocations(int64_t* allocs, int64_t* frees);

/* ---- context ------------------------------------------------------------ */
/* Replaces the Teuchos::Comm / rank plumbing of the managers: one context per
 * device.  `device` < 0 selects the current device. */
int mclsgpu_context_create(int device, mclsgpu_context** out);
int mclsgpu_context_destroy(mclsgpu_context* ctx);
const char* mclsgpu_last_error(const mclsgpu_context* ctx);
/* Synchronise the context stream and report any pending device error. */
int mclsgpu_context_sync(mclsgpu_context* ctx);
/* Failure detection, no counterpart in the reference.  The library's kernels
 * wait on tensor-core completion barriers with a bounded number of polls
 * (default 1,048,576); a wait that runs out ends its kernel early, the call
 * returns MCLSGPU_ERR_TIMEOUT and the context stays usable.  This sets that
 * bound on the context's device for every later launch (polls < 0 restores
 * the default; 0 makes every such wait give up at once, which failure-
 * detection tests use). */
int mclsgpu_set_wait_limit(mclsgpu_context* ctx, int32_t polls);

/* ---- operator (LinearProblem's A) --------------------------------------- */
/* Replaces LinearProblem(A, x, b)'s operator handle
 * (src/MCLS_LinearProblem.hpp:73-80): a square FP64 CSR matrix with sorted
 * column indices, copied to the device. */
int mclsgpu_operator_upload(mclsgpu_context* ctx, int64_t n,
                            const int64_t* rowptr, const int64_t* colind,
                            const double* values, mclsgpu_operator** out);
int mclsgpu_operator_destroy(mclsgpu_operator* op);
int64_t mclsgpu_operator_rows(const mclsgpu_operator* op);
int64_t mclsgpu_operator_nnz(const mclsgpu_operator* op);
/* y = A x with host vectors (MatrixTraits::apply,
 * tpetra/src/MCLS_TpetraCrsMatrixAdapter.hpp:366-371). */
int mclsgpu_operator_apply(mclsgpu_operator* op, const double* x, double* y);
/* y = A x with host vectors, allocating no device memory.  No counterpart in
 * the reference: it exists for callers that cannot let a library call
 * cudaMalloc/cudaFree (a thread under a real-time budget, since those calls
 * can synchronise the device; an application whose pool owns all device
 * memory).  x and y are staged through one static device array built into
 * the library (16 MiB, held on every GPU that loads it until exit), so the
 * operator may have at most 1,048,576 rows; larger ones get
 * MCLSGPU_ERR_INVALID_ARG.  All calls on a device share that array: calls
 * that overlap on the GPU race and must be serialised by the caller.  The
 * first call on a device looks up the array's address; make it before any
 * stream capture begins. */
int mclsgpu_operator_apply_static(mclsgpu_operator* op, const double* x, double* y);

/* ---- preconditioner ------------------------------------------------------ */
/* Replaces Preconditioner<Matrix>::buildPreconditioner / getLeftPreconditioner
 * (src/MCLS_Preconditioner.hpp:75-100;
 *  tpetra/src/MCLS_TpetraPointJacobiPreconditioner_impl.hpp:104-139;
 *  tpetra/src/MCLS_TpetraBlockJacobiPreconditioner_impl.hpp:122-223). */
int mclsgpu_precond_build(mclsgpu_context* ctx, mclsgpu_operator* op,
                          const mclsgpu_precond_params* params,
                          mclsgpu_precond** out);
int mclsgpu_precond_destroy(mclsgpu_precond* pc);
/* Copies the preconditioner's CSR to host arrays (NULL arrays query sizes:
 * *nnz_out receives the entry count). */
int mclsgpu_precond_export(mclsgpu_precond* pc, int64_t* nnz_out,
                           int64_t* rowptr, int64_t* colind, double* values);

/* ---- learned SPAI network ------------------------------------------------- */
/* No counterpart in the reference (its preconditioner slot for ParaSails is
 * the nearest relative).  A per-row MLP (16 stencil features -> 64 -> 64 ->
 * 16, ReLU, BF16 tensor-core products with FP32 accumulation) emits row i of
 * a sparse approximate inverse M on A's pattern for operators stored by
 * diagonal offsets with `slots` (3..9) offsets.  It is trained on the GPU to
 * minimise (1/R) sum_v |v - M A v|^2 / |v|^2 over vectors v (MCSA residual
 * snapshots and random vectors) and used through mclsgpu_precond_build with
 * kind MCLSGPU_PREC_LEARNED_SPAI, where point Jacobi replaces it when its
 * rho(I - M A) reaches both rho_fallback and the Jacobi rho. */
typedef struct mclsgpu_spai mclsgpu_spai;
typedef struct {
    uint32_t size;            /* sizeof(mclsgpu_spai_adam) */
    double lr;                /* step size */
    double beta1, beta2, eps; /* Adam moments and denominator guard */
    double grad_clip;         /* per-component gradient clip; <= 0 = off */
} mclsgpu_spai_adam;
/* Number of FP32 parameters (W1[64][16], b1, W2[64][64], b2, W3[16][64], b3). */
int mclsgpu_spai_num_params(void);
/* He-uniform hidden layers from `seed`, zero output layer (= point Jacobi). */
int mclsgpu_spai_create(mclsgpu_context* ctx, int slots, uint64_t seed, mclsgpu_spai** out);
int mclsgpu_spai_destroy(mclsgpu_spai* net);
/* Training loss term weight/n * sum_i max(0, W_i - threshold)^2 with W_i
 * the row sum of |I - M A|: the factor by which a forward walk's weight
 * grows at state i, which sets the variance of the Monte Carlo correction.
 * weight 0 (the default) turns it off. */
int mclsgpu_spai_set_penalty(mclsgpu_spai* net, double weight, double threshold);
int mclsgpu_spai_get_params(mclsgpu_spai* net, float* host);
/* Replaces the parameters and clears the optimiser state. */
int mclsgpu_spai_set_params(mclsgpu_spai* net, const float* host);
/* Inference on every row of op: raw outputs out[n][16] and/or the values of
 * M on A's CSR pattern (either may be NULL, not both). */
int mclsgpu_spai_infer(mclsgpu_spai* net, mclsgpu_operator* op, float* out, double* mvals);
/* The same into device arrays (out_dev [n][16] FP32, mvals_dev [nnz] FP64;
 * either may be NULL, not both); *ms (may be NULL) receives the forward
 * kernel's device time. */
int mclsgpu_spai_infer_dev(mclsgpu_spai* net, mclsgpu_operator* op, float* out_dev,
                           double* mvals_dev, float* ms);
/* Loss and parameter gradient (host, may be NULL) for nvec device vectors
 * stored one after another (v_dev[k*n + i]). */
int mclsgpu_spai_gradient(mclsgpu_spai* net, mclsgpu_operator* op, const double* v_dev,
                          int nvec, double* loss, float* grad);
/* One Adam step on that gradient; *loss receives the loss before the step. */
int mclsgpu_spai_train_step(mclsgpu_spai* net, mclsgpu_operator* op, const double* v_dev,
                            int nvec, const mclsgpu_spai_adam* opt, double* loss);
/* In place, for each of nvec device vectors (v_dev[k*n + i]): `iters`
 * applications of H = I - M A with the network's current M, normalised to
 * unit 2-norm after each: the error modes the learned-preconditioner
 * iteration damps slowest, used as on-policy training vectors. */
int mclsgpu_spai_smooth_vectors(mclsgpu_spai* net, mclsgpu_operator* op, double* v_dev, int nvec,
                                int iters);
/* Power-iteration estimates of rho(I - M A) for the network's M and for
 * point Jacobi (either output may be NULL). */
int mclsgpu_spai_rho(mclsgpu_spai* net, mclsgpu_operator* op, int iters, double* rho_learned,
                     double* rho_jacobi);

/* ---- Monte Carlo domain --------------------------------------------------- */
/* Replaces MonteCarloSolverManager::buildMonteCarloDomain + the
 * AlmostOptimalDomain constructor (src/MCLS_MonteCarloSolverManager_impl.hpp:
 * 308-340, src/MCLS_AlmostOptimalDomain_impl.hpp:70-366): builds the
 * (transposed, for ADJOINT) composite operator PL*A*PR, the iteration matrix
 * H = I - w*M on its pattern, the per-row CDFs and weights, and the packed
 * FP32 walk records.  `right` may be NULL (no right preconditioner). */
int mclsgpu_domain_build(mclsgpu_context* ctx, mclsgpu_operator* op,
                         mclsgpu_precond* left, mclsgpu_precond* right,
                         const mclsgpu_mc_params* params,
                         mclsgpu_domain** out);
int mclsgpu_domain_destroy(mclsgpu_domain* dom);
/* Copies the FP64 domain (rowptr[n+1], col[nnz], h[nnz], cdf[nnz],
 * weights[n]) to host arrays; NULL arrays query *nnz_out only. */
int mclsgpu_domain_export(mclsgpu_domain* dom, int64_t* nnz_out,
                          int64_t* rowptr, int64_t* col, double* h,
                          double* cdf, double* weights);
/* Layout of a built domain (no counterpart in the reference: the device
 * record format replaces AlmostOptimalDomain's per-row arrays). */
typedef struct {
    uint32_t size;            /* sizeof(mclsgpu_domain_info) */
    int32_t record_format;    /* MCLSGPU_RECORD_PACKED, _STENCIL or _STENCIL16 */
    int64_t rows;
    int64_t entries;          /* retained H entries */
    int32_t record_bytes;     /* bytes of one FP32 walk record (0: FP64 walk only) */
    int32_t max_row_entries;
    int32_t stencil_offsets;  /* distinct column offsets (stencil records) */
    int32_t operator_dia;     /* operator stored by diagonal offsets */
    int32_t histories_per_lane;  /* FP32 walk launch shape */
    int32_t block_size;
    int32_t record_cache_l1;  /* record loads allocated in L1 */
    int32_t reserved0;
} mclsgpu_domain_info;
int mclsgpu_domain_query(mclsgpu_domain* dom, mclsgpu_domain_info* info);

/* FP32 walk launch shape: histories carried per lane (1, 2, 4 or 8; 2
 * applies to fixed-length histories on records of at most 64 bytes, 4 and 8
 * to fixed-length histories on 32-byte records, others fall back to fewer) and
 * threads per block (128 or 256).  No counterpart in the reference. */
int mclsgpu_domain_set_launch(mclsgpu_domain* dom, int histories_per_lane,
                              int block_size);
/* Record loads of the FP32 walk allocated in L1 (1) or bypassing it (0, the
 * default).  No counterpart in the reference. */
int mclsgpu_domain_set_record_cache(mclsgpu_domain* dom, int allocate_l1);
/* Autotuner: times every launch shape on `reps` Monte Carlo solves of the
 * device vector rhs_dev (n entries), with the record loads bypassing and
 * allocated in L1, keeps the fastest walk and reports it.
 * The random stream position is restored afterwards.  No counterpart in the
 * reference. */
int mclsgpu_domain_autotune(mclsgpu_domain* dom, const double* rhs_dev, int reps,
                            int* histories_per_lane, int* block_size,
                            double* walk_ms);

/* Precision check of the FP32 walk, no counterpart in the reference: runs
 * `histories` histories of History Length transitions (history e starts at
 * state e mod n on its own counter stream keyed by `seed`) along the FP64
 * domain, selecting each transition with std::lower_bound over the FP64 CDF
 * for u = the 53-bit canonical uniform of the draw, as the reference
 * samples (src/MCLS_SamplingTools.hpp:67-80); at every transition the FP32
 * record of the same state is searched as the production walk does, with
 * the 24-bit uniform of the same draw.  Reports the histories with at least
 * one transition where the two select a different column or sign, and the
 * number of such transitions (of histories * History Length).  Needs an
 * FP32 domain. */
int mclsgpu_domain_walk_agreement(mclsgpu_domain* dom, int64_t histories, uint64_t seed,
                                  int64_t* histories_differing, int64_t* transitions_differing);

/* Replace the stream seed/position (restart the reproducible stream). */
int mclsgpu_domain_reseed(mclsgpu_domain* dom, uint64_t seed);
/* Per-rank Xorshift seed as PRNG<RNG>(rank) derives it
 * (src/MCLS_PRNG_impl.hpp:56-75) with std::random_device replaced by
 * `master_seed`. */
uint64_t mclsgpu_rank_seed(uint64_t master_seed, int rank);

/* ---- Monte Carlo solve ---------------------------------------------------- */
/* Replaces MonteCarloSolverManager::solve (src/MCLS_MonteCarloSolverManager_
 * impl.hpp:199-235) and MCSolver::solve (src/MCLS_MCSolver_impl.hpp:82-112):
 * x = MC estimate of (I-H)^-1 (PL rhs, x w).  `internal` = 1 skips the left
 * preconditioning of the source and the right recovery (the MCSA inner
 * solve).  Host vectors of length n. */
int mclsgpu_mc_solve(mclsgpu_domain* dom, const double* rhs, double* x,
                     int internal, mclsgpu_stats* stats);
/* Same with device vectors. */
int mclsgpu_mc_solve_dev(mclsgpu_domain* dom, const double* rhs_dev,
                         double* x_dev, int internal, mclsgpu_stats* stats);
/* Parity instrument: one MC solve recording, per history in emission order
 * (up to max_trace histories), the state before each step
 * (states[e*(L+1)+k], -1 after termination), the final weight, the
 * termination event (2 = CUTOFF) and the starting state. */
int mclsgpu_mc_trace(mclsgpu_domain* dom, const double* rhs, double* x,
                     int internal, int64_t max_trace, int64_t* states,
                     double* final_weight, int32_t* events,
                     int64_t* start_state, int64_t* num_histories);

/* ---- MCSA solve ------------------------------------------------------------ */
/* Replaces MCSASolverManager::solve (src/MCLS_MCSASolverManager_impl.hpp:
 * 278-432) including RichardsonIteration::doOneIteration
 * (src/MCLS_RichardsonIteration_impl.hpp:134-147) and
 * LinearProblem::updatePrecResidual (src/MCLS_LinearProblem_impl.hpp:
 * 410-442).  x is updated in place.  Returns MCLSGPU_OK whether or not the
 * tolerance was met; stats->converged carries the converged status. */
int mclsgpu_mcsa_solve(mclsgpu_domain* dom, const double* b, double* x,
                       const mclsgpu_mcsa_params* params,
                       mclsgpu_stats* stats);
int mclsgpu_mcsa_solve_dev(mclsgpu_domain* dom, const double* b_dev,
                           double* x_dev, const mclsgpu_mcsa_params* params,
                           mclsgpu_stats* stats);
/* ---- fixed-point solve ------------------------------------------------------ */
/* Replaces FixedPointSolverManager::solve (src/MCLS_FixedPointSolverManager_
 * impl.hpp:208-321): params->fixed_point_type iterations alone, no Monte
 * Carlo, until |rp|_inf <= tolerance |PL b|_inf (checked every check_freq
 * iterations) or max_iters.  The iterations are
 *   Richardson        x += w rp; rp = PL (b - A PR x)
 *                     (src/MCLS_RichardsonIteration_impl.hpp:134-147)
 *   Steepest Descent  p = Op rp; a = <rp,rp>/<p,rp>; x += a rp; rp -= a p
 *                     (src/MCLS_SteepestDescentIteration_impl.hpp:114-136)
 *   MINRES            p = Op rp; a = <p,rp>/<p,p>;   x += a rp; rp -= a p
 *                     (src/MCLS_MinimalResidualIteration_impl.hpp:114-136)
 *   RNSD              v = Op^T rp; w = Op v; a = <v,v>/<w,w>; x += a v;
 *                     rp -= a w  (src/MCLS_RNSDIteration_impl.hpp:118-142)
 * with Op = PL A PR (LinearProblem::apply / applyTranspose,
 * src/MCLS_LinearProblem_impl.hpp:251-315).  A zero denominator gives a = 0
 * (the reference divides by it).  left and right may be NULL.  Host
 * vectors (b, x: x holds the initial guess and receives PR x) or, in the
 * _dev form, device vectors.  stats->iterations, converged, residual_norm
 * (|rp|_inf) and achieved_tol (|rp|_inf / |PL b|_inf) are filled. */
int mclsgpu_fixed_point_solve(mclsgpu_context* ctx, mclsgpu_operator* op,
                              mclsgpu_precond* left, mclsgpu_precond* right,
                              const double* b, double* x,
                              const mclsgpu_mcsa_params* params,
                              mclsgpu_stats* stats);
int mclsgpu_fixed_point_solve_dev(mclsgpu_context* ctx, mclsgpu_operator* op,
                                  mclsgpu_precond* left, mclsgpu_precond* right,
                                  const double* b_dev, double* x_dev,
                                  const mclsgpu_mcsa_params* params,
                                  mclsgpu_stats* stats);

/* ---- Anderson-accelerated MCSA --------------------------------------------- */
/* Replaces AndersonSolverManager::solve (src/MCLS_AndersonSolverManager_
 * impl.hpp:186-284): NOX's "Anderson Accelerated Fixed-Point" solver on the
 * MCSAModelEvaluator map (src/MCLS_MCSAModelEvaluator_impl.hpp:306-350)
 *   F(x) = f + delta - x,  f = x smoothed by smoother_steps steps f += r,
 *   r = PL (b - A f), delta = the Monte Carlo estimate of (I-H)^-1 r,
 * accelerated as Walker & Ni (SIAM J. Numer. Anal. 49, 2011) state it:
 *   x_{k+1} = x_k + beta F_k - (dX + beta dF) gamma,
 *   gamma = argmin |F_k - dF gamma|_2 over the last storage_depth
 *   differences, solved through a QR factorisation of dF that is updated in
 *   place (modified Gram-Schmidt to add a column, Givens rotations to drop
 *   the oldest; with adjust_condition, older columns are also dropped while
 *   the reciprocal 1-norm condition number of R is below drop_tolerance).
 * Stops when |PL (b - A x)|_2 < tolerance |b|_2 (MCSAStatusTest,
 * src/MCLS_MCSAStatusTest_impl.hpp:65-110; checked on x0 too) or after
 * max_iters steps.  NOX is not part of the reference tree; its parameter
 * names are kept.  The whole loop runs on the device (a captured graph
 * with a WHILE node).  The domain must have no right preconditioner (the
 * model evaluator applies the left one only).  x is updated in place;
 * stats->iterations = steps taken, achieved_tol = |rp|_2 / |b|_2. */
typedef struct {
    uint32_t size;            /* sizeof(mclsgpu_anderson_params) */
    int32_t max_iters;        /* "Maximum Iterations" (1000)                 */
    double tolerance;         /* "Convergence Tolerance" (1e-8)              */
    int32_t smoother_steps;   /* "Smoother Steps" (1)                        */
    int32_t storage_depth;    /* "Anderson Parameters" sublist: "Storage
                               * Depth" (2), 0..16                           */
    double mixing;            /* "Mixing Parameter" (1.0)                    */
    int32_t start_iteration;  /* "Acceleration Start Iteration" (1), >= 1    */
    int32_t adjust_condition; /* "Adjust Matrix for Condition Number" (0)    */
    double drop_tolerance;    /* "Condition Number Drop Tolerance" (1e-12)   */
    int32_t host_loop;        /* 1: host-driven loop instead of the graph   */
    int32_t reserved0;
} mclsgpu_anderson_params;

int mclsgpu_anderson_solve(mclsgpu_domain* dom, const double* b, double* x,
                           const mclsgpu_anderson_params* params, mclsgpu_stats* stats);
int mclsgpu_anderson_solve_dev(mclsgpu_domain* dom, const double* b_dev, double* x_dev,
                               const mclsgpu_anderson_params* params, mclsgpu_stats* stats);
/* The same solve one step at a time, for drivers that combine the Monte
 * Carlo corrections of several sets (one set per GPU): the model
 * evaluator's MultiSetLinearProblem::blockConstantVectorSum between the
 * Monte Carlo solve and F (src/MCLS_MCSAModelEvaluator_impl.hpp:338-345).
 *   begin:      x = x0; *rnorm = |PL (b - A x0)|_2, *bnorm = |b|_2,
 *               *done = 1 when x0 already passes the status test
 *   correction: smoothing, then delta_dev = this set's Monte Carlo correction
 *   apply:      F = f + scale * delta_dev - x (scale = 1 / number of sets
 *               after the caller summed delta over the sets), the
 *               accelerated update, the new residual and the status test;
 *               *done = 1 when the loop must stop
 *   finish:     x_dev = x; stats of the steps since begin
 * Device vectors of length n.  Every set takes the same steps: the update
 * uses fixed-order reductions, so equal inputs give equal iterates. */
int mclsgpu_anderson_begin(mclsgpu_domain* dom, const double* b_dev, const double* x0_dev,
                           const mclsgpu_anderson_params* params, double* rnorm, double* bnorm,
                           int32_t* done);
int mclsgpu_anderson_correction(mclsgpu_domain* dom, double* delta_dev);
int mclsgpu_anderson_apply(mclsgpu_domain* dom, const double* delta_dev, double scale,
                           double* rnorm, int32_t* done);
int mclsgpu_anderson_finish(mclsgpu_domain* dom, double* x_dev, mclsgpu_stats* stats);

/* MCSA one iteration at a time, for drivers that combine the Monte Carlo
 * corrections of several sets (one set per GPU): the loop of
 * MCSASolverManager::solve with MultiSetLinearProblem::blockConstantVectorSum
 * between the Monte Carlo solve and the update
 * (src/MCLS_MCSASolverManager_impl.hpp:344-400,
 *  src/MCLS_MultiSetLinearProblem_impl.hpp:102-120).
 *   begin:      x = x0, rp = PL (b - A PR x); *rnorm = |rp|_2, *bnorm = |PL b|_2
 *   correction: smoother_steps fixed-point steps, then delta_dev = the Monte
 *               Carlo estimate of the correction (this set's histories)
 *   apply:      x += scale * delta_dev (scale = 1 / number of sets after the
 *               caller summed delta over the sets), new rp; *rnorm = |rp|_2
 *   finish:     x_dev = PR x; stats of the walks since begin
 * Device vectors of length n. */
int mclsgpu_mcsa_begin(mclsgpu_domain* dom, const double* b_dev, const double* x0_dev,
                       const mclsgpu_mcsa_params* params, double* rnorm, double* bnorm);
int mclsgpu_mcsa_correction(mclsgpu_domain* dom, double* delta_dev);
int mclsgpu_mcsa_apply(mclsgpu_domain* dom, const double* delta_dev, double scale,
                       double* rnorm);
int mclsgpu_mcsa_finish(mclsgpu_domain* dom, double* x_dev, mclsgpu_stats* stats);
/* ---- multi-set MCSA ---------------------------------------------------------- */
/* Replaces MCSASolverManager::solve on a MultiSetLinearProblem with more than
 * one set (src/MCLS_MCSASolverManager_impl.hpp:344-400 with
 * MultiSetLinearProblem::blockConstantVectorSum,
 * src/MCLS_MultiSetLinearProblem_impl.hpp:102-120): every set (one call per
 * set, typically one process and GPU each, all with the same b, x0, domain
 * parameters and MCSA parameters but their own random streams) transports
 * its own histories; each iteration the sets' Monte Carlo corrections are
 * summed by `reduce` and divided by num_sets.  The sets apply the same sum,
 * so their iterates, residuals and stopping decisions are identical; the sum
 * is the only exchange.
 *   reduce(user, data_dev, n, stream): sum the n doubles at data_dev over
 *   all sets, in place, identically on every set, either enqueued on the
 *   CUDA stream `stream` (a cudaStream_t) or finished before returning;
 *   returns 0 on success.
 *   capturable = 1: reduce only enqueues stream work that a CUDA graph
 *   capture may record (NCCL); the whole loop then runs on the device in a
 *   captured WHILE graph, with no host round trip per iteration.  Otherwise
 *   (a host reduction such as MPI or gloo on host copies) the loop runs from
 *   the host.  *device_loop (may be NULL) receives which one ran. */
typedef int (*mclsgpu_set_reduce_fn)(void* user, double* data_dev, int64_t n, void* stream);
typedef struct {
    uint32_t size;                  /* sizeof(mclsgpu_set_params) */
    int32_t num_sets;               /* "Number of Sets" */
    mclsgpu_set_reduce_fn reduce;
    void* user;
    int32_t capturable;
    int32_t reserved0;
} mclsgpu_set_params;
int mclsgpu_mcsa_solve_sets(mclsgpu_domain* dom, const mclsgpu_set_params* sets, const double* b,
                            double* x, const mclsgpu_mcsa_params* params, mclsgpu_stats* stats,
                            int32_t* device_loop);
int mclsgpu_mcsa_solve_sets_dev(mclsgpu_domain* dom, const mclsgpu_set_params* sets,
                                const double* b_dev, double* x_dev,
                                const mclsgpu_mcsa_params* params, mclsgpu_stats* stats,
                                int32_t* device_loop);
/* The Anderson-accelerated solve of a multi-set problem (AndersonSolverManager
 * on a MultiSetLinearProblem: the model evaluator sums the sets' corrections
 * before F, src/MCLS_MCSAModelEvaluator_impl.hpp:338-345), host vectors, the
 * loop run from the host around mclsgpu_anderson_begin / _correction / the
 * set reducer / _apply (scale 1 / num_sets) / _finish. */
int mclsgpu_anderson_solve_sets(mclsgpu_domain* dom, const mclsgpu_set_params* sets,
                                const double* b, double* x,
                                const mclsgpu_anderson_params* params, mclsgpu_stats* stats);
/* An NCCL communicator of nranks sets (no counterpart in the reference, whose
 * sets talk over MPI): the library loads libnccl.so.2 at run time.  One rank
 * makes the 128-byte unique id and the caller sends it to the others (any
 * channel); every rank then creates its communicator with its own context's
 * device.  mclsgpu_comm_set_params fills set params whose reducer is an
 * in-place ncclAllReduce (sum) on the solve's stream, capturable. */
typedef struct mclsgpu_comm mclsgpu_comm;
int mclsgpu_comm_unique_id(uint8_t* id128);
int mclsgpu_comm_create(mclsgpu_context* ctx, int nranks, int rank, const uint8_t* id128,
                        mclsgpu_comm** out);
int mclsgpu_comm_destroy(mclsgpu_comm* comm);
int mclsgpu_comm_set_params(mclsgpu_comm* comm, mclsgpu_set_params* out);

/* The preconditioned residual PL (b - A x) at the end of the last MCSA
 * solve, copied to the device vector rp_dev (LinearProblem::getPrecResidual,
 * src/MCLS_LinearProblem.hpp:121-122). */
int mclsgpu_domain_residual(mclsgpu_domain* dom, double* rp_dev);

/* ---- batched MCSA: many systems, many right-hand sides -------------------- */
/* No single counterpart in the reference, which solves one system per
 * manager (MCSASolverManager::solve, src/MCLS_MCSASolverManager_impl.hpp:
 * 278-432).  m square systems (host int64 CSR each) with 1..16 right-hand
 * sides each are solved in one MCSA loop: one block-diagonal point-Jacobi
 * domain, one shared set of forward FP32 walks per iteration whose histories
 * carry a tally per right-hand side of their system, and a separate
 * convergence test |rp|_2 <= tol |D^-1 b|_2 for every (system, right-hand
 * side) pair.  The loop (four kernels per iteration) runs in a captured CUDA
 * graph.  params must ask for forward FP32 walks without a weight cutoff. */
typedef struct mclsgpu_batch mclsgpu_batch;
int mclsgpu_batch_build(mclsgpu_context* ctx, int nsys, const int64_t* n,
                        const int64_t* const* rowptr, const int64_t* const* colind,
                        const double* const* values, const int32_t* nrhs,
                        const mclsgpu_mc_params* params, mclsgpu_batch** out);
int mclsgpu_batch_destroy(mclsgpu_batch* b);
/* Vector layout: FP64 arrays of `elements` entries.  System s owns the
 * row-major [n_s][widths[s]] block starting at elem_offsets[s]; widths[s] is
 * nrhs[s] rounded up to a power of two, and columns nrhs[s] .. widths[s]-1
 * are ignored.  Systems are placed grouped by width (not in argument order),
 * with unused padding elements between the groups.  Per-pair outputs are
 * [nsys][max_width].  elem_offsets and widths have nsys entries; any output
 * may be NULL. */
int mclsgpu_batch_layout(mclsgpu_batch* b, int64_t* elem_offsets, int32_t* widths,
                         int64_t* elements, int32_t* max_width);
/* The batch's block-diagonal domain (for mclsgpu_domain_query/reseed). */
int mclsgpu_batch_domain(mclsgpu_batch* b, mclsgpu_domain** dom);
/* Walk launch shape: threads per block (128 or 256) and the work-queue grab
 * (each warp takes 32 * grab histories per grab, 1..8).  The autotuner times
 * block sizes {256, 128} x grabs {1, 2, 4} on `reps` iterations of b_dev
 * (x_dev is overwritten) and keeps the fastest walk. */
int mclsgpu_batch_set_launch(mclsgpu_batch* b, int block_size, int grab);
int mclsgpu_batch_autotune(mclsgpu_batch* b, const double* b_dev, double* x_dev, int reps,
                           int* block_size, int* grab, double* walk_ms);
/* x_dev holds the initial guesses and receives the solutions.  Optional host
 * outputs, [nsys][max_width]: conv_iters = the iteration at which each pair
 * first met the tolerance (-1: never, or an unused column), rel_resid = the
 * final |rp|_2 / |D^-1 b|_2.  params->smoother_steps must be 1. */
int mclsgpu_batch_mcsa_solve_dev(mclsgpu_batch* b, const double* b_dev, double* x_dev,
                                 const mclsgpu_mcsa_params* params, int32_t* conv_iters,
                                 double* rel_resid, mclsgpu_stats* stats);

/* ---- row-partitioned domains (domain-decomposed transport) ---------------- */
/* Replaces the reference's domain decomposition over MPI ranks
 * (DomainTransporter's BOUNDARY events, src/MCLS_DomainTransporter_impl.hpp:
 * 70-119; DomainCommunicator and SourceTransporter buffering histories to the
 * owning rank, src/MCLS_DomainCommunicator_impl.hpp,
 * src/MCLS_SourceTransporter_impl.hpp; the packed history,
 * src/MCLS_History_impl.hpp:56-89) for systems whose domain does not fit one
 * GPU.  A part holds rows [bounds[part], bounds[part+1]) of the domain (FP32
 * records, FP64 domain, tallies).  Histories that step into another part's
 * rows and go on (steps left, weight above the cutoff) are written to that
 * part's outbox as 32-byte mclsgpu_history_wire records and continue there in
 * the next round on the same random stream, so every transition and tally is
 * the one the whole-domain walk makes.  Adjoint histories tally where they
 * stand; a forward history's sum belongs to its start row, so when it ends
 * outside the part that owns that row, the sum goes there as a tally return
 * (state -1) in the next round.  The caller runs the rounds and moves outboxes
 * to inboxes (NCCL all-to-all between GPUs, device copies within one GPU)
 * until no part has departures; no kernel waits on another part. */
typedef struct {
    uint64_t rng;     /* Xorshift state after the last draw */
    int32_t state;    /* the global state the history moved to; -1: a forward
                         tally return */
    int32_t step;     /* transitions taken */
    float weight;
    int32_t id;       /* its index in the global source */
    float acc;        /* forward: the history's Kahan-compensated sum so far */
    float comp;       /* forward: its compensation */
} mclsgpu_history_wire;
int32_t mclsgpu_history_wire_size(void);

typedef struct mclsgpu_subdomain mclsgpu_subdomain;
/* Part `part` of nparts (<= 64).  bounds: nparts + 1 global row bounds from
 * 0 to n_global.  The part's rows of the composite operator the walks
 * follow -- (PL A PR)^T for adjoint walks, PL A PR for forward walks -- as a
 * host CSR (bounds[part+1] - bounds[part] rows, global column indices),
 * filtered by params->composite_threshold.  params: FP32 walks on the
 * counter-based stream, adjoint collision or forward (collision or expected
 * value), of History Length steps or ended earlier by the Weight Cutoff; all
 * parts of one solve take the same params (seed included). */
int mclsgpu_subdomain_build(mclsgpu_context* ctx, int64_t n_global, int32_t nparts,
                            const int64_t* bounds, int32_t part, const int64_t* rowptr,
                            const int64_t* colind, const double* values,
                            const mclsgpu_mc_params* params, mclsgpu_subdomain** out);
int mclsgpu_subdomain_destroy(mclsgpu_subdomain* sd);
int mclsgpu_subdomain_info(const mclsgpu_subdomain* sd, int64_t* row_begin, int64_t* rows,
                           int32_t* record_bytes);
/* Start of one Monte Carlo solve of rhs_dev (the whole source vector,
 * n_global, device; already left preconditioned as an MCSA residual is).
 * Adjoint: the global source is built as the whole-domain solve builds it
 * and the part keeps the histories starting in its rows.  Forward: history e
 * starts at row e / ceil(Sample Ratio), and the part's records take the tally
 * source of its rows.  *n_start = the part's starting histories, *n_total =
 * histories in the solve. */
int mclsgpu_subdomain_begin(mclsgpu_subdomain* sd, const double* rhs_dev, int64_t* n_start,
                            int64_t* n_total);
/* One round: walk the part's starting histories (inbox_dev NULL) or the
 * n_in histories of inbox_dev (device); departures for part q go to
 * outbox_dev[q * capacity + i], i < out_counts[q] (host array of nparts).
 * Fails if a destination needs more than `capacity` slots. */
int mclsgpu_subdomain_transport(mclsgpu_subdomain* sd, const mclsgpu_history_wire* inbox_dev,
                                int64_t n_in, mclsgpu_history_wire* outbox_dev,
                                int64_t capacity, int64_t* out_counts);
/* End of the solve: x_part_dev (the part's rows, device) = the normalised
 * tallies (adjoint: / total histories; forward: / histories per row, plus the
 * source for the expected-value estimator); stats->walk_steps = steps walked
 * in this part. */
int mclsgpu_subdomain_finish(mclsgpu_subdomain* sd, double* x_part_dev, mclsgpu_stats* stats);

/* ---- spectral radius ------------------------------------------------------- */
/* Replaces AlmostOptimalDomain::computeConvergenceCriteria
 * (src/MCLS_AlmostOptimalDomain_impl.hpp:437-635): FP64 power iteration
 * estimates of rho(H) (which = 0), rho(|H|) (which = 1) and rho(H*)
 * (which = 2, |h_ij| * W_i). */
int mclsgpu_domain_spectral_radius(mclsgpu_domain* dom, int which,
                                   int max_iters, double tol, uint64_t seed,
                                   double* rho);

/* Replaces AlmostOptimalDomain::computeConvergenceCriteria and the
 * "Compute Convergence Criteria" printout (src/MCLS_AlmostOptimalDomain_
 * impl.hpp:95-113, 437-635): rho(H), rho(H+ = |H|) and rho(H*) by power
 * iteration, |H|_inf and the smallest row sum of |H|, and the balance
 * parameters max_j |h_ij| / max_j |h_ji| over the states (min, max, mean;
 * states that no row transitions into are left out). */
typedef struct {
    uint32_t size;            /* sizeof(mclsgpu_criteria) */
    int32_t reserved0;
    double rho_h, rho_abs, rho_star;
    double row_sum_max;       /* ||H||_inf */
    double row_sum_min;       /* sum|H|_min */
    double balance_min, balance_max, balance_ave;
} mclsgpu_criteria;
int mclsgpu_domain_convergence_criteria(mclsgpu_domain* dom, int max_iters, double tol,
                                        uint64_t seed, mclsgpu_criteria* out);

#ifdef __cplusplus
}
#endif
#endif /* MCLSGPU_H */
