// MCLS_GpuBackend.hpp -- device handles and ParameterList mapping shared by
// the GPU solver managers (MCLS_MonteCarloSolverManager.hpp,
// MCLS_MCSASolverManager.hpp) and preconditioners (MCLS_GpuPreconditioners.hpp).
//
// Everything here is a thin owner around the C ABI in mclsgpu.h: every call
// that fails throws MCLS::Assertion with the library's message, as the
// reference's MCLS_INSIST does (src/MCLS_DBC.hpp:162).
#ifndef MCLS_GPUBACKEND_HPP
#define MCLS_GPUBACKEND_HPP

#include <cstdint>
#include <map>
#include <cstdio>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "MCLS_GpuTraits.hpp"
#include "MCLS_LinearProblem.hpp"
#include "mclsgpu.h"

namespace MCLS {
namespace gpu {

inline const char* status_name(int rc) {
    switch (rc) {
        case MCLSGPU_OK: return "OK";
        case MCLSGPU_ERR_INVALID_ARG: return "invalid argument";
        case MCLSGPU_ERR_CUDA: return "CUDA error";
        case MCLSGPU_ERR_DIVERGED: return "diverged";
        case MCLSGPU_ERR_TIMEOUT: return "device wait timed out";
        case MCLSGPU_ERR_NOT_CONVERGED: return "not converged";
        case MCLSGPU_ERR_DEGENERATE: return "degenerate domain";
        case MCLSGPU_ERR_NO_DEVICE: return "no usable CUDA device";
        case MCLSGPU_ERR_UNSUPPORTED: return "unsupported configuration";
        default: return "unknown status";
    }
}

// One library context (one CUDA stream) per device, shared by every manager
// and preconditioner of the process that uses that device.
class Context {
  public:
    explicit Context(int device) : d_device(device) {
        int rc = mclsgpu_context_create(device, &d_h);
        if (rc != MCLSGPU_OK)
            throw Assertion(std::string("mclsgpu_context_create: ") + status_name(rc));
    }
    ~Context() { mclsgpu_context_destroy(d_h); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    mclsgpu_context* get() const { return d_h; }
    int device() const { return d_device; }
    void check(int rc, const char* what) const {
        if (rc != MCLSGPU_OK && rc != MCLSGPU_ERR_NOT_CONVERGED)
            throw Assertion(std::string(what) + ": " + status_name(rc) + ": " +
                            mclsgpu_last_error(d_h));
    }

    static std::shared_ptr<Context> on(int device) {
        static std::mutex m;
        static std::map<int, std::weak_ptr<Context>> live;
        std::lock_guard<std::mutex> lock(m);
        if (auto c = live[device].lock()) return c;
        auto c = std::make_shared<Context>(device);
        live[device] = c;
        return c;
    }

  private:
    int d_device;
    mclsgpu_context* d_h = nullptr;
};

class Operator {
  public:
    Operator(std::shared_ptr<Context> ctx, std::int64_t n, const std::vector<std::int64_t>& rp,
             const std::vector<std::int64_t>& ci, const std::vector<double>& v)
        : d_ctx(std::move(ctx)) {
        if (std::int64_t(rp.size()) != n + 1 || ci.size() != v.size())
            throw Assertion("operator CSR arrays have inconsistent sizes");
        d_ctx->check(mclsgpu_operator_upload(d_ctx->get(), n, rp.data(), ci.data(), v.data(), &d_h),
                     "mclsgpu_operator_upload");
    }
    ~Operator() { mclsgpu_operator_destroy(d_h); }
    Operator(const Operator&) = delete;
    Operator& operator=(const Operator&) = delete;
    mclsgpu_operator* get() const { return d_h; }
    const std::shared_ptr<Context>& context() const { return d_ctx; }

  private:
    std::shared_ptr<Context> d_ctx;
    mclsgpu_operator* d_h = nullptr;
};

class Precond {
  public:
    Precond(std::shared_ptr<Operator> op, const mclsgpu_precond_params& p)
        : d_op(std::move(op)) {
        const Context& c = *d_op->context();
        c.check(mclsgpu_precond_build(c.get(), d_op->get(), &p, &d_h), "mclsgpu_precond_build");
    }
    ~Precond() { mclsgpu_precond_destroy(d_h); }
    Precond(const Precond&) = delete;
    Precond& operator=(const Precond&) = delete;
    mclsgpu_precond* get() const { return d_h; }
    const std::shared_ptr<Operator>& op() const { return d_op; }
    // Host copy of the preconditioner matrix.
    void exportCsr(std::vector<std::int64_t>& rp, std::vector<std::int64_t>& ci,
                   std::vector<double>& v) const {
        const Context& c = *d_op->context();
        std::int64_t nnz = 0;
        c.check(mclsgpu_precond_export(d_h, &nnz, nullptr, nullptr, nullptr),
                "mclsgpu_precond_export");
        rp.resize(size_t(mclsgpu_operator_rows(d_op->get()) + 1));
        ci.resize(size_t(nnz));
        v.resize(size_t(nnz));
        c.check(mclsgpu_precond_export(d_h, &nnz, rp.data(), ci.data(), v.data()),
                "mclsgpu_precond_export");
    }

  private:
    std::shared_ptr<Operator> d_op;
    mclsgpu_precond* d_h = nullptr;
};

class Domain {
  public:
    Domain(std::shared_ptr<Operator> op, std::shared_ptr<Precond> left,
           std::shared_ptr<Precond> right, const mclsgpu_mc_params& p)
        : d_op(std::move(op)), d_left(std::move(left)), d_right(std::move(right)) {
        const Context& c = *d_op->context();
        c.check(mclsgpu_domain_build(c.get(), d_op->get(), d_left ? d_left->get() : nullptr,
                                     d_right ? d_right->get() : nullptr, &p, &d_h),
                "mclsgpu_domain_build");
    }
    ~Domain() { mclsgpu_domain_destroy(d_h); }
    Domain(const Domain&) = delete;
    Domain& operator=(const Domain&) = delete;
    mclsgpu_domain* get() const { return d_h; }
    const Context& context() const { return *d_op->context(); }

  private:
    std::shared_ptr<Operator> d_op;
    std::shared_ptr<Precond> d_left, d_right;
    mclsgpu_domain* d_h = nullptr;
};

// Device operators keyed by the host matrix they were uploaded from.  The
// managers reuse an upload while the same matrix object is alive, the
// identity test the reference applies to decide whether to rebuild its
// domain (src/MCLS_MonteCarloSolverManager_impl.hpp:161-178).
class Registry {
  public:
    static Registry& instance() {
        static Registry r;
        return r;
    }
    std::shared_ptr<Operator> findOperator(const std::shared_ptr<const void>& key, int device) {
        std::lock_guard<std::mutex> lock(d_m);
        for (auto& e : d_ops)
            if (!e.key.expired() && e.key.lock() == key && e.device == device)
                if (auto h = e.handle.lock()) return h;
        return nullptr;
    }
    void addOperator(const std::shared_ptr<const void>& key, int device,
                     const std::shared_ptr<Operator>& h) {
        std::lock_guard<std::mutex> lock(d_m);
        prune();
        d_ops.push_back({key, device, h});
    }
    // A preconditioner matrix built on the device by an MCLS GPU
    // preconditioner: the managers use the device copy directly.
    std::shared_ptr<Precond> findPrecond(const std::shared_ptr<const void>& key) {
        std::lock_guard<std::mutex> lock(d_m);
        for (auto& e : d_precs)
            if (!e.key.expired() && e.key.lock() == key)
                if (auto h = e.handle.lock()) return h;
        return nullptr;
    }
    void addPrecond(const std::shared_ptr<const void>& key, const std::shared_ptr<Precond>& h) {
        std::lock_guard<std::mutex> lock(d_m);
        prune();
        d_precs.push_back({key, 0, h});
    }

  private:
    template <class H>
    struct Entry {
        std::weak_ptr<const void> key;
        int device;
        std::weak_ptr<H> handle;
    };
    void prune() {
        auto dead = [](const auto& e) { return e.key.expired() || e.handle.expired(); };
        for (size_t i = d_ops.size(); i-- > 0;)
            if (dead(d_ops[i])) d_ops.erase(d_ops.begin() + long(i));
        for (size_t i = d_precs.size(); i-- > 0;)
            if (dead(d_precs[i])) d_precs.erase(d_precs.begin() + long(i));
    }
    std::mutex d_m;
    std::vector<Entry<Operator>> d_ops;
    std::vector<Entry<Precond>> d_precs;
};

// Device operator for host matrix A (uploaded once while A is alive).
template <class Vector, class Matrix>
std::shared_ptr<Operator> operatorFor(const std::shared_ptr<Context>& ctx,
                                      const Teuchos::RCP<const Matrix>& A) {
    std::shared_ptr<const void> key = A;
    if (auto h = Registry::instance().findOperator(key, ctx->device())) return h;
    std::vector<std::int64_t> rp, ci;
    std::vector<double> v;
    MatrixTraits<Vector, Matrix>::getCsr(*A, rp, ci, v);
    auto h = std::make_shared<Operator>(ctx, MatrixTraits<Vector, Matrix>::getGlobalNumRows(*A),
                                        rp, ci, v);
    Registry::instance().addOperator(key, ctx->device(), h);
    return h;
}

// Device preconditioner for a preconditioner matrix given to LinearProblem:
// the device copy when an MCLS GPU preconditioner built it, else an upload
// of the host matrix.
template <class Vector, class Matrix>
std::shared_ptr<Precond> precondFor(const std::shared_ptr<Operator>& op,
                                    const Teuchos::RCP<const Matrix>& P) {
    if (!Teuchos::nonnull(P)) return nullptr;
    std::shared_ptr<const void> key = P;
    if (auto h = Registry::instance().findPrecond(key)) return h;
    std::vector<std::int64_t> rp, ci;
    std::vector<double> v;
    MatrixTraits<Vector, Matrix>::getCsr(*P, rp, ci, v);
    mclsgpu_precond_params pp{};
    pp.size = sizeof(pp);
    pp.kind = MCLSGPU_PREC_USER_CSR;
    pp.user_n = MatrixTraits<Vector, Matrix>::getGlobalNumRows(*P);
    pp.user_rowptr = rp.data();
    pp.user_colind = ci.data();
    pp.user_values = v.data();
    return std::make_shared<Precond>(op, pp);
}

// ---- ParameterList -> parameter structs ----------------------------------

// Numeric entry read as double whatever numeric type it was set with.
inline bool readNumeric(const Teuchos::ParameterList& pl, const std::string& key, double& out) {
    if (!pl.isParameter(key)) return false;
    if (pl.isType<double>(key)) out = pl.get<double>(key);
    else if (pl.isType<int>(key)) out = pl.get<int>(key);
    else if (pl.isType<float>(key)) out = pl.get<float>(key);
    else if (pl.isType<long>(key)) out = double(pl.get<long>(key));
    else if (pl.isType<long long>(key)) out = double(pl.get<long long>(key));
    else if (pl.isType<unsigned>(key)) out = pl.get<unsigned>(key);
    else throw Assertion("parameter \"" + key + "\" must be numeric");
    return true;
}
inline double numeric(const Teuchos::ParameterList& pl, const std::string& key, double def) {
    double v = def;
    readNumeric(pl, key, v);
    return v;
}
inline std::string text(const Teuchos::ParameterList& pl, const std::string& key,
                        const std::string& def) {
    if (!pl.isParameter(key)) return def;
    if (!pl.isType<std::string>(key)) throw Assertion("parameter \"" + key + "\" must be a string");
    return pl.get<std::string>(key);
}
inline bool flag(const Teuchos::ParameterList& pl, const std::string& key, bool def) {
    if (!pl.isParameter(key)) return def;
    if (pl.isType<bool>(key)) return pl.get<bool>(key);
    return numeric(pl, key, def ? 1.0 : 0.0) != 0.0;
}

// Monte Carlo keys (src/MCLS_MonteCarloSolverManager_impl.hpp:96-110,
// src/MCLS_AlmostOptimalDomain_impl.hpp:88-146,
// src/MCLS_UniformAdjointSource_impl.hpp:82-101,
// src/MCLS_UniformForwardSource_impl.hpp:84-86) plus this library's own:
// "Estimator Type", "Weight Cutoff", "Walk Precision", "Reproducible MC
// Mode", "Random Seed", "Walk Record Format".
inline mclsgpu_mc_params mcParams(const Teuchos::ParameterList& pl, int direction) {
    mclsgpu_mc_params p{};
    p.size = sizeof(p);
    p.direction = direction;
    p.history_length = int(numeric(pl, "History Length", 10.0));
    p.sample_ratio = numeric(pl, "Sample Ratio", 1.0);
    p.neumann_relaxation = numeric(pl, "Neumann Relaxation", 1.0);
    p.composite_threshold = numeric(pl, "Composite Operator Threshold", 0.0);
    p.weight_cutoff = numeric(pl, "Weight Cutoff", 0.0);
    const std::string sampling = text(pl, "Source Sampling Type", "Random");
    if (sampling == "Random") p.source_sampling = MCLSGPU_SOURCE_RANDOM;
    else if (sampling == "Stratified") p.source_sampling = MCLSGPU_SOURCE_STRATIFIED;
    else throw Assertion("Source Sampling Type \"" + sampling + "\" not supported");
    const std::string est = text(pl, "Estimator Type", "Collision");
    if (est == "Collision") p.estimator = MCLSGPU_COLLISION;
    else if (est == "Expected Value") p.estimator = MCLSGPU_EXPECTED_VALUE;
    else throw Assertion("Estimator Type \"" + est + "\" not supported");
    const std::string prec = text(pl, "Walk Precision", "FP64");
    if (prec == "FP64") p.precision = MCLSGPU_FP64;
    else if (prec == "FP32") p.precision = MCLSGPU_FP32;
    else throw Assertion("Walk Precision \"" + prec + "\" not supported");
    p.rng_mode = flag(pl, "Reproducible MC Mode", false) ? MCLSGPU_RNG_REFERENCE
                                                         : MCLSGPU_RNG_COUNTER;
    const std::string fmt = text(pl, "Walk Record Format", "Auto");
    if (fmt == "Auto") p.record_format = MCLSGPU_RECORD_AUTO;
    else if (fmt == "Packed") p.record_format = MCLSGPU_RECORD_PACKED;
    else if (fmt == "Stencil") p.record_format = MCLSGPU_RECORD_STENCIL;
    else if (fmt == "Stencil16") p.record_format = MCLSGPU_RECORD_STENCIL16;
    else throw Assertion("Walk Record Format \"" + fmt + "\" not supported");
    p.seed = std::uint64_t(numeric(pl, "Random Seed", 433494437.0));
    // "Transport Type" (Global | Subdomain), "MC Check Frequency" and "MC
    // Buffer Size" steer inter-rank history transport; one device holds the
    // whole domain, so they are accepted and have no effect.
    const std::string transport = text(pl, "Transport Type", "Global");
    if (transport != "Global" && transport != "Subdomain")
        throw Assertion("Transport Type \"" + transport + "\" not supported");
    return p;
}

// "Fixed Point Type" (src/MCLS_FixedPointIterationFactory_impl.hpp:56-107).
inline int fixedPointType(const Teuchos::ParameterList& pl) {
    const std::string fp = text(pl, "Fixed Point Type", "Richardson");
    if (fp == "Richardson") return MCLSGPU_FIXED_POINT_RICHARDSON;
    if (fp == "Steepest Descent") return MCLSGPU_FIXED_POINT_STEEPEST_DESCENT;
    if (fp == "MINRES") return MCLSGPU_FIXED_POINT_MINRES;
    if (fp == "RNSD") return MCLSGPU_FIXED_POINT_RNSD;
    throw Assertion("Iteration type not supported!");
}

// MCSA keys (src/MCLS_MCSASolverManager_impl.hpp:290-343,
// src/MCLS_RichardsonIteration_impl.hpp:56-99).
inline mclsgpu_mcsa_params mcsaParams(const Teuchos::ParameterList& pl) {
    mclsgpu_mcsa_params p{};
    p.size = sizeof(p);
    p.tolerance = numeric(pl, "Convergence Tolerance", 1.0);
    p.max_iters = int(numeric(pl, "Maximum Iterations", 1000.0));
    p.print_freq = int(numeric(pl, "Iteration Print Frequency", 10.0));
    p.check_freq = int(numeric(pl, "Iteration Check Frequency", 1.0));
    p.smoother_steps = int(numeric(pl, "Smoother Steps", 1.0));
    p.richardson_omega = numeric(pl, "Richardson Relaxation", 1.0);
    // The reference prints its banner and every print_freq-th residual on
    // rank 0; "Print Iterations" = false silences it.
    p.verbose = flag(pl, "Print Iterations", true) ? 1 : 0;
    p.fixed_point_type = fixedPointType(pl);
    return p;
}

// FixedPointSolverManager keys (src/MCLS_FixedPointSolverManager_impl.hpp:
// 214-268): the MCSA keys without the smoother count.
inline mclsgpu_mcsa_params fixedPointParams(const Teuchos::ParameterList& pl) {
    mclsgpu_mcsa_params p = mcsaParams(pl);
    p.smoother_steps = 1;
    return p;
}

// AndersonSolverManager keys (src/MCLS_AndersonSolverManager_impl.hpp:
// 232-247) and NOX's "Anderson Parameters" sublist.
inline mclsgpu_anderson_params andersonParams(const Teuchos::ParameterList& pl) {
    mclsgpu_anderson_params p{};
    p.size = sizeof(p);
    p.tolerance = numeric(pl, "Convergence Tolerance", 1.0e-8);
    p.max_iters = int(numeric(pl, "Maximum Iterations", 1000.0));
    p.smoother_steps = int(numeric(pl, "Smoother Steps", 1.0));
    p.storage_depth = 2;
    p.mixing = 1.0;
    p.start_iteration = 1;
    p.adjust_condition = 0;
    p.drop_tolerance = 1.0e-12;
    if (pl.isSublist("Anderson Parameters")) {
        const Teuchos::ParameterList& a = pl.sublist("Anderson Parameters");
        p.storage_depth = int(numeric(a, "Storage Depth", 2.0));
        p.mixing = numeric(a, "Mixing Parameter", 1.0);
        p.start_iteration = int(numeric(a, "Acceleration Start Iteration", 1.0));
        p.adjust_condition = flag(a, "Adjust Matrix for Condition Number", false) ? 1 : 0;
        p.drop_tolerance = numeric(a, "Condition Number Drop Tolerance", 1.0e-12);
    }
    if (p.storage_depth < 0 || p.storage_depth > 16)
        throw Assertion("Anderson Parameters: Storage Depth must be in 0..16");
    if (p.start_iteration < 1)
        throw Assertion("Anderson Parameters: Acceleration Start Iteration must be >= 1");
    return p;
}

inline bool sameParams(const mclsgpu_mc_params& a, const mclsgpu_mc_params& b) {
    return a.direction == b.direction && a.estimator == b.estimator &&
           a.history_length == b.history_length && a.weight_cutoff == b.weight_cutoff &&
           a.sample_ratio == b.sample_ratio && a.source_sampling == b.source_sampling &&
           a.precision == b.precision && a.neumann_relaxation == b.neumann_relaxation &&
           a.composite_threshold == b.composite_threshold && a.rng_mode == b.rng_mode &&
           a.record_format == b.record_format && a.seed == b.seed;
}

// The device state a manager keeps between solves: operator, preconditioners
// and domain, rebuilt only when the problem's operator or preconditioners or
// the Monte Carlo parameters change.
template <class Vector, class Matrix>
class DeviceProblem {
  public:
    typedef LinearProblem<Vector, Matrix> Problem;

    Domain& prepare(const Problem& problem, const Teuchos::ParameterList& pl, int direction) {
        const int device = int(numeric(pl, "GPU Device", 0.0));
        mclsgpu_mc_params mp = mcParams(pl, direction);
        const bool stale = !d_domain || d_device != device || !sameParams(mp, d_mp) ||
                           d_A.lock() != std::shared_ptr<const void>(problem.getOperator()) ||
                           d_PL.lock() != std::shared_ptr<const void>(problem.getLeftPrec()) ||
                           d_PR.lock() != std::shared_ptr<const void>(problem.getRightPrec()) ||
                           d_generation != problem.generation();
        if (stale) {
            d_domain.reset();
            auto ctx = Context::on(device);
            auto op = operatorFor<Vector, Matrix>(ctx, problem.getOperator());
            auto left = precondFor<Vector, Matrix>(op, problem.getLeftPrec());
            auto right = precondFor<Vector, Matrix>(op, problem.getRightPrec());
            d_domain = std::make_shared<Domain>(op, left, right, mp);
            // "Compute Convergence Criteria" prints the reference's report of
            // the new domain (src/MCLS_AlmostOptimalDomain_impl.hpp:95-113,
            // 530-541).
            if (flag(pl, "Compute Convergence Criteria", false)) {
                mclsgpu_criteria c{};
                c.size = sizeof(c);
                ctx->check(mclsgpu_domain_convergence_criteria(d_domain->get(), 2000, 1e-6, 7, &c),
                           "mclsgpu_domain_convergence_criteria");
                std::printf("\n||H||_inf = %g\nsum|H|_min = %g\n\nH Balance Parameters\n"
                            "min: %g\nmax: %g\nave: %g\n",
                            c.row_sum_max, c.row_sum_min, c.balance_min, c.balance_max,
                            c.balance_ave);
                std::printf("\nNeumann/Ulam Convergence Criteria\n"
                            "---------------------------------\n"
                            "rho(H)  = %g\nrho(H+) = %g\nrho(H*) = %g\n"
                            "---------------------------------\n\n",
                            c.rho_h, c.rho_abs, c.rho_star);
            }
            d_device = device;
            d_mp = mp;
            d_A = problem.getOperator();
            d_PL = problem.getLeftPrec();
            d_PR = problem.getRightPrec();
            d_generation = problem.generation();
        }
        // A kept domain continues its random stream where the last solve
        // left it, as the reference's one generator per rank does.
        return *d_domain;
    }

  private:
    std::shared_ptr<Domain> d_domain;
    int d_device = -1;
    mclsgpu_mc_params d_mp{};
    std::weak_ptr<const void> d_A, d_PL, d_PR;
    std::uint64_t d_generation = 0;
};

}  // namespace gpu
}  // namespace MCLS

#endif  // MCLS_GPUBACKEND_HPP
