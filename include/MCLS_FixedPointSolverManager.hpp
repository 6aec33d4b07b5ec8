// MCLS_FixedPointSolverManager.hpp -- "Fixed Point" on the GPU.
//
// Same constructors and SolverManager methods as the reference manager
// (src/MCLS_FixedPointSolverManager.hpp:68-140,
// src/MCLS_FixedPointSolverManager_impl.hpp:56-321).  solve() runs the
// "Fixed Point Type" iteration (Richardson, Steepest Descent, MINRES or RNSD)
// on the device until |rp|_inf <= tol * |PL b|_inf and updates x in place.
#ifndef MCLS_FIXEDPOINTSOLVERMANAGER_HPP
#define MCLS_FIXEDPOINTSOLVERMANAGER_HPP

#include "MCLS_GpuBackend.hpp"
#include "MCLS_SolverManager.hpp"

namespace MCLS {

template <class Vector, class Matrix>
class FixedPointSolverManager : public SolverManager<Vector, Matrix> {
  public:
    typedef VectorTraits<Vector> VT;
    typedef typename VT::scalar_type Scalar;
    typedef LinearProblem<Vector, Matrix> LinearProblemType;

    // Parameter constructor: setProblem() must be called before solve().
    explicit FixedPointSolverManager(const Teuchos::RCP<Teuchos::ParameterList>& plist)
        : d_plist(plist) {
        if (!Teuchos::nonnull(plist)) throw Assertion("FixedPointSolverManager: null parameters");
        gpu::fixedPointParams(*plist);  // "Iteration type not supported!" early
    }
    FixedPointSolverManager(const Teuchos::RCP<LinearProblemType>& problem,
                            const Teuchos::RCP<Teuchos::ParameterList>& plist)
        : FixedPointSolverManager(plist) {
        setProblem(problem);
    }

    const LinearProblem<Vector, Matrix>& getProblem() const override { return *d_problem; }
    std::string description() const override { return std::string("Fixed Point (GPU)"); }

    // src/MCLS_FixedPointSolverManager_impl.hpp:106-126 (with the
    // Richardson iteration's "Richardson Relaxation").
    Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const override {
        auto pl = Teuchos::parameterList();
        pl->set<double>("Richardson Relaxation", 1.0);
        pl->set<double>("Convergence Tolerance", 1.0);
        pl->set<int>("Maximum Iterations", 1000);
        pl->set<int>("Iteration Print Frequency", 10);
        pl->set<int>("Iteration Check Frequency", 1);
        pl->set<std::string>("Fixed Point Type", "Richardson");
        pl->set<bool>("Print Iterations", true);
        return pl;
    }
    Teuchos::RCP<const Teuchos::ParameterList> getCurrentParameters() const override {
        return d_plist;
    }

    // |rp|_inf / |PL b|_inf at the end of the last solve (:133-160).
    typename Teuchos::ScalarTraits<Scalar>::magnitudeType achievedTol() const override {
        return d_stats.achieved_tol;
    }
    int getNumIters() const override { return d_stats.iterations; }

    void setProblem(const Teuchos::RCP<LinearProblemType>& problem) override {
        if (!Teuchos::nonnull(problem)) throw Assertion("FixedPointSolverManager: null problem");
        d_problem = problem;
    }
    void setParameters(const Teuchos::RCP<Teuchos::ParameterList>& params) override {
        if (!Teuchos::nonnull(params)) throw Assertion("FixedPointSolverManager: null parameters");
        gpu::fixedPointParams(*params);
        d_plist = params;
    }

    bool solve() override {
        if (!Teuchos::nonnull(d_problem)) throw Assertion("FixedPointSolverManager: no problem set");
        const mclsgpu_mcsa_params p = gpu::fixedPointParams(*d_plist);
        const int device = int(gpu::numeric(*d_plist, "GPU Device", 0.0));
        auto ctx = gpu::Context::on(device);
        auto op = gpu::operatorFor<Vector, Matrix>(ctx, d_problem->getOperator());
        auto left = gpu::precondFor<Vector, Matrix>(op, d_problem->getLeftPrec());
        auto right = gpu::precondFor<Vector, Matrix>(op, d_problem->getRightPrec());
        d_stats = mclsgpu_stats{};
        d_stats.size = sizeof(d_stats);
        ctx->check(mclsgpu_fixed_point_solve(ctx->get(), op->get(), left ? left->get() : nullptr,
                                             right ? right->get() : nullptr,
                                             VT::view(*d_problem->getRHS()),
                                             VT::viewNonConst(*d_problem->getLHS()), &p,
                                             &d_stats),
                   "mclsgpu_fixed_point_solve");
        return d_stats.converged != 0;
    }
    bool getConvergedStatus() const override { return d_stats.converged != 0; }

    const mclsgpu_stats& lastStats() const { return d_stats; }

  private:
    Teuchos::RCP<LinearProblemType> d_problem;
    Teuchos::RCP<Teuchos::ParameterList> d_plist;
    mclsgpu_stats d_stats{};
};

}  // namespace MCLS

#endif  // MCLS_FIXEDPOINTSOLVERMANAGER_HPP
