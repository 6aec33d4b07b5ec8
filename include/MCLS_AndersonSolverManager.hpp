// MCLS_AndersonSolverManager.hpp -- "Adjoint Anderson" / "Forward Anderson"
// on the GPU.
//
// Same constructors and SolverManager methods as the reference manager
// (src/MCLS_AndersonSolverManager.hpp:70-160,
// src/MCLS_AndersonSolverManager_impl.hpp:65-284), which hands the
// MCSAModelEvaluator map to NOX's "Anderson Accelerated Fixed-Point"
// solver.  solve() runs the whole accelerated loop on the device
// (mclsgpu_anderson_solve): smoothing, the Monte Carlo correction, the
// least-squares update over the last "Storage Depth" differences and the
// status test |PL (b - A x)|_2 < tol * |b|_2.  The "Anderson Parameters"
// sublist keys are NOX's.  The left preconditioner is applied, the right one
// is not (as in the model evaluator).
#ifndef MCLS_ANDERSONSOLVERMANAGER_HPP
#define MCLS_ANDERSONSOLVERMANAGER_HPP

#include <type_traits>

#include "MCLS_GpuBackend.hpp"
#include "MCLS_MonteCarloSolverManager.hpp"
#include "MCLS_MultiSetLinearProblem.hpp"
#include "MCLS_SolverManager.hpp"

namespace MCLS {

template <class Vector, class Matrix, class MonteCarloTag = AdjointTag, class RNG = Xorshift<>>
class AndersonSolverManager : public SolverManager<Vector, Matrix> {
  public:
    typedef VectorTraits<Vector> VT;
    typedef typename VT::scalar_type Scalar;
    typedef LinearProblem<Vector, Matrix> LinearProblemType;
    typedef MultiSetLinearProblem<Vector, Matrix> MultiSetType;

    // Parameter constructor: setProblem() must be called before solve().
    explicit AndersonSolverManager(const Teuchos::RCP<Teuchos::ParameterList>& plist)
        : d_plist(plist) {
        if (!Teuchos::nonnull(plist)) throw Assertion("AndersonSolverManager: null parameters");
        d_plist->set<std::string>("Nonlinear Solver", "Anderson Accelerated Fixed-Point");
        gpu::andersonParams(*plist);
    }
    AndersonSolverManager(const Teuchos::RCP<MultiSetType>& multiset_problem,
                          const Teuchos::RCP<Teuchos::ParameterList>& plist)
        : AndersonSolverManager(plist) {
        setMultiSetProblem(multiset_problem);
    }

    const LinearProblem<Vector, Matrix>& getProblem() const override { return *d_problem; }
    std::string description() const override { return std::string(std::is_same<MonteCarloTag, ForwardTag>::value ? "Forward" : "Adjoint") + " Anderson (GPU)"; }

    // The Monte Carlo keys and the loop's own (the reference returns an empty
    // list here, :113-121).
    Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const override {
        auto pl = Teuchos::parameterList();
        pl->setParameters(
            *MonteCarloSolverManager<Vector, Matrix, MonteCarloTag, RNG>(Teuchos::parameterList())
                 .getValidParameters());
        pl->set<double>("Convergence Tolerance", 1.0e-8);
        pl->set<int>("Maximum Iterations", 1000);
        pl->set<int>("Smoother Steps", 1);
        auto& a = pl->sublist("Anderson Parameters");
        a.set<int>("Storage Depth", 2);
        a.set<double>("Mixing Parameter", 1.0);
        a.set<int>("Acceleration Start Iteration", 1);
        a.set<bool>("Adjust Matrix for Condition Number", false);
        a.set<double>("Condition Number Drop Tolerance", 1.0e-12);
        return pl;
    }
    Teuchos::RCP<const Teuchos::ParameterList> getCurrentParameters() const override {
        return d_plist;
    }

    // |PL (b - A x)|_2 / |b|_2 at the end of the last solve (the reference
    // returns 0 here, :128-135).
    typename Teuchos::ScalarTraits<Scalar>::magnitudeType achievedTol() const override {
        return d_stats.achieved_tol;
    }
    // Steps taken (NOX's iteration count).
    int getNumIters() const override { return d_stats.iterations; }

    void setMultiSetProblem(const Teuchos::RCP<MultiSetType>& multiset_problem) {
        if (!Teuchos::nonnull(multiset_problem))
            throw Assertion("AndersonSolverManager: null problem");
        if (multiset_problem->getNumSets() != 1 && !multiset_problem->hasSetReducer())
            throw Assertion("AndersonSolverManager: a problem of several sets needs a set "
                            "reducer (MultiSetLinearProblem::setSetReducer)");
        d_multiset = multiset_problem;
        setProblem(multiset_problem->getProblem());
    }
    void setProblem(const Teuchos::RCP<LinearProblemType>& problem) override {
        if (!Teuchos::nonnull(problem)) throw Assertion("AndersonSolverManager: null problem");
        d_problem = problem;
    }
    void setParameters(const Teuchos::RCP<Teuchos::ParameterList>& params) override {
        if (!Teuchos::nonnull(params)) throw Assertion("AndersonSolverManager: null parameters");
        gpu::andersonParams(*params);
        d_plist = params;
        d_plist->set<std::string>("Nonlinear Solver", "Anderson Accelerated Fixed-Point");
    }

    bool solve() override {
        if (!Teuchos::nonnull(d_problem)) throw Assertion("AndersonSolverManager: no problem set");
        const mclsgpu_anderson_params ap = gpu::andersonParams(*d_plist);
        // The model evaluator's residual problem carries A and the left
        // preconditioner only (src/MCLS_MCSAModelEvaluator_impl.hpp:358-380).
        LinearProblemType left_only(d_problem->getOperator(), d_problem->getLHS(),
                                    d_problem->getRHS());
        if (Teuchos::nonnull(d_problem->getLeftPrec()))
            left_only.setLeftPrec(d_problem->getLeftPrec());
        gpu::Domain& dom = d_device.prepare(left_only, *d_plist, direction());
        d_stats = mclsgpu_stats{};
        d_stats.size = sizeof(d_stats);
        const int sets = Teuchos::nonnull(d_multiset) ? d_multiset->getNumSets() : 1;
        if (d_plist->isParameter("Number of Sets") &&
            int(gpu::numeric(*d_plist, "Number of Sets", 1.0)) != sets)
            throw Assertion("AndersonSolverManager: \"Number of Sets\" differs from the "
                            "problem's");
        if (sets > 1) {
            dom.context().check(
                mclsgpu_anderson_solve_sets(dom.get(), &d_multiset->setReducer(),
                                            VT::view(*d_problem->getRHS()),
                                            VT::viewNonConst(*d_problem->getLHS()), &ap, &d_stats),
                "mclsgpu_anderson_solve_sets");
            return d_stats.converged != 0;
        }
        dom.context().check(mclsgpu_anderson_solve(dom.get(), VT::view(*d_problem->getRHS()),
                                                   VT::viewNonConst(*d_problem->getLHS()), &ap,
                                                   &d_stats),
                            "mclsgpu_anderson_solve");
        return d_stats.converged != 0;
    }
    bool getConvergedStatus() const override { return d_stats.converged != 0; }

    const mclsgpu_stats& lastStats() const { return d_stats; }

  private:
    static int direction() {
        return std::is_same<MonteCarloTag, ForwardTag>::value ? MCLSGPU_FORWARD : MCLSGPU_ADJOINT;
    }

    Teuchos::RCP<MultiSetType> d_multiset;
    Teuchos::RCP<LinearProblemType> d_problem;
    Teuchos::RCP<Teuchos::ParameterList> d_plist;
    gpu::DeviceProblem<Vector, Matrix> d_device;
    mclsgpu_stats d_stats{};
};

}  // namespace MCLS

#endif  // MCLS_ANDERSONSOLVERMANAGER_HPP
