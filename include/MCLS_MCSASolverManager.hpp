// MCLS_MCSASolverManager.hpp -- "Adjoint MCSA" / "Forward MCSA" on the GPU.
//
// Same constructors and SolverManager methods as the reference manager
// (src/MCLS_MCSASolverManager.hpp:85-135,
// src/MCLS_MCSASolverManager_impl.hpp:56-432).  solve() runs the whole MCSA
// loop on the device -- smoothing ("Fixed Point Type": Richardson, Steepest
// Descent, MINRES or RNSD), preconditioned residual, the
// Monte Carlo correction and the convergence test
// |rp|_2 <= tol * |PL b|_2 -- and updates x in place.
#ifndef MCLS_MCSASOLVERMANAGER_HPP
#define MCLS_MCSASOLVERMANAGER_HPP

#include <type_traits>

#include "MCLS_GpuBackend.hpp"
#include "MCLS_MonteCarloSolverManager.hpp"
#include "MCLS_MultiSetLinearProblem.hpp"
#include "MCLS_SolverManager.hpp"

namespace MCLS {

template <class Vector, class Matrix, class MonteCarloTag = AdjointTag, class RNG = Xorshift<>>
class MCSASolverManager : public SolverManager<Vector, Matrix> {
  public:
    typedef VectorTraits<Vector> VT;
    typedef typename VT::scalar_type Scalar;
    typedef LinearProblem<Vector, Matrix> LinearProblemType;
    typedef MultiSetLinearProblem<Vector, Matrix> MultiSetType;

    // Parameter constructor: setProblem() must be called before solve().
    explicit MCSASolverManager(const Teuchos::RCP<Teuchos::ParameterList>& plist)
        : d_plist(plist) {
        if (!Teuchos::nonnull(plist)) throw Assertion("MCSASolverManager: null parameters");
        gpu::mcsaParams(*plist);  // rejects an unsupported "Fixed Point Type" early
    }
    MCSASolverManager(const Teuchos::RCP<MultiSetType>& multiset_problem,
                      const Teuchos::RCP<Teuchos::ParameterList>& plist)
        : MCSASolverManager(plist) {
        setMultiSetProblem(multiset_problem);
    }

    const LinearProblem<Vector, Matrix>& getProblem() const override { return *d_problem; }
    std::string description() const override { return std::string(std::is_same<MonteCarloTag, ForwardTag>::value ? "Forward" : "Adjoint") + " MCSA (GPU)"; }

    // Monte Carlo keys plus the MCSA defaults
    // (src/MCLS_MCSASolverManager_impl.hpp:116-133).
    Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const override {
        auto pl = Teuchos::parameterList();
        pl->setParameters(
            *MonteCarloSolverManager<Vector, Matrix, MonteCarloTag, RNG>(Teuchos::parameterList())
                 .getValidParameters());
        pl->set<double>("Convergence Tolerance", 1.0);
        pl->set<int>("Maximum Iterations", 1000);
        pl->set<int>("Iteration Print Frequency", 10);
        pl->set<int>("Iteration Check Frequency", 1);
        pl->set<std::string>("Fixed Point Type", "Richardson");
        pl->set<double>("Richardson Relaxation", 1.0);
        pl->set<int>("Smoother Steps", 1);
        pl->set<bool>("Print Iterations", true);
        pl->set<int>("Number of Sets", 1);
        return pl;
    }
    Teuchos::RCP<const Teuchos::ParameterList> getCurrentParameters() const override {
        return d_plist;
    }

    // |rp|_2 / |PL b|_2 at the end of the last solve
    // (src/MCLS_MCSASolverManager_impl.hpp:142-173).
    typename Teuchos::ScalarTraits<Scalar>::magnitudeType achievedTol() const override {
        return d_stats.achieved_tol;
    }
    int getNumIters() const override { return d_stats.iterations; }

    // Several sets need the problem's set reducer, which sums the sets'
    // corrections each iteration (MultiSetLinearProblem::setSetReducer).
    void setMultiSetProblem(const Teuchos::RCP<MultiSetType>& multiset_problem) {
        if (!Teuchos::nonnull(multiset_problem)) throw Assertion("MCSASolverManager: null problem");
        if (multiset_problem->getNumSets() != 1 && !multiset_problem->hasSetReducer())
            throw Assertion("MCSASolverManager: a problem of several sets needs a set reducer "
                            "(MultiSetLinearProblem::setSetReducer)");
        d_multiset = multiset_problem;
        setProblem(multiset_problem->getProblem());
    }
    void setProblem(const Teuchos::RCP<LinearProblemType>& problem) override {
        if (!Teuchos::nonnull(problem)) throw Assertion("MCSASolverManager: null problem");
        d_problem = problem;
    }
    void setParameters(const Teuchos::RCP<Teuchos::ParameterList>& params) override {
        if (!Teuchos::nonnull(params)) throw Assertion("MCSASolverManager: null parameters");
        gpu::mcsaParams(*params);
        d_plist = params;
    }

    bool solve() override {
        if (!Teuchos::nonnull(d_problem)) throw Assertion("MCSASolverManager: no problem set");
        const mclsgpu_mcsa_params mp = gpu::mcsaParams(*d_plist);
        gpu::Domain& dom = d_device.prepare(*d_problem, *d_plist, direction());
        d_stats = mclsgpu_stats{};
        d_stats.size = sizeof(d_stats);
        const int sets = Teuchos::nonnull(d_multiset) ? d_multiset->getNumSets() : 1;
        // "Number of Sets", when given, must agree with the problem's layout.
        if (d_plist->isParameter("Number of Sets") &&
            int(gpu::numeric(*d_plist, "Number of Sets", 1.0)) != sets)
            throw Assertion("MCSASolverManager: \"Number of Sets\" differs from the problem's");
        if (sets > 1) {
            int32_t on_device = 0;
            dom.context().check(
                mclsgpu_mcsa_solve_sets(dom.get(), &d_multiset->setReducer(),
                                        VT::view(*d_problem->getRHS()),
                                        VT::viewNonConst(*d_problem->getLHS()), &mp, &d_stats,
                                        &on_device),
                "mclsgpu_mcsa_solve_sets");
            return d_stats.converged != 0;
        }
        dom.context().check(mclsgpu_mcsa_solve(dom.get(), VT::view(*d_problem->getRHS()),
                                               VT::viewNonConst(*d_problem->getLHS()), &mp,
                                               &d_stats),
                            "mclsgpu_mcsa_solve");
        return d_stats.converged != 0;
    }
    bool getConvergedStatus() const override { return d_stats.converged != 0; }

    // Statistics of the last solve (iterations, histories, device time).
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

#endif  // MCLS_MCSASOLVERMANAGER_HPP
