// MCLS_MonteCarloSolverManager.hpp -- "Adjoint MC" / "Forward MC" on the GPU.
//
// Same constructors and SolverManager methods as the reference manager
// (src/MCLS_MonteCarloSolverManager.hpp:95-136,
// src/MCLS_MonteCarloSolverManager_impl.hpp:96-235).  solve() builds the
// device domain when the problem's operator or preconditioners change
// (kept between solves otherwise), samples the source from the right-hand
// side and transports the histories on the GPU; x receives the Monte Carlo
// estimate, right-preconditioner recovery included unless the manager is an
// internal solver.
#ifndef MCLS_MONTECARLOSOLVERMANAGER_HPP
#define MCLS_MONTECARLOSOLVERMANAGER_HPP

#include <algorithm>
#include <cmath>
#include <type_traits>

#include "MCLS_GpuBackend.hpp"
#include "MCLS_SolverManager.hpp"

namespace MCLS {

template <class Vector, class Matrix, class MonteCarloTag = AdjointTag, class RNG = Xorshift<>>
class MonteCarloSolverManager : public SolverManager<Vector, Matrix> {
  public:
    typedef SolverManager<Vector, Matrix> Base;
    typedef VectorTraits<Vector> VT;
    typedef typename VT::scalar_type Scalar;
    typedef LinearProblem<Vector, Matrix> LinearProblemType;
    typedef MonteCarloTag Tag;
    typedef RNG rng_type;

    explicit MonteCarloSolverManager(const Teuchos::RCP<Teuchos::ParameterList>& plist,
                                     int global_rank = 0, bool internal_solver = false)
        : d_plist(plist), d_rank(global_rank), d_internal(internal_solver) {
        if (!Teuchos::nonnull(plist)) throw Assertion("MonteCarloSolverManager: null parameters");
    }
    MonteCarloSolverManager(const Teuchos::RCP<LinearProblemType>& problem,
                            const Teuchos::RCP<Teuchos::ParameterList>& plist,
                            int global_rank = 0, bool internal_solver = false)
        : MonteCarloSolverManager(plist, global_rank, internal_solver) {
        setProblem(problem);
    }

    const LinearProblem<Vector, Matrix>& getProblem() const override { return *d_problem; }
    std::string description() const override { return std::string(std::is_same<MonteCarloTag, ForwardTag>::value ? "Forward" : "Adjoint") + " MC (GPU)"; }

    // Defaults (src/MCLS_MonteCarloSolverManager_impl.hpp:99-110) and this
    // library's own keys.
    Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const override {
        auto pl = Teuchos::parameterList();
        pl->set<double>("Sample Ratio", 1.0);
        pl->set<int>("History Length", 10);
        pl->set<int>("MC Check Frequency", 1000);
        pl->set<int>("MC Buffer Size", 1000);
        pl->set<double>("Neumann Relaxation", 1.0);
        pl->set<double>("Composite Operator Threshold", 0.0);
        pl->set<std::string>("Source Sampling Type", "Random");
        pl->set<std::string>("Transport Type", "Global");
        pl->set<std::string>("Estimator Type", "Collision");
        pl->set<double>("Weight Cutoff", 0.0);
        pl->set<std::string>("Walk Precision", "FP64");
        pl->set<bool>("Reproducible MC Mode", false);
        pl->set<int>("Random Seed", 433494437);
        pl->set<std::string>("Walk Record Format", "Auto");
        pl->set<int>("GPU Device", 0);
        return pl;
    }
    Teuchos::RCP<const Teuchos::ParameterList> getCurrentParameters() const override {
        return d_plist;
    }

    // |b - A x|_inf / |b|_inf after the solve, the reference's measure of the
    // stochastic error (src/MCLS_MonteCarloSolverManager_impl.hpp:118-131).
    typename Teuchos::ScalarTraits<Scalar>::magnitudeType achievedTol() const override {
        d_problem->updateResidual();
        const auto& r = *d_problem->getResidual();
        const auto& b = *d_problem->getRHS();
        double rn = 0.0, bn = 0.0;
        for (std::int64_t i = 0; i < VT::getGlobalLength(r); ++i) {
            rn = std::max(rn, std::fabs(VT::view(r)[i]));
            bn = std::max(bn, std::fabs(VT::view(b)[i]));
        }
        return rn / bn;
    }
    int getNumIters() const override { return 0; }

    void setProblem(const Teuchos::RCP<LinearProblemType>& problem) override {
        if (!Teuchos::nonnull(problem)) throw Assertion("MonteCarloSolverManager: null problem");
        d_problem = problem;
    }
    void setParameters(const Teuchos::RCP<Teuchos::ParameterList>& params) override {
        if (!Teuchos::nonnull(params)) throw Assertion("MonteCarloSolverManager: null parameters");
        d_plist = params;
    }

    bool solve() override {
        if (!Teuchos::nonnull(d_problem)) throw Assertion("MonteCarloSolverManager: no problem set");
        gpu::Domain& dom = d_device.prepare(*d_problem, *d_plist, direction());
        Vector& x = *d_problem->getLHS();
        d_stats = mclsgpu_stats{};
        d_stats.size = sizeof(d_stats);
        dom.context().check(mclsgpu_mc_solve(dom.get(), VT::view(*d_problem->getRHS()),
                                             VT::viewNonConst(x), d_internal ? 1 : 0, &d_stats),
                            "mclsgpu_mc_solve");
        return true;  // a direct solve (src/MCLS_MonteCarloSolverManager_impl.hpp:231-234)
    }
    bool getConvergedStatus() const override { return true; }

    // Statistics of the last solve (histories, walk steps, device time).
    const mclsgpu_stats& lastStats() const { return d_stats; }
    int globalRank() const { return d_rank; }

  private:
    static int direction() {
        return std::is_same<MonteCarloTag, ForwardTag>::value ? MCLSGPU_FORWARD : MCLSGPU_ADJOINT;
    }

    Teuchos::RCP<LinearProblemType> d_problem;
    Teuchos::RCP<Teuchos::ParameterList> d_plist;
    int d_rank;
    bool d_internal;
    gpu::DeviceProblem<Vector, Matrix> d_device;
    mclsgpu_stats d_stats{};
};

}  // namespace MCLS

#endif  // MCLS_MONTECARLOSOLVERMANAGER_HPP
