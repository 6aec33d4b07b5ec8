// MCLS_SolverFactory.hpp -- name -> solver manager
// (src/MCLS_SolverFactory.hpp:61-95, src/MCLS_SolverFactory_impl.hpp:57-140).
//
// Every name the reference knows creates the GPU manager: "Adjoint MC",
// "Forward MC", "Adjoint MCSA", "Forward MCSA", "Adjoint Anderson",
// "Forward Anderson" and "Fixed Point".  Unknown names throw Assertion.
#ifndef MCLS_SOLVERFACTORY_HPP
#define MCLS_SOLVERFACTORY_HPP

#include <map>
#include <string>

#include "MCLS_AndersonSolverManager.hpp"
#include "MCLS_FixedPointSolverManager.hpp"
#include "MCLS_MCSASolverManager.hpp"
#include "MCLS_MonteCarloSolverManager.hpp"

namespace MCLS {

template <class Vector, class Matrix>
class SolverFactory {
  public:
    typedef SolverManager<Vector, Matrix> Solver;

    SolverFactory() = default;

    Teuchos::RCP<Solver> create(const std::string& solver_name,
                                const Teuchos::RCP<Teuchos::ParameterList>& solver_parameters) {
        if (!Teuchos::nonnull(solver_parameters)) throw Assertion("SolverFactory: null parameters");
        if (solver_name == "Adjoint MC")
            return Teuchos::rcp(
                new MonteCarloSolverManager<Vector, Matrix, AdjointTag>(solver_parameters));
        if (solver_name == "Forward MC")
            return Teuchos::rcp(
                new MonteCarloSolverManager<Vector, Matrix, ForwardTag>(solver_parameters));
        if (solver_name == "Adjoint MCSA")
            return Teuchos::rcp(new MCSASolverManager<Vector, Matrix, AdjointTag>(solver_parameters));
        if (solver_name == "Forward MCSA")
            return Teuchos::rcp(new MCSASolverManager<Vector, Matrix, ForwardTag>(solver_parameters));
        if (solver_name == "Fixed Point")
            return Teuchos::rcp(new FixedPointSolverManager<Vector, Matrix>(solver_parameters));
        if (solver_name == "Adjoint Anderson")
            return Teuchos::rcp(
                new AndersonSolverManager<Vector, Matrix, AdjointTag>(solver_parameters));
        if (solver_name == "Forward Anderson")
            return Teuchos::rcp(
                new AndersonSolverManager<Vector, Matrix, ForwardTag>(solver_parameters));
        throw Assertion("Solver type not supported!");
    }
};

}  // namespace MCLS

#endif  // MCLS_SOLVERFACTORY_HPP
