// MCLS_SolverManager.hpp -- the solver manager interface
// (src/MCLS_SolverManager.hpp:60-112).
#ifndef MCLS_SOLVERMANAGER_HPP
#define MCLS_SOLVERMANAGER_HPP

#include "MCLS_GpuTeuchos.hpp"
#include "MCLS_LinearProblem.hpp"

namespace MCLS {

template <class Vector, class Matrix>
class SolverManager : public virtual Teuchos::Describable {
  public:
    typedef Vector vector_type;
    typedef VectorTraits<Vector> VT;
    typedef typename VT::scalar_type Scalar;
    typedef Matrix matrix_type;

    virtual ~SolverManager() = default;
    virtual const LinearProblem<Vector, Matrix>& getProblem() const = 0;
    virtual Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const = 0;
    virtual Teuchos::RCP<const Teuchos::ParameterList> getCurrentParameters() const = 0;
    virtual typename Teuchos::ScalarTraits<Scalar>::magnitudeType achievedTol() const = 0;
    virtual int getNumIters() const = 0;
    virtual void setProblem(const Teuchos::RCP<LinearProblem<Vector, Matrix>>& problem) = 0;
    virtual void setParameters(const Teuchos::RCP<Teuchos::ParameterList>& params) = 0;
    virtual bool solve() = 0;
    virtual bool getConvergedStatus() const = 0;
};

}  // namespace MCLS

#endif  // MCLS_SOLVERMANAGER_HPP
