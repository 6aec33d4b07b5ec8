// MCLS_Preconditioner.hpp -- preconditioner interface of the MCLS managers
// (src/MCLS_Preconditioner.hpp:75-100).  Device-built implementations are in
// MCLS_GpuPreconditioners.hpp.
#ifndef MCLS_PRECONDITIONER_HPP
#define MCLS_PRECONDITIONER_HPP

#include "MCLS_GpuTeuchos.hpp"

namespace MCLS {

template <class Matrix>
class Preconditioner : public virtual Teuchos::Describable {
  public:
    typedef Matrix matrix_type;
    virtual ~Preconditioner() = default;
    virtual Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const = 0;
    virtual Teuchos::RCP<const Teuchos::ParameterList> getCurrentParameters() const = 0;
    virtual void setParameters(const Teuchos::RCP<Teuchos::ParameterList>& params) = 0;
    virtual void setOperator(const Teuchos::RCP<const Matrix>& A) = 0;
    virtual const Matrix& getOperator() const = 0;
    virtual void buildPreconditioner() = 0;
    virtual Teuchos::RCP<const Matrix> getLeftPreconditioner() const = 0;
    virtual Teuchos::RCP<const Matrix> getRightPreconditioner() const = 0;
};

}  // namespace MCLS

#endif  // MCLS_PRECONDITIONER_HPP
