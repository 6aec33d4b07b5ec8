// Stand-in for the part of Thyra's interface (and the Teuchos pieces it
// brings) that include/Thyra_MCLSGpuLinearOpWithSolveFactory.hpp uses:
// the operator / solve / factory base classes with Thyra's member names,
// the solve vocabulary, Teuchos::Ptr and Teuchos::dyn_cast.  It lets the
// Thyra layer be compiled and run without Trilinos; it is not Thyra.
#ifndef STANDIN_THYRA_LOWSFB_HPP
#define STANDIN_THYRA_LOWSFB_HPP

#include <stdexcept>
#include <string>
#include <typeinfo>

#include "MCLS_GpuTeuchos.hpp"

namespace Teuchos {

template <class T>
class Ptr {
  public:
    Ptr(std::nullptr_t = nullptr) {}
    explicit Ptr(T* p) : d_p(p) {}
    template <class U>
    Ptr(const Ptr<U>& o) : d_p(o.get()) {}
    T* get() const { return d_p; }
    T* getRawPtr() const { return d_p; }
    T* operator->() const { return d_p; }
    T& operator*() const { return *d_p; }
    bool is_null() const { return d_p == nullptr; }

  private:
    T* d_p = nullptr;
};
template <class T>
Ptr<T> ptr(T* p) { return Ptr<T>(p); }
template <class T>
Ptr<T> outArg(T& r) { return Ptr<T>(&r); }
template <class T>
bool nonnull(const Ptr<T>& p) { return !p.is_null(); }
template <class T>
bool is_null(const Ptr<T>& p) { return p.is_null(); }
template <class T>
RCP<T> rcpFromPtr(const Ptr<T>& p) { return rcp(p.get(), false); }

template <class T, class U>
T& dyn_cast(U& from) {
    T* p = dynamic_cast<T*>(&from);
    if (!p) throw std::bad_cast();
    return *p;
}

class ParameterListAcceptor {
  public:
    virtual ~ParameterListAcceptor() = default;
    virtual void setParameterList(const RCP<ParameterList>& paramList) = 0;
    virtual RCP<ParameterList> getNonconstParameterList() = 0;
    virtual RCP<ParameterList> unsetParameterList() = 0;
    virtual RCP<const ParameterList> getParameterList() const { return null; }
    virtual RCP<const ParameterList> getValidParameters() const { return null; }
};

}  // namespace Teuchos

namespace Thyra {

using Teuchos::Ptr;
using Teuchos::RCP;

enum EOpTransp { NOTRANS, CONJ, TRANS, CONJTRANS };
enum ESupportSolveUse {
    SUPPORT_SOLVE_UNSPECIFIED,
    SUPPORT_SOLVE_FORWARD_ONLY,
    SUPPORT_SOLVE_TRANSPOSE_ONLY,
    SUPPORT_SOLVE_FORWARD_AND_TRANSPOSE
};
enum EPreconditionerInputType {
    PRECONDITIONER_INPUT_TYPE_AS_OPERATOR,
    PRECONDITIONER_INPUT_TYPE_AS_MATRIX
};
enum ESolveMeasureNormType {
    SOLVE_MEASURE_ONE,
    SOLVE_MEASURE_NORM_RESIDUAL,
    SOLVE_MEASURE_NORM_SOLUTION,
    SOLVE_MEASURE_NORM_INIT_RESIDUAL,
    SOLVE_MEASURE_NORM_RHS
};
enum ESolveStatus { SOLVE_STATUS_CONVERGED, SOLVE_STATUS_UNCONVERGED, SOLVE_STATUS_UNKNOWN };

struct SolveMeasureType {
    ESolveMeasureNormType numerator = SOLVE_MEASURE_ONE;
    ESolveMeasureNormType denominator = SOLVE_MEASURE_ONE;
    SolveMeasureType() = default;
    SolveMeasureType(ESolveMeasureNormType n, ESolveMeasureNormType d)
        : numerator(n), denominator(d) {}
    bool useDefault() const {
        return numerator == SOLVE_MEASURE_ONE && denominator == SOLVE_MEASURE_ONE;
    }
};

template <class Scalar>
struct SolveCriteria {
    static Scalar unspecifiedTolerance() { return Scalar(-1); }
    SolveMeasureType solveMeasureType;
    Scalar requestedTol = unspecifiedTolerance();
    RCP<Teuchos::ParameterList> extraParameters;
    SolveCriteria() = default;
    SolveCriteria(SolveMeasureType m, Scalar tol,
                  const RCP<Teuchos::ParameterList>& extra = Teuchos::null)
        : solveMeasureType(m), requestedTol(tol), extraParameters(extra) {}
};

template <class Scalar>
struct SolveStatus {
    ESolveStatus solveStatus = SOLVE_STATUS_UNKNOWN;
    Scalar achievedTol = Scalar(-1);
    std::string message;
    RCP<Teuchos::ParameterList> extraParameters;
};

template <class Scalar>
class VectorSpaceBase {
  public:
    virtual ~VectorSpaceBase() = default;
    virtual long dim() const = 0;
};

template <class Scalar>
class MultiVectorBase {
  public:
    virtual ~MultiVectorBase() = default;
};

template <class Scalar>
class LinearOpBase : public virtual Teuchos::Describable {
  public:
    virtual RCP<const VectorSpaceBase<Scalar>> range() const = 0;
    virtual RCP<const VectorSpaceBase<Scalar>> domain() const = 0;
    bool opSupported(EOpTransp t) const { return opSupportedImpl(t); }
    void apply(EOpTransp t, const MultiVectorBase<Scalar>& X, const Ptr<MultiVectorBase<Scalar>>& Y,
               Scalar alpha, Scalar beta) const {
        applyImpl(t, X, Y, alpha, beta);
    }

  protected:
    virtual bool opSupportedImpl(EOpTransp t) const = 0;
    virtual void applyImpl(EOpTransp t, const MultiVectorBase<Scalar>& X,
                           const Ptr<MultiVectorBase<Scalar>>& Y, Scalar alpha,
                           Scalar beta) const = 0;
};

template <class Scalar>
class LinearOpWithSolveBase : public virtual LinearOpBase<Scalar> {
  public:
    bool solveSupports(EOpTransp t) const { return solveSupportsImpl(t); }
    bool solveSupports(EOpTransp t, const Ptr<const SolveCriteria<Scalar>> c) const {
        return solveSupportsNewImpl(t, c);
    }
    bool solveSupportsSolveMeasureType(EOpTransp t, const SolveMeasureType& m) const {
        return solveSupportsSolveMeasureTypeImpl(t, m);
    }
    SolveStatus<Scalar> solve(EOpTransp t, const MultiVectorBase<Scalar>& B,
                              const Ptr<MultiVectorBase<Scalar>>& X,
                              const Ptr<const SolveCriteria<Scalar>> c = nullptr) const {
        return solveImpl(t, B, X, c);
    }

  protected:
    virtual bool solveSupportsImpl(EOpTransp t) const { return t == NOTRANS; }
    virtual bool solveSupportsNewImpl(EOpTransp t, const Ptr<const SolveCriteria<Scalar>>) const {
        return solveSupportsImpl(t);
    }
    virtual bool solveSupportsSolveMeasureTypeImpl(EOpTransp t, const SolveMeasureType&) const {
        return solveSupportsImpl(t);
    }
    virtual SolveStatus<Scalar> solveImpl(EOpTransp t, const MultiVectorBase<Scalar>& B,
                                          const Ptr<MultiVectorBase<Scalar>>& X,
                                          const Ptr<const SolveCriteria<Scalar>> c) const = 0;
};

template <class Scalar>
class LinearOpSourceBase : public virtual Teuchos::Describable {
  public:
    virtual RCP<const LinearOpBase<Scalar>> getOp() const = 0;
};

template <class Scalar>
class DefaultLinearOpSource : public LinearOpSourceBase<Scalar> {
  public:
    explicit DefaultLinearOpSource(const RCP<const LinearOpBase<Scalar>>& op) : d_op(op) {}
    RCP<const LinearOpBase<Scalar>> getOp() const override { return d_op; }

  private:
    RCP<const LinearOpBase<Scalar>> d_op;
};
template <class Scalar>
RCP<const LinearOpSourceBase<Scalar>> defaultLinearOpSource(
    const RCP<const LinearOpBase<Scalar>>& op) {
    return Teuchos::rcp(new DefaultLinearOpSource<Scalar>(op));
}

template <class Scalar>
class PreconditionerBase : public virtual Teuchos::Describable {
  public:
    virtual RCP<const LinearOpBase<Scalar>> getLeftPrecOp() const = 0;
    virtual RCP<const LinearOpBase<Scalar>> getRightPrecOp() const = 0;
    virtual RCP<const LinearOpBase<Scalar>> getUnspecifiedPrecOp() const = 0;
};

template <class Scalar>
class DefaultPreconditioner : public PreconditionerBase<Scalar> {
  public:
    DefaultPreconditioner(const RCP<const LinearOpBase<Scalar>>& left,
                          const RCP<const LinearOpBase<Scalar>>& right)
        : d_left(left), d_right(right) {}
    RCP<const LinearOpBase<Scalar>> getLeftPrecOp() const override { return d_left; }
    RCP<const LinearOpBase<Scalar>> getRightPrecOp() const override { return d_right; }
    RCP<const LinearOpBase<Scalar>> getUnspecifiedPrecOp() const override { return Teuchos::null; }

  private:
    RCP<const LinearOpBase<Scalar>> d_left, d_right;
};

template <class Scalar>
class LinearOpWithSolveFactoryBase : public virtual Teuchos::Describable,
                                     public virtual Teuchos::ParameterListAcceptor {
  public:
    virtual bool isCompatible(const LinearOpSourceBase<Scalar>& fwdOpSrc) const = 0;
    virtual RCP<LinearOpWithSolveBase<Scalar>> createOp() const = 0;
    virtual void initializeOp(const RCP<const LinearOpSourceBase<Scalar>>& fwdOpSrc,
                              LinearOpWithSolveBase<Scalar>* Op,
                              const ESupportSolveUse use = SUPPORT_SOLVE_UNSPECIFIED) const = 0;
    virtual void initializeAndReuseOp(const RCP<const LinearOpSourceBase<Scalar>>& fwdOpSrc,
                                      LinearOpWithSolveBase<Scalar>* Op) const {
        initializeOp(fwdOpSrc, Op);
    }
    virtual void uninitializeOp(LinearOpWithSolveBase<Scalar>* Op,
                                RCP<const LinearOpSourceBase<Scalar>>* fwdOpSrc = nullptr,
                                RCP<const PreconditionerBase<Scalar>>* prec = nullptr,
                                RCP<const LinearOpSourceBase<Scalar>>* approxFwdOpSrc = nullptr,
                                ESupportSolveUse* use = nullptr) const = 0;
    virtual bool supportsPreconditionerInputType(const EPreconditionerInputType) const {
        return false;
    }
    virtual void initializePreconditionedOp(const RCP<const LinearOpSourceBase<Scalar>>&,
                                            const RCP<const PreconditionerBase<Scalar>>&,
                                            LinearOpWithSolveBase<Scalar>*,
                                            const ESupportSolveUse = SUPPORT_SOLVE_UNSPECIFIED) const {
        throw std::logic_error("initializePreconditionedOp not supported");
    }
};

}  // namespace Thyra

#endif
