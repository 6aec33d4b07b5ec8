// Thyra_MCLSGpuLinearOpWithSolveFactory.hpp -- the Stratimikos linear-solve
// strategy over the GPU managers.
//
// Replaces Thyra::MCLSLinearOpWithSolveFactory and
// Thyra::MCLSLinearOpWithSolve (thyra/src/Thyra_MCLSLinearOpWithSolveFactory_impl.hpp:58-615,
// thyra/src/Thyra_MCLSLinearOpWithSolve_impl.hpp:52-430), which no longer
// compile against the library: they create AdjointSolverManager and
// ForwardSolverManager (Thyra_MCLSLinearOpWithSolveFactory_impl.hpp:499-531).
// The classes here only translate -- Thyra operators, preconditioners and
// multi-vectors to the Tpetra objects inside them
// (TpetraOperatorVectorExtraction), Thyra's solve criteria and statuses to
// and from MCLS's -- and forward to MCLS::LinearOpWithSolveFactory /
// MCLS::LinearOpWithSolve (MCLS_LinearOpWithSolve.hpp) over the traits of
// MCLS_TpetraAdapter.hpp.  Each MCLS solve enum has Thyra's enumerators in
// Thyra's order, so the conversions are casts.
//
// Needs Thyra and Tpetra (compile with -DMCLSGPU_USE_TEUCHOS).  Register with
// a Stratimikos builder as
//   builder.setLinearSolveStrategyFactory(
//       Teuchos::abstractFactoryStd<Thyra::LinearOpWithSolveFactoryBase<double>,
//                                   Thyra::MCLSGpuLinearOpWithSolveFactory<LO, GO, Node>>(),
//       "MCLS");
#ifndef THYRA_MCLSGPULINEAROPWITHSOLVEFACTORY_HPP
#define THYRA_MCLSGPULINEAROPWITHSOLVEFACTORY_HPP

#include <string>

#include <Thyra_LinearOpWithSolveFactoryBase.hpp>
#include <Thyra_TpetraThyraWrappers.hpp>

#include "MCLS_TpetraAdapter.hpp"

namespace Thyra {

template <class LO, class GO, class Node>
class MCLSGpuLinearOpWithSolve : public LinearOpWithSolveBase<double> {
  public:
    typedef Tpetra::MultiVector<double, LO, GO, Node> TMV;
    typedef Tpetra::CrsMatrix<double, LO, GO, Node> TM;
    typedef TpetraOperatorVectorExtraction<double, LO, GO, Node> TOVE;
    typedef MCLS::LinearOpWithSolve<TMV, TM> Core;

    Core& core() { return d_core; }
    const Core& core() const { return d_core; }

    // What the factory keeps beside the core (handed back by uninitializeOp).
    void setSources(const RCP<const LinearOpSourceBase<double>>& fwd,
                    const RCP<const PreconditionerBase<double>>& prec, ESupportSolveUse use) {
        d_fwd = fwd;
        d_prec = prec;
        d_use = use;
        d_space = Teuchos::nonnull(fwd) ? fwd->getOp()->range() : Teuchos::null;
    }
    RCP<const LinearOpSourceBase<double>> fwdOpSrc() const { return d_fwd; }
    RCP<const PreconditionerBase<double>> prec() const { return d_prec; }
    ESupportSolveUse supportSolveUse() const { return d_use; }

    RCP<const VectorSpaceBase<double>> range() const override { return d_space; }
    RCP<const VectorSpaceBase<double>> domain() const override { return d_space; }
    std::string description() const override {
        return "Thyra::MCLSGpuLinearOpWithSolve{" + d_core.description() + "}";
    }

    static MCLS::SolveMeasureType measure(const SolveMeasureType& m) {
        return MCLS::SolveMeasureType(MCLS::ESolveMeasureNormType(m.numerator),
                                      MCLS::ESolveMeasureNormType(m.denominator));
    }

  protected:
    bool opSupportedImpl(EOpTransp t) const override {
        return d_core.opSupported(MCLS::EOpTransp(t));
    }
    void applyImpl(EOpTransp t, const MultiVectorBase<double>& X,
                   const Ptr<MultiVectorBase<double>>& Y, double alpha,
                   double beta) const override {
        auto x = TOVE::getConstTpetraMultiVector(Teuchos::rcpFromRef(X));
        auto y = TOVE::getTpetraMultiVector(Teuchos::rcpFromPtr(Y));
        d_core.apply(MCLS::EOpTransp(t), *x, y.get(), alpha, beta);
    }
    bool solveSupportsImpl(EOpTransp t) const override {
        return d_core.solveSupports(MCLS::EOpTransp(t));
    }
    bool solveSupportsNewImpl(EOpTransp t, const Ptr<const SolveCriteria<double>> c) const override {
        if (Teuchos::is_null(c)) return solveSupportsImpl(t);
        return d_core.solveSupportsSolveMeasureType(MCLS::EOpTransp(t), measure(c->solveMeasureType));
    }
    bool solveSupportsSolveMeasureTypeImpl(EOpTransp t, const SolveMeasureType& m) const override {
        return d_core.solveSupportsSolveMeasureType(MCLS::EOpTransp(t), measure(m));
    }
    SolveStatus<double> solveImpl(EOpTransp t, const MultiVectorBase<double>& B,
                                  const Ptr<MultiVectorBase<double>>& X,
                                  const Ptr<const SolveCriteria<double>> c) const override {
        auto b = TOVE::getConstTpetraMultiVector(Teuchos::rcpFromRef(B));
        auto x = TOVE::getTpetraMultiVector(Teuchos::rcpFromPtr(X));
        MCLS::SolveCriteria mc;
        if (!Teuchos::is_null(c)) {
            mc.solveMeasureType = measure(c->solveMeasureType);
            mc.requestedTol = c->requestedTol == SolveCriteria<double>::unspecifiedTolerance()
                                  ? MCLS::SolveCriteria::unspecifiedTolerance()
                                  : double(c->requestedTol);
            mc.extraParameters = c->extraParameters;
        }
        const MCLS::SolveStatus s =
            d_core.solve(MCLS::EOpTransp(t), *b, x.get(), Teuchos::is_null(c) ? nullptr : &mc);
        SolveStatus<double> out;
        out.solveStatus = ESolveStatus(s.solveStatus);
        out.achievedTol = s.achievedTol;
        out.message = s.message;
        out.extraParameters = s.extraParameters;
        return out;
    }

  private:
    Core d_core;
    RCP<const LinearOpSourceBase<double>> d_fwd;
    RCP<const PreconditionerBase<double>> d_prec;
    ESupportSolveUse d_use = SUPPORT_SOLVE_UNSPECIFIED;
    RCP<const VectorSpaceBase<double>> d_space;
};

template <class LO, class GO, class Node>
class MCLSGpuLinearOpWithSolveFactory : public LinearOpWithSolveFactoryBase<double> {
  public:
    typedef MCLSGpuLinearOpWithSolve<LO, GO, Node> Op;
    typedef typename Op::TMV TMV;
    typedef typename Op::TM TM;
    typedef TpetraOperatorVectorExtraction<double, LO, GO, Node> TOVE;
    typedef MCLS::LinearOpWithSolveFactory<TMV, TM> Core;

    Core& core() { return d_core; }

    bool isCompatible(const LinearOpSourceBase<double>& src) const override {
        auto A = matrix(src.getOp());
        return Teuchos::nonnull(A) && d_core.isCompatible(*A);
    }
    RCP<LinearOpWithSolveBase<double>> createOp() const override { return Teuchos::rcp(new Op()); }
    void initializeOp(const RCP<const LinearOpSourceBase<double>>& src,
                      LinearOpWithSolveBase<double>* op,
                      const ESupportSolveUse use = SUPPORT_SOLVE_UNSPECIFIED) const override {
        Op& o = Teuchos::dyn_cast<Op>(*op);
        d_core.initializeOp(required(src), &o.core(), MCLS::ESupportSolveUse(use));
        o.setSources(src, Teuchos::null, use);
    }
    void initializeAndReuseOp(const RCP<const LinearOpSourceBase<double>>& src,
                              LinearOpWithSolveBase<double>* op) const override {
        Op& o = Teuchos::dyn_cast<Op>(*op);
        d_core.initializeAndReuseOp(required(src), &o.core());
        o.setSources(src, Teuchos::null, o.supportSolveUse());
    }
    // A Thyra preconditioner (Ifpack2, MueLu, ...) whose left and right
    // operators are Tpetra CRS matrices: they become PL and PR.
    bool supportsPreconditionerInputType(const EPreconditionerInputType t) const override {
        return t == PRECONDITIONER_INPUT_TYPE_AS_OPERATOR;
    }
    void initializePreconditionedOp(const RCP<const LinearOpSourceBase<double>>& src,
                                    const RCP<const PreconditionerBase<double>>& prec,
                                    LinearOpWithSolveBase<double>* op,
                                    const ESupportSolveUse use = SUPPORT_SOLVE_UNSPECIFIED) const override {
        if (Teuchos::is_null(prec))
            throw MCLS::Assertion("MCLSGpuLinearOpWithSolveFactory: null preconditioner");
        Op& o = Teuchos::dyn_cast<Op>(*op);
        d_core.initializePreconditionedOp(required(src), matrix(prec->getLeftPrecOp()),
                                          matrix(prec->getRightPrecOp()), &o.core(),
                                          MCLS::ESupportSolveUse(use));
        o.setSources(src, prec, use);
    }
    void uninitializeOp(LinearOpWithSolveBase<double>* op,
                        RCP<const LinearOpSourceBase<double>>* fwdOpSrc = nullptr,
                        RCP<const PreconditionerBase<double>>* prec = nullptr,
                        RCP<const LinearOpSourceBase<double>>* approxFwdOpSrc = nullptr,
                        ESupportSolveUse* use = nullptr) const override {
        Op& o = Teuchos::dyn_cast<Op>(*op);
        if (fwdOpSrc) *fwdOpSrc = o.fwdOpSrc();
        if (prec) *prec = o.prec();
        if (approxFwdOpSrc) *approxFwdOpSrc = Teuchos::null;
        if (use) *use = o.supportSolveUse();
        d_core.uninitializeOp(&o.core());
        o.setSources(Teuchos::null, Teuchos::null, SUPPORT_SOLVE_UNSPECIFIED);
    }

    void setParameterList(const RCP<Teuchos::ParameterList>& pl) override {
        d_core.setParameterList(pl);
    }
    RCP<Teuchos::ParameterList> getNonconstParameterList() override {
        return d_core.getNonconstParameterList();
    }
    RCP<Teuchos::ParameterList> unsetParameterList() override { return d_core.unsetParameterList(); }
    RCP<const Teuchos::ParameterList> getParameterList() const override {
        return d_core.getParameterList();
    }
    RCP<const Teuchos::ParameterList> getValidParameters() const override {
        return d_core.getValidParameters();
    }
    std::string description() const override { return "Thyra::MCLSGpuLinearOpWithSolveFactory"; }

  private:
    // The Tpetra CRS matrix inside a Thyra operator, or null.
    static RCP<const TM> matrix(const RCP<const LinearOpBase<double>>& op) {
        if (Teuchos::is_null(op)) return Teuchos::null;
        return Teuchos::rcp_dynamic_cast<const TM>(TOVE::getConstTpetraOperator(op));
    }
    static RCP<const TM> required(const RCP<const LinearOpSourceBase<double>>& src) {
        auto A = Teuchos::is_null(src) ? RCP<const TM>() : matrix(src->getOp());
        if (Teuchos::is_null(A))
            throw MCLS::Assertion("MCLSGpuLinearOpWithSolveFactory: the operator is not a "
                                  "Tpetra::CrsMatrix");
        return A;
    }

    Core d_core;
};

}  // namespace Thyra

#endif  // THYRA_MCLSGPULINEAROPWITHSOLVEFACTORY_HPP
