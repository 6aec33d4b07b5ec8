// Stand-in for Thyra's Tpetra wrappers (Thyra_TpetraThyraWrappers.hpp):
// a Thyra operator around a Tpetra operator, a Thyra multi-vector around a
// Tpetra multi-vector, and TpetraOperatorVectorExtraction to get them back.
#ifndef STANDIN_THYRA_TPETRA_WRAPPERS_HPP
#define STANDIN_THYRA_TPETRA_WRAPPERS_HPP

#include "Thyra_LinearOpWithSolveFactoryBase.hpp"
#include "Tpetra_CrsMatrix.hpp"

namespace Thyra {

template <class Scalar>
class TpetraVectorSpace : public VectorSpaceBase<Scalar> {
  public:
    explicit TpetraVectorSpace(long dim) : d_dim(dim) {}
    long dim() const override { return d_dim; }

  private:
    long d_dim;
};

template <class Scalar, class LO, class GO, class Node>
class TpetraMultiVector : public MultiVectorBase<Scalar> {
  public:
    typedef Tpetra::MultiVector<Scalar, LO, GO, Node> TMV;
    explicit TpetraMultiVector(const RCP<TMV>& mv) : d_mv(mv) {}
    RCP<TMV> tpetra() const { return d_mv; }

  private:
    RCP<TMV> d_mv;
};

template <class Scalar, class LO, class GO, class Node>
class TpetraLinearOp : public LinearOpBase<Scalar> {
  public:
    typedef Tpetra::Operator<Scalar, LO, GO, Node> TOp;
    typedef Tpetra::CrsMatrix<Scalar, LO, GO, Node> TM;
    explicit TpetraLinearOp(const RCP<const TOp>& op) : d_op(op) {
        auto A = Teuchos::rcp_dynamic_cast<const TM>(op);
        d_space = Teuchos::rcp(new TpetraVectorSpace<Scalar>(A ? long(A->getGlobalNumRows()) : 0));
    }
    RCP<const TOp> tpetra() const { return d_op; }
    RCP<const VectorSpaceBase<Scalar>> range() const override { return d_space; }
    RCP<const VectorSpaceBase<Scalar>> domain() const override { return d_space; }

  protected:
    bool opSupportedImpl(EOpTransp t) const override { return t == NOTRANS; }
    void applyImpl(EOpTransp, const MultiVectorBase<Scalar>& X,
                   const Ptr<MultiVectorBase<Scalar>>& Y, Scalar alpha, Scalar beta) const override {
        auto A = Teuchos::rcp_dynamic_cast<const TM>(d_op);
        auto x = dynamic_cast<const TpetraMultiVector<Scalar, LO, GO, Node>&>(X).tpetra();
        auto y = dynamic_cast<TpetraMultiVector<Scalar, LO, GO, Node>&>(*Y).tpetra();
        Tpetra::MultiVector<Scalar, LO, GO, Node> ax(x->getMap(), x->getNumVectors());
        A->apply(*x, ax);
        for (std::size_t j = 0; j < x->getNumVectors(); ++j)
            for (std::size_t i = 0; i < x->getGlobalLength(); ++i)
                y->at(i, j) = alpha * ax.at(i, j) + (beta == Scalar(0) ? Scalar(0) : beta * y->at(i, j));
    }

  private:
    RCP<const TOp> d_op;
    RCP<const VectorSpaceBase<Scalar>> d_space;
};

template <class Scalar, class LO, class GO, class Node>
RCP<const LinearOpBase<Scalar>> createConstLinearOp(
    const RCP<const Tpetra::Operator<Scalar, LO, GO, Node>>& op) {
    return Teuchos::rcp(new TpetraLinearOp<Scalar, LO, GO, Node>(op));
}
template <class Scalar, class LO, class GO, class Node>
RCP<MultiVectorBase<Scalar>> createMultiVector(
    const RCP<Tpetra::MultiVector<Scalar, LO, GO, Node>>& mv) {
    return Teuchos::rcp(new TpetraMultiVector<Scalar, LO, GO, Node>(mv));
}

template <class Scalar, class LO, class GO, class Node>
struct TpetraOperatorVectorExtraction {
    typedef Tpetra::Operator<Scalar, LO, GO, Node> TOp;
    typedef Tpetra::MultiVector<Scalar, LO, GO, Node> TMV;
    static RCP<const TOp> getConstTpetraOperator(const RCP<const LinearOpBase<Scalar>>& op) {
        return dynamic_cast<const TpetraLinearOp<Scalar, LO, GO, Node>&>(*op).tpetra();
    }
    static RCP<TMV> getTpetraMultiVector(const RCP<MultiVectorBase<Scalar>>& mv) {
        return dynamic_cast<TpetraMultiVector<Scalar, LO, GO, Node>&>(*mv).tpetra();
    }
    static RCP<const TMV> getConstTpetraMultiVector(const RCP<const MultiVectorBase<Scalar>>& mv) {
        return dynamic_cast<const TpetraMultiVector<Scalar, LO, GO, Node>&>(*mv).tpetra();
    }
};

}  // namespace Thyra

#endif
