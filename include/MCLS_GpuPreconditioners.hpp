// MCLS_GpuPreconditioners.hpp -- preconditioners built on the device.
//
// PointJacobiPreconditioner and BlockJacobiPreconditioner replace
// TpetraPointJacobiPreconditioner and TpetraBlockJacobiPreconditioner
// (tpetra/src/MCLS_TpetraPointJacobiPreconditioner_impl.hpp:104-139,
// tpetra/src/MCLS_TpetraBlockJacobiPreconditioner_impl.hpp:122-223).  The
// matrix returned by getLeftPreconditioner() is a host copy; when it is
// handed to LinearProblem::setLeftPrec the managers find and use the device
// copy instead of uploading it again.
#ifndef MCLS_GPUPRECONDITIONERS_HPP
#define MCLS_GPUPRECONDITIONERS_HPP

#include "MCLS_GpuBackend.hpp"
#include "MCLS_Preconditioner.hpp"

namespace MCLS {

template <class Vector, class Matrix>
class GpuPreconditionerBase : public Preconditioner<Matrix> {
  public:
    typedef MatrixTraits<Vector, Matrix> MT;

    Teuchos::RCP<const Teuchos::ParameterList> getCurrentParameters() const override {
        return d_plist;
    }
    void setParameters(const Teuchos::RCP<Teuchos::ParameterList>& params) override {
        if (!Teuchos::nonnull(params)) throw Assertion("preconditioner: null parameters");
        d_plist = params;
    }
    void setOperator(const Teuchos::RCP<const Matrix>& A) override {
        if (!Teuchos::nonnull(A)) throw Assertion("preconditioner: null operator");
        d_A = A;
    }
    const Matrix& getOperator() const override { return *d_A; }
    Teuchos::RCP<const Matrix> getLeftPreconditioner() const override { return d_M; }
    Teuchos::RCP<const Matrix> getRightPreconditioner() const override { return Teuchos::null; }

  protected:
    explicit GpuPreconditionerBase(const Teuchos::RCP<Teuchos::ParameterList>& params)
        : d_plist(params ? params : Teuchos::parameterList()) {}

    void buildWith(mclsgpu_precond_params pp) {
        if (!Teuchos::nonnull(d_A)) throw Assertion("preconditioner: setOperator() first");
        auto ctx = gpu::Context::on(int(gpu::numeric(*d_plist, "GPU Device", 0.0)));
        auto op = gpu::operatorFor<Vector, Matrix>(ctx, d_A);
        d_pc = std::make_shared<gpu::Precond>(op, pp);
        std::vector<std::int64_t> rp, ci;
        std::vector<double> v;
        d_pc->exportCsr(rp, ci, v);
        auto M = MT::fromCsr(MT::getGlobalNumRows(*d_A), std::move(rp), std::move(ci),
                             std::move(v));
        d_M = M;
        gpu::Registry::instance().addPrecond(std::shared_ptr<const void>(d_M), d_pc);
    }

    Teuchos::RCP<Teuchos::ParameterList> d_plist;
    Teuchos::RCP<const Matrix> d_A;
    Teuchos::RCP<const Matrix> d_M;
    std::shared_ptr<gpu::Precond> d_pc;
};

// M^-1 = diag(A)^-1.
template <class Vector, class Matrix>
class PointJacobiPreconditioner : public GpuPreconditionerBase<Vector, Matrix> {
  public:
    explicit PointJacobiPreconditioner(
        const Teuchos::RCP<Teuchos::ParameterList>& params = Teuchos::null)
        : GpuPreconditionerBase<Vector, Matrix>(params) {}
    Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const override {
        auto pl = Teuchos::parameterList();
        pl->set<int>("GPU Device", 0);
        return pl;
    }
    void buildPreconditioner() override {
        mclsgpu_precond_params pp{};
        pp.size = sizeof(pp);
        pp.kind = MCLSGPU_PREC_POINT_JACOBI;
        this->buildWith(pp);
    }
};

// Inverse of the contiguous diagonal blocks of A ("Jacobi Block Size").
template <class Vector, class Matrix>
class BlockJacobiPreconditioner : public GpuPreconditionerBase<Vector, Matrix> {
  public:
    explicit BlockJacobiPreconditioner(
        const Teuchos::RCP<Teuchos::ParameterList>& params = Teuchos::null)
        : GpuPreconditionerBase<Vector, Matrix>(params) {}
    Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const override {
        auto pl = Teuchos::parameterList();
        pl->set<int>("Jacobi Block Size", 1);
        pl->set<int>("GPU Device", 0);
        return pl;
    }
    void buildPreconditioner() override {
        mclsgpu_precond_params pp{};
        pp.size = sizeof(pp);
        pp.kind = MCLSGPU_PREC_BLOCK_JACOBI;
        pp.block_size = int(gpu::numeric(*this->d_plist, "Jacobi Block Size", 1.0));
        this->buildWith(pp);
    }
};

}  // namespace MCLS

#endif  // MCLS_GPUPRECONDITIONERS_HPP
