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

#include <algorithm>
#include <vector>

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

// Learned sparse approximate inverse on A's pattern (mclsgpu_spai_*): M from
// a trained per-row network; point Jacobi replaces it when its
// power-iteration rho(I - M A) reaches both "Rho Fallback" and the Jacobi
// rho, or when A has no fixed stencil.  The network is either a trained
// handle given with setNetwork() (owned by the caller) or the flat FP32
// parameters in "SPAI Weights" (std::vector<float>, mclsgpu_spai_num_params()
// values, e.g. saved by `python -m mcls_b200.spai --out`).  No counterpart in
// the reference.
template <class Vector, class Matrix>
class LearnedSpaiPreconditioner : public GpuPreconditionerBase<Vector, Matrix> {
  public:
    typedef MatrixTraits<Vector, Matrix> MT;

    explicit LearnedSpaiPreconditioner(
        const Teuchos::RCP<Teuchos::ParameterList>& params = Teuchos::null)
        : GpuPreconditionerBase<Vector, Matrix>(params) {}
    Teuchos::RCP<const Teuchos::ParameterList> getValidParameters() const override {
        auto pl = Teuchos::parameterList();
        pl->set<std::vector<float>>("SPAI Weights", std::vector<float>());
        pl->set<double>("Rho Fallback", 0.95);
        pl->set<int>("GPU Device", 0);
        return pl;
    }
    void setNetwork(mclsgpu_spai* net) { d_net = net; }
    void buildPreconditioner() override {
        if (!Teuchos::nonnull(this->d_A)) throw Assertion("preconditioner: setOperator() first");
        mclsgpu_spai* net = d_net;
        mclsgpu_spai* own = nullptr;
        std::shared_ptr<gpu::Context> ctx;
        if (!net && this->d_plist->isParameter("SPAI Weights")) {
            const auto& w = this->d_plist->template get<std::vector<float>>("SPAI Weights");
            if (!w.empty()) {
                if (int(w.size()) != mclsgpu_spai_num_params())
                    throw Assertion("SPAI Weights: wrong parameter count");
                ctx = gpu::Context::on(int(gpu::numeric(*this->d_plist, "GPU Device", 0.0)));
                ctx->check(mclsgpu_spai_create(ctx->get(), stencilSlots(), 0, &own),
                           "mclsgpu_spai_create");
                int rc = mclsgpu_spai_set_params(own, w.data());
                if (rc != MCLSGPU_OK) {
                    mclsgpu_spai_destroy(own);
                    ctx->check(rc, "mclsgpu_spai_set_params");
                }
                net = own;
            }
        }
        mclsgpu_precond_params pp{};
        pp.size = sizeof(pp);
        pp.kind = MCLSGPU_PREC_LEARNED_SPAI;
        pp.spai_net = net;
        pp.rho_fallback = gpu::numeric(*this->d_plist, "Rho Fallback", 0.95);
        try {
            this->buildWith(pp);
        } catch (...) {
            if (own) mclsgpu_spai_destroy(own);
            throw;
        }
        if (own) mclsgpu_spai_destroy(own);  // M is built; the network is no longer needed
    }

  private:
    // Distinct column offsets of A: the network's stencil slots.
    int stencilSlots() const {
        std::vector<std::int64_t> rp, ci;
        std::vector<double> v;
        MT::getCsr(*this->d_A, rp, ci, v);
        std::vector<std::int64_t> offs;
        for (size_t i = 0; i + 1 < rp.size(); ++i)
            for (std::int64_t p = rp[i]; p < rp[i + 1]; ++p) offs.push_back(ci[p] - std::int64_t(i));
        std::sort(offs.begin(), offs.end());
        return int(std::unique(offs.begin(), offs.end()) - offs.begin());
    }

    mclsgpu_spai* d_net = nullptr;
};

}  // namespace MCLS

#endif  // MCLS_GPUPRECONDITIONERS_HPP
