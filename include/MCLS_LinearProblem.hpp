// MCLS_LinearProblem.hpp -- A x = b with optional left/right preconditioners.
//
// Same constructor, setters and getters as the reference's LinearProblem
// (src/MCLS_LinearProblem.hpp:73-154).  The composite operators
// PL*A*PR and (PL*A*PR)^T (src/MCLS_LinearProblem_impl.hpp:141-221) are not
// formed on the host: mclsgpu_domain_build forms them on the device.  The
// host-side apply/residual helpers below serve callers that inspect the
// problem; the solve itself runs on the GPU.
#ifndef MCLS_LINEARPROBLEM_HPP
#define MCLS_LINEARPROBLEM_HPP

#include <cmath>
#include <cstdint>

#include "MCLS_GpuTraits.hpp"

namespace MCLS {

template <class Vector, class Matrix>
class LinearProblem {
  public:
    typedef Vector vector_type;
    typedef Matrix matrix_type;
    typedef VectorTraits<Vector> VT;
    typedef MatrixTraits<Vector, Matrix> MT;
    typedef typename VT::scalar_type Scalar;

    LinearProblem(const Teuchos::RCP<const Matrix>& A, const Teuchos::RCP<Vector>& x,
                  const Teuchos::RCP<const Vector>& b)
        : d_A(A), d_x(x), d_b(b) {
        if (!Teuchos::nonnull(A) || !Teuchos::nonnull(x) || !Teuchos::nonnull(b))
            throw Assertion("LinearProblem: A, x and b must be non-null");
        d_r = VT::clone(*x);
        d_rp = VT::clone(*x);
    }

    void setOperator(const Teuchos::RCP<const Matrix>& A) { d_A = A; ++d_generation; }
    void setLHS(const Teuchos::RCP<Vector>& x) { d_x = x; }
    void setRHS(const Teuchos::RCP<const Vector>& b) { d_b = b; }
    void setLeftPrec(const Teuchos::RCP<const Matrix>& PL) { d_PL = PL; ++d_generation; }
    void setRightPrec(const Teuchos::RCP<const Matrix>& PR) { d_PR = PR; ++d_generation; }

    Teuchos::RCP<const Matrix> getOperator() const { return d_A; }
    Teuchos::RCP<Vector> getLHS() const { return d_x; }
    Teuchos::RCP<const Vector> getRHS() const { return d_b; }
    Teuchos::RCP<const Matrix> getLeftPrec() const { return d_PL; }
    Teuchos::RCP<const Matrix> getRightPrec() const { return d_PR; }
    Teuchos::RCP<const Vector> getResidual() const { return d_r; }
    Teuchos::RCP<const Vector> getPrecResidual() const { return d_rp; }
    Teuchos::RCP<Vector> getPrecResidual() { return d_rp; }
    bool isLeftPrec() const { return Teuchos::nonnull(d_PL); }
    bool isRightPrec() const { return Teuchos::nonnull(d_PR); }

    // Bumped whenever the operator or a preconditioner is replaced; the
    // managers rebuild their device domain when it changes.
    std::uint64_t generation() const { return d_generation; }

    // y = PL A PR x (src/MCLS_LinearProblem_impl.hpp:252-287).
    void apply(const Vector& x, Vector& y) const {
        Vector t = x;
        if (isRightPrec()) MT::apply(*d_PR, x, t);
        MT::apply(*d_A, t, y);
        if (isLeftPrec()) {
            Vector u = y;
            MT::apply(*d_PL, u, y);
        }
    }
    void applyOp(const Vector& x, Vector& y) const { MT::apply(*d_A, x, y); }
    void applyLeftPrec(const Vector& x, Vector& y) const { MT::apply(*d_PL, x, y); }
    void applyRightPrec(const Vector& x, Vector& y) const { MT::apply(*d_PR, x, y); }

    // r = b - A x (src/MCLS_LinearProblem_impl.hpp:390-405).
    void updateResidual() {
        Vector ax = *d_r;
        MT::apply(*d_A, *d_x, ax);
        const double* b = VT::view(*d_b);
        const double* a = VT::view(ax);
        double* r = VT::viewNonConst(*d_r);
        for (std::int64_t i = 0; i < VT::getGlobalLength(*d_r); ++i) r[i] = b[i] - a[i];
    }
    // rp = PL (b - A x) (src/MCLS_LinearProblem_impl.hpp:410-442).
    void updatePrecResidual() {
        updateResidual();
        if (isLeftPrec())
            MT::apply(*d_PL, *d_r, *d_rp);
        else
            *d_rp = *d_r;
    }
    // x += PR update (src/MCLS_LinearProblem_impl.hpp:228-247).
    void updateSolution(const Teuchos::RCP<Vector>& update) {
        Vector u = *update;
        if (isRightPrec()) MT::apply(*d_PR, *update, u);
        double* x = VT::viewNonConst(*d_x);
        const double* p = VT::view(u);
        for (std::int64_t i = 0; i < VT::getGlobalLength(*d_x); ++i) x[i] += p[i];
    }

  private:
    Teuchos::RCP<const Matrix> d_A;
    Teuchos::RCP<Vector> d_x;
    Teuchos::RCP<const Vector> d_b;
    Teuchos::RCP<const Matrix> d_PL;
    Teuchos::RCP<const Matrix> d_PR;
    Teuchos::RCP<Vector> d_r;
    Teuchos::RCP<Vector> d_rp;
    std::uint64_t d_generation = 0;
};

}  // namespace MCLS

#endif  // MCLS_LINEARPROBLEM_HPP
