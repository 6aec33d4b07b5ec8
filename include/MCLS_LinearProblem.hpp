// MCLS_LinearProblem.hpp -- A x = b with optional left/right preconditioners.
//
// Same constructor, setters and getters as the reference's LinearProblem
// (src/MCLS_LinearProblem.hpp:73-154).  The solvers never form the
// composite operators PL*A*PR and (PL*A*PR)^T on the host:
// mclsgpu_domain_build forms them on the device.  getCompositeOperator /
// getTransposeCompositeOperator and the apply/residual helpers below serve
// callers that inspect the problem; the solve itself runs on the GPU.
#ifndef MCLS_LINEARPROBLEM_HPP
#define MCLS_LINEARPROBLEM_HPP

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "MCLS_GpuTraits.hpp"

namespace MCLS {

namespace detail {

// Square host CSR used by the composite-operator helpers.
struct Csr {
    std::int64_t n = 0;
    std::vector<std::int64_t> rp{0}, ci;
    std::vector<double> v;
};

// C = A B row by row: the products of row i of A, taken in A's column order,
// accumulate into a dense row; columns come out sorted.  Then the reference
// filter (tpetra/src/MCLS_TpetraHelpers.hpp:196-259): entries with
// |c| <= threshold * (signed row max) and exact zeros are dropped.
inline Csr multiply(const Csr& A, const Csr& B, double threshold) {
    Csr C;
    C.n = A.n;
    std::vector<double> acc(size_t(A.n), 0.0);
    std::vector<char> used(size_t(A.n), 0);
    std::vector<std::int64_t> cols;
    for (std::int64_t i = 0; i < A.n; ++i) {
        cols.clear();
        for (std::int64_t p = A.rp[i]; p < A.rp[i + 1]; ++p) {
            const std::int64_t k = A.ci[p];
            for (std::int64_t q = B.rp[k]; q < B.rp[k + 1]; ++q) {
                const std::int64_t j = B.ci[q];
                if (!used[j]) {
                    used[j] = 1;
                    acc[j] = 0.0;
                    cols.push_back(j);
                }
                acc[j] += A.v[p] * B.v[q];
            }
        }
        std::sort(cols.begin(), cols.end());
        double rmax = 0.0;
        for (size_t t = 0; t < cols.size(); ++t)
            rmax = t == 0 ? acc[cols[t]] : std::max(rmax, acc[cols[t]]);
        const double row_threshold = rmax * threshold;
        for (std::int64_t j : cols) {
            used[j] = 0;
            if (std::abs(acc[j]) <= row_threshold || acc[j] == 0.0) continue;
            C.ci.push_back(j);
            C.v.push_back(acc[j]);
        }
        C.rp.push_back(std::int64_t(C.ci.size()));
    }
    return C;
}

inline Csr transpose(const Csr& A) {
    Csr T;
    T.n = A.n;
    T.rp.assign(size_t(A.n) + 1, 0);
    for (std::int64_t j : A.ci) ++T.rp[size_t(j) + 1];
    for (std::int64_t i = 0; i < A.n; ++i) T.rp[i + 1] += T.rp[i];
    T.ci.resize(A.ci.size());
    T.v.resize(A.v.size());
    std::vector<std::int64_t> next(T.rp.begin(), T.rp.end() - 1);
    for (std::int64_t i = 0; i < A.n; ++i)
        for (std::int64_t p = A.rp[i]; p < A.rp[i + 1]; ++p) {
            const std::int64_t q = next[size_t(A.ci[p])]++;
            T.ci[q] = i;
            T.v[q] = A.v[p];
        }
    return T;
}

}  // namespace detail

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

    // PL A PR, the products filtered with `threshold` (no preconditioner:
    // A itself) (src/MCLS_LinearProblem_impl.hpp:141-176).
    Teuchos::RCP<const Matrix> getCompositeOperator(double threshold = 0.0) const {
        if (!isLeftPrec() && !isRightPrec()) return d_A;
        detail::Csr C = csr(*d_A);
        if (isRightPrec()) C = detail::multiply(C, csr(*d_PR), threshold);
        if (isLeftPrec()) C = detail::multiply(csr(*d_PL), C, threshold);
        return fromCsr(std::move(C));
    }
    // (PL A PR)^T = PR^T A^T PL^T, formed from the transposes as the
    // reference does (src/MCLS_LinearProblem_impl.hpp:182-221); no
    // preconditioner: a copy of A^T.
    Teuchos::RCP<const Matrix> getTransposeCompositeOperator(double threshold = 0.0) const {
        detail::Csr C = detail::transpose(csr(*d_A));
        if (isLeftPrec()) C = detail::multiply(C, detail::transpose(csr(*d_PL)), threshold);
        if (isRightPrec()) C = detail::multiply(detail::transpose(csr(*d_PR)), C, threshold);
        return fromCsr(std::move(C));
    }

    // y = PL A PR x (src/MCLS_LinearProblem_impl.hpp:252-287).  The
    // intermediate vectors are VT::clone'd, never copy-constructed: a
    // vector type may copy by view (Tpetra does).
    void apply(const Vector& x, Vector& y) const {
        const Vector* in = &x;
        Teuchos::RCP<Vector> t;
        if (isRightPrec()) {
            t = VT::clone(x);
            MT::apply(*d_PR, x, *t);
            in = t.get();
        }
        if (isLeftPrec()) {
            auto u = VT::clone(y);
            MT::apply(*d_A, *in, *u);
            MT::apply(*d_PL, *u, y);
        } else {
            MT::apply(*d_A, *in, y);
        }
    }
    void applyOp(const Vector& x, Vector& y) const { MT::apply(*d_A, x, y); }
    void applyLeftPrec(const Vector& x, Vector& y) const { MT::apply(*d_PL, x, y); }
    void applyRightPrec(const Vector& x, Vector& y) const { MT::apply(*d_PR, x, y); }

    // r = b - A x (src/MCLS_LinearProblem_impl.hpp:390-405).
    void updateResidual() {
        auto ax = VT::clone(*d_r);
        MT::apply(*d_A, *d_x, *ax);
        const double* b = VT::view(*d_b);
        const double* a = VT::view(*ax);
        double* r = VT::viewNonConst(*d_r);
        for (std::int64_t i = 0; i < VT::getGlobalLength(*d_r); ++i) r[i] = b[i] - a[i];
    }
    // rp = PL (b - A x) (src/MCLS_LinearProblem_impl.hpp:410-442).
    void updatePrecResidual() {
        updateResidual();
        if (isLeftPrec()) {
            MT::apply(*d_PL, *d_r, *d_rp);
        } else {
            const double* r = VT::view(*d_r);
            double* rp = VT::viewNonConst(*d_rp);
            for (std::int64_t i = 0; i < VT::getGlobalLength(*d_r); ++i) rp[i] = r[i];
        }
    }
    // x += PR update (src/MCLS_LinearProblem_impl.hpp:228-247).
    void updateSolution(const Teuchos::RCP<Vector>& update) {
        Teuchos::RCP<Vector> u;
        if (isRightPrec()) {
            u = VT::clone(*update);
            MT::apply(*d_PR, *update, *u);
        }
        const double* p = VT::view(isRightPrec() ? *u : *update);
        double* x = VT::viewNonConst(*d_x);
        for (std::int64_t i = 0; i < VT::getGlobalLength(*d_x); ++i) x[i] += p[i];
    }

  private:
    static detail::Csr csr(const Matrix& M) {
        detail::Csr c;
        c.n = MT::getGlobalNumRows(M);
        MT::getCsr(M, c.rp, c.ci, c.v);
        return c;
    }
    static Teuchos::RCP<const Matrix> fromCsr(detail::Csr c) {
        return MT::fromCsr(c.n, std::move(c.rp), std::move(c.ci), std::move(c.v));
    }

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
