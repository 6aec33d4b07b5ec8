// MCLS_GpuTraits.hpp -- vector/matrix access for the GPU solver managers.
//
// The reference reaches vectors and matrices through the static-function
// traits VectorTraits<Vector> and MatrixTraits<Vector,Matrix>
// (src/MCLS_VectorTraits.hpp:95-349, src/MCLS_MatrixTraits.hpp:95-401).  The
// GPU managers need far less of them: the length and contiguous host storage
// of a vector, and a matrix as 64-bit CSR (to upload it) and back (to hand a
// device-built preconditioner to LinearProblem::setLeftPrec).  Adapting a
// vector/matrix type (Tpetra, a user's own) means specialising these two
// templates; HostVector and HostCrsMatrix below are ready-made host types.
#ifndef MCLS_GPUTRAITS_HPP
#define MCLS_GPUTRAITS_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "MCLS_GpuTeuchos.hpp"

namespace MCLS {

// Failure of a precondition or of the device library (src/MCLS_DBC.hpp:59-75).
class Assertion : public std::logic_error {
  public:
    explicit Assertion(const std::string& msg) : std::logic_error(msg) {}
};

// Monte Carlo direction tags (src/MCLS_MonteCarloSolverManager.hpp:71-72).
class ForwardTag {};
class AdjointTag {};

// The reference's default random number generator type
// (src/MCLS_Xorshift.hpp:57-109).  On the GPU path it selects nothing: the
// walk kernels carry their own Xorshift(13,7,17) streams.
template <class uint_type = std::uint64_t, uint_type a = 13, uint_type b = 7, uint_type c = 17>
class Xorshift {};

template <class Vector>
struct VectorTraits;  // specialise: see HostVector below

template <class Vector, class Matrix>
struct MatrixTraits;  // specialise: see HostCrsMatrix below

// Dense host vector.
typedef std::vector<double> HostVector;

// Square host CSR matrix with sorted 64-bit column indices.
struct HostCrsMatrix {
    std::int64_t n = 0;
    std::vector<std::int64_t> rowptr{0};
    std::vector<std::int64_t> colind;
    std::vector<double> values;
};

template <>
struct VectorTraits<HostVector> {
    typedef double scalar_type;
    static std::int64_t getGlobalLength(const HostVector& v) { return std::int64_t(v.size()); }
    static const double* view(const HostVector& v) { return v.data(); }
    static double* viewNonConst(HostVector& v) { return v.data(); }
    static Teuchos::RCP<HostVector> clone(const HostVector& v) {
        return Teuchos::rcp(new HostVector(v.size(), 0.0));
    }
};

template <>
struct MatrixTraits<HostVector, HostCrsMatrix> {
    static std::int64_t getGlobalNumRows(const HostCrsMatrix& A) { return A.n; }
    static void getCsr(const HostCrsMatrix& A, std::vector<std::int64_t>& rowptr,
                       std::vector<std::int64_t>& colind, std::vector<double>& values) {
        rowptr = A.rowptr;
        colind = A.colind;
        values = A.values;
    }
    static Teuchos::RCP<HostCrsMatrix> fromCsr(std::int64_t n, std::vector<std::int64_t> rowptr,
                                               std::vector<std::int64_t> colind,
                                               std::vector<double> values) {
        auto M = Teuchos::rcp(new HostCrsMatrix);
        M->n = n;
        M->rowptr = std::move(rowptr);
        M->colind = std::move(colind);
        M->values = std::move(values);
        return M;
    }
    // y = A x (MatrixTraits::apply, tpetra/src/MCLS_TpetraCrsMatrixAdapter.hpp:366-371).
    static void apply(const HostCrsMatrix& A, const HostVector& x, HostVector& y) {
        y.assign(size_t(A.n), 0.0);
        for (std::int64_t i = 0; i < A.n; ++i) {
            double s = 0.0;
            for (std::int64_t p = A.rowptr[i]; p < A.rowptr[i + 1]; ++p)
                s += A.values[p] * x[size_t(A.colind[p])];
            y[size_t(i)] = s;
        }
    }
};

}  // namespace MCLS

#endif  // MCLS_GPUTRAITS_HPP
