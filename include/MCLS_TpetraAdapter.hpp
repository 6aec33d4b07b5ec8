// MCLS_TpetraAdapter.hpp -- the facade's traits for Tpetra::Vector,
// Tpetra::CrsMatrix and Tpetra::MultiVector.
//
// Replaces the reference's Tpetra adapters for the GPU path
// (tpetra/src/MCLS_TpetraVectorAdapter.hpp:68-340,
// tpetra/src/MCLS_TpetraCrsMatrixAdapter.hpp:73-498) and the Tpetra
// multi-vector traits of its Thyra layer (thyra/src/MCLS_MultiVectorTraits.hpp:
// 95-395).  The GPU managers need far less than the reference's traits: a
// vector's length and host storage, a matrix as 64-bit CSR (rows sorted by
// global column) and back, y = A x, and the columns of a multi-vector.
//
// Scope: one MPI rank holds the whole system on a contiguous row map (local
// row i is global row g0 + i) -- the GPU path has one domain per device, and
// several sets go through the multi-set driver -- so getCsr rejects a matrix
// distributed over more than one rank or on a permuted map.  Vectors are
// reached through getData / getDataNonConst, host views of a host-resident
// (Serial or OpenMP node) vector.  fromCsr builds its matrices on a
// contiguous map with index base 0.
//
// Needs Tpetra; compile with -DMCLSGPU_USE_TEUCHOS so the real Teuchos
// headers serve the facade as well.  Include it before the managers are
// instantiated.
#ifndef MCLS_TPETRAADAPTER_HPP
#define MCLS_TPETRAADAPTER_HPP

#include <algorithm>
#include <cstdint>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include <Tpetra_Core.hpp>
#include <Tpetra_CrsMatrix.hpp>
#include <Tpetra_MultiVector.hpp>
#include <Tpetra_Vector.hpp>

#include "MCLS_GpuTraits.hpp"
#include "MCLS_LinearOpWithSolve.hpp"

namespace MCLS {

template <class Scalar, class LO, class GO, class Node>
struct VectorTraits<Tpetra::Vector<Scalar, LO, GO, Node>> {
    static_assert(std::is_same<Scalar, double>::value,
                  "the GPU path computes in FP64: use Tpetra::Vector<double, ...>");
    typedef Tpetra::Vector<Scalar, LO, GO, Node> vector_type;
    typedef Scalar scalar_type;
    static std::int64_t getGlobalLength(const vector_type& v) {
        return std::int64_t(v.getGlobalLength());
    }
    static const Scalar* view(const vector_type& v) { return v.getData().getRawPtr(); }
    static Scalar* viewNonConst(vector_type& v) { return v.getDataNonConst().getRawPtr(); }
    // A zero vector on v's map.
    static Teuchos::RCP<vector_type> clone(const vector_type& v) {
        return Teuchos::rcp(new vector_type(v.getMap()));
    }
};

template <class Scalar, class LO, class GO, class Node>
struct MatrixTraits<Tpetra::Vector<Scalar, LO, GO, Node>, Tpetra::CrsMatrix<Scalar, LO, GO, Node>> {
    typedef Tpetra::Vector<Scalar, LO, GO, Node> vector_type;
    typedef Tpetra::CrsMatrix<Scalar, LO, GO, Node> matrix_type;
    typedef Tpetra::Map<LO, GO, Node> map_type;

    static std::int64_t getGlobalNumRows(const matrix_type& A) {
        return std::int64_t(A.getGlobalNumRows());
    }
    // Rows in order, each sorted by column; indices relative to the first
    // global row, so row and column i are vector entry i.
    static void getCsr(const matrix_type& A, std::vector<std::int64_t>& rowptr,
                       std::vector<std::int64_t>& colind, std::vector<double>& values) {
        if (A.getComm()->getSize() != 1)
            throw Assertion("MCLS Tpetra adapter: the matrix must be held by one rank");
        const std::size_t n = A.getLocalNumRows();
        const auto rows = A.getRowMap();
        const auto cols = A.getColMap();
        const std::int64_t g0 = n ? std::int64_t(rows->getGlobalElement(LO(0))) : 0;
        for (std::size_t r = 0; r < n; ++r)
            if (std::int64_t(rows->getGlobalElement(LO(r))) != g0 + std::int64_t(r))
                throw Assertion("MCLS Tpetra adapter: the row map must be contiguous");
        rowptr.assign(1, 0);
        colind.clear();
        values.clear();
        typename matrix_type::local_inds_host_view_type idx;
        typename matrix_type::values_host_view_type val;
        std::vector<std::pair<std::int64_t, double>> row;
        for (std::size_t r = 0; r < n; ++r) {
            A.getLocalRowView(LO(r), idx, val);
            row.clear();
            for (std::size_t k = 0; k < std::size_t(idx.extent(0)); ++k) {
                const std::int64_t c = std::int64_t(cols->getGlobalElement(idx(k))) - g0;
                if (c < 0 || c >= std::int64_t(n))
                    throw Assertion("MCLS Tpetra adapter: a column outside the row range");
                row.emplace_back(c, double(val(k)));
            }
            std::sort(row.begin(), row.end(),
                      [](const std::pair<std::int64_t, double>& a,
                         const std::pair<std::int64_t, double>& b) { return a.first < b.first; });
            for (const auto& e : row) {
                colind.push_back(e.first);
                values.push_back(e.second);
            }
            rowptr.push_back(std::int64_t(colind.size()));
        }
    }
    // An n x n matrix on a contiguous map of the default communicator (the
    // row map of a one-rank system), fill-completed.
    static Teuchos::RCP<matrix_type> fromCsr(std::int64_t n, std::vector<std::int64_t> rowptr,
                                             std::vector<std::int64_t> colind,
                                             std::vector<double> values) {
        auto map = Teuchos::rcp(new map_type(n, GO(0), Tpetra::getDefaultComm()));
        std::size_t max_row = 0;
        for (std::int64_t i = 0; i < n; ++i)
            max_row = std::max(max_row, std::size_t(rowptr[i + 1] - rowptr[i]));
        auto M = Teuchos::rcp(new matrix_type(map, max_row));
        std::vector<GO> c;
        std::vector<Scalar> v;
        for (std::int64_t i = 0; i < n; ++i) {
            c.assign(colind.begin() + rowptr[i], colind.begin() + rowptr[i + 1]);
            v.assign(values.begin() + rowptr[i], values.begin() + rowptr[i + 1]);
            M->insertGlobalValues(GO(i), LO(c.size()), v.data(), c.data());
        }
        M->fillComplete();
        return M;
    }
    // y = A x.
    static void apply(const matrix_type& A, const vector_type& x, vector_type& y) {
        A.apply(x, y);
    }
};

template <class Scalar, class LO, class GO, class Node>
struct MultiVectorTraits<Tpetra::MultiVector<Scalar, LO, GO, Node>,
                         Tpetra::CrsMatrix<Scalar, LO, GO, Node>> {
    typedef Tpetra::MultiVector<Scalar, LO, GO, Node> multivector_type;
    typedef Tpetra::Vector<Scalar, LO, GO, Node> vector_type;
    typedef Scalar scalar_type;
    static int getNumVectors(const multivector_type& X) { return int(X.getNumVectors()); }
    // Column `id` as a vector sharing X's storage.
    static Teuchos::RCP<const vector_type> getVector(const multivector_type& X, int id) {
        return X.getVector(std::size_t(id));
    }
    static Teuchos::RCP<vector_type> getVectorNonConst(multivector_type& X, int id) {
        return X.getVectorNonConst(std::size_t(id));
    }
};

}  // namespace MCLS

#endif  // MCLS_TPETRAADAPTER_HPP
