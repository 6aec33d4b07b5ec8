// Stand-in for Tpetra::CrsMatrix on one rank.  Entries go in by global
// indices; fillComplete builds the column map in order of first appearance
// (rows in local order) and keeps each row in insertion order, so neither
// local rows nor local columns come out sorted by global index.
#ifndef STANDIN_TPETRA_CRSMATRIX_HPP
#define STANDIN_TPETRA_CRSMATRIX_HPP

#include <map>
#include <stdexcept>
#include <vector>

#include "Tpetra_MultiVector.hpp"

namespace Tpetra {

// The operator base a Thyra wrapper holds (Tpetra_Operator.hpp).
template <class S = double, class LO = int, class GO = long long, class Node = DefaultNode>
class Operator {
  public:
    virtual ~Operator() = default;
};

template <class S = double, class LO = int, class GO = long long, class Node = DefaultNode>
class CrsMatrix : public Operator<S, LO, GO, Node> {
  public:
    typedef Map<LO, GO, Node> map_type;
    typedef MultiVector<S, LO, GO, Node> mv_type;

    template <class T>
    struct HostView {  // the Kokkos::View calls the adapter makes
        const T* p = nullptr;
        std::size_t n = 0;
        std::size_t extent(int) const { return n; }
        const T& operator()(std::size_t k) const { return p[k]; }
    };
    typedef HostView<LO> local_inds_host_view_type;
    typedef HostView<S> values_host_view_type;

    CrsMatrix(const Teuchos::RCP<const map_type>& rowMap, std::size_t /*maxEntriesPerRow*/)
        : d_rows(rowMap), d_gcol(rowMap->getLocalNumElements()),
          d_val(rowMap->getLocalNumElements()), d_lcol(rowMap->getLocalNumElements()) {}

    void insertGlobalValues(GO row, LO numEnt, const S vals[], const GO inds[]) {
        if (d_filled) throw std::logic_error("CrsMatrix: insert after fillComplete");
        const LO r = d_rows->getLocalElement(row);
        for (LO k = 0; k < numEnt; ++k) {
            d_gcol[r].push_back(inds[k]);
            d_val[r].push_back(vals[k]);
        }
    }
    void fillComplete() {
        std::vector<GO> order;
        std::map<GO, LO> seen;
        for (auto& row : d_gcol)
            for (GO g : row)
                if (!seen.count(g)) {
                    seen[g] = LO(order.size());
                    order.push_back(g);
                }
        d_cols = Teuchos::rcp(new map_type(order.size(), order, GO(0), d_rows->getComm()));
        for (std::size_t r = 0; r < d_gcol.size(); ++r) {
            d_lcol[r].clear();
            for (GO g : d_gcol[r]) d_lcol[r].push_back(seen[g]);
        }
        d_filled = true;
    }

    std::size_t getGlobalNumRows() const { return d_rows->getGlobalNumElements(); }
    std::size_t getLocalNumRows() const { return d_rows->getLocalNumElements(); }
    Teuchos::RCP<const map_type> getRowMap() const { return d_rows; }
    Teuchos::RCP<const map_type> getColMap() const { return d_cols; }
    Teuchos::RCP<const Teuchos::Comm<int>> getComm() const { return d_rows->getComm(); }

    void getLocalRowView(LO r, local_inds_host_view_type& idx, values_host_view_type& val) const {
        if (!d_filled) throw std::logic_error("CrsMatrix: local view before fillComplete");
        idx.p = d_lcol.at(std::size_t(r)).data();
        idx.n = d_lcol[std::size_t(r)].size();
        val.p = d_val[std::size_t(r)].data();
        val.n = d_val[std::size_t(r)].size();
    }

    // Y = A X; X and Y live on the row map (square, one rank).
    void apply(const mv_type& X, mv_type& Y) const {
        if (!d_filled) throw std::logic_error("CrsMatrix: apply before fillComplete");
        for (std::size_t j = 0; j < X.getNumVectors(); ++j)
            for (std::size_t r = 0; r < getLocalNumRows(); ++r) {
                S s = 0;
                for (std::size_t k = 0; k < d_lcol[r].size(); ++k) {
                    const GO g = d_cols->getGlobalElement(d_lcol[r][k]);
                    s += d_val[r][k] * X.at(std::size_t(d_rows->getLocalElement(g)), j);
                }
                Y.at(r, j) = s;
            }
    }

  private:
    Teuchos::RCP<const map_type> d_rows, d_cols;
    std::vector<std::vector<GO>> d_gcol;
    std::vector<std::vector<S>> d_val;
    std::vector<std::vector<LO>> d_lcol;
    bool d_filled = false;
};

}  // namespace Tpetra

#endif
