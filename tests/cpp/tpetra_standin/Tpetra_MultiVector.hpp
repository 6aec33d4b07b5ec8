// Stand-in for Tpetra::MultiVector and Tpetra::Vector: column-major storage
// by local index; copies and column views share the storage, as Tpetra's do.
#ifndef STANDIN_TPETRA_MULTIVECTOR_HPP
#define STANDIN_TPETRA_MULTIVECTOR_HPP

#include <memory>
#include <vector>

#include "Teuchos_ArrayRCP.hpp"
#include "Tpetra_Map.hpp"

namespace Tpetra {

template <class S = double, class LO = int, class GO = long long, class Node = DefaultNode>
class Vector;

template <class S = double, class LO = int, class GO = long long, class Node = DefaultNode>
class MultiVector {
  public:
    typedef Map<LO, GO, Node> map_type;
    typedef Vector<S, LO, GO, Node> vector_type;

    MultiVector(const Teuchos::RCP<const map_type>& map, std::size_t ncols)
        : d_map(map),
          d_n(map->getLocalNumElements()),
          d_ncols(ncols),
          d_data(std::make_shared<std::vector<S>>(d_n * ncols, S(0))) {}
    MultiVector(const MultiVector&) = default;  // a view, as in Tpetra
    virtual ~MultiVector() = default;

    std::size_t getNumVectors() const { return d_ncols; }
    std::size_t getGlobalLength() const { return d_map->getGlobalNumElements(); }
    Teuchos::RCP<const map_type> getMap() const { return d_map; }
    Teuchos::RCP<const vector_type> getVector(std::size_t j) const {
        return Teuchos::rcp(new vector_type(d_map, d_data, d_offset + j * d_n));
    }
    Teuchos::RCP<vector_type> getVectorNonConst(std::size_t j) {
        return Teuchos::rcp(new vector_type(d_map, d_data, d_offset + j * d_n));
    }
    // Entry (local row i, column j).
    S& at(std::size_t i, std::size_t j) const { return (*d_data)[d_offset + j * d_n + i]; }

  protected:
    MultiVector(const Teuchos::RCP<const map_type>& map, std::shared_ptr<std::vector<S>> data,
                std::size_t offset)
        : d_map(map), d_n(map->getLocalNumElements()), d_ncols(1), d_data(std::move(data)),
          d_offset(offset) {}

    Teuchos::RCP<const map_type> d_map;
    std::size_t d_n, d_ncols;
    std::shared_ptr<std::vector<S>> d_data;
    std::size_t d_offset = 0;
};

template <class S, class LO, class GO, class Node>
class Vector : public MultiVector<S, LO, GO, Node> {
    typedef MultiVector<S, LO, GO, Node> Base;
    friend class MultiVector<S, LO, GO, Node>;

  public:
    typedef typename Base::map_type map_type;
    explicit Vector(const Teuchos::RCP<const map_type>& map) : Base(map, 1) {}
    Vector(const Vector&) = default;  // a view, as in Tpetra

    Teuchos::ArrayRCP<const S> getData() const {
        return Teuchos::ArrayRCP<const S>(this->d_data->data() + this->d_offset, this->d_data);
    }
    Teuchos::ArrayRCP<S> getDataNonConst() {
        return Teuchos::ArrayRCP<S>(this->d_data->data() + this->d_offset, this->d_data);
    }

  private:
    Vector(const Teuchos::RCP<const map_type>& map, std::shared_ptr<std::vector<S>> data,
           std::size_t offset)
        : Base(map, std::move(data), offset) {}
};

}  // namespace Tpetra

#endif
