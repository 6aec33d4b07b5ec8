// Stand-in for Tpetra::Map: one rank, global indices in local order.
#ifndef STANDIN_TPETRA_MAP_HPP
#define STANDIN_TPETRA_MAP_HPP

#include <cstddef>
#include <map>
#include <stdexcept>
#include <vector>

#include "MCLS_GpuTeuchos.hpp"

namespace Tpetra {

struct DefaultNode {};

template <class LO = int, class GO = long long, class Node = DefaultNode>
class Map {
  public:
    typedef LO local_ordinal_type;
    typedef GO global_ordinal_type;
    typedef Node node_type;
    // Contiguous: local i holds global indexBase + i.
    Map(std::size_t numGlobal, GO indexBase, const Teuchos::RCP<const Teuchos::Comm<int>>& comm)
        : d_comm(comm) {
        for (std::size_t i = 0; i < numGlobal; ++i) add(indexBase + GO(i));
    }
    // The given global indices in local order (Tpetra's ArrayView form).
    Map(std::size_t numGlobal, const std::vector<GO>& gids, GO /*indexBase*/,
        const Teuchos::RCP<const Teuchos::Comm<int>>& comm)
        : d_comm(comm) {
        if (gids.size() != numGlobal) throw std::logic_error("Map: size mismatch");
        for (GO g : gids) add(g);
    }
    GO getGlobalElement(LO i) const { return d_gids.at(std::size_t(i)); }
    LO getLocalElement(GO g) const {
        auto it = d_local.find(g);
        if (it == d_local.end()) throw std::logic_error("Map: global index not on this rank");
        return it->second;
    }
    std::size_t getGlobalNumElements() const { return d_gids.size(); }
    std::size_t getLocalNumElements() const { return d_gids.size(); }
    Teuchos::RCP<const Teuchos::Comm<int>> getComm() const { return d_comm; }

  private:
    void add(GO g) {
        d_local[g] = LO(d_gids.size());
        d_gids.push_back(g);
    }
    std::vector<GO> d_gids;
    std::map<GO, LO> d_local;
    Teuchos::RCP<const Teuchos::Comm<int>> d_comm;
};

}  // namespace Tpetra

#endif
