// Stand-in for Tpetra_Core.hpp: the default (serial) communicator.
#ifndef STANDIN_TPETRA_CORE_HPP
#define STANDIN_TPETRA_CORE_HPP

#include "MCLS_GpuTeuchos.hpp"

namespace Tpetra {
inline Teuchos::RCP<const Teuchos::Comm<int>> getDefaultComm() {
    return Teuchos::DefaultComm<int>::getComm();
}
}  // namespace Tpetra

#endif
