// Stand-in for Teuchos::ArrayRCP: a raw pointer that keeps its storage alive.
#ifndef STANDIN_TEUCHOS_ARRAYRCP_HPP
#define STANDIN_TEUCHOS_ARRAYRCP_HPP

#include <memory>

#include "MCLS_GpuTeuchos.hpp"

namespace Teuchos {

template <class T>
class ArrayRCP {
  public:
    ArrayRCP(T* p, std::shared_ptr<const void> keep) : d_p(p), d_keep(std::move(keep)) {}
    T* getRawPtr() const { return d_p; }
    T& operator[](std::size_t i) const { return d_p[i]; }

  private:
    T* d_p;
    std::shared_ptr<const void> d_keep;
};

}  // namespace Teuchos

#endif
