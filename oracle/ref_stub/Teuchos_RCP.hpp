// Minimal stand-in for Teuchos_RCP.hpp so that the reference's RNG and
// sampling headers compile without Trilinos (oracle/_ref build only).
#ifndef ORACLE_REF_STUB_TEUCHOS_RCP_HPP
#define ORACLE_REF_STUB_TEUCHOS_RCP_HPP
#include <memory>
namespace Teuchos {
template <class T> using RCP = std::shared_ptr<T>;
template <class T> RCP<T> rcp(T* p) { return RCP<T>(p); }
struct NullRCP {
    template <class T> operator std::shared_ptr<T>() const { return nullptr; }
};
static const NullRCP null = NullRCP();
}  // namespace Teuchos
#endif
