// MCLS_GpuTeuchos.hpp -- the slice of Teuchos the MCLS manager API uses.
//
// The MCLS solver managers take Teuchos::RCP handles and Teuchos::
// ParameterList settings (src/MCLS_SolverManager.hpp:80-112).  Where Trilinos
// is installed, define MCLSGPU_USE_TEUCHOS and the real Teuchos headers are
// used.  Otherwise this header supplies a small stand-in with the same
// spelling for what user code of the managers touches: RCP / rcp / null /
// nonnull / is_null, ParameterList (set, get, get-with-default,
// isParameter, isType, sublist, setParameters, validateParameters and
// validateParametersAndSetDefaults without validators), parameterList(),
// sublist(), ScalarTraits, Describable, as<>, and a serial Comm<int>.
#ifndef MCLS_GPUTEUCHOS_HPP
#define MCLS_GPUTEUCHOS_HPP

#ifdef MCLSGPU_USE_TEUCHOS
#include <Teuchos_Comm.hpp>
#include <Teuchos_DefaultComm.hpp>
#include <Teuchos_Describable.hpp>
#include <Teuchos_ParameterList.hpp>
#include <Teuchos_RCP.hpp>
#include <Teuchos_ScalarTraits.hpp>
#else

#include <any>
#include <cstddef>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <typeinfo>
#include <vector>

namespace Teuchos {

// Reference-counted handle with the RCP spellings on top of shared_ptr.
template <class T>
class RCP : public std::shared_ptr<T> {
  public:
    using std::shared_ptr<T>::shared_ptr;
    RCP() = default;
    RCP(std::nullptr_t) {}
    RCP(const std::shared_ptr<T>& p) : std::shared_ptr<T>(p) {}
    template <class U>
    RCP(const RCP<U>& p) : std::shared_ptr<T>(p) {}
    T* getRawPtr() const { return this->get(); }
    bool is_null() const { return this->get() == nullptr; }
};

constexpr std::nullptr_t null = nullptr;

template <class T>
RCP<T> rcp(T* p, bool owns = true) {
    if (owns) return RCP<T>(p);
    return RCP<T>(p, [](T*) {});
}
template <class T>
RCP<T> rcpFromRef(T& r) {
    return RCP<T>(&r, [](T*) {});
}
template <class T>
bool nonnull(const RCP<T>& p) { return p.get() != nullptr; }
template <class T>
bool is_null(const RCP<T>& p) { return p.get() == nullptr; }
template <class T, class U>
RCP<T> rcp_dynamic_cast(const RCP<U>& p) {
    return RCP<T>(std::dynamic_pointer_cast<T>(std::shared_ptr<U>(p)));
}

template <class T, class U>
T as(const U& u) { return static_cast<T>(u); }

template <class S>
struct ScalarTraits {
    typedef S magnitudeType;
};

class Describable {
  public:
    virtual ~Describable() = default;
    virtual std::string description() const { return "MCLS GPU object"; }
};

namespace Exceptions {
struct InvalidParameter : std::logic_error {
    using std::logic_error::logic_error;
};
struct InvalidParameterName : InvalidParameter {
    using InvalidParameter::InvalidParameter;
};
struct InvalidParameterType : InvalidParameter {
    using InvalidParameter::InvalidParameter;
};
struct InvalidParameterValue : InvalidParameter {
    using InvalidParameter::InvalidParameter;
};
}  // namespace Exceptions

// Name -> typed value map.  Typing is strict as in Teuchos: get<int> on an
// entry set as double throws InvalidParameterType.
class ParameterList {
  public:
    ParameterList() = default;
    explicit ParameterList(const std::string& name) : name_(name) {}

    const std::string& name() const { return name_; }

    template <class T>
    ParameterList& set(const std::string& key, const T& value) {
        entries_[key] = value;
        order(key);
        return *this;
    }
    ParameterList& set(const std::string& key, const char* value) {
        return set<std::string>(key, std::string(value));
    }

    template <class T>
    T& get(const std::string& key) {
        return cast<T>(key, find(key));
    }
    template <class T>
    const T& get(const std::string& key) const {
        return cast<T>(key, const_cast<ParameterList*>(this)->find(key));
    }
    // Returns the entry, first setting it to `def` when absent.
    template <class T>
    T& get(const std::string& key, const T& def) {
        if (!isParameter(key)) set<T>(key, def);
        return get<T>(key);
    }
    std::string& get(const std::string& key, const char* def) {
        return get<std::string>(key, std::string(def));
    }

    // Nested list `key`, created empty when absent (Teuchos::ParameterList::sublist).
    ParameterList& sublist(const std::string& key) {
        if (!isParameter(key)) set<ParameterList>(key, ParameterList(key));
        return get<ParameterList>(key);
    }
    const ParameterList& sublist(const std::string& key) const {
        return get<ParameterList>(key);
    }
    bool isSublist(const std::string& key) const { return isType<ParameterList>(key); }

    bool isParameter(const std::string& key) const { return entries_.count(key) != 0; }
    template <class T>
    bool isType(const std::string& key) const {
        auto it = entries_.find(key);
        return it != entries_.end() && it->second.type() == typeid(T);
    }
    bool remove(const std::string& key) {
        if (!entries_.erase(key)) return false;
        for (auto it = names_.begin(); it != names_.end(); ++it)
            if (*it == key) { names_.erase(it); break; }
        return true;
    }
    // Copies every entry of `other` over this list.
    ParameterList& setParameters(const ParameterList& other) {
        for (const auto& k : other.names_) {
            entries_[k] = other.entries_.at(k);
            order(k);
        }
        return *this;
    }
    int numParams() const { return static_cast<int>(names_.size()); }
    const std::vector<std::string>& names() const { return names_; }

    // Every entry must be named in `valid` with the same type
    // (InvalidParameterName / InvalidParameterType otherwise); sublists
    // present in both lists are checked `depth` levels further down.
    void validateParameters(const ParameterList& valid, int depth = 1000) const {
        for (const auto& k : names_) {
            const std::any& a = entries_.at(k);
            const std::any& v = valid.checked(name_, k, a);
            if (depth > 0 && a.type() == typeid(ParameterList))
                std::any_cast<const ParameterList&>(a).validateParameters(
                    std::any_cast<const ParameterList&>(v), depth - 1);
        }
    }
    // validateParameters, then copies in every entry of `valid` missing here
    // (a missing sublist arrives whole, with all its defaults).
    void validateParametersAndSetDefaults(const ParameterList& valid, int depth = 1000) {
        for (const auto& k : names_) {
            std::any& a = entries_.at(k);
            const std::any& v = valid.checked(name_, k, a);
            if (depth > 0 && a.type() == typeid(ParameterList))
                std::any_cast<ParameterList&>(a).validateParametersAndSetDefaults(
                    std::any_cast<const ParameterList&>(v), depth - 1);
        }
        for (const auto& k : valid.names_)
            if (!isParameter(k)) {
                entries_[k] = valid.entries_.at(k);
                order(k);
            }
    }

  private:
    // The entry of this (valid) list that `value`, named `key` in the list
    // `owner`, must match by name and type.
    const std::any& checked(const std::string& owner, const std::string& key,
                            const std::any& value) const {
        auto it = entries_.find(key);
        if (it == entries_.end())
            throw Exceptions::InvalidParameterName("ParameterList '" + owner + "': parameter \"" +
                                                   key + "\" is not a valid parameter");
        if (it->second.type() != value.type())
            throw Exceptions::InvalidParameterType("ParameterList '" + owner + "': parameter \"" +
                                                   key + "\" has the wrong type");
        return it->second;
    }
    std::any& find(const std::string& key) {
        auto it = entries_.find(key);
        if (it == entries_.end())
            throw Exceptions::InvalidParameterName("ParameterList '" + name_ +
                                                   "': no parameter \"" + key + "\"");
        return it->second;
    }
    template <class T>
    static T& cast(const std::string& key, std::any& a) {
        T* p = std::any_cast<T>(&a);
        if (!p)
            throw Exceptions::InvalidParameterType("parameter \"" + key +
                                                   "\" was requested with a different type");
        return *p;
    }
    void order(const std::string& key) {
        for (const auto& k : names_)
            if (k == key) return;
        names_.push_back(key);
    }

    std::string name_ = "ANONYMOUS";
    std::map<std::string, std::any> entries_;
    std::vector<std::string> names_;
};

inline RCP<ParameterList> parameterList() { return RCP<ParameterList>(new ParameterList); }
inline RCP<ParameterList> parameterList(const std::string& name) {
    return RCP<ParameterList>(new ParameterList(name));
}
// Handle to the sublist `name` of `parent` that keeps `parent` alive.
inline RCP<ParameterList> sublist(const RCP<ParameterList>& parent, const std::string& name,
                                  bool mustAlreadyExist = false) {
    if (mustAlreadyExist && !parent->isSublist(name))
        throw Exceptions::InvalidParameterName("ParameterList '" + parent->name() +
                                               "': no sublist \"" + name + "\"");
    return RCP<ParameterList>(std::shared_ptr<ParameterList>(parent, &parent->sublist(name)));
}

// Serial communicator: one process, rank 0.
template <class Ordinal>
class Comm {
  public:
    virtual ~Comm() = default;
    virtual int getRank() const { return 0; }
    virtual int getSize() const { return 1; }
    virtual void barrier() const {}
};
template <class Ordinal>
struct DefaultComm {
    static RCP<const Comm<Ordinal>> getComm() {
        return RCP<const Comm<Ordinal>>(new Comm<Ordinal>);
    }
};

}  // namespace Teuchos

#endif  // MCLSGPU_USE_TEUCHOS
#endif  // MCLS_GPUTEUCHOS_HPP
