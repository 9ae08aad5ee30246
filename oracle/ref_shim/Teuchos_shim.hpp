// The few Teuchos pieces the reference's BiCGStab2 (MatrixSystem/BiCGStab2.h,
// .inl) names -- RCP, rcp, Ptr, ParameterList with get<T>, ScalarTraits,
// Comm, the exception macros -- for the parity checker (oracle/_ref).  Test
// infrastructure only: single rank, no reference counting beyond
// std::shared_ptr.
#pragma once

#include <any>
#include <cstddef>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>

#define TEUCHOS_TEST_FOR_EXCEPTION(cond, Exc, msg) \
    do {                                           \
        if (cond) {                                \
            std::ostringstream teuchos_os_;        \
            teuchos_os_ << msg;                    \
            throw Exc(teuchos_os_.str());          \
        }                                          \
    } while (0)
#define TEUCHOS_TEST_FOR_EXCEPT_MSG(cond, msg) TEUCHOS_TEST_FOR_EXCEPTION(cond, std::logic_error, msg)

namespace Teuchos {
template <class T>
class Ptr {
public:
    explicit Ptr(T* p = nullptr) : p_(p) {}
    T* operator->() const { return p_; }
    T& operator*() const { return *p_; }
    T* get() const { return p_; }

private:
    T* p_;
};

template <class T>
class RCP {
public:
    RCP() = default;
    RCP(std::nullptr_t) {}
    explicit RCP(T* p) : p_(p) {}
    explicit RCP(std::shared_ptr<T> p) : p_(std::move(p)) {}
    template <class U>
    RCP(const RCP<U>& o) : p_(o.shared()) {}
    T* operator->() const { return p_.get(); }
    T& operator*() const { return *p_; }
    T* get() const { return p_.get(); }
    bool is_null() const { return !p_; }
    Ptr<T> ptr() const { return Ptr<T>(p_.get()); }
    const std::shared_ptr<T>& shared() const { return p_; }

private:
    std::shared_ptr<T> p_;
};
template <class T>
RCP<T> rcp(T* p) {
    return RCP<T>(p);
}

namespace Exceptions {
struct InvalidParameterName : std::logic_error {
    using std::logic_error::logic_error;
};
struct InvalidParameterType : std::logic_error {
    using std::logic_error::logic_error;
};
}  // namespace Exceptions

class ParameterList {
public:
    template <class T>
    ParameterList& set(const std::string& name, const T& value) {
        m_[name] = value;
        return *this;
    }
    ParameterList& set(const std::string& name, const char* value) { return set(name, std::string(value)); }
    template <class T>
    const T& get(const std::string& name) const {
        auto it = m_.find(name);
        if (it == m_.end()) throw Exceptions::InvalidParameterName("parameter \"" + name + "\" not found");
        const T* v = std::any_cast<T>(&it->second);
        if (!v) throw Exceptions::InvalidParameterType("parameter \"" + name + "\" has another type");
        return *v;
    }

private:
    std::map<std::string, std::any> m_;
};
template <class T>
T get(const ParameterList& l, const std::string& name) {
    return l.template get<T>(name);
}

template <class T>
struct ScalarTraits {
    using magnitudeType = T;
    static T one() { return T(1); }
    static T zero() { return T(0); }
};

template <class Ordinal>
class Comm {
public:
    virtual ~Comm() = default;
    virtual int getRank() const { return 0; }
    virtual int getSize() const { return 1; }
};
}  // namespace Teuchos
