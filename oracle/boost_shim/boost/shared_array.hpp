// Test infrastructure: boost::shared_array (shared owner of a new[] array)
// over std::shared_ptr with an array deleter, for the reference's host code.
#pragma once
#include <cstddef>
#include <memory>
namespace boost {
template <class T> class shared_array {
public:
    shared_array() = default;
    explicit shared_array(T* p) : p_(p, std::default_delete<T[]>()) {}
    void reset(T* p = nullptr) { p_.reset(p, std::default_delete<T[]>()); }
    T& operator[](std::ptrdiff_t i) const { return p_.get()[i]; }
    T* get() const { return p_.get(); }
    explicit operator bool() const { return (bool)p_; }
private:
    std::shared_ptr<T> p_;
};
}
