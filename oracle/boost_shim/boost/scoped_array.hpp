// Test infrastructure: boost::scoped_array (sole owner of a new[] array)
// over std::unique_ptr<T[]>, for the reference's host code.
#pragma once
#include <cstddef>
#include <memory>
namespace boost {
template <class T> class scoped_array {
public:
    explicit scoped_array(T* p = nullptr) : p_(p) {}
    scoped_array(const scoped_array&) = delete;
    scoped_array& operator=(const scoped_array&) = delete;
    void reset(T* p = nullptr) { p_.reset(p); }
    T& operator[](std::ptrdiff_t i) const { return p_[i]; }
    T* get() const { return p_.get(); }
private:
    std::unique_ptr<T[]> p_;
};
}
