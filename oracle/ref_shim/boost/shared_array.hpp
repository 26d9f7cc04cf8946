// boost::shared_array<T>: an array owned by a shared pointer, indexed with [].
// The reference holds its per-device mutexes in one (cudaDeviceManager.cpp).
#pragma once
#include <cstddef>
#include <memory>
namespace boost {
template <class T> class shared_array {
  public:
    shared_array() = default;
    explicit shared_array(T *p) : p_(p, std::default_delete<T[]>()) {}
    T &operator[](std::ptrdiff_t i) const { return p_.get()[i]; }
    T *get() const { return p_.get(); }

  private:
    std::shared_ptr<T> p_;
};
}  // namespace boost
