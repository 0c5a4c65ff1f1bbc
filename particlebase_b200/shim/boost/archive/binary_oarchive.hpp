#pragma once
#include "archive_common.hpp"

namespace boost {
namespace archive {

class binary_oarchive {
  std::ostream &os_;

 public:
  explicit binary_oarchive(std::ostream &os, unsigned int = 0) : os_(os) {}
  template <class T>
  binary_oarchive &operator<<(const serialization::nvp<T> &x) {
    save(x.value());
    return *this;
  }
  template <class T>
  binary_oarchive &operator&(const serialization::nvp<T> &x) {
    return *this << x;
  }

 private:
  template <class T>
  void save(const T &t) {
    if constexpr (detail::has_pb_save<T>::value) {
      t.pb_save(os_);
    } else {
      static_assert(std::is_trivially_copyable<T>::value, "not archivable");
      os_.write(reinterpret_cast<const char *>(&t), sizeof(T));
    }
  }
};

}  // namespace archive
}  // namespace boost
