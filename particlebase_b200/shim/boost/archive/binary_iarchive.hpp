#pragma once
#include "archive_common.hpp"

namespace boost {
namespace archive {

class binary_iarchive {
  std::istream &is_;

 public:
  explicit binary_iarchive(std::istream &is, unsigned int = 0) : is_(is) {}
  template <class T>
  binary_iarchive &operator>>(const serialization::nvp<T> &x) {
    load(x.value());
    return *this;
  }
  template <class T>
  binary_iarchive &operator&(const serialization::nvp<T> &x) {
    return *this >> x;
  }

 private:
  template <class T>
  void load(T &t) {
    if constexpr (detail::has_pb_save<T>::value) {
      t.pb_load(is_);
    } else {
      static_assert(std::is_trivially_copyable<T>::value, "not archivable");
      is_.read(reinterpret_cast<char *>(&t), sizeof(T));
    }
  }
};

}  // namespace archive
}  // namespace boost
