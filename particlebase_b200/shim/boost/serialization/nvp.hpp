// Stand-in for the part of Boost.Serialization the reference's drivers use
// (make_nvp with the archives in boost/archive/): names are ignored, values
// go to the shim classes' own checkpoint format.
#pragma once

namespace boost {
namespace serialization {

template <class T>
struct nvp {
  const char *name;
  T *ptr;
  T &value() const { return *ptr; }
};

template <class T>
inline nvp<T> make_nvp(const char *name, T &t) {
  return nvp<T>{name, &t};
}

class access {};

}  // namespace serialization
}  // namespace boost
