// Binary archives of the Boost stand-in: an object with pb_save / pb_load
// members writes its own checkpoint; trivially copyable values are written
// as raw bytes.  Not compatible with real Boost archive files.
#pragma once

// Boost's archive headers make these available to the files that include
// them, and drivers rely on that.
#include <algorithm>
#include <cassert>
#include <climits>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <vector>

#include <istream>
#include <ostream>
#include <type_traits>
#include <utility>

#include "../serialization/nvp.hpp"

namespace boost {
namespace archive {
namespace detail {

template <class T, class = void>
struct has_pb_save : std::false_type {};
template <class T>
struct has_pb_save<T, std::void_t<decltype(std::declval<const T &>().pb_save(
                          std::declval<std::ostream &>()))>> : std::true_type {};

}  // namespace detail
}  // namespace archive
}  // namespace boost
