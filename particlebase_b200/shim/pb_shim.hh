// Common support of the drop-in C++ classes: the scalar type, error handling
// and the checkpoint stream helpers.  The classes keep the reference's names,
// public fields and method signatures (cudaFrame.hh:20-112,
// cudaParticleBase.hh:29-226, cudaParticleMD.hh:32-194, cudaParticleVV.hh:14-57,
// GaussianThermo.hh:14-90, CUDAenv.hh:19-89) and forward every call to the
// C ABI in pb/pb.h, so drivers written against the reference compile and run
// unchanged on one B200.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include "pb/pb.h"

#if !defined(REAL)
#define REAL float
#endif
typedef REAL real;

namespace pb_shim {

// The reference reports CUDA errors and exits (cudaFrame::ErrorInfo,
// cudaFrame.cu:20-32); the shim does the same with the library's message.
inline void check(int rc, const char *what, const pb_md *h) {
  if (rc == PB_OK) return;
  std::cerr << "particlebase_b200: " << what << " failed (" << rc << ")"
            << (h ? std::string(": ") + pb_md_last_error(h) : std::string()) << std::endl;
  std::exit(1);
}

template <typename T>
inline void put(std::ostream &o, const T &x) {
  o.write(reinterpret_cast<const char *>(&x), sizeof(T));
}
template <typename T>
inline void get(std::istream &i, T &x) {
  i.read(reinterpret_cast<char *>(&x), sizeof(T));
}
template <typename T>
inline void put_vec(std::ostream &o, const std::vector<T> &v) {
  const uint64_t n = v.size();
  put(o, n);
  if (n) o.write(reinterpret_cast<const char *>(v.data()), sizeof(T) * n);
}
template <typename T>
inline void get_vec(std::istream &i, std::vector<T> &v) {
  uint64_t n = 0;
  get(i, n);
  v.resize(n);
  if (n) i.read(reinterpret_cast<char *>(v.data()), sizeof(T) * n);
}

}  // namespace pb_shim
