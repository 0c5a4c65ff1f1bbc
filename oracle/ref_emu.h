// CUDA execution-model emulation for compiling the reference's kernel sources
// (kernelfuncs.cu, kerneltemplate.hh, kernelinline.hh of particlelover/ParticleBase)
// as plain host C++ with g++.
//
// TEST INFRASTRUCTURE ONLY: this header is part of the oracle. It lets the
// reference's own __global__ kernels run on the CPU so that the FP64
// restatement in oracle.cpp can be checked against the reference's actual
// arithmetic.  Nothing in the product library includes it.
//
// Emulation model: every "CUDA block" has exactly one thread (blockDim = 1), so
// __syncthreads() is a no-op.  Shared memory becomes ordinary globals:
// every kernel that uses it is launched as a single block and run serially.  The reference's kernels are all written with grid-stride
// loops, so a grid of G one-thread blocks covers the whole index range.
// Blocks may be run in parallel by OpenMP when they write disjoint outputs.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <climits>
#include <cassert>
#include <algorithm>
#include <numeric>
#include <vector>
#include <valarray>
#include <string>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __constant__
#define __shared__

struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct double2 { double x, y; };
struct uint2 { uint32_t x, y; };
struct uint3 { uint32_t x, y, z; };
struct uint4 { uint32_t x, y, z, w; };
struct dim3 {
  uint32_t x, y, z;
  dim3(uint32_t a = 1, uint32_t b = 1, uint32_t c = 1) : x(a), y(b), z(c) {}
};

inline uint2 make_uint2(uint32_t a, uint32_t b) { return uint2{a, b}; }
inline float4 make_float4(float a, float b, float c, float d) { return float4{a, b, c, d}; }

// CUDA's reciprocal square root overloads.  The device versions are
// approximate (about 2 ulp); the emulation uses the correctly rounded
// quotient, so emulated results may differ from a GPU run in the last bits.
inline float rsqrt(float x) { return 1.0f / std::sqrt(x); }
inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
using std::sqrt;
using std::isnan;

// The built-in index variables.  thread_local so that OpenMP threads can each
// emulate a different block.
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

inline void __syncthreads() {}

enum cudaMemcpyKind { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2 };
template <typename T>
inline int cudaMemcpyToSymbol(T &symbol, const void *src, size_t bytes) {
  std::memcpy(&symbol, src, bytes);
  return 0;
}
