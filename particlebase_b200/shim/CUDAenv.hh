// CUDAenv<T> (CUDAenv.hh:19-89): device query and one particle object per
// GPU.  This library runs on one GPU: nDevices() is 1, the force exchange
// between GPUs is a no-op, and setThnum fills the launch-shape fields the
// drivers may read.
#if !defined(CUDAENV)
#define CUDAENV

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <string>
#include <vector>

#include <boost/archive/binary_iarchive.hpp>
#include <boost/archive/binary_oarchive.hpp>

#include "ExchangeMode.hh"
#include "pb_shim.hh"

template <typename T>
class CUDAenv {
 public:
  CUDAenv() {
    std::cerr << "checking GPU devices" << std::endl;
    int count = 0;
    cudaError_t t = cudaGetDeviceCount(&count);
    std::cerr << "GPU status: " << cudaGetErrorString(t) << std::endl;
    if (t != cudaSuccess || count < 1) std::exit(1);
    ndev = 1;  // one GPU
    cudaDeviceProp p;
    cudaGetDeviceProperties(&p, 0);
    name = p.name;
    capability = p.major + 0.1 * p.minor;
    numMP = p.multiProcessorCount;
    numCpMP = 128;  // FP32 lanes per SM on sm_100
    globalMemSize = (uint32_t)std::min<size_t>(p.totalGlobalMem, 0xffffffffu);
    numTh = p.maxThreadsPerBlock;
    maxGrid = p.maxGridSize[0];
    shMem = (uint32_t)p.sharedMemPerBlock;
    if (count > 1) std::cerr << "using GPU 0 of " << count << std::endl;
  }
  ~CUDAenv() {
    for (T *q : P) delete q;
  }

  void display(std::ostream &o) const {
    o << "GPU 0: " << name << ", compute capability " << capability << ", " << numMP
      << " multiprocessors" << std::endl;
  }
  void setGPU(int i) {
    if (i != 0) {
      std::cerr << "particlebase_b200: one GPU (asked for " << i << ")" << std::endl;
      std::exit(1);
    }
    cudaSetDevice(0);
  }

  std::string getName(void) const { return name; }
  double getCapability(void) const { return capability; }
  uint32_t getNumMP(void) const { return numMP; }
  uint32_t getNumCpMP(void) const { return numCpMP; }
  uint32_t getMemSize(void) const { return globalMemSize; }
  uint32_t getNumTh(void) const { return numTh; }
  uint32_t getMaxGrid(void) const { return maxGrid; }
  uint32_t getShMem(void) const { return shMem; }

  void setThnum(T &p) {
    const int th2d = (int)std::min(getNumCpMP() / 4, (uint32_t)std::sqrt((double)getNumTh()));
    p.MPnum = getNumMP();
    p.THnum1D = (int)std::min(1024u, getNumTh());
    p.THnum1DX = getNumCpMP() * 4;
    p.THnum2D = th2d;
    p.threadsMax = getNumTh();
    p.maxGrid = getMaxGrid();
    std::cerr << "CUDA thread parameters: MPnum: " << p.MPnum << ", THnum1D: " << p.THnum1D
              << ", THnum1DX: " << p.THnum1DX << ", THnum2D: " << th2d << std::endl;
  }

  int nDevices(void) { return ndev; }
  T &operator[](int i) { return *P[i]; }

  void setup(void) {
    for (T *q : P) delete q;
    P.assign(ndev, nullptr);
    for (int i = 0; i < ndev; ++i) {
      P[i] = new T;
      setThnum(*P[i]);
    }
  }

  // one GPU holds every force already
  void exchangeForce(void) {}
  void exchangeAccelerations(void) {}
  void exchangeForceSelected(const ExchangeMode = ExchangeMode::force) {}

  void readSerialization(std::string filename) {
    std::ifstream ifs(filename, std::ios::binary);
    boost::archive::binary_iarchive ia(ifs);
    ia >> boost::serialization::make_nvp("cudaParticles", *P[0]);
  }
  void writeSerialization(std::string filename) const {
    std::ofstream ofs(filename, std::ios::binary);
    boost::archive::binary_oarchive oa(ofs);
    oa << boost::serialization::make_nvp("cudaParticles", *P[0]);
  }

 protected:
  int ndev = 1;
  int currentGPU = 0;

 private:
  std::string name;
  double capability = 0;
  uint32_t numMP = 0, numCpMP = 0, globalMemSize = 0, numTh = 0, maxGrid = 0, shMem = 0;
  std::vector<T *> P;
};

#endif /* CUDAENV */
