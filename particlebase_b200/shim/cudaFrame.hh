// cudaFrame (cudaFrame.hh:20-112): launch-shape fields, the host staging
// buffer TMP and the LAMMPS dump writer.
#if !defined(CUDAFRAME)
#define CUDAFRAME

#include <ctime>
#include <iostream>
#include <mutex>
#include <string>
#include <valarray>

#include "pb_shim.hh"

class cudaFrame {
 protected:
  bool withInfo = false;
  std::valarray<real> TMP;             // 4 floats per particle after getPosition()
  std::valarray<unsigned short> TMP2;  // type id per particle after getTypeID()
  real cell[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  std::mutex mutTMP;
  time_t starttime = time(nullptr);

 public:
  // launch shapes of the reference's kernels; set by CUDAenv::setThnum and
  // kept for source compatibility (this library sizes its own launches)
  int MPnum = 0, THnum1D = 0, THnum1DX = 0, THnum2D = 0;
  uint32_t threadsMax = 0, maxGrid = 0;
  uint32_t timestep = 0;

  cudaFrame() = default;
  virtual ~cudaFrame() = default;

  void ErrorInfo(const std::string &s) const {
    (void)s;  // library calls report their own errors
  }

  // LAMMPS dump of the staged positions and type ids (cudaFrame.cu:34-83).
  // Written before the call returns; waitPutTMP() is kept for compatibility.
  void putTMP(std::ostream &o = std::cout) {
    std::lock_guard<std::mutex> lk(mutTMP);
    std::cerr << "output in TMPthread: " << timestep << " elapsed " << (time(nullptr) - starttime)
              << " sec" << std::endl;
    const uint32_t n = (uint32_t)TMP2.size();
    o << "ITEM: TIMESTEP" << std::endl << timestep << std::endl
      << "ITEM: NUMBER OF ATOMS" << std::endl << n << std::endl
      << "ITEM: BOX BOUNDS" << std::endl
      << cell[0] << " " << cell[1] << std::endl
      << cell[2] << " " << cell[3] << std::endl
      << cell[4] << " " << cell[5] << std::endl
      << "ITEM: ATOMS id type x y z" << additionalTag() << std::endl;
    for (uint32_t i = 0; i < n; ++i) {
      o << i << "  " << TMP2[i] << " ";
      if (TMP.size() >= 4 * (size_t)n)
        o << TMP[i * 4] << " " << TMP[i * 4 + 1] << " " << TMP[i * 4 + 2];
      o << additionalOutput(i) << std::endl;
    }
  }

  void waitPutTMP(void) { std::lock_guard<std::mutex> lk(mutTMP); }

  // cudaFrame::setCell (cudaFrame.cu:85-91)
  virtual void setCell(real *_cell) {
    for (int i = 0; i < 6; ++i) cell[i] = _cell[i];
    for (int i = 0; i < 3; ++i) {
      cell[i + 6] = (cell[i * 2 + 1] - cell[i * 2]) / 2;
      cell[i + 6] *= cell[i + 6];
    }
  }

  // the box as setCell stored it: xmin, xmax, ymin, ymax, zmin, zmax, (L/2)^2 x 3
  const real *cellData(void) const { return cell; }

  virtual std::string additionalTag(void) const { return ""; }
  virtual std::string additionalOutput(uint32_t) const { return ""; }

 protected:
  void frame_save(std::ostream &o) const {
    for (int i = 0; i < 9; ++i) pb_shim::put(o, cell[i]);
    pb_shim::put(o, timestep);
  }
  void frame_load(std::istream &in) {
    for (int i = 0; i < 9; ++i) pb_shim::get(in, cell[i]);
    pb_shim::get(in, timestep);
  }
};

#endif /* CUDAFRAME */
