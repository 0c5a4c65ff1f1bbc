// cudaCalcGR (cudaCalcGR.hh:9-69, cudaCalcGR.cu:1-145): radial distribution
// function of a particle system, over every pair of its atoms.  The pair
// counts come from pb_md_gr on the system's own device positions; the
// normalisation of igr2gr and the text of getGr are the reference's.
#if !defined(CUDACALCGR)
#define CUDACALCGR

#include <cmath>
#include <cstdint>
#include <iostream>
#include <vector>

#include "cudaFrame.hh"
#include "cudaParticleMD.hh"

class cudaCalcGR : public cudaFrame {
 public:
  cudaCalcGR() = default;
  virtual ~cudaCalcGR() = default;

  // cudaCalcGR::setup (cudaCalcGR.hh:27-40): bin width and range
  void setup(const real rstep, const real rmax) {
    rstep_ = rstep;
    rmax_ = rmax;
    rstepinv = 1.0 / rstep;
    rnum = static_cast<uint32_t>(rmax * rstepinv);
    igr.assign(rnum, 0);
    gr.assign(rnum, 0);
    TMP.resize(rnum);
  }

  void copyCell(const cudaParticleMD &P) {
    const real *c = P.cellData();
    real c6[6];
    for (int i = 0; i < 6; ++i) c6[i] = c[i];
    setCell(c6);
  }

  // every pair is counted directly: no pair list to prepare
  void makePairInfo(const cudaParticleMD &) {}

  void cleargr(void) { std::fill(igr.begin(), igr.end(), 0); }

  // cudaCalcGR::calcgr (cudaCalcGR.cu:85-116): add this configuration's pair
  // counts to igr
  void calcgr(const cudaParticleMD &part) {
    uint32_t n = 0;
    pb_shim::check(pb_md_gr(part.handle(), rstep_, rmax_, nullptr, &n), "calcgr", part.handle());
    std::vector<uint64_t> c(n);
    pb_shim::check(pb_md_gr(part.handle(), rstep_, rmax_, c.data(), &n), "calcgr",
                   part.handle());
    for (uint32_t k = 0; k < n && k < rnum; ++k) igr[k] += c[k];
  }

  // cudaCalcGR::igr2gr (cudaCalcGR.cu:118-136): g_j = igr_j Q / (4 j^2 + 1/3)
  // with Q = 2 / N / (pi rstep^3) * V / N, the shell of (j - 1/2, j + 1/2) rstep
  void igr2gr(const cudaParticleMD &part) {
    const real *c = part.cellData();
    const real N = (real)part.size();
    const real rhoinv = (c[1] - c[0]) * (c[3] - c[2]) * (c[5] - c[4]) / N;
    const real Vinv = M_1_PI * rstepinv * rstepinv * rstepinv;
    const real Q = 2.0 / N * Vinv * rhoinv;
    const real onethird = 1.0 / 3.0;
    for (uint32_t j = 1; j < rnum; ++j) gr[j] = (real)igr[j] * Q / (4 * j * j + onethird);
    if (rnum) gr[0] = 0;
  }

  // cudaCalcGR::getGr (cudaCalcGR.cu:138-145): "r  g(r)" per bin
  void getGr(std::ostream &o = std::cout) {
    for (uint32_t i = 0; i < rnum; ++i) {
      const real r = i / rstepinv;
      o << r << "  " << gr[i] << std::endl;
    }
  }

 private:
  real rstep_ = 0, rmax_ = 0, rstepinv = 0;
  uint32_t rnum = 0;
  std::vector<uint64_t> igr;
  std::vector<real> gr;
};

#endif /* CUDACALCGR */
