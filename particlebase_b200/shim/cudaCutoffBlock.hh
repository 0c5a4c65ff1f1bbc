// cudaCutoffBlock (cudaCutoffBlock.hh:28-133): the cell list.
#if !defined(CUDACUTOFFBLOCK)
#define CUDACUTOFFBLOCK

#include "cudaParticleBase.hh"

class cudaCutoffBlock : public virtual cudaParticleBase {
 protected:
  real rmax_cells = 0;  // rmax of the last setupCutoffBlock (0: none yet)
  bool periodic_cells = true;

 public:
  void setupCutoffBlock(real rmax, bool periodic = true) {
    need("setupCutoffBlock");
    before_cells();
    pb_shim::check(pb_md_setup_cells(h, rmax, periodic ? 1 : 0), "setupCutoffBlock", h);
    rmax_cells = rmax;
    periodic_cells = periodic;
  }

  void calcBlockID(void) {
    need("calcBlockID");
    pb_shim::check(pb_md_build_cells(h), "calcBlockID", h);
  }

  uint32_t numBlocks(void) const {
    uint32_t c = 0;
    if (h) pb_md_grid(h, nullptr, nullptr, &c);
    return c;
  }

  // cudaCutoffBlock::setBlockRange (cudaCutoffBlock.hh:54-70): the range of
  // cells one GPU handles.  One GPU handles all of them.
  void setBlockRange(uint32_t blocknum, uint32_t N_GPU, uint32_t thisGPU) {
    if (N_GPU != 1 || thisGPU != 0 || blocknum != numBlocks()) {
      std::cerr << "particlebase_b200: setBlockRange supports one GPU with all cells" << std::endl;
      std::exit(1);
    }
  }

 protected:
  virtual void before_cells(void) {}
};

#endif /* CUDACUTOFFBLOCK */
