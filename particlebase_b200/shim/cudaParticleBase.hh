// cudaParticleBase (cudaParticleBase.hh:29-226): one particle system on the
// GPU.  Here it owns a pb_md handle; the device arrays live in the library.
#if !defined(CUDAPARTICLEBASE)
#define CUDAPARTICLEBASE

#include <cstring>
#include <vector>

#include "ParticleBase.hh"
#include "cudaFrame.hh"

static_assert(sizeof(ParticleBase) == sizeof(pb_particle), "ParticleBase layout");

class cudaParticleBase : public virtual cudaFrame {
 protected:
  pb_md *h = nullptr;
  uint32_t N = 0;
  bool cell_set = false;

  // creation flags of the handle (GaussianThermo keeps FP64 velocities)
  virtual uint32_t handle_flags(void) const { return 0; }

  void need(const char *what) const {
    if (!h) {
      std::cerr << "particlebase_b200: " << what << " before setup()" << std::endl;
      std::exit(1);
    }
  }

 public:
  cudaParticleBase() = default;
  cudaParticleBase(const cudaParticleBase &) = delete;
  cudaParticleBase &operator=(const cudaParticleBase &) = delete;
  virtual ~cudaParticleBase() {
    if (h) pb_md_destroy(h);
  }

  // cudaParticleBase::setup (cudaParticleBase.cu:18-66)
  virtual void setup(int n) {
    if (h) pb_md_destroy(h);
    h = nullptr;
    N = (uint32_t)n;
    pb_shim::check(pb_md_create(N, handle_flags(), &h), "setup", nullptr);
    if (cell_set) pb_shim::check(pb_md_set_cell(h, cell), "setCell", h);
  }

  void setCell(real *_cell) override {
    cudaFrame::setCell(_cell);
    cell_set = true;
    if (h) pb_shim::check(pb_md_set_cell(h, cell), "setCell", h);
  }

  // cudaParticleBase::import (cudaParticleBase.cu:68-117)
  virtual void import(const std::vector<ParticleBase> &P) {
    need("import");
    pb_shim::check(pb_md_import(h, reinterpret_cast<const pb_particle *>(P.data()),
                                (uint32_t)P.size()),
                   "import", h);
  }

  // getPosition / getForce / getTypeID (cudaParticleBase.cu:119-149): stage
  // the array in TMP / TMP2 for putTMP()
  void getPosition(void) {
    need("getPosition");
    std::lock_guard<std::mutex> lk(mutTMP);
    TMP.resize(4 * (size_t)N);
    pb_shim::check(pb_md_get(h, PB_FIELD_R, &TMP[0], 16 * (size_t)N), "getPosition", h);
  }
  void getForce(void) {
    need("getForce");
    std::lock_guard<std::mutex> lk(mutTMP);
    TMP.resize(4 * (size_t)N);
    pb_shim::check(pb_md_get(h, PB_FIELD_F, &TMP[0], 16 * (size_t)N), "getForce", h);
  }
  void getTypeID(void) {
    need("getTypeID");
    std::lock_guard<std::mutex> lk(mutTMP);
    TMP2.resize(N);
    pb_shim::check(pb_md_get(h, PB_FIELD_TYPE, &TMP2[0], 2 * (size_t)N), "getTypeID", h);
  }

  // cudaParticleBase::treatPeriodicCondition (cudaParticleBase.cu:175-184)
  void treatPeriodicCondition(void) {
    need("treatPeriodicCondition");
    pb_shim::check(pb_md_wrap(h), "treatPeriodicCondition", h);
  }

  uint32_t size(void) const { return N; }
  pb_md *handle(void) const { return h; }
};

#endif /* CUDAPARTICLEBASE */
