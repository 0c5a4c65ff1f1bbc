// cudaParticleVV (cudaParticleVV.hh:14-57): velocity Verlet.
#if !defined(CUDAPARTICLEVV)
#define CUDAPARTICLEVV

#include "cudaParticleBase.hh"

class cudaParticleVV : public virtual cudaParticleBase {
 public:
  // F = Fold = 0 (cudaParticleVV.cu:10-15)
  void clearForce(void) {
    need("clearForce");
    pb_shim::check(pb_md_clear_force(h), "clearForce", h);
  }

  // propagateVelocityVerlet_F4 (cudaParticleVV.cu:17-34)
  virtual void TimeEvolution(real dt) {
    need("TimeEvolution");
    pb_shim::check(pb_md_step_vv(h, dt), "TimeEvolution", h);
  }
};

#endif /* CUDAPARTICLEVV */
