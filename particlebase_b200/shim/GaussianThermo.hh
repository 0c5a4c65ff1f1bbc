// GaussianThermo (GaussianThermo.hh:14-90): isokinetic velocity Verlet with
// FP64 velocities.
#if !defined(GAUSSIANTHERMO)
#define GAUSSIANTHERMO

#include "cudaParticleMD.hh"

class GaussianThermo : public virtual cudaParticleMD {
 protected:
  double xi = 0;  // friction of the last step (kept on the device)
  real _e = 1e-8; // Newton-Raphson tolerance of the reference (solved in closed form here)

  uint32_t handle_flags(void) const override { return PB_MD_VEL_FP64; }

 public:
  GaussianThermo() = default;

  void setup(int n) override { cudaParticleMD::setup(n); }

  // GaussianThermo::TimeEvolution (GaussianThermo.cu:29-77)
  void TimeEvolution(real dt) override {
    need("TimeEvolution");
    pb_shim::check(pb_md_step_gauss(h, dt, _e), "TimeEvolution", h);
  }

  void setE(real _e0) { _e = _e0; }

  void pb_save(std::ostream &o) const override {
    cudaParticleMD::pb_save(o);
    pb_md_sums s;
    pb_md_reduce(h, &s);
    pb_shim::put(o, s.xi);
    pb_shim::put(o, _e);
  }

  void pb_load(std::istream &in) override {
    cudaParticleMD::pb_load(in);
    pb_shim::get(in, xi);
    pb_shim::get(in, _e);
    pb_shim::check(pb_md_set_xi(h, xi), "load", h);
  }
};

#endif /* GAUSSIANTHERMO */
