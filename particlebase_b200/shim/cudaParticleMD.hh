// cudaParticleMD (cudaParticleMD.hh:32-194): Lennard-Jones MD over the cell
// list.  The public fields kB and rmax2 are plain members, as in the
// reference, and reach the library before the next call that uses them.
#if !defined(CUDAPARTICLEMD)
#define CUDAPARTICLEMD

#include <cmath>
#include <istream>
#include <ostream>
#include <vector>

#include "cudaCutoffBlock.hh"
#include "cudaParticleVV.hh"
#include "cudaSortedPositions.hh"

class cudaParticleMD : public cudaParticleVV,
                       public virtual cudaCutoffBlock,
                       public virtual cudaSortedPositions {
 protected:
  real m0 = 1;       // mean particle mass
  bool useNlist = false;
  real pushed_kB = -1, pushed_rmax2 = -1;

  // kB and rmax2 are public fields: send the values the caller last wrote
  void sync_params(void) {
    if (kB != pushed_kB && kB > 0) {
      pb_shim::check(pb_md_set_kB(h, kB), "kB", h);
      pushed_kB = kB;
    }
    if (rmax2 != pushed_rmax2 && rmax2 > 0) {
      pb_shim::check(pb_md_set_rmax2(h, rmax2), "rmax2", h);
      pushed_rmax2 = rmax2;
    }
  }
  void before_cells(void) override { sync_params(); }

 public:
  real mv2 = 0.0;     // cached value of the last calcMV2()
  real kB = 1;        // Boltzmann constant in simulation units
  real rmax2 = 0;     // square of the LJ cutoff
  real thickness = 0; // neighbour-list skin: list radius sqrt(rmax2) + thickness

  void setup(int n) override {
    cudaParticleBase::setup(n);
    pushed_kB = pushed_rmax2 = -1;
  }

  // cudaParticleMD::calcForce (cudaParticleMD.cu:24-69)
  void calcForce(void) {
    need("calcForce");
    sync_params();
    pb_shim::check(pb_md_force(h, 0), "calcForce", h);
  }

  // m = 1/minv is computed at import (cudaParticleMD.cu:135-138)
  void setM(void) {}

  void import(const std::vector<ParticleBase> &P) override {
    cudaParticleBase::import(P);
    double m = 1;
    pb_md_mean_mass(h, &m);
    m0 = (real)m;
  }

  // sum m v^2 (cudaParticleMD.cu:124-133), accumulated in FP64
  virtual real calcMV2(void) {
    need("calcMV2");
    sync_params();
    double T = 0;
    pb_shim::check(pb_md_temperature(h, &T), "calcMV2", h);
    return (real)(T * 3.0 * N * (double)kB);
  }

  real calcTemp(void) {
    mv2 = calcMV2();
    return mv2 / (N * 3 * kB);
  }

  // sum_{i<j} 4 eps [(s/r)^12 - (s/r)^6] over pairs inside the cutoff at the
  // positions of the last calcBlockID (cudaParticleMD.cu:71-122 computes the
  // same quantity with an assignment where a sum is meant)
  real calcPotentialE(void) {
    need("calcPotentialE");
    sync_params();
    pb_shim::check(pb_md_force(h, PB_FORCE_ENERGY), "calcPotentialE", h);
    pb_md_sums s;
    pb_shim::check(pb_md_reduce(h, &s), "calcPotentialE", h);
    return (real)s.pe;
  }

  real calcKineticE(void) const { return mv2 / 2.0; }

  // cudaParticleMD::constTemp (cudaParticleMD.cu:140-155):
  // lambda = sum F.v / sum m v^2, F -= lambda m v; returns the temperature
  real constTemp(void) {
    need("constTemp");
    sync_params();
    pb_md_sums s;
    pb_shim::check(pb_md_reduce(h, &s), "constTemp", h);
    const real t = (real)s.mv2;
    const double lambda = s.mv2 > 0 ? s.fv / s.mv2 : 0.0;
    std::cerr << "[l=" << (real)lambda << "]";
    if (lambda != 0) pb_shim::check(pb_md_correct_force(h, lambda), "constTemp", h);
    return t / (3 * N * kB);
  }

  // cudaParticleMD::scaleTemp (cudaParticleMD.cu:168-175)
  virtual real scaleTemp(real Temp) {
    const real T0 = calcTemp();
    const real s = std::sqrt(static_cast<real>(3 * N - 1) / static_cast<real>(3 * N) * Temp / T0);
    pb_shim::check(pb_md_scale_velocities(h, s), "scaleTemp", h);
    return s;
  }

  // cudaParticleMD::adjustVelocities (cudaParticleMD.cu:177-198)
  virtual void adjustVelocities(real Temp, bool debug = false) {
    need("adjustVelocities");
    const real v1 = std::sqrt(kB * Temp / m0);
    if (debug)
      std::cerr << std::endl << std::endl << "adjustVelocity currentTemp\t" << calcTemp()
                << "\tTarget Temp " << Temp << std::endl;
    pb_shim::check(pb_md_adjust_velocities(h, v1), "adjustVelocities", h);
    if (debug) std::cerr << "after adjusted T=" << calcTemp() << std::endl;
  }

  // cudaParticleMD::setLJparams (cudaParticleMD.cu:200-202)
  void setLJparams(const std::vector<real> &p, uint32_t elemnum) {
    need("setLJparams");
    sync_params();
    std::vector<float> q(p.begin(), p.end());
    pb_shim::check(pb_md_set_lj(h, q.data(), elemnum), "setLJparams", h);
  }

  // cudaParticleMD::initialAnnealing (cudaParticleMD.cu:205-325): anealstep
  // Euler steps under a soft-core repulsion whose range grows to _rc, each
  // with the constTemp force correction, a temperature rescale, then anealstep
  // velocity-Verlet LJ steps with constTemp, and a final rescale.
  void initialAnnealing(uint32_t anealstep, real dt, real _rc, real _f0, real T) {
    need("initialAnnealing");
    sync_params();
    std::cerr << "performs initial annealing by soft core potential to rmax= " << _rc
              << " with steps " << anealstep << std::endl;
    for (uint32_t i = 0; i < anealstep; ++i) {
      const real rc = _rc * (i + 1) / anealstep;
      std::cerr << "\r" << rc << "\t" << std::flush;
      calcBlockID();
      pb_shim::check(pb_md_force_softcore(h, rc, _f0), "initialAnnealing", h);
      constTemp();
      pb_shim::check(pb_md_step_euler(h, dt), "initialAnnealing", h);
      std::cerr << "T= " << calcTemp() << std::flush;
    }
    std::cerr << std::endl;
    std::cerr << "temperature scaling: " << scaleTemp(T) << std::endl;
    std::cerr << "with LJ " << std::endl;
    clearForce();  // Fold = 0 before the LJ stage
    for (uint32_t i = 0; i < anealstep; ++i) {
      std::cerr << i << "\t" << calcTemp() << "\t";
      calcBlockID();
      calcForce();
      std::cerr << constTemp() << std::endl;
      pb_shim::check(pb_md_step_vv(h, dt), "initialAnnealing", h);
      treatPeriodicCondition();
    }
    std::cerr << "temperature scaling: " << scaleTemp(T) << std::endl;
  }

  // per-particle m v^2, one line each (cudaParticleMD.cu:157-166)
  void statMV2(std::ostream &o = std::cout) {
    need("statMV2");
    calcMV2();
    std::vector<float> m(N);
    pb_shim::check(pb_md_get(h, PB_FIELD_MASS, m.data(), 4 * (size_t)N), "statMV2", h);
    std::vector<double> v2(N);
    if (handle_flags() & PB_MD_VEL_FP64) {
      std::vector<double> vd(3 * (size_t)N);
      pb_shim::check(pb_md_get(h, PB_FIELD_VD, vd.data(), 24 * (size_t)N), "statMV2", h);
      for (uint32_t i = 0; i < N; ++i)
        v2[i] = vd[i] * vd[i] + vd[N + i] * vd[N + i] + vd[2 * (size_t)N + i] * vd[2 * (size_t)N + i];
    } else {
      std::vector<float> v(4 * (size_t)N);
      pb_shim::check(pb_md_get(h, PB_FIELD_V, v.data(), 16 * (size_t)N), "statMV2", h);
      for (uint32_t i = 0; i < N; ++i)
        v2[i] = (double)v[4 * i] * v[4 * i] + (double)v[4 * i + 1] * v[4 * i + 1] +
                (double)v[4 * i + 2] * v[4 * i + 2];
    }
    std::lock_guard<std::mutex> lk(mutTMP);
    o << std::endl << std::endl;
    for (uint32_t i = 0; i < N; ++i) o << i << "\t" << (real)(m[i] * v2[i]) << std::endl;
  }

  // Neighbour lists (cudaParticleMD.hh:167-179, cudaParticleMD.cu:338-394):
  // useNList switches force calls to a Verlet list of the atoms within
  // sqrt(rmax2) + thickness; makeNList rebuilds the cell list and that list,
  // with the thickness set at the time of the call.
  void useNList(void) { useNlist = true; }
  void makeNList(void) {
    if (!useNlist) return;
    need("makeNList");
    sync_params();
    pb_shim::check(pb_md_use_nlist(h, thickness), "useNList", h);
    pb_shim::check(pb_md_make_nlist(h), "makeNList", h);
  }

  // checkpoint: frame, particle arrays, cell grid, kB, rmax2
  virtual void pb_save(std::ostream &o) const {
    need("save");
    const uint32_t magic = 0x4b434250u;  // "PBCK"
    pb_shim::put(o, magic);
    pb_shim::put(o, handle_flags());
    frame_save(o);
    pb_shim::put(o, N);
    std::vector<float> r(4 * (size_t)N), F(4 * (size_t)N), Fo(4 * (size_t)N), minv(N);
    std::vector<uint16_t> type(N);
    pb_md_get(h, PB_FIELD_R, r.data(), 16 * (size_t)N);
    pb_md_get(h, PB_FIELD_F, F.data(), 16 * (size_t)N);
    pb_md_get(h, PB_FIELD_FOLD, Fo.data(), 16 * (size_t)N);
    pb_md_get(h, PB_FIELD_MINV, minv.data(), 4 * (size_t)N);
    pb_md_get(h, PB_FIELD_TYPE, type.data(), 2 * (size_t)N);
    pb_shim::put_vec(o, r);
    pb_shim::put_vec(o, F);
    pb_shim::put_vec(o, Fo);
    pb_shim::put_vec(o, minv);
    pb_shim::put_vec(o, type);
    if (handle_flags() & PB_MD_VEL_FP64) {
      std::vector<double> vd(3 * (size_t)N);
      pb_md_get(h, PB_FIELD_VD, vd.data(), 24 * (size_t)N);
      pb_shim::put_vec(o, vd);
    } else {
      std::vector<float> v(4 * (size_t)N);
      pb_md_get(h, PB_FIELD_V, v.data(), 16 * (size_t)N);
      pb_shim::put_vec(o, v);
    }
    pb_shim::put(o, rmax_cells);
    pb_shim::put(o, periodic_cells);
    pb_shim::put(o, kB);
    pb_shim::put(o, rmax2);
    pb_shim::put(o, m0);
  }

  virtual void pb_load(std::istream &in) {
    uint32_t magic = 0, flags = 0, n = 0;
    pb_shim::get(in, magic);
    pb_shim::get(in, flags);
    if (magic != 0x4b434250u || flags != handle_flags()) {
      std::cerr << "particlebase_b200: not a checkpoint of this class" << std::endl;
      std::exit(1);
    }
    frame_load(in);
    pb_shim::get(in, n);
    setup((int)n);
    pb_shim::check(pb_md_set_cell(h, cell), "load", h);
    cell_set = true;
    std::vector<float> r, F, Fo, minv;
    std::vector<uint16_t> type;
    pb_shim::get_vec(in, r);
    pb_shim::get_vec(in, F);
    pb_shim::get_vec(in, Fo);
    pb_shim::get_vec(in, minv);
    pb_shim::get_vec(in, type);
    pb_shim::check(pb_md_set(h, PB_FIELD_R, r.data(), 4 * r.size()), "load", h);
    pb_shim::check(pb_md_set(h, PB_FIELD_F, F.data(), 4 * F.size()), "load", h);
    pb_shim::check(pb_md_set(h, PB_FIELD_FOLD, Fo.data(), 4 * Fo.size()), "load", h);
    pb_shim::check(pb_md_set(h, PB_FIELD_MINV, minv.data(), 4 * minv.size()), "load", h);
    pb_shim::check(pb_md_set(h, PB_FIELD_TYPE, type.data(), 2 * type.size()), "load", h);
    if (flags & PB_MD_VEL_FP64) {
      std::vector<double> vd;
      pb_shim::get_vec(in, vd);
      pb_shim::check(pb_md_set(h, PB_FIELD_VD, vd.data(), 8 * vd.size()), "load", h);
    } else {
      std::vector<float> v;
      pb_shim::get_vec(in, v);
      pb_shim::check(pb_md_set(h, PB_FIELD_V, v.data(), 4 * v.size()), "load", h);
    }
    pb_shim::get(in, rmax_cells);
    pb_shim::get(in, periodic_cells);
    pb_shim::get(in, kB);
    pb_shim::get(in, rmax2);
    pb_shim::get(in, m0);
    if (!in) {
      std::cerr << "particlebase_b200: truncated checkpoint" << std::endl;
      std::exit(1);
    }
    sync_params();
    if (rmax_cells > 0)
      pb_shim::check(pb_md_setup_cells(h, rmax_cells, periodic_cells ? 1 : 0), "load", h);
  }
};

#endif /* CUDAPARTICLEMD */
