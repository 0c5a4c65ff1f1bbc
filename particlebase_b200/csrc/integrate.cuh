// Time integration and reductions for one system (particle order).
#pragma once

#include "common.cuh"

namespace pb {

// Device-resident scalars of one system.  Reductions are finished on the
// device (last-block pattern), so a step never needs a host round trip.
struct DevScalars {
  double xi_old;      // Gaussian friction used by the current step's A term
  double xi_new;      // friction solved this step
  double sum_fa;      // sum F . A
  double sum_ma2;     // sum m A^2
  double mv2;         // sum m v^2 after the last update
  double pe, pe_shift, virial;   // from the last force call with energy
  double vstat[6];    // sum v, sum v^2 per axis (adjustVelocities)
  double fv;          // sum F . v (constTemp)
  double npairs;      // ordered pairs inside the cutoff (last force with energy)
  unsigned int counter[4];
};

struct IntegrateArgs {
  float4 *r;
  float4 *v;          // FP32 velocities (nullptr when vd is used)
  double *vd;         // FP64 velocities, SoA planes x[N], y[N], z[N]
  const float4 *F;    // F(t)
  const float4 *Fold; // F(t - dt)
  const float *minv;
  const float *mass;
  uint32_t N;
  float dt;
  float c0[3], c1[3], L[3];  // box for the wrap
  int wrap;
  DevScalars *sc;
  double *partials;   // >= 8 doubles per block
  uint32_t *status;   // status bits (non-finite sums)
};

cudaError_t launch_vv(const IntegrateArgs &a, cudaStream_t s);
cudaError_t launch_gauss(const IntegrateArgs &a, cudaStream_t s);
cudaError_t launch_wrap(const IntegrateArgs &a, cudaStream_t s);
cudaError_t launch_mv2(const IntegrateArgs &a, cudaStream_t s);
cudaError_t launch_fv(const IntegrateArgs &a, cudaStream_t s);
cudaError_t launch_scale(const IntegrateArgs &a, double factor, cudaStream_t s);
cudaError_t launch_adjust(const IntegrateArgs &a, double v1, cudaStream_t s);
cudaError_t launch_energy_total(const double *partials, uint32_t nparts, DevScalars *sc,
                                cudaStream_t s);
uint32_t integrate_blocks(uint32_t N);

}  // namespace pb
