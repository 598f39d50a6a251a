// integrate.cuh -- integrator helpers shared by the free functions
// (integrate.cu) and the scheduler (scheduler.cu).
#pragma once

#include "common.cuh"

namespace tdmd_b200 {

constexpr int kMaxChain = 16;

// Single-image wrap of fused_kick_drift_kernel
// (src/integrator/device_velocity_verlet.cu:111-122): one shift of L, bound
// written as lo + L exactly as the reference does.
__device__ __forceinline__ double wrap_single(double p, double lo, double L, int periodic) {
  if (periodic) {
    if (p < lo)
      p += L;
    else if (p >= lo + L)
      p -= L;
  }
  return p;
}

// --------------------------------------------------------------------------
// Nose-Hoover chain half step, NoseHooverChain::half_step
// (src/integrator/device_nose_hoover.cu:206-289): masses refreshed from the
// target temperature, chain integrated from the outermost thermostat inward
// with exp(-v_{k+1} dt/8) factors around each update, returns the velocity
// scale exp(-v_0 dt/2).  Runs on the host (tdmd_nhc) and on the device (the
// scheduler's control kernel).
// --------------------------------------------------------------------------
inline __host__ __device__ double nhc_half_step(double* eta, double* eta_v, double* eta_m, int M,
                                                double t_target, double t_period, int n_dof,
                                                double dt, double ke) {
  if (M <= 0) return 1.0;
  const double half_dt = 0.5 * dt;
  const double kt = kBoltzmann * t_target;
  const double tau2 = t_period * t_period;
  const double ke_target = 0.5 * static_cast<double>(n_dof) * kBoltzmann * t_target;
  eta_m[0] = static_cast<double>(n_dof) * kt * tau2;
  for (int k = 1; k < M; ++k) eta_m[k] = kt * tau2;
  if (M > 1) {
    const int last = M - 1;
    const double g =
        (eta_m[last - 1] * eta_v[last - 1] * eta_v[last - 1] - kBoltzmann * t_target) / eta_m[last];
    eta_v[last] += g * half_dt;
  }
  for (int k = M - 2; k >= 1; --k) {
    const double ef = exp(-eta_v[k + 1] * half_dt / 4.0);
    eta_v[k] *= ef;
    const double g = (eta_m[k - 1] * eta_v[k - 1] * eta_v[k - 1] - kBoltzmann * t_target) / eta_m[k];
    eta_v[k] += g * half_dt;
    eta_v[k] *= ef;
  }
  {
    const double ef = M > 1 ? exp(-eta_v[1] * half_dt / 4.0) : 1.0;
    eta_v[0] *= ef;
    const double g0 = (2.0 * ke - 2.0 * ke_target) / eta_m[0];
    eta_v[0] += g0 * half_dt;
    eta_v[0] *= ef;
  }
  const double scale = exp(-eta_v[0] * half_dt);
  for (int k = 0; k < M; ++k) eta[k] += eta_v[k] * half_dt;
  return scale;
}

void nhc_init(double* eta, double* eta_v, double* eta_m, int M, double t_target, double t_period,
              int n_dof);

__global__ void k_ke_vmax_partials(const double* __restrict__ v, const int* __restrict__ types,
                                   const double* __restrict__ masses, int n,
                                   double* __restrict__ partials);
__global__ void k_ke_vmax_finish(const double* __restrict__ partials, int nblk,
                                 double* __restrict__ out);

}  // namespace tdmd_b200
