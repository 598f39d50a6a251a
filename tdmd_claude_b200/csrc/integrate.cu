// integrate.cu -- velocity-Verlet kernels on the reference's array layouts,
// FP64 reductions (kinetic energy, v_max) and the Nose-Hoover chain.
//
// Reference: src/integrator/device_velocity_verlet.cu:14-198 (half kick,
// drift, fused kick+drift with the single-image wrap, zero forces) and
// src/integrator/device_nose_hoover.cu:24-289 (KE / v_max block reductions
// finished on the host, velocity scaling, NoseHooverChain).  Here every
// reduction finishes on the device in a fixed order (no atomics, no host
// partial sums).
#include <cmath>
#include <vector>

#include "buffers.cuh"
#include "common.cuh"
#include "integrate.cuh"

namespace tdmd_b200 {

namespace {

template <class F>
__global__ void k_half_kick(double* __restrict__ v, const F* __restrict__ f,
                            const int* __restrict__ types, const double* __restrict__ masses,
                            int n, double half_dt) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double factor = half_dt / (masses[types[i]] * kMvv2e);
#pragma unroll
  for (int a = 0; a < 3; ++a) v[3ll * i + a] += factor * static_cast<double>(f[3ll * i + a]);
}

__global__ void k_drift(double* __restrict__ x, const double* __restrict__ v, int n, double dt,
                        DevBox b) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double p = x[3ll * i + a] + dt * v[3ll * i + a];
    x[3ll * i + a] = wrap_single(p, b.lo[a], b.L[a], b.periodic[a]);
  }
}

template <class F, bool FULL>
__global__ void k_fused_kick_drift(double* __restrict__ v, double* __restrict__ x,
                                   const F* __restrict__ f, const int* __restrict__ types,
                                   const double* __restrict__ masses, int n, double dt, DevBox b) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double kick_dt = FULL ? dt : 0.5 * dt;
  const double factor = kick_dt / (masses[types[i]] * kMvv2e);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double vv = v[3ll * i + a] + factor * static_cast<double>(f[3ll * i + a]);
    v[3ll * i + a] = vv;
    x[3ll * i + a] = wrap_single(x[3ll * i + a] + dt * vv, b.lo[a], b.L[a], b.periodic[a]);
  }
}

template <class F>
__global__ void k_zero(F* __restrict__ f, long long m) {
  dependent_launch_prologue();
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < m) f[i] = F(0);
}

__global__ void k_scale(double* __restrict__ v, long long m, double s) {
  dependent_launch_prologue();
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < m) v[i] *= s;
}

}  // namespace

// KE = sum 1/2 m mvv2e |v|^2 and max |v|^2 per block -> partials[b*2 + {0,1}].
__global__ void k_ke_vmax_partials(const double* __restrict__ v, const int* __restrict__ types,
                                   const double* __restrict__ masses, int n,
                                   double* __restrict__ partials) {
  dependent_launch_prologue();
  __shared__ double red[32 * 2];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double ke = 0.0, v2 = 0.0;
  if (i < n) {
    const double vx = v[3ll * i], vy = v[3ll * i + 1], vz = v[3ll * i + 2];
    v2 = vx * vx + vy * vy + vz * vz;
    ke = 0.5 * masses[types[i]] * kMvv2e * v2;
  }
  ke = warp_sum(ke);
  v2 = warp_max(v2);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[2 * warp] = ke;
    red[2 * warp + 1] = v2;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    ke = lane < nw ? red[2 * lane] : 0.0;
    v2 = lane < nw ? red[2 * lane + 1] : 0.0;
    ke = warp_sum(ke);
    v2 = warp_max(v2);
    if (lane == 0) {
      partials[2ll * blockIdx.x] = ke;
      partials[2ll * blockIdx.x + 1] = v2;
    }
  }
}

// Sums/maxes nblk (ke, v2) records in block order -> out[0] = KE,
// out[1] = max |v|^2.
__global__ void k_ke_vmax_finish(const double* __restrict__ partials, int nblk,
                                 double* __restrict__ out) {
  dependent_launch_prologue();
  __shared__ double red[32 * 2];
  double ke = 0.0, v2 = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    ke += partials[2ll * b];
    v2 = fmax(v2, partials[2ll * b + 1]);
  }
  ke = warp_sum(ke);
  v2 = warp_max(v2);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[2 * warp] = ke;
    red[2 * warp + 1] = v2;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    ke = lane < nw ? red[2 * lane] : 0.0;
    v2 = lane < nw ? red[2 * lane + 1] : 0.0;
    ke = warp_sum(ke);
    v2 = warp_max(v2);
    if (lane == 0) {
      out[0] = ke;
      out[1] = v2;
    }
  }
}

void nhc_init(double* eta, double* eta_v, double* eta_m, int M, double t_target, double t_period,
              int n_dof) {
  const double kt = kBoltzmann * t_target;
  const double tau2 = t_period * t_period;
  for (int k = 0; k < M; ++k) {
    eta[k] = 0.0;
    eta_v[k] = 0.0;
    eta_m[k] = k == 0 ? static_cast<double>(n_dof) * kt * tau2 : kt * tau2;
  }
}

}  // namespace tdmd_b200

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace tdmd_b200;

struct tdmd_nhc {
  double t_target, t_period, dt;
  int M, n_dof;
  std::vector<double> eta, eta_v, eta_m;
};

namespace {

constexpr int kThreads = 256;

template <class Fn>
int32_t with_forces(int32_t prec, const void* f, Fn&& fn) {
  if (prec == TDMD_FP64) return fn(static_cast<const double*>(f));
  if (prec == TDMD_MIXED) return fn(static_cast<const float*>(f));
  throw Error{TDMD_ERR_INVALID_ARGUMENT, "unknown force precision"};
}

void ke_vmax(const double* v, const int* types, const double* masses, int n, double* h2,
             cudaStream_t s) {
  const int nblk = ceil_div(n, kThreads);
  double* buf = nullptr;
  TDMD_CU(cudaMallocAsync(reinterpret_cast<void**>(&buf), sizeof(double) * (2ll * nblk + 2), s));
  launch(k_ke_vmax_partials, nblk, kThreads, 0, s, v, types, masses, n, buf);
  cudaError_t e1 = cudaGetLastError();
  launch(k_ke_vmax_finish, 1, 256, 0, s, buf, nblk, buf + 2ll * nblk);
  cudaError_t e2 = cudaGetLastError();
  cudaError_t e3 = cudaMemcpyAsync(h2, buf + 2ll * nblk, 2 * sizeof(double),
                                   cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(buf, s);
  TDMD_CU(e1);
  TDMD_CU(e2);
  TDMD_CU(e3);
  TDMD_CU(cudaStreamSynchronize(s));
}

}  // namespace

extern "C" {

int32_t tdmd_vv_half_kick(double* d_velocities, const void* d_forces, int32_t force_precision,
                          const int32_t* d_types, const double* d_masses, int32_t natoms,
                          double dt, void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(natoms >= 0, "natoms must be non-negative");
    if (natoms == 0) return;
    TDMD_REQUIRE(d_velocities && d_forces && d_types && d_masses, "null device array");
    with_forces(force_precision, d_forces, [&](auto f) {
      using F = std::remove_cv_t<std::remove_pointer_t<decltype(f)>>;
      launch(k_half_kick<F>, ceil_div(natoms, kThreads), kThreads, 0, as_stream(stream),
             d_velocities, f, d_types, d_masses, natoms, 0.5 * dt);
      TDMD_LAUNCH_CHECK();
      return 0;
    });
  });
}

int32_t tdmd_vv_drift(double* d_positions, const double* d_velocities, int32_t natoms, double dt,
                      const tdmd_box* box, void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(box && natoms >= 0, "bad arguments");
    if (natoms == 0) return;
    TDMD_REQUIRE(d_positions && d_velocities, "null device array");
    launch(k_drift, ceil_div(natoms, kThreads), kThreads, 0, as_stream(stream), d_positions,
           d_velocities, natoms, dt, make_devbox(*box, 0.0));
    TDMD_LAUNCH_CHECK();
  });
}

int32_t tdmd_vv_fused_kick_drift(double* d_velocities, double* d_positions, const void* d_forces,
                                 int32_t force_precision, const int32_t* d_types,
                                 const double* d_masses, int32_t natoms, double dt,
                                 const tdmd_box* box, int32_t full_kick, void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(box && natoms >= 0, "bad arguments");
    if (natoms == 0) return;
    TDMD_REQUIRE(d_velocities && d_positions && d_forces && d_types && d_masses,
                 "null device array");
    const DevBox b = make_devbox(*box, 0.0);
    with_forces(force_precision, d_forces, [&](auto f) {
      using F = std::remove_cv_t<std::remove_pointer_t<decltype(f)>>;
      if (full_kick)
        launch(k_fused_kick_drift<F, true>, ceil_div(natoms, kThreads), kThreads, 0,
               as_stream(stream), d_velocities, d_positions, f, d_types, d_masses, natoms, dt, b);
      else
        launch(k_fused_kick_drift<F, false>, ceil_div(natoms, kThreads), kThreads, 0,
               as_stream(stream), d_velocities, d_positions, f, d_types, d_masses, natoms, dt, b);
      TDMD_LAUNCH_CHECK();
      return 0;
    });
  });
}

int32_t tdmd_vv_zero_forces(void* d_forces, int32_t force_precision, int32_t natoms,
                            void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(natoms >= 0, "natoms must be non-negative");
    if (natoms == 0) return;
    TDMD_REQUIRE(d_forces, "null device array");
    const long long m = 3ll * natoms;
    if (force_precision == TDMD_FP64)
      launch(k_zero<double>, ceil_div(m, kThreads), kThreads, 0, as_stream(stream),
             static_cast<double*>(d_forces), m);
    else
      launch(k_zero<float>, ceil_div(m, kThreads), kThreads, 0, as_stream(stream),
             static_cast<float*>(d_forces), m);
    TDMD_LAUNCH_CHECK();
  });
}

int32_t tdmd_reduce_ke(const double* d_velocities, const int32_t* d_types,
                       const double* d_masses, int32_t natoms, double* h_ke, void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(h_ke && natoms >= 0, "bad arguments");
    *h_ke = 0.0;
    if (natoms == 0) return;
    TDMD_REQUIRE(d_velocities && d_types && d_masses, "null device array");
    double h2[2];
    ke_vmax(d_velocities, d_types, d_masses, natoms, h2, as_stream(stream));
    *h_ke = h2[0];
  });
}

int32_t tdmd_reduce_vmax(const double* d_velocities, int32_t natoms, double* h_vmax,
                         void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(h_vmax && natoms >= 0, "bad arguments");
    *h_vmax = 0.0;
    if (natoms == 0) return;
    TDMD_REQUIRE(d_velocities, "null device array");
    // Types/masses are not needed for |v|; reuse the fused kernel with a
    // unit mass table.
    const double one[2] = {1.0, 1.0};
    double* dm = nullptr;
    int* dt = nullptr;
    cudaStream_t s = as_stream(stream);
    TDMD_CU(cudaMallocAsync(reinterpret_cast<void**>(&dm), sizeof(one), s));
    TDMD_CU(cudaMallocAsync(reinterpret_cast<void**>(&dt), sizeof(int) * natoms, s));
    cudaError_t e1 = cudaMemcpyAsync(dm, one, sizeof(one), cudaMemcpyHostToDevice, s);
    cudaError_t e2 = cudaMemsetAsync(dt, 0, sizeof(int) * natoms, s);
    double h2[2] = {0, 0};
    if (e1 == cudaSuccess && e2 == cudaSuccess) ke_vmax(d_velocities, dt, dm, natoms, h2, s);
    cudaFreeAsync(dm, s);
    cudaFreeAsync(dt, s);
    TDMD_CU(e1);
    TDMD_CU(e2);
    TDMD_CU(cudaStreamSynchronize(s));
    *h_vmax = std::sqrt(h2[1]);
  });
}

int32_t tdmd_scale_velocities(double* d_velocities, int32_t natoms, double factor, void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(natoms >= 0, "natoms must be non-negative");
    if (natoms == 0) return;
    TDMD_REQUIRE(d_velocities, "null device array");
    const long long m = 3ll * natoms;
    launch(k_scale, ceil_div(m, kThreads), kThreads, 0, as_stream(stream), d_velocities, m, factor);
    TDMD_LAUNCH_CHECK();
  });
}

int32_t tdmd_nhc_create(double t_target, double t_period, int32_t chain_length, double dt,
                        int32_t n_dof, tdmd_nhc** out) {
  return guarded([&] {
    TDMD_REQUIRE(out, "out is null");
    TDMD_REQUIRE(chain_length >= 0 && chain_length <= kMaxChain, "chain length out of range");
    auto* h = new tdmd_nhc();
    h->t_target = t_target;
    h->t_period = t_period;
    h->dt = dt;
    h->M = chain_length;
    h->n_dof = n_dof;
    h->eta.assign(static_cast<size_t>(chain_length), 0.0);
    h->eta_v.assign(static_cast<size_t>(chain_length), 0.0);
    h->eta_m.assign(static_cast<size_t>(chain_length), 0.0);
    if (chain_length > 0)
      nhc_init(h->eta.data(), h->eta_v.data(), h->eta_m.data(), chain_length, t_target, t_period,
               n_dof);
    *out = h;
  });
}

int32_t tdmd_nhc_destroy(tdmd_nhc* nhc) {
  delete nhc;
  return TDMD_OK;
}

int32_t tdmd_nhc_half_step(tdmd_nhc* h, double ke_current, double* scale) {
  return guarded([&] {
    TDMD_REQUIRE(h && scale, "null argument");
    *scale = h->M > 0 ? nhc_half_step(h->eta.data(), h->eta_v.data(), h->eta_m.data(), h->M,
                                      h->t_target, h->t_period, h->n_dof, h->dt, ke_current)
                      : 1.0;
  });
}

int32_t tdmd_nhc_set_t_target(tdmd_nhc* h, double t_target) {
  return guarded([&] {
    TDMD_REQUIRE(h, "null handle");
    h->t_target = t_target;  // chain masses keep their construction-time value
  });
}

int32_t tdmd_nhc_state(const tdmd_nhc* h, double* eta, double* eta_v, double* eta_m) {
  return guarded([&] {
    TDMD_REQUIRE(h, "null handle");
    for (int k = 0; k < h->M; ++k) {
      if (eta) eta[k] = h->eta[static_cast<size_t>(k)];
      if (eta_v) eta_v[k] = h->eta_v[static_cast<size_t>(k)];
      if (eta_m) eta_m[k] = h->eta_m[static_cast<size_t>(k)];
    }
  });
}

}  // extern "C"
