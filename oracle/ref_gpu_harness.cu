// ref_gpu_harness.cu -- drives the reference's own GPU path (tdmd_Claude,
// compiled from its unmodified sources by oracle/Makefile into oracle/_ref/,
// once per build: FP64, mixed, and FP64 with TDMD_DETERMINISTIC_REDUCE):
//  * refgpu_run_eam times its FastPipelineScheduler on an EAM system, for a
//    same-box comparison in bench.py;
//  * refgpu_morse_forces / refgpu_eam_forces build its DeviceNeighborList
//    and evaluate compute_morse_gpu / DeviceEam::compute with an energy, for
//    the bit-parity tests of the ID-ordered energy mode.
// Test/measurement infrastructure only; no product code loads it.
//
// The reference synchronizes the host inside a rebuild (its cell list scans
// on the host), so the time is host wall clock around whole run_until
// windows, after a cudaDeviceSynchronize on both sides.
#include <chrono>
#include <cstdint>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "core/box.hpp"
#include "core/types.hpp"
#include "neighbors/device_neighbor_list.cuh"
#include "potentials/device_eam.cuh"
#include "potentials/device_morse.cuh"
#include "potentials/eam_alloy.hpp"
#include "scheduler/fast_pipeline_scheduler.cuh"

namespace {
std::string g_err;
}

extern "C" {

const char* refgpu_last_error() { return g_err.c_str(); }

// Runs `warm` then `windows` run_until windows of `window` steps on an EAM
// system (positions/velocities double[3n], types int32[n] 1-based, masses
// double[n_types]) and returns the wall seconds of the timed windows
// (negative on error).
double refgpu_run_eam(const char* setfl, const double* pos, const double* vel, const int32_t* types,
                      const double* masses, int32_t n_types, int32_t natoms, const double* lo,
                      const double* hi, double dt, double skin, int32_t rebuild_every,
                      int32_t window, int32_t warm, int32_t windows) {
  try {
    using namespace tdmd;
    potentials::EamAlloy eam;
    eam.read_setfl(setfl);
    Box box;
    box.lo = {lo[0], lo[1], lo[2]};
    box.hi = {hi[0], hi[1], hi[2]};
    scheduler::FastPipelineConfig cfg;
    cfg.dt = static_cast<real>(dt);
    cfg.r_skin = static_cast<real>(skin);
    cfg.rebuild_every = rebuild_every;
    const size_t n = static_cast<size_t>(natoms);
    std::vector<PositionVec> p(n);
    std::vector<VelocityVec> v(n);
    std::vector<ForceVec> f(n);
    std::vector<i32> ids(n);
    std::vector<real> m(static_cast<size_t>(n_types));
    for (size_t i = 0; i < n; ++i) {
      p[i] = PositionVec{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
      v[i] = VelocityVec{vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
      f[i] = ForceVec{0, 0, 0};
      ids[i] = static_cast<i32>(i + 1);
    }
    for (int t = 0; t < n_types; ++t) m[static_cast<size_t>(t)] = static_cast<real>(masses[t]);
    scheduler::FastPipelineScheduler s(box, natoms, eam, cfg);
    s.upload(p.data(), v.data(), f.data(), types, ids.data(), m.data(), n_types);
    int step = 0;
    s.run_until(step);
    for (int k = 0; k < warm; ++k) s.run_until(step += window);
    cudaDeviceSynchronize();
    const auto t0 = std::chrono::steady_clock::now();
    for (int k = 0; k < windows; ++k) s.run_until(step += window);
    cudaDeviceSynchronize();
    const auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1.0;
  }
}

}  // extern "C"

// Positions double[3n] (and 1-based types int32[n] for EAM) on a periodic
// box: the reference's DeviceNeighborList (r_cut, skin), then one force call
// with an energy accumulator starting at 0.  Forces (ForceVec of the build,
// written as double[3n]) and the energy come back to the host.  Returns 0,
// or -1 with refgpu_last_error set.
namespace {
template <class Fn>
int32_t with_list(const double* pos, int32_t natoms, const double* lo, const double* hi,
                  double r_cut, double skin, double* forces_out, double* energy_out, Fn&& call) {
  using namespace tdmd;
  try {
    Box box;
    box.lo = {lo[0], lo[1], lo[2]};
    box.hi = {hi[0], hi[1], hi[2]};
    const size_t n = static_cast<size_t>(natoms);
    PositionVec* d_pos = nullptr;
    ForceVec* d_f = nullptr;
    accum_t* d_e = nullptr;
    std::vector<PositionVec> hp(n);
    for (size_t i = 0; i < n; ++i) hp[i] = PositionVec{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    if (cudaMalloc(&d_pos, n * sizeof(PositionVec)) != cudaSuccess ||
        cudaMalloc(&d_f, n * sizeof(ForceVec)) != cudaSuccess ||
        cudaMalloc(&d_e, sizeof(accum_t)) != cudaSuccess)
      throw std::runtime_error("cudaMalloc failed");
    cudaMemcpy(d_pos, hp.data(), n * sizeof(PositionVec), cudaMemcpyHostToDevice);
    cudaMemset(d_e, 0, sizeof(accum_t));
    neighbors::DeviceNeighborList nl;
    nl.build(d_pos, natoms, box, static_cast<real>(r_cut), static_cast<real>(skin));
    call(d_pos, d_f, d_e, nl, box);
    std::vector<ForceVec> hf(n);
    accum_t e = 0;
    cudaMemcpy(hf.data(), d_f, n * sizeof(ForceVec), cudaMemcpyDeviceToHost);
    cudaMemcpy(&e, d_e, sizeof(accum_t), cudaMemcpyDeviceToHost);
    const cudaError_t err = cudaDeviceSynchronize();
    cudaFree(d_pos);
    cudaFree(d_f);
    cudaFree(d_e);
    if (err != cudaSuccess) throw std::runtime_error(cudaGetErrorString(err));
    for (size_t i = 0; i < n; ++i) {
      forces_out[3 * i] = static_cast<double>(hf[i].x);
      forces_out[3 * i + 1] = static_cast<double>(hf[i].y);
      forces_out[3 * i + 2] = static_cast<double>(hf[i].z);
    }
    *energy_out = static_cast<double>(e);
    return 0;
  } catch (const std::exception& ex) {
    g_err = ex.what();
    return -1;
  }
}
}  // namespace

extern "C" {

int32_t refgpu_morse_forces(const double* pos, int32_t natoms, const double* lo, const double* hi,
                            double d, double alpha, double r0, double rc, double skin,
                            double* forces_out, double* energy_out) {
  using namespace tdmd;
  return with_list(pos, natoms, lo, hi, rc, skin, forces_out, energy_out,
                   [&](PositionVec* d_pos, ForceVec* d_f, accum_t* d_e,
                       neighbors::DeviceNeighborList& nl, const Box& box) {
                     potentials::MorseParams p{static_cast<real>(d), static_cast<real>(alpha),
                                               static_cast<real>(r0), static_cast<real>(rc),
                                               static_cast<real>(rc * rc)};
                     potentials::compute_morse_gpu(d_pos, d_f, nl.d_neighbors(), nl.d_offsets(),
                                                   nl.d_counts(), natoms, box, p, d_e);
                   });
}

int32_t refgpu_eam_forces(const char* setfl, const double* pos, const int32_t* types,
                          int32_t natoms, const double* lo, const double* hi, double skin,
                          double* forces_out, double* energy_out) {
  using namespace tdmd;
  try {
    potentials::EamAlloy eam;
    eam.read_setfl(setfl);
    potentials::DeviceEam de;
    de.upload_tables(eam);
    int32_t* d_types = nullptr;
    if (cudaMalloc(&d_types, sizeof(int32_t) * static_cast<size_t>(natoms)) != cudaSuccess)
      throw std::runtime_error("cudaMalloc failed");
    cudaMemcpy(d_types, types, sizeof(int32_t) * static_cast<size_t>(natoms),
               cudaMemcpyHostToDevice);
    const int32_t rc = with_list(
        pos, natoms, lo, hi, static_cast<double>(eam.cutoff()), skin, forces_out, energy_out,
        [&](PositionVec* d_pos, ForceVec* d_f, accum_t* d_e, neighbors::DeviceNeighborList& nl,
            const Box& box) {
          de.compute(d_pos, d_f, d_types, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(),
                     natoms, box, d_e);
        });
    cudaFree(d_types);
    return rc;
  } catch (const std::exception& ex) {
    g_err = ex.what();
    return -1;
  }
}

}  // extern "C"
