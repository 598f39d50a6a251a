// ref_gpu_harness.cu -- times the reference's own GPU FastPipelineScheduler
// (tdmd_Claude, src/scheduler/fast_pipeline_scheduler.cu, compiled from its
// unmodified sources by oracle/Makefile into oracle/_ref/, once per
// precision build) on an EAM system, for a same-box comparison in
// bench.py.  Test/measurement infrastructure only; no product code loads it.
//
// The reference synchronizes the host inside a rebuild (its cell list scans
// on the host), so the time is host wall clock around whole run_until
// windows, after a cudaDeviceSynchronize on both sides.
#include <chrono>
#include <cstdint>
#include <exception>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "core/box.hpp"
#include "core/types.hpp"
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
