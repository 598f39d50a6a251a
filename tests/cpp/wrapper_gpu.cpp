// Runs the GPU path through include/tdmd_b200.hpp with the reference's class
// and function names, as code written for the reference would: a
// FastPipelineScheduler (Morse) for 20 steps, then DeviceNeighborList +
// compute_morse_gpu on the final positions.  Input: "n lo hi" then n lines
// "x y z vx vy vz"; output: final positions, velocities and scheduler forces
// (17 significant digits), then the free-function energy and forces.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "tdmd_b200.hpp"

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  using namespace tdmd;
  std::FILE* in = std::fopen(argv[1], "r");
  if (!in) return 3;
  int n = 0;
  double lo = 0, hi = 0;
  if (std::fscanf(in, "%d %lf %lf", &n, &lo, &hi) != 3) return 4;
  std::vector<PositionVec> pos(static_cast<size_t>(n));
  std::vector<VelocityVec> vel(static_cast<size_t>(n));
  for (int i = 0; i < n; ++i)
    if (std::fscanf(in, "%lf %lf %lf %lf %lf %lf", &pos[i].x, &pos[i].y, &pos[i].z, &vel[i].x,
                    &vel[i].y, &vel[i].z) != 6)
      return 5;
  std::fclose(in);
  std::vector<i32> types(static_cast<size_t>(n), 1), ids(static_cast<size_t>(n));
  for (int i = 0; i < n; ++i) ids[i] = i + 1;
  std::vector<real> masses = {real(1.0), real(63.546)};

  Box box;
  box.lo = {lo, lo, lo};
  box.hi = {hi, hi, hi};
  const real rc = real(6.0);
  potentials::MorseParams mp{real(0.3429), real(1.3588), real(2.866), rc, rc * rc};
  scheduler::FastPipelineConfig cfg{real(0.001), real(0.3), 10};
  cfg.lanes_per_atom = 4;
  std::vector<ForceVec> forces(static_cast<size_t>(n));
  try {
    scheduler::FastPipelineScheduler sched(box, n, mp, cfg);
    sched.upload(pos.data(), vel.data(), nullptr, types.data(), ids.data(), masses.data(),
                 static_cast<i32>(masses.size()));
    sched.run_until(20);
    sched.download(pos.data(), vel.data(), forces.data(), nullptr, nullptr, n);
    if (sched.current_step() != 20 || sched.potential_kind() != scheduler::PotentialKind::Morse)
      return 6;
  } catch (const Error& e) {
    std::fprintf(stderr, "error %d: %s\n", e.status(), e.what());
    return 7;
  }
  std::FILE* out = std::fopen(argv[2], "w");
  for (int i = 0; i < n; ++i)
    std::fprintf(out, "%.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g\n", pos[i].x,
                 pos[i].y, pos[i].z, vel[i].x, vel[i].y, vel[i].z,
                 static_cast<double>(forces[i].x), static_cast<double>(forces[i].y),
                 static_cast<double>(forces[i].z));
  // free functions on device buffers
  PositionVec* d_pos = nullptr;
  ForceVec* d_f = nullptr;
  accum_t* d_e = nullptr;
  cudaMalloc(reinterpret_cast<void**>(&d_pos), sizeof(PositionVec) * n);
  cudaMalloc(reinterpret_cast<void**>(&d_f), sizeof(ForceVec) * n);
  cudaMalloc(reinterpret_cast<void**>(&d_e), sizeof(accum_t));
  cudaMemcpy(d_pos, pos.data(), sizeof(PositionVec) * n, cudaMemcpyHostToDevice);
  cudaMemset(d_e, 0, sizeof(accum_t));
  try {
    neighbors::DeviceNeighborList nl;
    nl.build(d_pos, n, box, rc, real(0.3));
    potentials::compute_morse_gpu(d_pos, d_f, nl.d_neighbors(), nl.d_offsets(), nl.d_counts(), n,
                                  box, mp, d_e);
  } catch (const Error& e) {
    std::fprintf(stderr, "error %d: %s\n", e.status(), e.what());
    return 8;
  }
  accum_t e = 0;
  cudaMemcpy(&e, d_e, sizeof(e), cudaMemcpyDeviceToHost);
  cudaMemcpy(forces.data(), d_f, sizeof(ForceVec) * n, cudaMemcpyDeviceToHost);
  std::fprintf(out, "%.17g\n", e);
  for (int i = 0; i < n; ++i)
    std::fprintf(out, "%.17g %.17g %.17g\n", static_cast<double>(forces[i].x),
                 static_cast<double>(forces[i].y), static_cast<double>(forces[i].z));
  // cell list of the same positions at r_list = rc + skin: grid and cell size
  try {
    domain::DeviceCellList cl;
    cl.build(d_pos, n, box, rc + real(0.3));
    const Vec3D cs = cl.cell_size();
    std::fprintf(out, "%d %d %d %.17g %.17g %.17g\n", cl.ncells_x(), cl.ncells_y(),
                 cl.ncells_z(), cs.x, cs.y, cs.z);
  } catch (const Error& e) {
    std::fprintf(stderr, "error %d: %s\n", e.status(), e.what());
    return 9;
  }
  // the zone calls of the TD pipeline on the same list: two zones' forces
  // added into zeroed forces equal the whole-system forces; a zone half kick
  // moves only its zone
  try {
    ForceVec* d_fz = nullptr;
    VelocityVec* d_v = nullptr;
    i32* d_t = nullptr;
    real* d_m = nullptr;
    accum_t* d_ez = nullptr;
    cudaMalloc(reinterpret_cast<void**>(&d_fz), sizeof(ForceVec) * n);
    cudaMalloc(reinterpret_cast<void**>(&d_v), sizeof(VelocityVec) * n);
    cudaMalloc(reinterpret_cast<void**>(&d_t), sizeof(i32) * n);
    cudaMalloc(reinterpret_cast<void**>(&d_m), sizeof(real) * masses.size());
    cudaMalloc(reinterpret_cast<void**>(&d_ez), sizeof(accum_t));
    cudaMemset(d_ez, 0, sizeof(accum_t));
    cudaMemset(d_v, 0, sizeof(VelocityVec) * n);
    cudaMemcpy(d_t, types.data(), sizeof(i32) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(d_m, masses.data(), sizeof(real) * masses.size(), cudaMemcpyHostToDevice);
    neighbors::DeviceNeighborList nl;
    nl.build(d_pos, n, box, rc, real(0.3));
    const i32 half = n / 2;
    integrator::device_zero_forces_zone(d_fz, 0, half, nullptr);
    integrator::device_zero_forces_zone(d_fz, half, n - half, nullptr);
    potentials::compute_morse_gpu_zone(d_pos, d_fz, nl.d_neighbors(), nl.d_offsets(),
                                       nl.d_counts(), 0, half, box, mp, d_ez, nullptr);
    potentials::compute_morse_gpu_zone(d_pos, d_fz, nl.d_neighbors(), nl.d_offsets(),
                                       nl.d_counts(), half, n - half, box, mp, d_ez, nullptr);
    integrator::device_half_kick_zone(d_v, d_fz, d_t, d_m, half, n - half, real(0.001), nullptr);
    std::vector<ForceVec> fz(static_cast<size_t>(n));
    std::vector<VelocityVec> vz(static_cast<size_t>(n));
    accum_t ez = 0;
    cudaMemcpy(fz.data(), d_fz, sizeof(ForceVec) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(vz.data(), d_v, sizeof(VelocityVec) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(&ez, d_ez, sizeof(ez), cudaMemcpyDeviceToHost);
    double df = 0, vlo = 0, vhi = 0;
    for (int i = 0; i < n; ++i) {
      df = std::max(df, std::abs(static_cast<double>(fz[i].x) - static_cast<double>(forces[i].x)));
      (i < half ? vlo : vhi) += std::abs(vz[i].x) + std::abs(vz[i].y) + std::abs(vz[i].z);
    }
    std::fprintf(out, "%.17g %.17g %.17g %.17g\n", ez, df, vlo, vhi);
    cudaFree(d_fz);
    cudaFree(d_v);
    cudaFree(d_t);
    cudaFree(d_m);
    cudaFree(d_ez);
  } catch (const Error& e) {
    std::fprintf(stderr, "error %d: %s\n", e.status(), e.what());
    return 10;
  }
  std::fclose(out);
  cudaFree(d_pos);
  cudaFree(d_f);
  cudaFree(d_e);
  return 0;
}
