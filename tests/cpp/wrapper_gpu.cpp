// Runs the GPU path through include/tdmd_b200.hpp with the reference's class
// and function names, as code written for the reference would: a
// FastPipelineScheduler (Morse) for 20 steps, then DeviceNeighborList +
// compute_morse_gpu on the final positions.  Input: "n lo hi" then n lines
// "x y z vx vy vz"; output: final positions, velocities and scheduler forces
// (17 significant digits), then the free-function energy and forces.
#include <cuda_runtime_api.h>

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
  std::fclose(out);
  cudaFree(d_pos);
  cudaFree(d_f);
  cudaFree(d_e);
  return 0;
}
