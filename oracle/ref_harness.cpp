// ref_harness.cpp -- extern "C" entry points around the reference's own CPU
// path (tdmd_Claude, compiled from its unmodified sources by oracle/Makefile
// into oracle/_ref/libtdmd_ref.so).  Test infrastructure only: the tests use
// it to pin the C restatement in tdmd_oracle.c, and bench.py's reference arm
// times run_cpu() below as the CPU baseline.  No product code loads it.
//
// Reference classes used (paths relative to the tdmd_Claude tree):
//   io::read_lammps_data          src/io/lammps_data_reader.cpp:33
//   domain::CellList              src/domain/cell_list.cpp:13
//   neighbors::NeighborList       src/neighbors/neighbor_list.cpp:14,91
//   potentials::MorsePair         src/potentials/morse.hpp:21
//   potentials::compute_pair_forces src/potentials/force_compute.cpp:10
//   potentials::EamAlloy          src/potentials/eam_alloy.cpp:90,196
//   integrator::VelocityVerlet    src/integrator/velocity_verlet.cpp:11,29
//   integrator::NoseHooverChain   src/integrator/device_nose_hoover.cu:187,206
#include <chrono>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "core/box.hpp"
#include "core/constants.hpp"
#include "core/system_state.hpp"
#include "domain/cell_list.hpp"
#include "integrator/device_nose_hoover.cuh"
#include "integrator/velocity_verlet.hpp"
#include "io/lammps_data_reader.hpp"
#include "neighbors/neighbor_list.hpp"
#include "potentials/eam_alloy.hpp"
#include "potentials/force_compute.hpp"
#include "potentials/morse.hpp"

using namespace tdmd;

namespace {

thread_local std::string g_err;

Box make_box(const double* lo, const double* hi, const int32_t* periodic) {
  Box b;
  b.lo = {lo[0], lo[1], lo[2]};
  b.hi = {hi[0], hi[1], hi[2]};
  b.periodic = {periodic[0] != 0, periodic[1] != 0, periodic[2] != 0};
  return b;
}

SystemState make_state(const double* pos, const double* vel, const int32_t* types,
                       const double* masses, int32_t ntypes, int64_t n, const Box& box) {
  SystemState s;
  s.resize(n);
  s.box = box;
  for (int64_t i = 0; i < n; ++i) {
    s.positions[size_t(i)] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    if (vel) s.velocities[size_t(i)] = {vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
    s.types[size_t(i)] = types ? types[i] : 1;
    s.ids[size_t(i)] = int32_t(i + 1);
  }
  if (masses) s.masses.assign(masses, masses + ntypes + 1);
  return s;
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// read_lammps_data: natoms/ntypes query (positions == nullptr) or fill.
int32_t ref_read_data(const char* path, int64_t* natoms, int32_t* ntypes, double* lo, double* hi,
                      double* pos, double* vel, int32_t* types, int32_t* ids, double* masses) {
  try {
    SystemState s = io::read_lammps_data(path);
    *natoms = s.natoms;
    *ntypes = int32_t(s.masses.size()) - 1;
    lo[0] = s.box.lo.x; lo[1] = s.box.lo.y; lo[2] = s.box.lo.z;
    hi[0] = s.box.hi.x; hi[1] = s.box.hi.y; hi[2] = s.box.hi.z;
    if (!pos) return 0;
    for (int64_t i = 0; i < s.natoms; ++i) {
      auto& p = s.positions[size_t(i)];
      auto& v = s.velocities[size_t(i)];
      pos[3 * i] = p.x; pos[3 * i + 1] = p.y; pos[3 * i + 2] = p.z;
      vel[3 * i] = v.x; vel[3 * i + 1] = v.y; vel[3 * i + 2] = v.z;
      types[i] = s.types[size_t(i)];
      ids[i] = s.ids[size_t(i)];
    }
    for (size_t t = 0; t < s.masses.size(); ++t) masses[t] = s.masses[t];
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

// CellList::build -> grid, counts, offsets (from atoms_in_cell), atoms.
int32_t ref_cell_list(const double* pos, int64_t n, const double* lo, const double* hi,
                      const int32_t* periodic, double r_list, int32_t* nc, int32_t* counts,
                      int32_t* offsets, int32_t* atoms) {
  Box b = make_box(lo, hi, periodic);
  std::vector<PositionVec> p(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) p[size_t(i)] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
  domain::CellList cl;
  cl.build(p.data(), n, b, r_list);
  nc[0] = cl.ncells_x(); nc[1] = cl.ncells_y(); nc[2] = cl.ncells_z();
  if (!counts) return cl.ncells_total();
  const int32_t* base = cl.atoms_in_cell(0);
  for (int32_t c = 0; c < cl.ncells_total(); ++c) {
    counts[c] = cl.count(c);
    offsets[c] = int32_t(cl.atoms_in_cell(c) - base);
  }
  std::memcpy(atoms, base, sizeof(int32_t) * size_t(n));
  return cl.ncells_total();
}

// NeighborList::build (half list).  Returns total pairs; entries past cap
// are not written.
int64_t ref_half_list(const double* pos, int64_t n, const double* lo, const double* hi,
                      const int32_t* periodic, double r_cut, double r_skin, int32_t* counts,
                      int32_t* offsets, int32_t* nbrs, int64_t cap) {
  Box b = make_box(lo, hi, periodic);
  std::vector<PositionVec> p(static_cast<size_t>(n));
  for (int64_t i = 0; i < n; ++i) p[size_t(i)] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
  neighbors::NeighborList nl;
  nl.build(p.data(), n, b, r_cut, r_skin);
  int64_t total = 0;
  for (int64_t i = 0; i < n; ++i) {
    counts[i] = nl.count(i);
    offsets[i] = int32_t(total);
    const int32_t* nb = nl.neighbors_of(i);
    for (int32_t k = 0; k < nl.count(i); ++k)
      if (total + k < cap) nbrs[total + k] = nb[k];
    total += nl.count(i);
  }
  return total;
}

// Morse forces + PE via NeighborList + compute_pair_forces.
double ref_morse_forces(const double* pos, int64_t n, const double* lo, const double* hi,
                        const int32_t* periodic, double D, double alpha, double r0, double rc,
                        double r_skin, double* forces) {
  Box b = make_box(lo, hi, periodic);
  SystemState s = make_state(pos, nullptr, nullptr, nullptr, 1, n, b);
  neighbors::NeighborList nl;
  nl.build(s.positions.data(), n, b, rc, r_skin);
  potentials::MorsePair m(D, alpha, r0, rc);
  double pe = potentials::compute_pair_forces(s, nl, m);
  for (int64_t i = 0; i < n; ++i) {
    forces[3 * i] = s.forces[size_t(i)].x;
    forces[3 * i + 1] = s.forces[size_t(i)].y;
    forces[3 * i + 2] = s.forces[size_t(i)].z;
  }
  return pe;
}

// MorsePair::compute for one r^2.
void ref_morse_pair(double D, double alpha, double r0, double rc, double r2, double* e,
                    double* fpair) {
  potentials::MorsePair m(D, alpha, r0, rc);
  m.compute(r2, *e, *fpair);
}

// EamAlloy handle.
void* ref_eam_load(const char* path) {
  try {
    auto* e = new potentials::EamAlloy();
    e->read_setfl(path);
    return e;
  } catch (const std::exception& ex) {
    g_err = ex.what();
    return nullptr;
  }
}

void ref_eam_free(void* h) { delete static_cast<potentials::EamAlloy*>(h); }

double ref_eam_cutoff(void* h) { return static_cast<potentials::EamAlloy*>(h)->cutoff(); }
int32_t ref_eam_ntypes(void* h) { return static_cast<potentials::EamAlloy*>(h)->ntypes(); }

// Packed a|b|c|d coefficients of one spline (kind 0=F, 1=rho, 2=phi).
int32_t ref_eam_coeffs(void* h, int32_t kind, int32_t idx, double* out) {
  auto* e = static_cast<potentials::EamAlloy*>(h);
  const auto& v = kind == 0 ? e->embedding() : (kind == 1 ? e->density() : e->phi());
  const auto& s = v[size_t(idx)];
  const size_t ns = size_t(s.n - 1);
  if (out) {
    for (size_t i = 0; i < ns; ++i) {
      out[i] = s.a[i];
      out[ns + i] = s.b[i];
      out[2 * ns + i] = s.c[i];
      out[3 * ns + i] = s.d[i];
    }
  }
  return int32_t(4 * ns);
}

double ref_eam_spline(void* h, int32_t kind, int32_t idx, int32_t deriv, double r) {
  auto* e = static_cast<potentials::EamAlloy*>(h);
  const auto& v = kind == 0 ? e->embedding() : (kind == 1 ? e->density() : e->phi());
  return deriv ? v[size_t(idx)].eval_deriv(r) : v[size_t(idx)].eval(r);
}

double ref_eam_forces(void* h, const double* pos, const int32_t* types, int64_t n,
                      const double* lo, const double* hi, const int32_t* periodic, double r_skin,
                      double* forces) {
  auto* e = static_cast<potentials::EamAlloy*>(h);
  Box b = make_box(lo, hi, periodic);
  SystemState s = make_state(pos, nullptr, types, nullptr, 1, n, b);
  neighbors::NeighborList nl;
  nl.build(s.positions.data(), n, b, e->cutoff(), r_skin);
  double pe = e->compute_forces(s, nl);
  for (int64_t i = 0; i < n; ++i) {
    forces[3 * i] = s.forces[size_t(i)].x;
    forces[3 * i + 1] = s.forces[size_t(i)].y;
    forces[3 * i + 2] = s.forces[size_t(i)].z;
  }
  return pe;
}

// NoseHooverChain handle.
void* ref_nhc_create(double t_target, double t_period, int32_t chain, double dt, int32_t n_dof) {
  integrator::NHCConfig c;
  c.t_target = t_target;
  c.t_period = t_period;
  c.chain_length = chain;
  return new integrator::NoseHooverChain(c, dt, n_dof);
}
double ref_nhc_half_step(void* h, double ke) {
  return static_cast<integrator::NoseHooverChain*>(h)->half_step(ke);
}
void ref_nhc_free(void* h) { delete static_cast<integrator::NoseHooverChain*>(h); }

// The reference CPU MD loop (tdmd_main.cpp:237-254) with the neighbor list
// rebuilt every `rebuild_every` steps instead of on the skin check (the
// GPU scheduler's schedule).  eam == nullptr selects Morse.  Returns the
// wall seconds of the step loop (std::chrono::steady_clock, setup excluded)
// and leaves the final state in pos/vel/forces.
double ref_run_cpu(void* eam, double D, double alpha, double r0, double rc, double* pos,
                   double* vel, double* forces, const int32_t* types, const double* masses,
                   int32_t ntypes, int64_t n, const double* lo, const double* hi,
                   const int32_t* periodic, double dt, double r_skin, int32_t rebuild_every,
                   int32_t nsteps, double* pe_out) {
  Box b = make_box(lo, hi, periodic);
  SystemState s = make_state(pos, vel, types, masses, ntypes, n, b);
  auto* e = static_cast<potentials::EamAlloy*>(eam);
  potentials::MorsePair m(D, alpha, r0, rc);
  const double cut = e ? e->cutoff() : rc;
  integrator::VelocityVerlet vv(dt);
  neighbors::NeighborList nl;
  nl.build(s.positions.data(), n, b, cut, r_skin);
  auto force = [&]() {
    return e ? e->compute_forces(s, nl) : potentials::compute_pair_forces(s, nl, m);
  };
  double pe = force();
  int32_t since = 0;
  const auto t0 = std::chrono::steady_clock::now();
  for (int32_t step = 0; step < nsteps; ++step) {
    vv.half_kick(s);
    vv.drift(s);
    if (++since >= rebuild_every) {
      nl.build(s.positions.data(), n, b, cut, r_skin);
      since = 0;
    }
    pe = force();
    vv.half_kick(s);
  }
  const auto t1 = std::chrono::steady_clock::now();
  for (int64_t i = 0; i < n; ++i) {
    const auto& p = s.positions[size_t(i)];
    const auto& v = s.velocities[size_t(i)];
    const auto& f = s.forces[size_t(i)];
    pos[3 * i] = p.x; pos[3 * i + 1] = p.y; pos[3 * i + 2] = p.z;
    vel[3 * i] = v.x; vel[3 * i + 1] = v.y; vel[3 * i + 2] = v.z;
    forces[3 * i] = f.x; forces[3 * i + 1] = f.y; forces[3 * i + 2] = f.z;
  }
  if (pe_out) *pe_out = pe;
  return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"
