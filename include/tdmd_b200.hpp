// tdmd_b200.hpp -- header-only C++ layer over the C ABI in tdmd_b200.h that
// restores the reference's class and function names, namespaces and
// signatures (tdmd_Claude, src/...), so code written against the reference's
// GPU path compiles against this library with its includes swapped.
//
// Precision follows the reference's build switch (src/core/types.hpp:9-15,
// 44-61): define TDMD_PRECISION_MIXED for `real = float` and float forces,
// otherwise (or with TDMD_PRECISION_FP64) everything is double.
//
// Core types: by default this header defines the reference's core types
// itself (src/core/{types,box,system_state,constants,error}.hpp, same names
// and layouts).  A caller that keeps the reference's own core headers on its
// include path defines TDMD_B200_REFERENCE_CORE instead, and this layer uses
// those headers' types; the reference's CPU classes (NeighborList,
// MorsePair, EamAlloy::compute_forces, ...) then link beside it unchanged.
//
// Errors: every non-zero status becomes a tdmd::StatusError carrying the
// status code, a tdmd::Error (std::runtime_error, as src/core/error.hpp:13);
// without TDMD_B200_REFERENCE_CORE the two names are one class.  The
// reference aborts on CUDA failures instead (src/core/device_buffer.cuh:16-24);
// TDMD_CUDA_CHECK here throws.
//
// Needs <cuda_runtime_api.h>; callers link the CUDA runtime (DeviceBuffer).
#pragma once

#include <cuda_runtime_api.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "tdmd_b200.h"

#if defined(TDMD_B200_REFERENCE_CORE)
// The caller's tree supplies the reference's own core headers; this layer
// uses those types as they are.
#include "core/box.hpp"
#include "core/constants.hpp"
#include "core/error.hpp"
#include "core/system_state.hpp"
#include "core/types.hpp"
#include "domain/zone_partition.hpp"
#include "potentials/eam_alloy.hpp"
#endif

namespace tdmd {

#if !defined(TDMD_B200_REFERENCE_CORE)
// --- src/core/types.hpp -----------------------------------------------------
#if defined(TDMD_PRECISION_MIXED)
using real = float;
#else
using real = double;
#endif
using i32 = std::int32_t;
using i64 = std::int64_t;
using u32 = std::uint32_t;
using u64 = std::uint64_t;

template <class T>
struct Vec3T {
  T x;
  T y;
  T z;
};
using Vec3D = Vec3T<double>;
using Vec3F = Vec3T<float>;
using Vec3 = Vec3T<real>;

struct Aabb {
  Vec3D lo;
  Vec3D hi;
};

using pos_t = double;
using vel_t = double;
using accum_t = double;
using PositionVec = Vec3D;
using VelocityVec = Vec3D;
#if defined(TDMD_PRECISION_MIXED)
using force_t = float;
using ForceVec = Vec3F;
#else
using force_t = double;
using ForceVec = Vec3D;
#endif

// --- src/core/constants.hpp:15,28 (metal units) -----------------------------
inline constexpr real kBoltzmann = real{8.617333262e-5};
inline constexpr real kMvv2e = real{1.0364269e-4};

// --- src/core/error.hpp -----------------------------------------------------
class Error : public std::runtime_error {
 public:
  Error(int32_t status, const std::string& what) : std::runtime_error(what), status_(status) {}
  int32_t status() const noexcept { return status_; }

 private:
  int32_t status_;
};
using StatusError = Error;

// --- src/core/box.hpp -------------------------------------------------------
struct Box {
  Vec3D lo{0, 0, 0};
  Vec3D hi{0, 0, 0};
  std::array<bool, 3> periodic{true, true, true};

  Vec3D size() const noexcept { return Vec3D{hi.x - lo.x, hi.y - lo.y, hi.z - lo.z}; }
};

// --- src/core/system_state.hpp: the host SoA state of a simulation ----------
struct SystemState {
  i64 natoms{0};
  Box box;
  std::vector<PositionVec> positions;
  std::vector<VelocityVec> velocities;
  std::vector<ForceVec> forces;
  std::vector<i32> types;
  std::vector<i32> ids;
  std::vector<real> masses;  // indexed by the 1-based type: size ntypes + 1
  std::vector<std::string> type_names;
  i64 step{0};
  real time{0};

  void resize(i64 n) {
    natoms = n;
    const size_t k = static_cast<size_t>(n);
    positions.resize(k);
    velocities.resize(k);
    forces.resize(k);
    types.resize(k);
    ids.resize(k);
  }
};
#else
// The reference's tdmd::Error (a std::runtime_error) is the base; the status
// code of the failing call rides in this subclass.
class StatusError : public Error {
 public:
  StatusError(int32_t status, const std::string& what) : Error(what), status_(status) {}
  int32_t status() const noexcept { return status_; }

 private:
  int32_t status_;
};
#endif  // TDMD_B200_REFERENCE_CORE

#if defined(TDMD_PRECISION_MIXED)
constexpr int32_t kForcePrecision = TDMD_MIXED;
#else
constexpr int32_t kForcePrecision = TDMD_FP64;
#endif

namespace detail {
inline void check(int32_t rc) {
  if (rc != TDMD_OK) throw StatusError(rc, tdmd_last_error());
}
inline void* stream_ptr(cudaStream_t s) { return reinterpret_cast<void*>(s); }
inline tdmd_box to_c(const Box& box) noexcept {
  tdmd_box b{};
  b.lo[0] = box.lo.x;
  b.lo[1] = box.lo.y;
  b.lo[2] = box.lo.z;
  b.hi[0] = box.hi.x;
  b.hi[1] = box.hi.y;
  b.hi[2] = box.hi.z;
  for (int k = 0; k < 3; ++k) b.periodic[k] = box.periodic[static_cast<size_t>(k)] ? 1 : 0;
  return b;
}
}  // namespace detail

// --- src/core/determinism.hpp:20-24 ----------------------------------------
// The reference selects ID-ordered energy sums at build time
// (kDeterministicReduce); here it is a process-wide run-time switch.
inline void set_deterministic_reduce(bool on) {
  detail::check(tdmd_set_deterministic_reduce(on ? 1 : 0));
}
inline bool deterministic_reduce() {
  int32_t on = 0;
  detail::check(tdmd_get_deterministic_reduce(&on));
  return on != 0;
}

// --- src/core/device_buffer.cuh:16-112 ---------------------------------------
// A CUDA call that fails throws StatusError (TDMD_ERR_CUDA, or
// TDMD_ERR_OUT_OF_MEMORY for an allocation).
inline void check_cuda(cudaError_t err, const char* file, int line) {
  if (err != cudaSuccess)
    throw StatusError(err == cudaErrorMemoryAllocation ? TDMD_ERR_OUT_OF_MEMORY : TDMD_ERR_CUDA,
                      std::string(cudaGetErrorString(err)) + " at " + file + ":" +
                          std::to_string(line));
}
#define TDMD_CUDA_CHECK(call) ::tdmd::check_cuda((call), __FILE__, __LINE__)

// Device array of n elements (uninitialised), move-only; resize discards the
// contents; copies are synchronous.
template <typename T>
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(std::size_t n) { resize(n); }
  ~DeviceBuffer() { release(); }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept : ptr_(o.ptr_), size_(o.size_) {
    o.ptr_ = nullptr;
    o.size_ = 0;
  }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    if (this != &o) {
      release();
      ptr_ = o.ptr_;
      size_ = o.size_;
      o.ptr_ = nullptr;
      o.size_ = 0;
    }
    return *this;
  }

  void resize(std::size_t n) {
    if (n == size_) return;
    release();
    if (n > 0) TDMD_CUDA_CHECK(cudaMalloc(reinterpret_cast<void**>(&ptr_), n * sizeof(T)));
    size_ = n;
  }
  void copy_from_host(const T* src, std::size_t n, std::size_t offset = 0) {
    in_range(n, offset);
    if (n) TDMD_CUDA_CHECK(cudaMemcpy(ptr_ + offset, src, n * sizeof(T), cudaMemcpyHostToDevice));
  }
  void copy_to_host(T* dst, std::size_t n, std::size_t offset = 0) const {
    in_range(n, offset);
    if (n) TDMD_CUDA_CHECK(cudaMemcpy(dst, ptr_ + offset, n * sizeof(T), cudaMemcpyDeviceToHost));
  }
  void zero() {
    if (size_) TDMD_CUDA_CHECK(cudaMemset(ptr_, 0, size_ * sizeof(T)));
  }
  T* data() noexcept { return ptr_; }
  const T* data() const noexcept { return ptr_; }
  std::size_t size() const noexcept { return size_; }

 private:
  void release() noexcept {
    if (ptr_) cudaFree(ptr_);
    ptr_ = nullptr;
    size_ = 0;
  }
  void in_range(std::size_t n, std::size_t offset) const {
    if (offset > size_ || n > size_ - offset)
      throw StatusError(TDMD_ERR_INVALID_ARGUMENT, "DeviceBuffer copy out of range");
  }

  T* ptr_ = nullptr;
  std::size_t size_ = 0;
};

// --- src/core/device_system_state.cuh:18-42 ----------------------------------
// Device copy of a SystemState's per-atom arrays and per-type masses.
struct DeviceSystemState {
  i64 natoms{0};
  Box box;
  DeviceBuffer<PositionVec> positions;
  DeviceBuffer<VelocityVec> velocities;
  DeviceBuffer<ForceVec> forces;
  DeviceBuffer<i32> types;
  DeviceBuffer<i32> ids;
  DeviceBuffer<real> masses;

  void resize(i64 n, i32 ntypes = 0) {
    natoms = n;
    const std::size_t k = static_cast<std::size_t>(n);
    positions.resize(k);
    velocities.resize(k);
    forces.resize(k);
    types.resize(k);
    ids.resize(k);
    if (ntypes > 0) masses.resize(static_cast<std::size_t>(ntypes));
  }
  void upload(const SystemState& host) {
    const std::size_t k = static_cast<std::size_t>(host.natoms);
    if (positions.size() != k || masses.size() < host.masses.size())
      resize(host.natoms, static_cast<i32>(host.masses.size()));
    natoms = host.natoms;
    box = host.box;
    positions.copy_from_host(host.positions.data(), k);
    velocities.copy_from_host(host.velocities.data(), k);
    forces.copy_from_host(host.forces.data(), k);
    types.copy_from_host(host.types.data(), k);
    ids.copy_from_host(host.ids.data(), k);
    masses.copy_from_host(host.masses.data(), host.masses.size());
  }
  void download(SystemState& host) const {
    const std::size_t k = static_cast<std::size_t>(natoms);
    host.resize(natoms);
    host.box = box;
    positions.copy_to_host(host.positions.data(), k);
    velocities.copy_to_host(host.velocities.data(), k);
    forces.copy_to_host(host.forces.data(), k);
    types.copy_to_host(host.types.data(), k);
    ids.copy_to_host(host.ids.data(), k);
    if (masses.size() > 0) {
      host.masses.resize(masses.size());
      masses.copy_to_host(host.masses.data(), masses.size());
    }
  }
  void zero_forces() { forces.zero(); }
};

// --- src/potentials -----------------------------------------------------------
namespace potentials {

// device_morse.cuh:14-20
struct MorseParams {
  real d;
  real alpha;
  real r0;
  real rc;
  real rc_sq;

  tdmd_morse_params to_c() const noexcept {
    return tdmd_morse_params{d, alpha, r0, rc, rc_sq};
  }
};

// device_morse.cuh:37-41: forces stored, *d_energy accumulated.
inline void compute_morse_gpu(const PositionVec* d_positions, ForceVec* d_forces,
                              const i32* d_neighbors, const i32* d_offsets, const i32* d_counts,
                              i32 natoms, const Box& box, const MorseParams& params,
                              accum_t* d_energy, cudaStream_t stream = 0) {
  const tdmd_box b = detail::to_c(box);
  const tdmd_morse_params p = params.to_c();
  detail::check(tdmd_morse_compute(reinterpret_cast<const double*>(d_positions), d_forces,
                                   kForcePrecision, d_neighbors, d_offsets, d_counts, natoms, &b,
                                   &p, d_energy, nullptr, detail::stream_ptr(stream)));
}

// device_morse_zone.cuh:13-23: forces of atoms [first_atom, first_atom +
// atom_count) ADDED to d_forces (zero the zone first), from the global
// positions and list; *d_energy accumulated.
inline void compute_morse_gpu_zone(const PositionVec* d_positions, ForceVec* d_forces,
                                   const i32* d_neighbors, const i32* d_offsets,
                                   const i32* d_counts, i32 first_atom, i32 atom_count,
                                   const Box& box, const MorseParams& params, accum_t* d_energy,
                                   cudaStream_t stream) {
  const tdmd_box b = detail::to_c(box);
  const tdmd_morse_params p = params.to_c();
  detail::check(tdmd_morse_compute_zone(reinterpret_cast<const double*>(d_positions), d_forces,
                                        kForcePrecision, d_neighbors, d_offsets, d_counts,
                                        first_atom, atom_count, &b, &p, d_energy, nullptr,
                                        detail::stream_ptr(stream)));
}

#if !defined(TDMD_B200_REFERENCE_CORE)
// eam_alloy.hpp:47-93 (tables; the CPU compute_forces stays in the reference).
class EamAlloy {
 public:
  EamAlloy() = default;
  EamAlloy(const EamAlloy&) = delete;
  EamAlloy& operator=(const EamAlloy&) = delete;
  EamAlloy(EamAlloy&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
  ~EamAlloy() {
    if (h_) tdmd_eam_destroy(h_);
  }

  // eam_alloy.cpp:90-192
  void read_setfl(const std::string& filename) {
    tdmd_eam* h = nullptr;
    detail::check(tdmd_eam_read_setfl(filename.c_str(), &h));
    if (h_) tdmd_eam_destroy(h_);
    h_ = h;
  }
  real cutoff() const {
    double c = 0;
    detail::check(tdmd_eam_info(h_, nullptr, nullptr, nullptr, nullptr, nullptr, &c));
    return static_cast<real>(c);
  }
  i32 ntypes() const {
    int32_t n = 0;
    detail::check(tdmd_eam_info(h_, &n, nullptr, nullptr, nullptr, nullptr, nullptr));
    return n;
  }
  const tdmd_eam* handle() const noexcept { return h_; }

 private:
  tdmd_eam* h_ = nullptr;
};
#endif  // !TDMD_B200_REFERENCE_CORE

// The library's tables of an EamAlloy: its own handle, or, with the
// reference's EamAlloy (TDMD_B200_REFERENCE_CORE), a temporary set built from
// that class's sampled F(rho), rho(r) and phi(r) (eam_alloy.hpp:65-73) and
// freed once the consumer has copied it.
class EamTables {
 public:
#if defined(TDMD_B200_REFERENCE_CORE)
  explicit EamTables(const EamAlloy& eam) {
    const auto& F = eam.embedding();
    const auto& rho = eam.density();
    const auto& phi = eam.phi();
    const i32 nt = eam.ntypes();
    const size_t npairs = static_cast<size_t>(nt) * static_cast<size_t>(nt + 1) / 2;
    if (nt < 1 || F.size() != static_cast<size_t>(nt) || rho.size() != static_cast<size_t>(nt) ||
        phi.size() != npairs)
      throw StatusError(TDMD_ERR_INVALID_ARGUMENT, "EamAlloy has no tables (read_setfl first)");
    const i32 nrho = F[0].n, nr = rho[0].n;
    std::vector<double> f, r, p;
    for (const auto& t : F) f.insert(f.end(), t.values.begin(), t.values.end());
    for (const auto& t : rho) r.insert(r.end(), t.values.begin(), t.values.end());
    for (const auto& t : phi) p.insert(p.end(), t.values.begin(), t.values.end());
    if (f.size() != static_cast<size_t>(nt) * nrho || r.size() != static_cast<size_t>(nt) * nr ||
        p.size() != npairs * static_cast<size_t>(nr))
      throw StatusError(TDMD_ERR_INVALID_ARGUMENT, "EamAlloy tables of unequal lengths");
    detail::check(tdmd_eam_create_sampled(nt, nrho, F[0].dr, nr, rho[0].dr, eam.cutoff(),
                                          f.data(), r.data(), p.data(), &own_));
    h_ = own_;
  }
#else
  explicit EamTables(const EamAlloy& eam) : h_(eam.handle()) {}
#endif
  ~EamTables() {
    if (own_) tdmd_eam_destroy(own_);
  }
  EamTables(const EamTables&) = delete;
  EamTables& operator=(const EamTables&) = delete;
  const tdmd_eam* get() const noexcept { return h_; }

 private:
  const tdmd_eam* h_ = nullptr;
  tdmd_eam* own_ = nullptr;
};

// device_eam.cuh:26-50
class DeviceEam {
 public:
  DeviceEam() = default;
  DeviceEam(const DeviceEam&) = delete;
  DeviceEam& operator=(const DeviceEam&) = delete;
  ~DeviceEam() {
    if (h_) tdmd_device_eam_destroy(h_);
  }

  void upload_tables(const EamAlloy& eam) {
    tdmd_device_eam* h = nullptr;
    detail::check(tdmd_device_eam_create(EamTables(eam).get(), &h));
    if (h_) tdmd_device_eam_destroy(h_);
    h_ = h;
    cutoff_ = eam.cutoff();
  }
  void compute(const PositionVec* d_positions, ForceVec* d_forces, const i32* d_types,
               const i32* d_neighbors, const i32* d_offsets, const i32* d_counts, i32 natoms,
               const Box& box, accum_t* d_energy, cudaStream_t stream = 0) {
    const tdmd_box b = detail::to_c(box);
    detail::check(tdmd_device_eam_compute(h_, reinterpret_cast<const double*>(d_positions),
                                          d_forces, kForcePrecision, d_types, d_neighbors,
                                          d_offsets, d_counts, natoms, &b, d_energy, nullptr,
                                          nullptr, nullptr, detail::stream_ptr(stream)));
  }
  real cutoff() const noexcept { return cutoff_; }

 private:
  tdmd_device_eam* h_ = nullptr;
  real cutoff_ = 0;
};

}  // namespace potentials

// --- src/io: LAMMPS data files and force dumps, setfl ------------------------
namespace io {

// lammps_data_reader.hpp / .cpp:33-204
inline SystemState read_lammps_data(const std::string& filename) {
  tdmd_system* h = nullptr;
  detail::check(tdmd_read_lammps_data(filename.c_str(), &h));
  struct Owner {
    tdmd_system* h;
    ~Owner() { tdmd_system_destroy(h); }
  } own{h};
  int64_t n = 0;
  int32_t nt = 0;
  tdmd_box b{};
  const double *p = nullptr, *v = nullptr, *m = nullptr;
  const int32_t *t = nullptr, *id = nullptr;
  detail::check(tdmd_system_get(h, &n, &nt, &b, &p, &v, &t, &id, &m));
  SystemState s;
  s.box.lo = Vec3D{b.lo[0], b.lo[1], b.lo[2]};
  s.box.hi = Vec3D{b.hi[0], b.hi[1], b.hi[2]};
  s.resize(n);
  for (i64 i = 0; i < n; ++i) {
    const size_t k = static_cast<size_t>(i);
    s.positions[k] = PositionVec{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
    s.velocities[k] = VelocityVec{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
    s.forces[k] = ForceVec{0, 0, 0};
    s.types[k] = t[i];
    s.ids[k] = id[i];
  }
  s.masses.assign(m, m + nt + 1);
  s.type_names.resize(static_cast<size_t>(nt) + 1);
  return s;
}

// dump_reader.hpp:14-26
struct DumpAtom {
  i32 id;
  i32 type;
  PositionVec pos;
  ForceVec force;
};

inline std::vector<DumpAtom> read_lammps_dump(const std::string& filename) {
  int64_t n = 0;
  detail::check(tdmd_read_force_dump(filename.c_str(), &n, 0, nullptr, nullptr, nullptr,
                                     nullptr));
  const size_t k = static_cast<size_t>(n);
  std::vector<int32_t> id(k), ty(k);
  std::vector<double> p(3 * k), f(3 * k);
  detail::check(tdmd_read_force_dump(filename.c_str(), &n, n, id.data(), ty.data(), p.data(),
                                     f.data()));
  std::vector<DumpAtom> out(k);
  for (size_t i = 0; i < k; ++i)
    out[i] = DumpAtom{id[i], ty[i], PositionVec{p[3 * i], p[3 * i + 1], p[3 * i + 2]},
                      ForceVec{static_cast<force_t>(f[3 * i]), static_cast<force_t>(f[3 * i + 1]),
                               static_cast<force_t>(f[3 * i + 2])}};
  return out;
}

// No reference counterpart (the reference only reads data files).
inline void write_lammps_data(const SystemState& s, const std::string& path,
                              const std::string& title = "tdmd_claude_b200 data") {
  const tdmd_box b = detail::to_c(s.box);
  std::vector<double> m(s.masses.begin(), s.masses.end());
  const int32_t nt = s.masses.empty() ? 1 : static_cast<int32_t>(s.masses.size()) - 1;
  detail::check(tdmd_write_lammps_data(
      path.c_str(), title.c_str(), s.natoms, nt, &b,
      reinterpret_cast<const double*>(s.positions.data()),
      reinterpret_cast<const double*>(s.velocities.data()), s.types.data(), s.ids.data(),
      m.empty() ? nullptr : m.data()));
}

// tdmd_main.cpp:65-95 (the reference driver's dump writer)
inline void write_lammps_force_dump(const SystemState& s, const std::string& path) {
  const tdmd_box b = detail::to_c(s.box);
  detail::check(tdmd_write_force_dump(path.c_str(), s.step, s.natoms, &b, s.ids.data(),
                                      s.types.data(),
                                      reinterpret_cast<const double*>(s.positions.data()),
                                      s.forces.data(), kForcePrecision));
}

// No reference counterpart (the reference only reads setfl).
inline void write_setfl(const potentials::EamAlloy& eam, const std::string& path) {
  detail::check(tdmd_write_setfl(path.c_str(), potentials::EamTables(eam).get(), nullptr, nullptr,
                                 nullptr));
}

}  // namespace io

// --- src/domain/device_cell_list.cuh:16-60 -------------------------------------
namespace domain {

class DeviceCellList {
 public:
  DeviceCellList() { detail::check(tdmd_cell_list_create(&h_)); }
  DeviceCellList(const DeviceCellList&) = delete;
  DeviceCellList& operator=(const DeviceCellList&) = delete;
  ~DeviceCellList() { tdmd_cell_list_destroy(h_); }

  void build(const PositionVec* d_positions, i64 natoms, const Box& box, real r_list) {
    const tdmd_box b = detail::to_c(box);
    detail::check(tdmd_cell_list_build(h_, reinterpret_cast<const double*>(d_positions), natoms,
                                       &b, r_list, nullptr));
    detail::check(tdmd_cell_list_get(h_, &atoms_, &offsets_, &counts_, &atom_cells_, nc_));
    const Vec3D L = box.size();
    cell_size_ = Vec3D{L.x / nc_[0], L.y / nc_[1], L.z / nc_[2]};  // cell_list.cpp:21-23
  }
  i32 ncells_x() const noexcept { return nc_[0]; }
  i32 ncells_y() const noexcept { return nc_[1]; }
  i32 ncells_z() const noexcept { return nc_[2]; }
  i32 ncells_total() const noexcept { return nc_[0] * nc_[1] * nc_[2]; }
  const i32* d_cell_offsets() const noexcept { return offsets_; }
  const i32* d_cell_counts() const noexcept { return counts_; }
  const i32* d_cell_atoms() const noexcept { return atoms_; }
  const i32* d_atom_cells() const noexcept { return atom_cells_; }
  Vec3D cell_size() const noexcept { return cell_size_; }

 private:
  tdmd_cell_list* h_ = nullptr;
  const int32_t* atoms_ = nullptr;
  const int32_t* offsets_ = nullptr;
  const int32_t* counts_ = nullptr;
  const int32_t* atom_cells_ = nullptr;
  int32_t nc_[3] = {0, 0, 0};
  Vec3D cell_size_{0, 0, 0};
};

}  // namespace domain

// --- src/neighbors/device_neighbor_list.cuh:20-65 ------------------------------
namespace neighbors {

class DeviceNeighborList {
 public:
  DeviceNeighborList() { detail::check(tdmd_nlist_create(&h_)); }
  DeviceNeighborList(const DeviceNeighborList&) = delete;
  DeviceNeighborList& operator=(const DeviceNeighborList&) = delete;
  ~DeviceNeighborList() { tdmd_nlist_destroy(h_); }

  void build(const PositionVec* d_positions, i64 natoms, const Box& box, real r_cut, real r_skin,
             cudaStream_t stream = 0) {
    const tdmd_box b = detail::to_c(box);
    detail::check(tdmd_nlist_build(h_, reinterpret_cast<const double*>(d_positions), natoms, &b,
                                   r_cut, r_skin, detail::stream_ptr(stream)));
    int64_t total = 0;
    detail::check(tdmd_nlist_get(h_, &nbrs_, &offsets_, &counts_, &max_neighbors_, &total));
    r_cut_ = r_cut;
    r_skin_ = r_skin;
  }
  const i32* d_neighbors() const noexcept { return nbrs_; }
  const i32* d_counts() const noexcept { return counts_; }
  const i32* d_offsets() const noexcept { return offsets_; }
  real cutoff() const noexcept { return r_cut_; }
  real skin() const noexcept { return r_skin_; }
  i32 max_neighbors() const noexcept { return max_neighbors_; }

 private:
  tdmd_nlist* h_ = nullptr;
  const int32_t* nbrs_ = nullptr;
  const int32_t* offsets_ = nullptr;
  const int32_t* counts_ = nullptr;
  int32_t max_neighbors_ = 0;
  real r_cut_ = 0;
  real r_skin_ = 0;
};

}  // namespace neighbors

// --- src/integrator -----------------------------------------------------------
namespace integrator {

namespace detail_masses {
// The C ABI takes FP64 device masses.  In the FP64 build `real` is double
// and the pointer passes through.  In the mixed build (float masses, as the
// reference's `real`) the entries up to the largest type in d_types are
// widened into a small per-thread device array first; that costs a read of
// the types and two small copies per call, which the scheduler path never
// pays (it keeps its own FP64 masses).
#if defined(TDMD_PRECISION_MIXED)
struct Widened {
  double* d = nullptr;
  size_t cap = 0;
  ~Widened() {
    if (d) cudaFree(d);
  }
};
inline const double* masses(const real* d_masses, const i32* d_types, i32 natoms,
                            cudaStream_t stream) {
  thread_local Widened w;
  void* s = ::tdmd::detail::stream_ptr(stream);
  std::vector<int32_t> types(static_cast<size_t>(natoms > 0 ? natoms : 0));
  if (!types.empty())
    ::tdmd::detail::check(tdmd_copy(types.data(), d_types, sizeof(int32_t) * types.size(), s));
  int32_t tmax = 0;
  for (int32_t t : types) tmax = t > tmax ? t : tmax;
  std::vector<float> hf(static_cast<size_t>(tmax) + 1);
  ::tdmd::detail::check(tdmd_copy(hf.data(), d_masses, sizeof(float) * hf.size(), s));
  std::vector<double> hd(hf.begin(), hf.end());
  if (w.cap < hd.size()) {
    if (w.d) cudaFree(w.d);
    w.d = nullptr;
    w.cap = 0;
    if (cudaMalloc(reinterpret_cast<void**>(&w.d), sizeof(double) * hd.size()) != cudaSuccess)
      throw StatusError(TDMD_ERR_OUT_OF_MEMORY, "mass buffer allocation failed");
    w.cap = hd.size();
  }
  ::tdmd::detail::check(tdmd_copy(w.d, hd.data(), sizeof(double) * hd.size(), s));
  return w.d;
}
#else
inline const double* masses(const real* d_masses, const i32*, i32, cudaStream_t) {
  return d_masses;
}
#endif
}  // namespace detail_masses

// device_velocity_verlet.cuh:13-59
inline void device_half_kick(VelocityVec* d_velocities, const ForceVec* d_forces,
                             const i32* d_types, const real* d_masses, i32 natoms, real dt,
                             cudaStream_t stream = 0) {
  ::tdmd::detail::check(tdmd_vv_half_kick(
      reinterpret_cast<double*>(d_velocities), d_forces, kForcePrecision, d_types,
      detail_masses::masses(d_masses, d_types, natoms, stream), natoms, dt, ::tdmd::detail::stream_ptr(stream)));
}
inline void device_drift(PositionVec* d_positions, const VelocityVec* d_velocities, i32 natoms,
                         real dt, const Box& box, cudaStream_t stream = 0) {
  const tdmd_box b = detail::to_c(box);
  ::tdmd::detail::check(tdmd_vv_drift(reinterpret_cast<double*>(d_positions),
                                      reinterpret_cast<const double*>(d_velocities), natoms, dt,
                                      &b, ::tdmd::detail::stream_ptr(stream)));
}
inline void device_fused_half_kick_drift(VelocityVec* d_velocities, PositionVec* d_positions,
                                         const ForceVec* d_forces, const i32* d_types,
                                         const real* d_masses, i32 natoms, real dt,
                                         const Box& box, cudaStream_t stream = 0) {
  const tdmd_box b = detail::to_c(box);
  ::tdmd::detail::check(tdmd_vv_fused_kick_drift(
      reinterpret_cast<double*>(d_velocities), reinterpret_cast<double*>(d_positions), d_forces,
      kForcePrecision, d_types, detail_masses::masses(d_masses, d_types, natoms, stream), natoms, dt, &b, 0,
      ::tdmd::detail::stream_ptr(stream)));
}
inline void device_fused_full_kick_drift(VelocityVec* d_velocities, PositionVec* d_positions,
                                         const ForceVec* d_forces, const i32* d_types,
                                         const real* d_masses, i32 natoms, real dt,
                                         const Box& box, cudaStream_t stream = 0) {
  const tdmd_box b = detail::to_c(box);
  ::tdmd::detail::check(tdmd_vv_fused_kick_drift(
      reinterpret_cast<double*>(d_velocities), reinterpret_cast<double*>(d_positions), d_forces,
      kForcePrecision, d_types, detail_masses::masses(d_masses, d_types, natoms, stream), natoms, dt, &b, 1,
      ::tdmd::detail::stream_ptr(stream)));
}
inline void device_zero_forces(ForceVec* d_forces, i32 natoms, cudaStream_t stream = 0) {
  ::tdmd::detail::check(
      tdmd_vv_zero_forces(d_forces, kForcePrecision, natoms, ::tdmd::detail::stream_ptr(stream)));
}

// device_velocity_verlet_zone.cuh:12-29: the same kernels on atoms
// [first_atom, first_atom + atom_count) of the arrays.
inline void device_half_kick_zone(VelocityVec* d_velocities, const ForceVec* d_forces,
                                  const i32* d_types, const real* d_masses, i32 first_atom,
                                  i32 atom_count, real dt, cudaStream_t stream) {
  device_half_kick(d_velocities + first_atom, d_forces + first_atom, d_types + first_atom,
                   d_masses, atom_count, dt, stream);
}
inline void device_drift_zone(PositionVec* d_positions, const VelocityVec* d_velocities,
                              i32 first_atom, i32 atom_count, real dt, const Box& box,
                              cudaStream_t stream) {
  device_drift(d_positions + first_atom, d_velocities + first_atom, atom_count, dt, box, stream);
}
inline void device_zero_forces_zone(ForceVec* d_forces, i32 first_atom, i32 atom_count,
                                    cudaStream_t stream) {
  device_zero_forces(d_forces + first_atom, atom_count, stream);
}

// device_nose_hoover.cuh:26-88
struct NHCConfig {
  real t_target{300.0};
  real t_period{0.1};
  i32 chain_length{3};
};

class NoseHooverChain {
 public:
  NoseHooverChain(const NHCConfig& cfg, real dt, i32 n_dof) : cfg_(cfg) {
    ::tdmd::detail::check(
        tdmd_nhc_create(cfg.t_target, cfg.t_period, cfg.chain_length, dt, n_dof, &h_));
  }
  NoseHooverChain(const NoseHooverChain&) = delete;
  NoseHooverChain& operator=(const NoseHooverChain&) = delete;
  ~NoseHooverChain() { tdmd_nhc_destroy(h_); }

  real half_step(accum_t ke_current) {
    double scale = 1.0;
    ::tdmd::detail::check(tdmd_nhc_half_step(h_, ke_current, &scale));
    return static_cast<real>(scale);
  }
  real t_target() const noexcept { return cfg_.t_target; }
  void set_t_target(real t) {
    ::tdmd::detail::check(tdmd_nhc_set_t_target(h_, t));
    cfg_.t_target = t;
  }

 private:
  NHCConfig cfg_;
  tdmd_nhc* h_ = nullptr;
};

inline accum_t device_compute_ke(const VelocityVec* d_velocities, const i32* d_types,
                                 const real* d_masses, i32 natoms) {
  double ke = 0;
  ::tdmd::detail::check(tdmd_reduce_ke(reinterpret_cast<const double*>(d_velocities), d_types,
                                       detail_masses::masses(d_masses, d_types, natoms, 0), natoms, &ke,
                                       nullptr));
  return ke;
}
inline void device_scale_velocities(VelocityVec* d_velocities, i32 natoms, real factor) {
  ::tdmd::detail::check(
      tdmd_scale_velocities(reinterpret_cast<double*>(d_velocities), natoms, factor, nullptr));
}
// The zone variant scales atoms [first_atom, first_atom + atom_count).
inline void device_scale_velocities_zone(VelocityVec* d_velocities, i32 first_atom,
                                         i32 atom_count, real factor,
                                         cudaStream_t stream = nullptr) {
  ::tdmd::detail::check(tdmd_scale_velocities(reinterpret_cast<double*>(d_velocities + first_atom),
                                              atom_count, factor,
                                              ::tdmd::detail::stream_ptr(stream)));
}
inline accum_t device_compute_vmax(const VelocityVec* d_velocities, i32 natoms) {
  double v = 0;
  ::tdmd::detail::check(
      tdmd_reduce_vmax(reinterpret_cast<const double*>(d_velocities), natoms, &v, nullptr));
  return v;
}

}  // namespace integrator

// --- src/scheduler/fast_pipeline_scheduler.cuh:36-192 --------------------------
namespace scheduler {

enum class PotentialKind {
  Morse,
  Eam,
};

// The reference's three fields first (so FastPipelineConfig{dt, skin, R}
// still works), then this library's additions with their defaults.
struct FastPipelineConfig {
  real dt{real{0.001}};
  real r_skin{real{1.0}};
  i32 rebuild_every{10};
  bool use_graphs{true};
  i32 lanes_per_atom{0};
  real t_target{0};
  real t_period{real{0.1}};
  i32 nhc_length{3};
  bool adaptive_dt{false};
  real dt_min{real{0.0001}};
  real dt_max{real{0.002}};
  real c2{real{0.05}};
  i32 energy_every{0};
  i32 energy_log_capacity{0};
  i32 nbr_batch{0};  // neighbors per lane sweep: 0 = autotuned, else 2 or 4

  tdmd_fast_pipeline_config to_c() const {
    tdmd_fast_pipeline_config c;
    tdmd_fast_pipeline_config_default(&c);
    c.dt = dt;
    c.r_skin = r_skin;
    c.rebuild_every = rebuild_every;
    c.precision = kForcePrecision;
    c.use_graphs = use_graphs ? 1 : 0;
    c.lanes_per_atom = lanes_per_atom;
    c.t_target = t_target;
    c.t_period = t_period;
    c.nhc_length = nhc_length;
    c.adaptive_dt = adaptive_dt ? 1 : 0;
    c.dt_min = dt_min;
    c.dt_max = dt_max;
    c.c2 = c2;
    c.energy_every = energy_every;
    c.energy_log_capacity = energy_log_capacity;
    c.nbr_batch = nbr_batch;
    return c;
  }
};

struct FastPipelineStats {
  i64 ticks{0};
  i64 kernel_launches{0};
  i64 rebuilds{0};
};

class FastPipelineScheduler {
 public:
  FastPipelineScheduler(const Box& box, i32 natoms, const potentials::MorseParams& params,
                        const FastPipelineConfig& cfg) {
    const tdmd_box b = detail::to_c(box);
    const tdmd_morse_params p = params.to_c();
    const tdmd_fast_pipeline_config c = cfg.to_c();
    ::tdmd::detail::check(tdmd_sched_create_morse(&b, natoms, &p, &c, &h_));
    refresh();
  }
  FastPipelineScheduler(const Box& box, i32 natoms, const potentials::EamAlloy& eam,
                        const FastPipelineConfig& cfg) {
    const tdmd_box b = detail::to_c(box);
    const tdmd_fast_pipeline_config c = cfg.to_c();
    ::tdmd::detail::check(
        tdmd_sched_create_eam(&b, natoms, potentials::EamTables(eam).get(), &c, &h_));
    refresh();
  }
  ~FastPipelineScheduler() { tdmd_sched_destroy(h_); }
  FastPipelineScheduler(const FastPipelineScheduler&) = delete;
  FastPipelineScheduler& operator=(const FastPipelineScheduler&) = delete;

  void upload(const PositionVec* positions, const VelocityVec* velocities, const ForceVec* forces,
              const i32* types, const i32* ids, const real* masses, i32 n_types) {
    std::vector<double> m(masses, masses + n_types);
    ::tdmd::detail::check(tdmd_sched_upload(h_, reinterpret_cast<const double*>(positions),
                                            reinterpret_cast<const double*>(velocities), forces,
                                            types, ids, m.data(), n_types));
    refresh();
  }
  void run_until(i32 target_step) {
    ::tdmd::detail::check(tdmd_sched_run_until(h_, target_step));
    refresh();
  }
  void download(PositionVec* positions, VelocityVec* velocities, ForceVec* forces, i32* types,
                i32* ids, i32 natoms) const {
    ::tdmd::detail::check(tdmd_sched_download(h_, reinterpret_cast<double*>(positions),
                                              reinterpret_cast<double*>(velocities), forces,
                                              types, ids, natoms));
  }
  const FastPipelineStats& stats() const noexcept { return stats_; }
  i32 current_step() const noexcept { return step_; }
  PotentialKind potential_kind() const noexcept { return kind_; }
  real interaction_cutoff() const noexcept { return cutoff_; }
  tdmd_sched* handle() const noexcept { return h_; }

 private:
  void refresh() {
    tdmd_fast_pipeline_stats s{};
    ::tdmd::detail::check(tdmd_sched_stats(h_, &s));
    stats_ = FastPipelineStats{s.ticks, s.kernel_launches, s.rebuilds};
    ::tdmd::detail::check(tdmd_sched_current_step(h_, &step_));
    int32_t k = 0;
    ::tdmd::detail::check(tdmd_sched_potential_kind(h_, &k));
    kind_ = k == TDMD_POT_EAM ? PotentialKind::Eam : PotentialKind::Morse;
    double c = 0;
    ::tdmd::detail::check(tdmd_sched_interaction_cutoff(h_, &c));
    cutoff_ = static_cast<real>(c);
  }

  tdmd_sched* h_ = nullptr;
  FastPipelineStats stats_{};
  i32 step_ = 0;
  PotentialKind kind_ = PotentialKind::Morse;
  real cutoff_ = 0;
};

}  // namespace scheduler

#if !defined(TDMD_B200_REFERENCE_CORE)
// --- src/scheduler/zone.hpp, src/domain/zone_partition.hpp (single rank) ----
namespace scheduler {
enum class ZoneState : std::uint8_t {
  Free = 0,
  Receiving = 1,
  Received = 2,
  Ready = 3,
  Computing = 4,
  Done = 5,
  Sending = 6,
};

// The zone life cycle (zone.hpp:22-40): Free -> Receiving -> Received ->
// Ready -> Computing -> Done -> Sending -> Free.
constexpr bool is_legal_transition(ZoneState from, ZoneState to) noexcept {
  switch (from) {
    case ZoneState::Free: return to == ZoneState::Receiving;
    case ZoneState::Receiving: return to == ZoneState::Received;
    case ZoneState::Received: return to == ZoneState::Ready;
    case ZoneState::Ready: return to == ZoneState::Computing;
    case ZoneState::Computing: return to == ZoneState::Done;
    case ZoneState::Done: return to == ZoneState::Sending;
    case ZoneState::Sending: return to == ZoneState::Free;
  }
  return false;
}

struct Zone {
  i32 id{-1};
  std::array<i32, 3> lattice_index{0, 0, 0};
  Aabb bbox{};
  i32 atom_offset{0};
  i32 natoms_in_zone{0};
  i32 time_step{0};
  ZoneState state{ZoneState::Free};
  i32 owner_rank{-1};

  // A step of the life cycle; reaching Done completes a time step.  An
  // illegal one throws (the reference asserts).
  void transition_to(ZoneState next) {
    if (!is_legal_transition(state, next))
      throw StatusError(TDMD_ERR_STATE, "illegal zone transition");
    state = next;
    if (next == ZoneState::Done) ++time_step;
  }
};
}  // namespace scheduler

namespace domain {
// Slabs of the box along x (zone_partition.cpp:12-40): n zones of width
// L_x / n, n = max(3, floor(L_x / r_cut)) unless given; a zone's neighbors
// are the zones within r_list of it, periodic in x.
class ZonePartition {
 public:
  void build(const Box& box, real r_cut, i32 n_zones = 0) {
    const Vec3D size = box.size();
    lo_x_ = box.lo.x;
    if (n_zones <= 0) n_zones = std::max(3, static_cast<i32>(std::floor(size.x / r_cut)));
    if (n_zones < 3) throw StatusError(TDMD_ERR_INVALID_ARGUMENT, "need at least 3 zones");
    width_ = size.x / n_zones;
    zones_.assign(static_cast<size_t>(n_zones), scheduler::Zone{});
    for (i32 i = 0; i < n_zones; ++i) {
      scheduler::Zone& z = zones_[static_cast<size_t>(i)];
      z.id = i;
      z.lattice_index = {i, 0, 0};
      z.bbox.lo = Vec3D{box.lo.x + i * width_, box.lo.y, box.lo.z};
      z.bbox.hi = Vec3D{box.lo.x + (i + 1) * width_, box.hi.y, box.hi.z};
      z.owner_rank = 0;
    }
    neighbors_.assign(static_cast<size_t>(n_zones), {});
  }
  void build_zone_neighbors(real r_list) {
    const i32 n = n_zones();
    const i32 reach = std::min(n / 2, static_cast<i32>(std::ceil(r_list / width_)));
    for (i32 i = 0; i < n; ++i) {
      std::vector<i32>& nb = neighbors_[static_cast<size_t>(i)];
      nb.clear();
      for (i32 d = -reach; d <= reach; ++d) {
        const i32 j = ((i + d) % n + n) % n;
        if (std::find(nb.begin(), nb.end(), j) == nb.end()) nb.push_back(j);
      }
      std::sort(nb.begin(), nb.end());
    }
  }
  i32 n_zones() const noexcept { return static_cast<i32>(zones_.size()); }
  const std::vector<scheduler::Zone>& zones() const noexcept { return zones_; }
  std::vector<scheduler::Zone>& zones() noexcept { return zones_; }
  i32 zone_of(real x) const noexcept {
    i32 z = static_cast<i32>((x - lo_x_) / width_);
    return z < 0 ? 0 : (z >= n_zones() ? n_zones() - 1 : z);
  }
  const std::vector<i32>& zone_neighbors(i32 z) const {
    return neighbors_[static_cast<size_t>(z)];
  }
  // Groups the host arrays by zone, in input order within a zone (a
  // counting sort on x), and records each zone's offset and count.
  void assign_atoms(PositionVec* positions, VelocityVec* velocities, ForceVec* forces, i32* types,
                    i32* ids, i64 natoms) {
    const size_t n = static_cast<size_t>(natoms), nz = static_cast<size_t>(n_zones());
    std::vector<i32> zone(n), count(nz, 0), offset(nz, 0), perm(n);
    for (size_t i = 0; i < n; ++i) {
      zone[i] = zone_of(static_cast<real>(positions[i].x));
      ++count[static_cast<size_t>(zone[i])];
    }
    for (size_t z = 1; z < nz; ++z) offset[z] = offset[z - 1] + count[z - 1];
    std::vector<i32> next(offset);
    for (size_t i = 0; i < n; ++i)
      perm[static_cast<size_t>(next[static_cast<size_t>(zone[i])]++)] = static_cast<i32>(i);
    permute(positions, perm);
    permute(velocities, perm);
    permute(forces, perm);
    permute(types, perm);
    permute(ids, perm);
    for (size_t z = 0; z < nz; ++z) {
      zones_[z].atom_offset = offset[z];
      zones_[z].natoms_in_zone = count[z];
    }
  }

 private:
  template <class T>
  static void permute(T* a, const std::vector<i32>& perm) {
    std::vector<T> tmp(perm.size());
    for (size_t i = 0; i < perm.size(); ++i) tmp[i] = a[static_cast<size_t>(perm[i])];
    std::copy(tmp.begin(), tmp.end(), a);
  }

  double lo_x_ = 0.0;
  double width_ = 1.0;
  std::vector<scheduler::Zone> zones_;
  std::vector<std::vector<i32>> neighbors_;
};
}  // namespace domain
#endif  // !TDMD_B200_REFERENCE_CORE

namespace scheduler {

// --- src/scheduler/pipeline_scheduler.cuh:18-44 -----------------------------
struct PipelineConfig {
  real dt{real{0.001}};
  real r_skin{real{1.0}};
  i32 n_zones{0};      // 0: max(3, floor(L_x / rc))
  i32 n_streams{4};    // accepted; one stream here
  i32 rebuild_every{10};
  bool deterministic{false};  // accepted; every run here is deterministic
  real t_target{0};    // > 0: NVT (Nose-Hoover chain)
  real t_period{real{0.1}};
  i32 nhc_length{3};
  bool adaptive_dt{false};
  real dt_max{real{0.002}};
  real dt_min{real{0.0001}};
  real c2{real{0.05}};
};

struct PipelineStats {
  i64 kernel_launches{0};
  i64 dep_check_calls{0};
  i64 dep_check_failures{0};
  i64 ticks{0};
};

// The reference's TD zone pipeline (pipeline_scheduler.cu:93-290) with its
// API and physics -- one velocity-Verlet step per zone step, NVT as the
// NHC half step around each step, adaptive dt from v_max -- run as whole-
// system windows on the library's scheduler: on one GPU the zones gain
// nothing from being stepped apart (the reference's own deterministic mode
// equals the plain sequential loop), so all zones advance together.  The
// partition is built as the reference builds it and reported (zone time
// steps follow the run); no zone waits on another, so no dependency checks
// are counted.
class PipelineScheduler {
 public:
  PipelineScheduler(const Box& box, i32 natoms, const potentials::MorseParams& params,
                    const PipelineConfig& cfg) {
    partition_.build(box, params.rc, cfg.n_zones);
    partition_.build_zone_neighbors(params.rc + cfg.r_skin);
    FastPipelineConfig f{};
    f.dt = cfg.dt;
    f.r_skin = cfg.r_skin;
    f.rebuild_every = cfg.rebuild_every;
    f.t_target = cfg.t_target;
    f.t_period = cfg.t_period;
    f.nhc_length = cfg.nhc_length;
    f.adaptive_dt = cfg.adaptive_dt;
    f.dt_min = cfg.dt_min;
    f.dt_max = cfg.dt_max;
    f.c2 = cfg.c2;
    sched_ = std::make_unique<FastPipelineScheduler>(box, natoms, params, f);
    natoms_ = natoms;
  }

  void upload(const PositionVec* positions, const VelocityVec* velocities, const ForceVec* forces,
              const i32* types, const i32* ids, const real* masses, i32 n_masses) {
    sched_->upload(positions, velocities, forces, types, ids, masses, n_masses);
    // zone populations as the reference's assign_atoms groups them
    const i32 nz = partition_.n_zones();
    std::vector<i32> count(static_cast<size_t>(nz), 0);
    for (i32 i = 0; i < natoms_; ++i)
      ++count[static_cast<size_t>(
          partition_.zone_of(static_cast<real>(positions[static_cast<size_t>(i)].x)))];
    i32 off = 0;
    for (i32 z = 0; z < nz; ++z) {
      Zone& zone = partition_.zones()[static_cast<size_t>(z)];
      zone.atom_offset = off;
      zone.natoms_in_zone = count[static_cast<size_t>(z)];
      off += zone.natoms_in_zone;
    }
    set_zones(0);
  }
  void run_until(i32 target_step) {
    sched_->run_until(target_step);
    set_zones(sched_->current_step());
    const FastPipelineStats& f = sched_->stats();
    stats_.kernel_launches = f.kernel_launches;
    stats_.ticks = f.ticks;
  }
  void download(PositionVec* positions, VelocityVec* velocities, ForceVec* forces, i32* types,
                i32* ids, i32 natoms) const {
    sched_->download(positions, velocities, forces, types, ids, natoms);
  }
  const domain::ZonePartition& partition() const noexcept { return partition_; }
  const PipelineStats& stats() const noexcept { return stats_; }
  i32 min_time_step() const noexcept {
    i32 m = std::numeric_limits<i32>::max();
    for (const Zone& z : partition_.zones()) m = std::min(m, z.time_step);
    return m;
  }

 private:
  void set_zones(i32 step) {
    for (Zone& z : partition_.zones()) {
      z.time_step = step;
      z.state = ZoneState::Ready;
    }
  }

  domain::ZonePartition partition_;
  std::unique_ptr<FastPipelineScheduler> sched_;
  PipelineStats stats_{};
  i32 natoms_ = 0;
};

}  // namespace scheduler
}  // namespace tdmd
