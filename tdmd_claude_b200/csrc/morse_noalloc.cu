// morse_noalloc.cu -- Morse forces, energy and virial with no device
// allocation: the per-block energy/virial partials that tdmd_morse_compute
// takes from the stream-ordered pool live here in a fixed, file-scope device
// array instead.
//
// Who needs it: a caller that sizes all of its device memory up front (a
// fixed arena handed to its own allocator, or a step loop in which any
// allocation is treated as an error) cannot let a force call draw on the
// CUDA memory pool, which may grow, block or fail at an arbitrary step.
//
// Limits and rules (also stated at the declaration in tdmd_b200.h):
//  * natoms <= TDMD_MORSE_NOALLOC_MAX_ATOMS; larger inputs are rejected with
//    TDMD_ERR_INVALID_ARGUMENT before anything is launched;
//  * the scratch holds at most kMaxBlocks partial records (1 MiB); every
//    block of the force kernel overwrites its own record before the
//    reduction reads it, so the scratch needs no zeroing.  The launch uses
//    tdmd_morse_compute's lanes per atom, halved while its blocks would
//    exceed kMaxBlocks (never at the default choice on a B200, whose lanes
//    give 16384 blocks at the atom limit; one lane per atom always fits);
//  * d_energy / d_virial are ADDED to, as in tdmd_morse_compute: zero them
//    first to get this call's totals alone; d_forces is overwritten;
//  * there is one scratch per device, so two calls in flight on the same
//    device at once (different streams, or different host threads without
//    ordering between them) race on it; order them on one stream;
//  * the first call on each device that asks for an energy or a virial
//    looks up the scratch's device address (cudaGetSymbolAddress, which may
//    load this module); make that first call before any stream capture
//    begins on that device.  Force-only and empty calls need no scratch and
//    do no look-up.
#include <mutex>

#include "common.cuh"
#include "forces.cuh"
#include "launch.cuh"
#include "tdmd_b200.h"

namespace tdmd_b200 {
namespace {

// Force blocks at the atom limit with the default 8 lanes per atom.
constexpr int kMaxBlocks =
    static_cast<int>(static_cast<long long>(TDMD_MORSE_NOALLOC_MAX_ATOMS) * 8 / kForceThreads);
constexpr int kMaxDevices = 64;

// One lane per atom fits at the atom limit, so halving the lanes always
// ends inside the scratch; the default 8 lanes of large inputs fit too.
static_assert(static_cast<long long>(TDMD_MORSE_NOALLOC_MAX_ATOMS) <=
                  static_cast<long long>(kMaxBlocks) * kForceThreads,
              "one lane per atom must fit the scratch at the atom limit");
static_assert(static_cast<long long>(TDMD_MORSE_NOALLOC_MAX_ATOMS) * 8 <=
                  static_cast<long long>(kMaxBlocks) * kForceThreads,
              "the default lanes of large inputs must fit the scratch at the atom limit");

// Per-block {energy, virial[6], pad} records of the force kernel.
static __device__ __align__(256) double g_morse_partials[kMaxBlocks * kEvStride];

std::mutex g_scratch_mutex;
double* g_scratch[kMaxDevices] = {};

// The scratch's address on the current device (set up once per device).
double* scratch_for_current_device() {
  int dev = -1;
  TDMD_CU(cudaGetDevice(&dev));
  TDMD_REQUIRE(dev >= 0 && dev < kMaxDevices, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch[dev]) {
    void* p = nullptr;
    TDMD_CU(cudaGetSymbolAddress(&p, g_morse_partials));
    TDMD_REQUIRE(p != nullptr, "scratch address lookup returned null");
    g_scratch[dev] = static_cast<double*>(p);
  }
  return g_scratch[dev];
}

}  // namespace
}  // namespace tdmd_b200

using namespace tdmd_b200;

extern "C" int32_t tdmd_morse_compute_noalloc(const double* d_positions, void* d_forces,
                                              int32_t precision, const int32_t* d_neighbors,
                                              const int32_t* d_offsets, const int32_t* d_counts,
                                              int32_t natoms, const tdmd_box* box,
                                              const tdmd_morse_params* params, double* d_energy,
                                              double* d_virial, void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(box && params, "null box or params");
    TDMD_REQUIRE(natoms >= 0, "natoms must be non-negative");
    TDMD_REQUIRE(natoms <= TDMD_MORSE_NOALLOC_MAX_ATOMS,
                 "natoms exceeds TDMD_MORSE_NOALLOC_MAX_ATOMS (fixed scratch size)");
    TDMD_REQUIRE(precision == TDMD_FP64 || precision == TDMD_MIXED, "unknown precision");
    if (natoms == 0) return;
    TDMD_REQUIRE(d_positions && d_forces && d_offsets && d_counts, "null device array");
    cudaStream_t s = as_stream(stream);
    const DevBox b = make_devbox(*box, 0.0);
    const NbrView nl{d_neighbors, d_offsets, d_counts, 0};
    const bool ev = d_energy || d_virial;
    int lpa = default_lpa(natoms);
    while (lpa > 1 && force_blocks(natoms, lpa) > kMaxBlocks) lpa >>= 1;
    const int nblk = force_blocks(natoms, lpa);
    TDMD_REQUIRE(nblk <= kMaxBlocks, "partial records exceed the fixed scratch");
    double* part = ev ? scratch_for_current_device() : nullptr;
    if (precision == TDMD_FP64) {
      GeoAoS64 g{d_positions, {b.L[0], b.L[1], b.L[2]}, {b.halfL[0], b.halfL[1], b.halfL[2]},
                 {b.periodic[0], b.periodic[1], b.periodic[2]}};
      MorseP<double> mp{params->d, params->alpha, params->r0, params->rc_sq, params->r0};
      launch_morse(g, nl, natoms, mp, static_cast<double*>(d_forces), ev, part, lpa, s);
    } else {
      const GeoAoS32 g = make_geo_aos32(d_positions, b);
      MorseP<float> mp{float(params->d), float(params->alpha), float(params->r0),
                       float(params->rc_sq), params->r0};
      launch_morse(g, nl, natoms, mp, static_cast<float*>(d_forces), ev, part, lpa, s);
    }
    if (ev) {
      launch(k_reduce_partials, 1, 256, 0, s, part, nblk, d_energy, d_virial);
      TDMD_LAUNCH_CHECK();
    }
  });
}
