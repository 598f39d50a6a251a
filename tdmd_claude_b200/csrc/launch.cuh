// launch.cuh -- host-side launchers of the force kernels: runtime LPA
// (lanes per atom) and energy/virial flags dispatched onto the template
// instantiations in forces.cuh.
#pragma once

#include "common.cuh"
#include "forces.cuh"

namespace tdmd_b200 {

constexpr int kForceThreads = 256;

int force_blocks(long long n, int lpa);
int default_lpa(long long n);

// VEC (16-byte aligned padded rows) is a runtime property of the view.
#define TDMD_VEC_DISPATCH(vec, ...)                               \
  if (vec) {                                                      \
    constexpr bool V = true;                                      \
    __VA_ARGS__;                                                  \
  } else {                                                        \
    constexpr bool V = false;                                     \
    __VA_ARGS__;                                                  \
  }

// MULTI: more than one atom type (per-neighbor type loads, pair-slot
// lookup); single-type alloys compile those out.
#define TDMD_MULTI_DISPATCH(multi, ...)                           \
  if (multi) {                                                    \
    constexpr bool M = true;                                      \
    __VA_ARGS__;                                                  \
  } else {                                                        \
    constexpr bool M = false;                                     \
    __VA_ARGS__;                                                  \
  }

inline bool vec_rows(const NbrView& nl) { return nl.row_off == nullptr && nl.cap % 4 == 0; }

#define TDMD_LPA_DISPATCH(lpa, ...)                              \
  switch (lpa) {                                                  \
    case 1: { constexpr int L = 1; __VA_ARGS__; } break;          \
    case 2: { constexpr int L = 2; __VA_ARGS__; } break;          \
    case 4: { constexpr int L = 4; __VA_ARGS__; } break;          \
    case 8: { constexpr int L = 8; __VA_ARGS__; } break;          \
    case 16: { constexpr int L = 16; __VA_ARGS__; } break;        \
    case 32: { constexpr int L = 32; __VA_ARGS__; } break;        \
    default: throw Error{TDMD_ERR_INVALID_ARGUMENT, "lanes per atom must be 1,2,4,8,16,32"}; \
  }

// Launch shape of the gather passes: lanes per atom and neighbors per lane
// per sweep.  A bare lanes count means the untuned sweep of kU.
struct Tune {
  int lpa;
  int nu;
  Tune(int lanes = 1, int batch = kU) : lpa(lanes), nu(batch) {}
};

#define TDMD_NU_DISPATCH(nu, ...)                                \
  switch (nu) {                                                   \
    case 2: { constexpr int U = 2; __VA_ARGS__; } break;          \
    case 4: { constexpr int U = 4; __VA_ARGS__; } break;          \
    default: throw Error{TDMD_ERR_INVALID_ARGUMENT, "neighbor batch must be 2 or 4"}; \
  }

// Defines L (lanes per atom) and U (neighbor batch) for the body.
#define TDMD_TUNE_DISPATCH(tn, ...) \
  TDMD_NU_DISPATCH((tn).nu, TDMD_LPA_DISPATCH((tn).lpa, __VA_ARGS__))

// Morse forces; with ev, per-block partials (force_blocks records; nullable)
// and per-atom energies (pe_atom, nullable).
template <class Geo, class F>
void launch_morse(const Geo& g, const NbrView& nl, int n, const MorseP<typename Geo::T>& mp,
                  F* forces, bool ev, double* partials, Tune tn, cudaStream_t s,
                  double* pe_atom = nullptr) {
  const int nblk = force_blocks(n, tn.lpa);
  TDMD_VEC_DISPATCH(vec_rows(nl), TDMD_TUNE_DISPATCH(tn, {
    if (ev && !partials && pe_atom)  // per-atom energies only
      launch(k_morse<Geo, L, U, 2, V, F>, nblk, kForceThreads, 0, s, g, nl, n, mp,
             ForceOut<F>{forces}, nullptr, pe_atom);
    else if (ev)
      launch(k_morse<Geo, L, U, 1, V, F>, nblk, kForceThreads, 0, s, g, nl, n, mp,
             ForceOut<F>{forces}, partials, pe_atom);
    else
      launch(k_morse<Geo, L, U, 0, V, F>, nblk, kForceThreads, 0, s, g, nl, n, mp,
             ForceOut<F>{forces}, nullptr, nullptr);
  }));
  TDMD_LAUNCH_CHECK();
}

// Morse forces of atoms [first, first + n) ADDED to forces[first ..], the
// neighbor j of a row read at its global index (the per-zone call).  nl's
// row offsets and counts are those of the range (shifted by the caller);
// dense CSR rows only, U = kU.
template <class Geo, class F>
void launch_morse_zone(const Geo& g, int first, const NbrView& nl, int n,
                       const MorseP<typename Geo::T>& mp, F* forces, bool ev, double* partials,
                       int lpa, cudaStream_t s) {
  const int nblk = force_blocks(n, lpa);
  const GeoShift<Geo> gs{g, first};
  const ForceAdd<F> out{forces + 3ll * first};
  TDMD_LPA_DISPATCH(lpa, {
    if (ev)
      launch(k_morse<GeoShift<Geo>, L, kU, 1, false, F, ForceAdd<F>>, nblk, kForceThreads, 0, s,
             gs, nl, n, mp, out, partials, nullptr);
    else
      launch(k_morse<GeoShift<Geo>, L, kU, 0, false, F, ForceAdd<F>>, nblk, kForceThreads, 0, s,
             gs, nl, n, mp, out, nullptr, nullptr);
  });
  TDMD_LAUNCH_CHECK();
}

// Density + embedding pass.  gout (fixed-point geometries only) receives
// the force pass's {q, F'} gather records, gout64 (GeoD4 / GeoD4B) its FP64
// records {x, y, z, F'}; e_out (nullable) each atom's embedding energy
// F(rho_i).
template <class Geo, class FP>
void launch_eam_density(const Geo& g, const NbrView& nl, int n,
                        const EamDev<typename Geo::T>& e, const int* types, FP* fp,
                        double* rho_out, double* fpd_out, int4* gout, bool ev, double* partials,
                        Tune tn, cudaStream_t s, double* e_out = nullptr,
                        double4* gout64 = nullptr) {
  const int nblk = force_blocks(n, tn.lpa);
  TDMD_MULTI_DISPATCH(types != nullptr, TDMD_VEC_DISPATCH(vec_rows(nl), TDMD_TUNE_DISPATCH(tn, {
    if (ev)
      launch(k_eam_density<Geo, L, U, true, V, M, FP>, nblk, kForceThreads, 0, s, g, nl, n, e,
             types, fp, rho_out, fpd_out, gout, partials, e_out, gout64);
    else
      launch(k_eam_density<Geo, L, U, false, V, M, FP>, nblk, kForceThreads, 0, s, g, nl, n, e,
             types, fp, rho_out, fpd_out, gout, nullptr, e_out, gout64);
  })));
  TDMD_LAUNCH_CHECK();
}

// Force pass.  FPG: the geometry reads gather records that carry F'(rho).
// kd (nullable; FPG only -- the pass then never reads the positions it
// updates): also apply the next step's kick + drift to each atom after its
// force.  With ev: per-block partials
// (nullable) and per-atom energies added to pe_atom (nullable; holds
// F(rho_i) from the density pass).
template <class Geo, bool FPG, class FP, class F>
void launch_eam_force(const Geo& g, const NbrView& nl, int n, const EamDev<typename Geo::T>& e,
                      const int* types, const FP* fp, F* forces, bool ev, double* partials,
                      Tune tn, cudaStream_t s, const KickDrift* kd = nullptr,
                      double* pe_atom = nullptr) {
  const int nblk = force_blocks(n, tn.lpa);
  TDMD_MULTI_DISPATCH(types != nullptr, TDMD_VEC_DISPATCH(vec_rows(nl), TDMD_TUNE_DISPATCH(tn, {
    if (ev && !partials && pe_atom)  // per-atom energies only
      launch(k_eam_force<Geo, L, U, 2, FPG, V, M, FP, F>, nblk, kForceThreads, 0, s, g, nl, n, e,
             types, fp, ForceOut<F>{forces}, nullptr, KickDrift{}, pe_atom);
    else if (ev)
      launch(k_eam_force<Geo, L, U, 1, FPG, V, M, FP, F>, nblk, kForceThreads, 0, s, g, nl, n, e,
             types, fp, ForceOut<F>{forces}, partials, KickDrift{}, pe_atom);
    else if constexpr (FPG) {
      if (kd)
        launch(k_eam_force<Geo, L, U, 0, FPG, V, M, FP, F, true>, nblk, kForceThreads, 0, s, g, nl,
               n, e, types, fp, ForceOut<F>{forces}, nullptr, *kd, nullptr);
      else
        launch(k_eam_force<Geo, L, U, 0, FPG, V, M, FP, F>, nblk, kForceThreads, 0, s, g, nl, n, e,
               types, fp, ForceOut<F>{forces}, nullptr, KickDrift{}, nullptr);
    } else {
      TDMD_REQUIRE(kd == nullptr, "fused kick-drift needs a gather-record force pass");
      launch(k_eam_force<Geo, L, U, 0, FPG, V, M, FP, F>, nblk, kForceThreads, 0, s, g, nl, n, e,
             types, fp, ForceOut<F>{forces}, nullptr, KickDrift{}, nullptr);
    }
  })));
  TDMD_LAUNCH_CHECK();
}

// Density then force on the same geometry (free functions).  With ev, the
// density pass writes records [0, nblk) and the force pass [nblk, 2*nblk).
template <class Geo, class FP, class F>
void launch_eam(const Geo& g, const NbrView& nl, int n, const EamDev<typename Geo::T>& e,
                const int* types, FP* fp, double* rho_out, double* fpd_out, F* forces, bool ev,
                double* partials, Tune tn, cudaStream_t s) {
  const int nblk = force_blocks(n, tn.lpa);
  launch_eam_density<Geo, FP>(g, nl, n, e, types, fp, rho_out, fpd_out, nullptr, ev, partials,
                              tn, s);
  launch_eam_force<Geo, false, FP, F>(
      g, nl, n, e, types, fp, forces, ev,
      ev ? partials + static_cast<long long>(nblk) * kEvStride : nullptr, tn, s);
}

}  // namespace tdmd_b200
