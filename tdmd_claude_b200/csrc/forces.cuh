// forces.cuh -- Morse and three-pass EAM force kernels (sm_100a), shared by
// the free-function C ABI (reference array layouts) and the scheduler
// (its own layouts).
//
// Reference kernels (tdmd_Claude): morse_force_kernel
// (src/potentials/device_morse.cu:32-132), eam_density_kernel /
// eam_embedding_kernel / eam_force_kernel (src/potentials/device_eam.cu:
// 72-278), spline_eval / spline_eval_deriv (device_eam.cu:41-66).
//
// Design (B200):
//  * LPA lanes per atom (1..32, a template parameter the autotuner picks):
//    the lanes of a group stride through the atom's neighbor row and merge
//    their partial sums with xor-shuffles; no atomics anywhere.
//  * Geometry policies: FP64 positions (double4 records or the reference's
//    Vec3D AoS, min-image in double), the reference's mixed form (FP64
//    delta cast to FP32), or fixed-point int32 positions whose wrapped
//    difference IS the minimum image (scheduler's mixed path, 16-byte
//    gathers).
//  * Mixed precision: FP32 distances/splines/forces with rsqrt-based 1/r,
//    an FP64-refined radius for the spline offset and the Morse exponent,
//    compensated FP32 per-atom sums (Kahan per lane, TwoSum across lanes);
//    energies and virial always accumulate in FP64.
//  * Energy/virial (template EV): per-block FP64 partials reduced later in a
//    fixed order by k_reduce_partials.
//  * EAM splines: the density pass reads rows (a,b,c,d) of rho_t; the force
//    pass reads derivative-ready rows (b, 2c, 3d, a) of every r-spline of one
//    interval side by side (density of each type, then phi of each pair), so
//    a single-type pair's lookups share one 32-byte sector.  The embedding
//    F(rho) is always evaluated in FP64 (one lookup per atom).
//  * Scheduler mixed EAM: the density pass emits a gather record
//    {qx, qy, qz, F'(rho)} per atom; the force pass reads position and F'
//    of a neighbor in one 16-byte load.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "common.cuh"
#include "integrate.cuh"
#include "replicas.cuh"

namespace tdmd_b200 {

constexpr int kEvStride = 8;  // doubles per block partial: e, w[6], pad

// --------------------------------------------------------------------------
// Neighbor rows: padded (row = i*cap) or dense CSR (row = row_off[i]).
// --------------------------------------------------------------------------
struct NbrView {
  const int* nbr;
  const int* row_off;  // nullable
  const int* cnt;
  int cap;
  __device__ __forceinline__ long long row(int i) const {
    return row_off ? static_cast<long long>(__ldg(row_off + i)) : static_cast<long long>(i) * cap;
  }
  __device__ __forceinline__ int count(int i) const {
    const int c = __ldg(cnt + i);
    return row_off ? c : (c < cap ? c : cap);
  }
};

// L1 eviction-priority loads: spline rows are re-read by every pair and
// stay resident (evict_last); neighbor indices are read once and bypass L1
// (no_allocate), so they do not push rows and position records out.
__device__ __forceinline__ float4 ld_keep(const float4* p) {
  float4 v;
  asm volatile("ld.global.nc.L1::evict_last.v4.f32 {%0, %1, %2, %3}, [%4];"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
      : "l"(p));
  return v;
}
__device__ __forceinline__ int4 ld_stream(const int4* p) {
  int4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0, %1, %2, %3}, [%4];"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
      : "l"(p));
  return v;
}

// Neighbors per lane per sweep (U): a lane fetches U indices, then U
// positions, then evaluates U pairs, so its loads overlap.  U is 2 or 4,
// chosen by the autotuner; kU is the choice without tuning.
constexpr int kU = 4;

__device__ __forceinline__ int2 ld_stream2(const int2* p) {
  int2 v;
  asm volatile("ld.global.nc.L1::no_allocate.v2.s32 {%0, %1}, [%2];"
               : "=r"(v.x), "=r"(v.y)
               : "l"(p));
  return v;
}

// Indices base .. base+U-1 of a row (base < c, base a multiple of U), -1
// past the count.  VEC: padded rows whose start is 16-byte aligned and whose
// capacity is a multiple of 4 (vec_rows), so the vector read stays inside
// the row: one int2 load for U = 2, one int4 load for U = 4.
template <bool VEC, int U>
__device__ __forceinline__ void nbr_batch(const NbrView& nl, long long row, int base, int c,
                                          int (&j)[U]) {
  static_assert(U == 2 || U == 4, "neighbor batch: 2 or 4");
  if constexpr (VEC && U == 2) {
    const int2 v = ld_stream2(reinterpret_cast<const int2*>(nl.nbr + row + base));
    j[0] = v.x;
    j[1] = base + 1 < c ? v.y : -1;
  } else if constexpr (VEC) {
    const int4 v = ld_stream(reinterpret_cast<const int4*>(nl.nbr + row + base));
    j[0] = v.x;
    j[1] = base + 1 < c ? v.y : -1;
    j[2] = base + 2 < c ? v.z : -1;
    j[3] = base + 3 < c ? v.w : -1;
  } else {
#pragma unroll
    for (int u = 0; u < U; ++u) j[u] = base + u < c ? __ldg(nl.nbr + row + base + u) : -1;
  }
}

// --------------------------------------------------------------------------
// Geometry policies.  own(i) loads atom i once; pair(own, j, p) fills p with
// r_i - r_j after the minimum image and r^2 in the policy's arithmetic type
// T; radius(own, p, r, rinv, rd) gives |r_i - r_j| and its inverse as T and as an
// FP64 value rd that the spline offset and the Morse exponent use.  In
// FP32, r itself carries an absolute error of ~ulp(r) = 2.4e-7 A at
// r ~ 2.5 A, which moves the spline argument and, through the large pair
// forces that cancel in each atom's net force, dominates the mixed-precision
// force error; rd removes that term (one Newton step in FP64 from the FP32
// root, with the residual r^2 - r_f^2 taken from FP64 r^2).
// --------------------------------------------------------------------------
struct PairD {
  double dx, dy, dz, r2;
};

struct PairF {
  float dx, dy, dz, r2;
  double r2d;  // FP64 r^2
};

// res: the FP64 r^2 of the exact fixed-point delta minus r2, rounded to
// float -- all that the radius refinement needs of the delta, so a pair in
// flight holds six words instead of eight.
struct PairQ {
  float dx, dy, dz, r2;
  float res;
  int w;  // the neighbor's 4th word
};

// |r| and 1/|r| in FP32 and the FP64-refined radius from a PairQ: with
// r = sqrt(r2) in FP32, r2d - r*r = res + (r2 - r*r), the second term exact
// by FMA; one Newton step rd = r + (r2d - r*r) / (2r).
// FP64 residual (exact r^2 of the fixed-point deltas) - r2.  When the
// three axes share one step (iso), the squares are summed exactly in 64-bit
// integers (|d| <= 2^31: each square <= 2^62, the sum < 2^64) and scaled
// once; otherwise each axis is scaled in FP64.
__device__ __forceinline__ float q_residual(int ix, int iy, int iz, int iso, double s2x,
                                            double s2y, double s2z, float r2) {
  if (iso) {
    const unsigned long long q2 = static_cast<unsigned long long>(static_cast<long long>(ix) * ix) +
                                  static_cast<unsigned long long>(static_cast<long long>(iy) * iy) +
                                  static_cast<unsigned long long>(static_cast<long long>(iz) * iz);
    return static_cast<float>(fma(__ull2double_rn(q2), s2x, -static_cast<double>(r2)));
  }
  const double x = ix, y = iy, z = iz;
  return static_cast<float>(x * x * s2x + y * y * s2y + z * z * s2z - static_cast<double>(r2));
}

__device__ __forceinline__ void radius_q(float r2, float res, float& r, float& rinv, double& rd) {
  rinv = rsqrtf(r2);
  r = r2 * rinv;
  const float corr = (res + fmaf(-r, r, r2)) * 0.5f * rinv;
  rd = static_cast<double>(r) + static_cast<double>(corr);
}

__device__ __forceinline__ void radius_f(float r2, double r2d, float& r, float& rinv, double& rd) {
  rinv = rsqrtf(r2);
  r = r2 * rinv;
  rd = static_cast<double>(r) +
       static_cast<double>(static_cast<float>(fma(-static_cast<double>(r), r, r2d)) * 0.5f * rinv);
}

// Geometries whose density pass may write FP64 gather records {x, y, z, F'}
// (their own atom's position as x, y, z members) declare kD4Out.
template <class G, class = void>
struct has_d4out : std::false_type {};
template <class G>
struct has_d4out<G, std::void_t<decltype(G::kD4Out)>> : std::bool_constant<G::kD4Out> {};

struct GeoD4 {  // FP64, scheduler layout double4 {x,y,z,type}
  using T = double;
  static constexpr bool kD4Out = true;
  static constexpr bool kRecords = false;  // no fixed-point gather records
  using Own = double3;
  using Pair = PairD;
  const double4* p;
  double L[3], halfL[3];
  int per[3];
  __device__ __forceinline__ double3 load(int i) const {
    const double4 a = ld_d4(p + i);
    return make_double3(a.x, a.y, a.z);
  }
  __device__ __forceinline__ Own own(int i) const { return load(i); }
  __device__ __forceinline__ void pair(const Own& o, int j, Pair& pr) const {
    const double3 q = load(j);
    pr.dx = min_image1(o.x - q.x, L[0], halfL[0], per[0]);
    pr.dy = min_image1(o.y - q.y, L[1], halfL[1], per[1]);
    pr.dz = min_image1(o.z - q.z, L[2], halfL[2], per[2]);
    pr.r2 = pr.dx * pr.dx + pr.dy * pr.dy + pr.dz * pr.dz;
  }
  __device__ __forceinline__ void radius(const Own&, const Pair& pr, T& r, T& rinv,
                                         double& rd) const {
    r = sqrt(pr.r2);
    rinv = 1.0 / r;
    rd = r;
  }
  __device__ __forceinline__ T radius_fast(const Pair& pr) const { return sqrt(pr.r2); }
};

// FP64 pair from a gather record: the neighbor's F'(rho) rides along.
struct PairDF {
  double dx, dy, dz, r2;
  double fw;
};

// FP64, scheduler gather records double4 {x, y, z, F'(rho)} written by the
// density pass: the force pass reads a neighbor's position and F' with one
// 32-byte load instead of a position record plus a separate F' gather.
struct GeoD4F {
  using T = double;
  static constexpr bool kRecords = false;
  using Own = double3;
  using Pair = PairDF;
  const double4* p;
  double L[3], halfL[3];
  int per[3];
  __device__ __forceinline__ Own own(int i) const {
    const double4 a = ld_d4(p + i);
    return make_double3(a.x, a.y, a.z);
  }
  __device__ __forceinline__ void pair(const Own& o, int j, Pair& pr) const {
    const double4 q = ld_d4(p + j);
    pr.dx = min_image1(o.x - q.x, L[0], halfL[0], per[0]);
    pr.dy = min_image1(o.y - q.y, L[1], halfL[1], per[1]);
    pr.dz = min_image1(o.z - q.z, L[2], halfL[2], per[2]);
    pr.r2 = pr.dx * pr.dx + pr.dy * pr.dy + pr.dz * pr.dz;
    pr.fw = q.w;
  }
  __device__ __forceinline__ void radius(const Own&, const Pair& pr, T& r, T& rinv,
                                         double& rd) const {
    r = sqrt(pr.r2);
    rinv = 1.0 / r;
    rd = r;
  }
  __device__ __forceinline__ T radius_fast(const Pair& pr) const { return sqrt(pr.r2); }
  // F'(rho_j) of a pair's record
  __device__ __forceinline__ double gather_fp(const Pair& pr, int /*tmask*/) const {
    return pr.fw;
  }
};

struct GeoAoS64 {  // FP64, reference Vec3D AoS
  using T = double;
  static constexpr bool kRecords = false;
  using Own = double3;
  using Pair = PairD;
  const double* p;
  double L[3], halfL[3];
  int per[3];
  __device__ __forceinline__ double3 load(int i) const {
    const double* q = p + 3ll * i;
    return make_double3(__ldg(q), __ldg(q + 1), __ldg(q + 2));
  }
  __device__ __forceinline__ Own own(int i) const { return load(i); }
  __device__ __forceinline__ void pair(const Own& o, int j, Pair& pr) const {
    const double3 q = load(j);
    pr.dx = min_image1(o.x - q.x, L[0], halfL[0], per[0]);
    pr.dy = min_image1(o.y - q.y, L[1], halfL[1], per[1]);
    pr.dz = min_image1(o.z - q.z, L[2], halfL[2], per[2]);
    pr.r2 = pr.dx * pr.dx + pr.dy * pr.dy + pr.dz * pr.dz;
  }
  __device__ __forceinline__ void radius(const Own&, const Pair& pr, T& r, T& rinv,
                                         double& rd) const {
    r = sqrt(pr.r2);
    rinv = 1.0 / r;
    rd = r;
  }
  __device__ __forceinline__ T radius_fast(const Pair& pr) const { return sqrt(pr.r2); }
};

// Mixed on the reference layout (free functions): the delta is formed in
// FP64 and min-imaged there, then cast to FP32 (the reference's
// relative-coordinate form, device_morse.cu:58-73, without its FP32
// min-image step).
struct GeoAoS32 {
  using T = float;
  static constexpr bool kRecords = false;
  using Own = double3;
  using Pair = PairF;
  const double* p;
  double L[3], halfL[3];
  int per[3];
  __device__ __forceinline__ double3 load(int i) const {
    const double* q = p + 3ll * i;
    return make_double3(__ldg(q), __ldg(q + 1), __ldg(q + 2));
  }
  __device__ __forceinline__ Own own(int i) const { return load(i); }
  __device__ __forceinline__ void pair(const Own& o, int j, Pair& pr) const {
    const double3 q = load(j);
    const double x = min_image1(o.x - q.x, L[0], halfL[0], per[0]);
    const double y = min_image1(o.y - q.y, L[1], halfL[1], per[1]);
    const double z = min_image1(o.z - q.z, L[2], halfL[2], per[2]);
    pr.dx = static_cast<float>(x);
    pr.dy = static_cast<float>(y);
    pr.dz = static_cast<float>(z);
    pr.r2d = x * x + y * y + z * z;
    pr.r2 = static_cast<float>(pr.r2d);
  }
  __device__ __forceinline__ void radius(const Own&, const Pair& pr, T& r, T& rinv,
                                         double& rd) const {
    radius_f(pr.r2, pr.r2d, r, rinv, rd);
  }
  __device__ __forceinline__ T radius_fast(const Pair& pr) const { return pr.r2 * rsqrtf(pr.r2); }
};

// Mixed, scheduler layout: fixed-point int4 records {qx,qy,qz,w}.  The
// wrapped int32 difference is the exact minimum-image delta in units of
// Lq/2^32; FP32 components come from one conversion each, the FP64 r^2 from
// the exact integers (only for pairs inside the cutoff).  w is the type
// (position records) or F'(rho) bits (the EAM force-pass gather records).
struct GeoQ {
  using T = float;
  using Own = int4;
  using Pair = PairQ;
  static constexpr bool kRecords = true;  // own() is the atom's fixed-point record
  const int4* q;
  float s[3];
  double s2[3];  // (Lq/2^32)^2 per axis
  int iso;       // one step on all three axes
  __device__ __forceinline__ Own own(int i) const { return __ldg(q + i); }
  __device__ __forceinline__ int4 record(const Own& o) const { return o; }
  __device__ __forceinline__ void pair(const Own& o, int j, Pair& pr) const {
    const int4 b = __ldg(q + j);
    const int ix = o.x - b.x, iy = o.y - b.y, iz = o.z - b.z;
    pr.w = b.w;
    pr.dx = __fmul_rn(__int2float_rn(ix), s[0]);
    pr.dy = __fmul_rn(__int2float_rn(iy), s[1]);
    pr.dz = __fmul_rn(__int2float_rn(iz), s[2]);
    pr.r2 = pr.dx * pr.dx + pr.dy * pr.dy + pr.dz * pr.dz;
    pr.res = q_residual(ix, iy, iz, iso, s2[0], s2[1], s2[2], pr.r2);
  }
  __device__ __forceinline__ void radius(const Own&, const Pair& pr, T& r, T& rinv,
                                         double& rd) const {
    radius_q(pr.r2, pr.res, r, rinv, rd);
  }
  __device__ __forceinline__ T radius_fast(const Pair& pr) const { return pr.r2 * rsqrtf(pr.r2); }
  // F'(rho_j) of a gather record: the 4th word's float bits, type bits cleared
  __device__ __forceinline__ float gather_fp(const Pair& pr, int tmask) const {
    return __int_as_float(pr.w & ~tmask);
  }
};

__host__ inline GeoQ make_geoq(const int4* q, const DevBox& b) {
  return GeoQ{q,
              {b.qscale[0], b.qscale[1], b.qscale[2]},
              {b.qstep[0] * b.qstep[0], b.qstep[1] * b.qstep[1], b.qstep[2] * b.qstep[2]},
              b.qstep[0] == b.qstep[1] && b.qstep[1] == b.qstep[2]};
}

__host__ inline GeoAoS32 make_geo_aos32(const double* p, const DevBox& b) {
  return GeoAoS32{p,
                  {b.L[0], b.L[1], b.L[2]},
                  {b.halfL[0], b.halfL[1], b.halfL[2]},
                  {b.periodic[0], b.periodic[1], b.periodic[2]}};
}

// --------------------------------------------------------------------------
// Accumulators: plain double (FP64) or compensated float (mixed: Kahan per
// lane -- 4 flops per term, error bounded by 2 eps sum|x| whatever the
// number of terms -- and error-free TwoSum when lanes merge).
// --------------------------------------------------------------------------
template <class T>
struct Acc;
template <>
struct Acc<double> {
  double s = 0.0;
  __device__ __forceinline__ void add(double x) { s += x; }
  __device__ __forceinline__ void shfl_merge(int o) { s += __shfl_xor_sync(0xffffffffu, s, o); }
  __device__ __forceinline__ double value() const { return s; }
};
template <>
struct Acc<float> {
  float s = 0.f, c = 0.f;  // running sum, compensation (subtracted)
  __device__ __forceinline__ void add(float x) {
    const float y = __fsub_rn(x, c);
    const float t = __fadd_rn(s, y);
    c = __fsub_rn(__fsub_rn(t, s), y);
    s = t;
  }
  __device__ __forceinline__ void shfl_merge(int o) {
    const float os = __shfl_xor_sync(0xffffffffu, s, o);
    const float oc = __shfl_xor_sync(0xffffffffu, c, o);
    // (s - c) + (os - oc) with TwoSum on the leading parts.
    const float t = __fadd_rn(s, os);
    const float z = __fsub_rn(t, s);
    const float e = __fadd_rn(__fsub_rn(s, __fsub_rn(t, z)), __fsub_rn(os, z));
    s = t;
    c = __fsub_rn(__fadd_rn(c, oc), e);
  }
  __device__ __forceinline__ double value() const {
    return static_cast<double>(s) - static_cast<double>(c);
  }
};

__device__ __forceinline__ double mul_rn(double a, double b) { return a * b; }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }

// FP64 keeps the reference's division by r; FP32 multiplies by rsqrt.
__device__ __forceinline__ double over_r(double x, double r, double /*rinv*/) { return x / r; }
__device__ __forceinline__ float over_r(float x, float /*r*/, float rinv) { return x * rinv; }

// Force output: AoS float3 or double3.
template <class F>
struct ForceOut {
  F* f;
  __device__ __forceinline__ void store(int i, double x, double y, double z) const {
    f[3ll * i] = static_cast<F>(x);
    f[3ll * i + 1] = static_cast<F>(y);
    f[3ll * i + 2] = static_cast<F>(z);
  }
};

// Accumulating force output (the per-zone form: a zone's forces are added to
// what the caller zeroed, compute_morse_gpu_zone, device_morse_zone.cu).
template <class F>
struct ForceAdd {
  F* f;
  __device__ __forceinline__ void store(int i, double x, double y, double z) const {
    f[3ll * i] += static_cast<F>(x);
    f[3ll * i + 1] += static_cast<F>(y);
    f[3ll * i + 2] += static_cast<F>(z);
  }
};

// A geometry whose own atoms start at `first` of the position array; the
// neighbors j of a row stay global indices.  A kernel over atoms
// [first, first + n) then reads its rows, counts and outputs through views
// shifted by first.
template <class G>
struct GeoShift : G {
  int first;
  __device__ __forceinline__ typename G::Own own(int i) const { return G::own(first + i); }
};

// Per-block FP64 energy/virial partials (thread 0 writes 8 doubles).
__device__ __forceinline__ void write_ev_partials(double e, const double (&w)[6],
                                                  double* __restrict__ partials) {
  __shared__ double red[32 * 7];
  double v[7] = {e, w[0], w[1], w[2], w[3], w[4], w[5]};
  block_sum<7>(v, red);
  if (threadIdx.x == 0) {
    double* o = partials + static_cast<long long>(blockIdx.x) * kEvStride;
#pragma unroll
    for (int k = 0; k < 7; ++k) o[k] = v[k];
    o[7] = 0.0;
  }
}

template <class T>
__device__ __forceinline__ void add_virial(double (&w)[6], T fpair, T dx, T dy, T dz) {
  const double hf = 0.5 * static_cast<double>(fpair);
  const double ddx = dx, ddy = dy, ddz = dz;
  w[0] += hf * ddx * ddx;
  w[1] += hf * ddy * ddy;
  w[2] += hf * ddz * ddz;
  w[3] += hf * ddx * ddy;
  w[4] += hf * ddx * ddz;
  w[5] += hf * ddy * ddz;
}

// --------------------------------------------------------------------------
// Morse, MorsePair::compute (src/potentials/morse.hpp:37-55) on the full
// list: F_i = sum_j fpair(r_ij) (r_i - r_j), energy 1/2 U per listed pair.
// --------------------------------------------------------------------------
template <class T>
struct MorseP {
  T d, alpha, r0, rc_sq;
  double r0d;
};

// EV: 0 forces only; 1 also energy + virial into per-block partials and,
// where pe_atom is given, per-atom energies; 2 forces + per-atom energies.
template <class Geo, int LPA, int U, int EV, bool VEC, class F, class Out = ForceOut<F>>
__global__ void __launch_bounds__(256) k_morse(Geo g, NbrView nl, int n,
                                               MorseP<typename Geo::T> mp, Out out,
                                               double* __restrict__ partials,
                                               double* __restrict__ pe_atom) {
  dependent_launch_prologue();
  using T = typename Geo::T;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = tid / LPA;
  const int sub = tid % LPA;
  const bool active = i < n;
  Acc<T> fx, fy, fz;
  double pe = 0.0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  if (active) {
    const typename Geo::Own o = g.own(i);
    const long long row = nl.row(i);
    const int c = nl.count(i);
    const T two_d_alpha = T(2) * mp.d * mp.alpha;
    for (int base = U * sub; base < c; base += U * LPA) {
      int jj[U];
      nbr_batch<VEC>(nl, row, base, c, jj);
      typename Geo::Pair pr[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (jj[u] >= 0)
          g.pair(o, jj[u], pr[u]);
        else
          pr[u].r2 = mp.rc_sq;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (pr[u].r2 < mp.rc_sq) {
          T r, rinv;
          double rd;
          g.radius(o, pr[u], r, rinv, rd);
          const T ex = exp(-mp.alpha * static_cast<T>(rd - mp.r0d));
          const T ome = T(1) - ex;
          const T fpair = -over_r(two_d_alpha * ome * ex, r, rinv);
          fx.add(mul_rn(fpair, pr[u].dx));
          fy.add(mul_rn(fpair, pr[u].dy));
          fz.add(mul_rn(fpair, pr[u].dz));
          if (EV) {
            pe += 0.5 * static_cast<double>(mp.d * (ome * ome - T(1)));
            if (EV == 1) add_virial(w, fpair, pr[u].dx, pr[u].dy, pr[u].dz);
          }
        }
      }
    }
  }
#pragma unroll
  for (int o = LPA / 2; o > 0; o >>= 1) {
    fx.shfl_merge(o);
    fy.shfl_merge(o);
    fz.shfl_merge(o);
  }
  if (active && sub == 0) out.store(i, fx.value(), fy.value(), fz.value());
  if (EV) {
    // per-atom energy (nullable): the lanes' sums merged pairwise
    if (pe_atom) {
      double pa = pe;
#pragma unroll
      for (int o = LPA / 2; o > 0; o >>= 1) pa += __shfl_xor_sync(0xffffffffu, pa, o);
      if (active && sub == 0) pe_atom[i] = pa;
    }
    if (EV == 1 && partials) write_ev_partials(pe, w, partials);
  }
}

// --------------------------------------------------------------------------
// EAM tables on the device.
// --------------------------------------------------------------------------
template <class T>
struct V4;
template <>
struct V4<double> {
  using type = double4;
};
template <>
struct V4<float> {
  using type = float4;
};

template <class T>
struct EamDev {
  const typename V4<T>::type* dtab;  // [(nr-1) * nt] (a, b, c, d) of rho_t
  const typename V4<T>::type* rtab;  // [(nr-1) * S]  (b, 2c, 3d, a), S = nt + npairs
  const double4* ftab;               // [nt * (nrho-1)] (a, b, c, d) of F_t, FP64
  int ntypes, S, nr, nrho;
  T dr, inv_dr, rc_sq;
  double drho;
  double dr_d;
  // FP32 path: dr_d - dr (the knot spacing's rounding), so that the
  // spline offset r - idx*dr carries no error proportional to idx (the
  // same sign for every pair of a neighbor shell, which summed into a
  // bias of the embedding energy).
  T dr_lo;
  // Multi-type mixed path: the low tbits mantissa bits of the gather
  // record's F'(rho) word hold the atom's 0-based type (a relative change of
  // F' below 2^(tbits-23)), so the force pass gathers no type; 0 = types are
  // gathered (one type, or more than 16).
  int tbits;
};

__device__ __forceinline__ int phi_slot(int ti, int tj, int nt) {
  if (ti > tj) {
    const int t = ti;
    ti = tj;
    tj = t;
  }
  return nt + ti * nt - ti * (ti + 1) / 2 + tj;
}

// Interval index and offset, SplineTable::eval (eam_alloy.cpp:52-61):
// idx = int((r - rmin)/dr) clamped to [0, n-2], dx = r - idx*dr (rmin = 0).
__device__ __forceinline__ int spline_idx(double r, double dr, int n, double& dx) {
  int idx = static_cast<int>(r / dr);
  idx = idx < 0 ? 0 : (idx > n - 2 ? n - 2 : idx);
  dx = r - static_cast<double>(idx) * dr;
  return idx;
}

// Interval from r in T, offset from the FP64 radius.
__device__ __forceinline__ int spline_at(double r, double /*rd*/, double dr, double /*inv*/,
                                         int n, double /*dr_d*/, double& sx) {
  return spline_idx(r, dr, n, sx);
}
__device__ __forceinline__ int spline_at(float r, double rd, float /*dr*/, float inv_dr, int n,
                                         double dr_d, float& sx) {
  int idx = static_cast<int>(r * inv_dr);
  idx = idx < 0 ? 0 : (idx > n - 2 ? n - 2 : idx);
  sx = static_cast<float>(fma(-static_cast<double>(idx), dr_d, rd));
  return idx;
}

// Interval and offset from r alone (density pass).
template <class T>
__device__ __forceinline__ int spline_fast(double r, const EamDev<T>& e, double& sx) {
  return spline_idx(r, e.dr, e.nr, sx);
}
template <class T>
__device__ __forceinline__ int spline_fast(float r, const EamDev<T>& e, float& sx) {
  int idx = static_cast<int>(r * e.inv_dr);
  idx = idx < 0 ? 0 : (idx > e.nr - 2 ? e.nr - 2 : idx);
  const float fi = static_cast<float>(idx);
  sx = fmaf(-fi, e.dr_lo, fmaf(-fi, e.dr, r));
  return idx;
}

// (a, b, c, d) rows: value a + x(b + x(c + x d)), derivative b + x(2c + 3d x).
template <class C, class T>
__device__ __forceinline__ T spl_val(const C& c, T dx) {
  return c.x + dx * (c.y + dx * (c.z + dx * c.w));
}
template <class C, class T>
__device__ __forceinline__ T spl_der(const C& c, T dx) {
  return c.y + dx * (T(2) * c.z + dx * T(3) * c.w);
}
// (b, 2c, 3d, a) rows.
template <class C, class T>
__device__ __forceinline__ T dspl_der(const C& c, T dx) {
  return c.x + dx * (c.y + dx * c.z);
}
template <class C, class T>
__device__ __forceinline__ T dspl_val(const C& c, T dx) {
  return c.w + dx * (c.x + dx * (T(0.5) * c.y + dx * (c.z * T(1.0 / 3.0))));
}

template <class T>
__device__ __forceinline__ typename V4<T>::type ldv4(const typename V4<T>::type* p);
template <>
__device__ __forceinline__ double4 ldv4<double>(const double4* p) {
  return ld_d4(p);
}
template <>
__device__ __forceinline__ float4 ldv4<float>(const float4* p) {
  return ld_keep(p);
}

// Both force rows of a single-type FP32 bin, (rho'_t) then (phi'), 32 bytes
// on a 32-byte boundary (one sector), in one 256-bit load: one L1 request per
// pair instead of two.
__device__ __forceinline__ void ld_rows2(const float4* p, float4& a, float4& b) {
  asm volatile("ld.global.nc.L1::evict_last.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}

// Embedding F(rho), F'(rho) in FP64 (SplineTable eval/eval_deriv on F).
__device__ __forceinline__ void embed_eval(const double4* ftab, int nrho, double drho, int t,
                                           double rho, double& F, double& dF) {
  double dx;
  const int idx = spline_idx(rho, drho, nrho, dx);
  const double4 c = ldv4<double>(ftab + static_cast<long long>(t) * (nrho - 1) + idx);
  F = spl_val(c, dx);
  dF = spl_der(c, dx);
}

// Pass 1 (+ fused pass 2): rho_i = sum_j f_tj(r_ij); then fp_i = F'(rho_i)
// and, with EV, the embedding energy F(rho_i) into the block partials.
// types == nullptr means a single-type alloy.  gout (GeoQ only, nullable)
// receives the force pass's gather records {qx, qy, qz, bits(F'(rho))}.
template <class Geo, int LPA, int U, bool EV, bool VEC, bool MULTI, class FP>
__global__ void __launch_bounds__(256) k_eam_density(Geo g, NbrView nl, int n,
                                                     EamDev<typename Geo::T> e,
                                                     const int* __restrict__ types,
                                                     FP* __restrict__ fp_out,
                                                     double* __restrict__ rho_out,
                                                     double* __restrict__ fpd_out,
                                                     int4* __restrict__ gout,
                                                     double* __restrict__ partials,
                                                     double* __restrict__ e_out,
                                                     double4* __restrict__ gout64) {
  dependent_launch_prologue();
  using T = typename Geo::T;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = tid / LPA;
  const int sub = tid % LPA;
  const bool active = i < n;
  Acc<T> rho;
  typename Geo::Own o{};
  if (active) {
    o = g.own(i);
    const long long row = nl.row(i);
    const int c = nl.count(i);
    for (int base = U * sub; base < c; base += U * LPA) {
      int jj[U];
      nbr_batch<VEC>(nl, row, base, c, jj);
      typename Geo::Pair pr[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (jj[u] >= 0)
          g.pair(o, jj[u], pr[u]);
        else
          pr[u].r2 = e.rc_sq;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (pr[u].r2 < e.rc_sq) {
          // No FP64-refined radius here: in the mixed path the density's
          // FP32 radius error is a few percent of the total force error
          // (the force pass's radius dominates), so it is not worth the
          // FP64 work.
          T sx;
          const int idx = spline_fast(g.radius_fast(pr[u]), e, sx);
          // fixed-point position records carry the atom's 1-based type in
          // their fourth word (the density pass always reads those)
          int tj = 0;
          if constexpr (MULTI) {
            if constexpr (Geo::kRecords)
              tj = pr[u].w - 1;
            else
              tj = __ldg(types + jj[u]) - 1;
          }
          const auto cf = ldv4<T>(e.dtab + static_cast<long long>(idx) * e.ntypes + tj);
          rho.add(spl_val(cf, sx));
        }
      }
    }
  }
#pragma unroll
  for (int s = LPA / 2; s > 0; s >>= 1) rho.shfl_merge(s);
  double Fi = 0.0;
  if (active && sub == 0) {
    const double rh = rho.value();
    const int ti = MULTI ? __ldg(types + i) - 1 : 0;
    double dF;
    embed_eval(e.ftab, e.nrho, e.drho, ti, rh, Fi, dF);
    fp_out[i] = static_cast<FP>(dF);
    if (rho_out) rho_out[i] = rh;
    if (fpd_out) fpd_out[i] = dF;
    if (e_out) e_out[i] = Fi;
    if constexpr (has_d4out<Geo>::value) {
      if (gout64) gout64[i] = make_double4(o.x, o.y, o.z, dF);
    }
    if constexpr (Geo::kRecords) {
      if (gout) {
        int4 rec = g.record(o);
        rec.w = __float_as_int(static_cast<float>(dF));
        if (MULTI && e.tbits) {
          const int mask = (1 << e.tbits) - 1;
          rec.w = (rec.w & ~mask) | ti;
        }
        gout[i] = rec;
      }
    }
  }
  if (EV && partials) {
    const double w[6] = {0, 0, 0, 0, 0, 0};
    write_ev_partials(Fi, w, partials);
  }
}

// The next step's fused kick + drift, applied by a force pass to each atom
// right after its force: v += dt F/(m mvv2e), x += dt v with the
// single-image wrap, fixed-point record refreshed (fused_kick_drift_kernel,
// device_velocity_verlet.cu:88-130, full kick).  Only for a force pass that
// reads gather records, never the positions it updates.
struct KickDrift {
  double4* pos4;
  int4* q;
  double* v;
  const int* types;
  const double* inv_mm;  // 1 / (m mvv2e) per type
  double dt;
  long long* step;       // device step counter, +1 per kick-drift (nullable)
  DevBox b;
  // Batched replicas: atom i's box is reps[rep[i]].box instead of b.
  const int* rep;
  const RepDesc* reps;
};

// FT: the force type (float: mixed, also refreshes the fixed-point record;
// double: FP64, which keeps no fixed-point copy).
template <class FT>
__device__ __forceinline__ void kick_drift_atom(const KickDrift& k, int i, FT fx, FT fy, FT fz) {
  const DevBox& b = k.reps ? k.reps[__ldg(k.rep + i)].box : k.b;
  const int t = __ldg(k.types + i);
  const double factor = k.dt * __ldg(k.inv_mm + t);
  double vx = k.v[3ll * i], vy = k.v[3ll * i + 1], vz = k.v[3ll * i + 2];
  vx += factor * static_cast<double>(fx);
  vy += factor * static_cast<double>(fy);
  vz += factor * static_cast<double>(fz);
  double4 p = k.pos4[i];
  p.x = wrap_single(p.x + k.dt * vx, b.lo[0], b.L[0], b.periodic[0]);
  p.y = wrap_single(p.y + k.dt * vy, b.lo[1], b.L[1], b.periodic[1]);
  p.z = wrap_single(p.z + k.dt * vz, b.lo[2], b.L[2], b.periodic[2]);
  k.v[3ll * i] = vx;
  k.v[3ll * i + 1] = vy;
  k.v[3ll * i + 2] = vz;
  k.pos4[i] = p;
  if constexpr (sizeof(FT) == sizeof(float))
    k.q[i] = make_int4(encode_q(p.x, b.qlo[0], b.qinv[0]), encode_q(p.y, b.qlo[1], b.qinv[1]),
                       encode_q(p.z, b.qlo[2], b.qinv[2]), t);
}

// Pass 3: f_ij = -(phi' + fp_i rho'_tj + fp_j rho'_ti)/r * (r_i - r_j).
// FPG: F'(rho_j) comes with the neighbor's gather record (pair w bits)
// instead of the fp array.  KD (FPG, float forces): then the next step's
// kick + drift of the same atom.
template <class Geo, int LPA, int U, int EV, bool FPG, bool VEC, bool MULTI, class FP, class F,
          bool KD = false>
__global__ void __launch_bounds__(256) k_eam_force(Geo g, NbrView nl, int n,
                                                   EamDev<typename Geo::T> e,
                                                   const int* __restrict__ types,
                                                   const FP* __restrict__ fp, ForceOut<F> out,
                                                   double* __restrict__ partials,
                                                   KickDrift kd = {},
                                                   double* __restrict__ pe_atom = nullptr) {
  dependent_launch_prologue();
  using T = typename Geo::T;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = tid / LPA;
  const int sub = tid % LPA;
  const bool active = i < n;
  Acc<T> fx, fy, fz;
  double pe = 0.0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  if (active) {
    const typename Geo::Own o = g.own(i);
    const long long row = nl.row(i);
    const int c = nl.count(i);
    const int ti = MULTI ? __ldg(types + i) - 1 : 0;
    // packed types (FPG, multi-type): F' of both atoms from the records with
    // the type bits cleared, so the pair term stays symmetric
    const bool packed = FPG && MULTI && e.tbits > 0;
    const int tmask = packed ? (1 << e.tbits) - 1 : 0;
    T fpi;
    if constexpr (FPG && MULTI && Geo::kRecords)
      fpi = packed ? __int_as_float(g.record(o).w & ~tmask) : static_cast<T>(__ldg(fp + i));
    else
      fpi = static_cast<T>(__ldg(fp + i));
    for (int base = U * sub; base < c; base += U * LPA) {
      int jj[U];
      nbr_batch<VEC>(nl, row, base, c, jj);
      typename Geo::Pair pr[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (jj[u] >= 0)
          g.pair(o, jj[u], pr[u]);
        else
          pr[u].r2 = e.rc_sq;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (pr[u].r2 < e.rc_sq) {
          T r, rinv, sx;
          double rd;
          g.radius(o, pr[u], r, rinv, rd);
          const int idx = spline_at(r, rd, e.dr, e.inv_dr, e.nr, e.dr_d, sx);
          const int j = jj[u];
          int tj = 0;
          if constexpr (MULTI && FPG && Geo::kRecords)
            tj = packed ? (pr[u].w & tmask) : __ldg(types + j) - 1;
          else if constexpr (MULTI)
            tj = __ldg(types + j) - 1;
          const auto* rowp = e.rtab + static_cast<long long>(idx) * e.S;
          typename V4<T>::type cphi, crho;
          if constexpr (!MULTI && sizeof(T) == sizeof(float)) {
            ld_rows2(rowp, crho, cphi);  // single type: S = 2, slots rho', phi'
          } else {
            cphi = ldv4<T>(rowp + (MULTI ? phi_slot(ti, tj, e.ntypes) : 1));
            crho = ldv4<T>(rowp + tj);
          }
          const T drj = dspl_der(crho, sx);
          T dri = drj;
          if (MULTI && tj != ti) dri = dspl_der(ldv4<T>(rowp + ti), sx);
          T fpj;
          if constexpr (FPG) {
            fpj = g.gather_fp(pr[u], tmask);
          } else {
            fpj = static_cast<T>(__ldg(fp + j));
          }
          const T fpair = -over_r(dspl_der(cphi, sx) + fpi * drj + fpj * dri, r, rinv);
          fx.add(mul_rn(fpair, pr[u].dx));
          fy.add(mul_rn(fpair, pr[u].dy));
          fz.add(mul_rn(fpair, pr[u].dz));
          if (EV) {
            pe += 0.5 * static_cast<double>(dspl_val(cphi, sx));
            if (EV == 1) add_virial(w, fpair, pr[u].dx, pr[u].dy, pr[u].dz);
          }
        }
      }
    }
  }
#pragma unroll
  for (int s = LPA / 2; s > 0; s >>= 1) {
    fx.shfl_merge(s);
    fy.shfl_merge(s);
    fz.shfl_merge(s);
  }
  if (active && sub == 0) {
    out.store(i, fx.value(), fy.value(), fz.value());
    if constexpr (KD) {
      static_assert(FPG, "fused kick-drift: a force pass that reads gather records");
      kick_drift_atom(kd, i, static_cast<F>(fx.value()), static_cast<F>(fy.value()),
                      static_cast<F>(fz.value()));
    }
  }
  if (KD && kd.step && blockIdx.x == 0 && threadIdx.x == 0) *kd.step += 1;
  if (EV) {
    // per-atom energy (nullable): the lanes' pair sums merged pairwise, plus
    // the embedding energy F(rho_i) the density pass stored there
    if (pe_atom) {
      double pa = pe;
#pragma unroll
      for (int o = LPA / 2; o > 0; o >>= 1) pa += __shfl_xor_sync(0xffffffffu, pa, o);
      if (active && sub == 0) pe_atom[i] = pa + pe_atom[i];
    }
    if (EV == 1 && partials) write_ev_partials(pe, w, partials);
  }
}

// Sums nblk partial records (kEvStride doubles each) in block order and
// ADDS them to energy[0] / virial[0..5] (either may be null).
__global__ void k_reduce_partials(const double* __restrict__ partials, int nblk,
                                  double* __restrict__ energy, double* __restrict__ virial);

int force_blocks(long long n, int lpa);

}  // namespace tdmd_b200
