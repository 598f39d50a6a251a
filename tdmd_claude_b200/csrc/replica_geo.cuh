// replica_geo.cuh -- force-kernel geometries over batched replicas (atoms of
// many independent boxes in one array; rep[i] names atom i's replica).
// Used by the batched replicas (batch.cu) and the force-matching adjoint
// (fit.cu).
#pragma once

#include "forces.cuh"
#include "replicas.cuh"

namespace tdmd_b200 {

// Per-replica minimum-image constants of the FP64 path.
struct RepImg {
  double L[3], halfL[3];
  int per[3];
  int pad;
};

// Mixed: fixed-point records, per-replica decode scales (the center atom's
// replica; all of its neighbors share it).
struct GeoQB {
  using T = float;
  struct Own {
    int4 q;
    float s0, s1, s2;
    double t0, t1, t2;
    int iso;
  };
  using Pair = PairQ;
  static constexpr bool kRecords = true;
  const int4* q;
  const int* rep;
  const RepScale* sc;
  __device__ __forceinline__ int4 record(const Own& o) const { return o.q; }
  __device__ __forceinline__ Own own(int i) const {
    Own o;
    o.q = __ldg(q + i);
    const RepScale* p = sc + __ldg(rep + i);
    o.s0 = __ldg(&p->s[0]);
    o.s1 = __ldg(&p->s[1]);
    o.s2 = __ldg(&p->s[2]);
    o.t0 = __ldg(&p->s2[0]);
    o.t1 = __ldg(&p->s2[1]);
    o.t2 = __ldg(&p->s2[2]);
    o.iso = __ldg(&p->iso);
    return o;
  }
  __device__ __forceinline__ void pair(const Own& o, int j, Pair& pr) const {
    const int4 b = __ldg(q + j);
    const int ix = o.q.x - b.x, iy = o.q.y - b.y, iz = o.q.z - b.z;
    pr.w = b.w;
    pr.dx = __fmul_rn(__int2float_rn(ix), o.s0);
    pr.dy = __fmul_rn(__int2float_rn(iy), o.s1);
    pr.dz = __fmul_rn(__int2float_rn(iz), o.s2);
    pr.r2 = pr.dx * pr.dx + pr.dy * pr.dy + pr.dz * pr.dz;
    pr.res = q_residual(ix, iy, iz, o.iso, o.t0, o.t1, o.t2, pr.r2);
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

// FP64: double4 positions, per-replica minimum image.
struct GeoD4B {
  using T = double;
  static constexpr bool kD4Out = true;  // the density pass may write {x, y, z, F'} records
  struct Own {
    double x, y, z;
    double L0, L1, L2, h0, h1, h2;
    int p0, p1, p2;
  };
  using Pair = PairD;
  static constexpr bool kRecords = false;
  const double4* p;
  const int* rep;
  const RepImg* img;
  __device__ __forceinline__ double3 load(int i) const {
    const double4 a = ld_d4(p + i);
    return make_double3(a.x, a.y, a.z);
  }
  __device__ __forceinline__ Own own(int i) const {
    const double3 a = load(i);
    const RepImg* m = img + __ldg(rep + i);
    Own o;
    o.x = a.x;
    o.y = a.y;
    o.z = a.z;
    o.L0 = __ldg(&m->L[0]);
    o.L1 = __ldg(&m->L[1]);
    o.L2 = __ldg(&m->L[2]);
    o.h0 = __ldg(&m->halfL[0]);
    o.h1 = __ldg(&m->halfL[1]);
    o.h2 = __ldg(&m->halfL[2]);
    o.p0 = __ldg(&m->per[0]);
    o.p1 = __ldg(&m->per[1]);
    o.p2 = __ldg(&m->per[2]);
    return o;
  }
  __device__ __forceinline__ void pair(const Own& o, int j, Pair& pr) const {
    const double3 q = load(j);
    pr.dx = min_image1(o.x - q.x, o.L0, o.h0, o.p0);
    pr.dy = min_image1(o.y - q.y, o.L1, o.h1, o.p1);
    pr.dz = min_image1(o.z - q.z, o.L2, o.h2, o.p2);
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

// FP64 gather records {x, y, z, F'(rho)} of a batch (written by the
// density pass), per-replica minimum image: the force pass reads a
// neighbor's position and F' with one 32-byte load.
struct GeoD4BF {
  using T = double;
  using Own = GeoD4B::Own;
  using Pair = PairDF;
  static constexpr bool kRecords = false;
  const double4* p;
  const int* rep;
  const RepImg* img;
  __device__ __forceinline__ Own own(int i) const {
    return GeoD4B{p, rep, img}.own(i);
  }
  __device__ __forceinline__ void pair(const Own& o, int j, Pair& pr) const {
    const double4 q = ld_d4(p + j);
    pr.dx = min_image1(o.x - q.x, o.L0, o.h0, o.p0);
    pr.dy = min_image1(o.y - q.y, o.L1, o.h1, o.p1);
    pr.dz = min_image1(o.z - q.z, o.L2, o.h2, o.p2);
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
  __device__ __forceinline__ double gather_fp(const Pair& pr, int /*tmask*/) const {
    return pr.fw;
  }
};

__host__ inline RepImg rep_img(const DevBox& b) {
  RepImg m{};
  for (int a = 0; a < 3; ++a) {
    m.L[a] = b.L[a];
    m.halfL[a] = b.halfL[a];
    m.per[a] = b.periodic[a];
  }
  return m;
}

__host__ inline RepScale rep_scale(const DevBox& b) {
  RepScale s{};
  for (int a = 0; a < 3; ++a) {
    s.s[a] = b.qscale[a];
    s.s2[a] = b.qstep[a] * b.qstep[a];
  }
  s.iso = b.qstep[0] == b.qstep[1] && b.qstep[1] == b.qstep[2];
  return s;
}

}  // namespace tdmd_b200
