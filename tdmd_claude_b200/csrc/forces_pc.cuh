// forces_pc.cuh -- single-type EAM with pair coefficients (sm_100a).
//
// The plain passes (forces.cuh) find each listed pair's radius and spline
// interval twice: the density pass for rho(r), the force pass again for
// phi'(r) and rho'(r), with the FP64-refined radius and a spline-row gather
// per pair.  Here the density pass does that work once: beside rho(r) it
// evaluates, at the refined radius, A = phi'(r)/r and B = rho'(r)/r from the
// same 32-byte row pair, and stores (A, B) in a coefficient array laid out
// like the neighbor rows (slot i*cap + k for the k-th neighbor of atom i;
// pairs at or beyond the cutoff and the padding of a row's last sweep get
// (0, 0)).  The force pass is then, per pair,
//   f_ij = -(A + (F'_i + F'_j) B) (r_i - r_j),
// the single-type form of eam_force_kernel's
// -(phi' + F'_i rho'_j + F'_j rho'_i)/r (src/potentials/device_eam.cu:
// 176-278): an index and a coefficient pair streamed from the row, the
// neighbor's 16-byte gather record (position, F'), no spline lookup and no
// radius.  Pairs whose coefficients are (0, 0) skip the gather.
//
// Energy steps: the density pass adds each pair's 1/2 phi(r) (same row) to
// its energy partials, the force pass the virial; their sum is the plain
// passes' energy and virial.  Per-atom energies (the replica log) stay on
// the plain passes.
#pragma once

#include "forces.cuh"

namespace tdmd_b200 {

template <class T>
struct PcPair;
template <>
struct PcPair<float> {
  using type = float2;
};
template <>
struct PcPair<double> {
  using type = double2;
};

// U consecutive coefficient slots starting at p (16-byte aligned: rows start
// at multiples of 8 slots and lanes at multiples of U).
template <int U>
__device__ __forceinline__ void pc_store(float2* p, const float2 (&v)[U]) {
  if constexpr (U == 2) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
  } else {
    reinterpret_cast<float4*>(p)[0] = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
    reinterpret_cast<float4*>(p)[1] = make_float4(v[2].x, v[2].y, v[3].x, v[3].y);
  }
}
template <int U>
__device__ __forceinline__ void pc_store(double2* p, const double2 (&v)[U]) {
#pragma unroll
  for (int u = 0; u < U; ++u) p[u] = v[u];
}

// Streamed once per step: no L1 allocation (as the index rows).
__device__ __forceinline__ float4 ld_stream_f4(const float4* p) {
  float4 v;
  asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
      : "l"(p));
  return v;
}
__device__ __forceinline__ double2 ld_stream_d2(const double2* p) {
  double2 v;
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}

template <int U>
__device__ __forceinline__ void pc_load(const float2* p, float2 (&v)[U]) {
#pragma unroll
  for (int h = 0; h < U / 2; ++h) {
    const float4 a = ld_stream_f4(reinterpret_cast<const float4*>(p) + h);
    v[2 * h] = make_float2(a.x, a.y);
    v[2 * h + 1] = make_float2(a.z, a.w);
  }
}
template <int U>
__device__ __forceinline__ void pc_load(const double2* p, double2 (&v)[U]) {
#pragma unroll
  for (int u = 0; u < U; ++u) v[u] = ld_stream_d2(p + u);
}

// Density + embedding pass that also writes the pair coefficients (padded
// rows, one type).  gout (fixed-point records only) gets {q, bits(F')}.
template <class Geo, int LPA, int U, bool EV, class FP>
__global__ void __launch_bounds__(256) k_eam_density_pc(
    Geo g, NbrView nl, int n, EamDev<typename Geo::T> e, FP* __restrict__ fp_out,
    int4* __restrict__ gout, typename PcPair<typename Geo::T>::type* __restrict__ pc,
    double* __restrict__ partials) {
  using T = typename Geo::T;
  using C2 = typename PcPair<T>::type;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = tid / LPA;
  const int sub = tid % LPA;
  const bool active = i < n;
  Acc<T> rho;
  double pe = 0.0;
  typename Geo::Own o{};
  if (active) {
    o = g.own(i);
    const long long row = nl.row(i);
    const int c = nl.count(i);
    for (int base = U * sub; base < c; base += U * LPA) {
      int jj[U];
      nbr_batch<true>(nl, row, base, c, jj);
      typename Geo::Pair pr[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (jj[u] >= 0)
          g.pair(o, jj[u], pr[u]);
        else
          pr[u].r2 = e.rc_sq;
      }
      C2 out[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        out[u].x = T(0);
        out[u].y = T(0);
        if (pr[u].r2 < e.rc_sq) {
          T r, rinv, sx;
          double rd;
          g.radius(o, pr[u], r, rinv, rd);
          const int idx = spline_at(r, rd, e.dr, e.inv_dr, e.nr, e.dr_d, sx);
          const auto* rowp = e.rtab + static_cast<long long>(idx) * e.S;
          typename V4<T>::type crho, cphi;
          if constexpr (sizeof(T) == sizeof(float)) {
            ld_rows2(rowp, crho, cphi);  // slots rho', phi' of one 32-byte sector
          } else {
            crho = ldv4<T>(rowp);
            cphi = ldv4<T>(rowp + 1);
          }
          rho.add(dspl_val(crho, sx));
          out[u].x = over_r(dspl_der(cphi, sx), r, rinv);
          out[u].y = over_r(dspl_der(crho, sx), r, rinv);
          if (EV) pe += 0.5 * static_cast<double>(dspl_val(cphi, sx));
        }
      }
      pc_store<U>(pc + row + base, out);
    }
  }
#pragma unroll
  for (int s = LPA / 2; s > 0; s >>= 1) rho.shfl_merge(s);
  double Fi = 0.0;
  if (active && sub == 0) {
    const double rh = rho.value();
    double dF;
    embed_eval(e.ftab, e.nrho, e.drho, 0, rh, Fi, dF);
    fp_out[i] = static_cast<FP>(dF);
    if constexpr (Geo::kRecords) {
      int4 rec = g.record(o);
      rec.w = __float_as_int(static_cast<float>(dF));
      gout[i] = rec;
    }
  }
  if (EV && partials) {
    const double w[6] = {0, 0, 0, 0, 0, 0};
    write_ev_partials(Fi + pe, w, partials);
  }
}

// r_i - r_j for the force pass: the fixed-point records' wrapped difference
// (mixed; w of the neighbor's record carries F'(rho_j)) or the FP64 minimum
// image (F'(rho_j) from the fp array).
__device__ __forceinline__ void pc_delta(const GeoQ& g, const int4& o, int j,
                                         const float* /*fp*/, float& dx, float& dy, float& dz,
                                         float& fpj) {
  const int4 b = __ldg(g.q + j);
  dx = __fmul_rn(__int2float_rn(o.x - b.x), g.s[0]);
  dy = __fmul_rn(__int2float_rn(o.y - b.y), g.s[1]);
  dz = __fmul_rn(__int2float_rn(o.z - b.z), g.s[2]);
  fpj = __int_as_float(b.w);
}
__device__ __forceinline__ void pc_delta(const GeoD4& g, const double3& o, int j,
                                         const double* fp, double& dx, double& dy, double& dz,
                                         double& fpj) {
  const double3 q = g.load(j);
  dx = min_image1(o.x - q.x, g.L[0], g.halfL[0], g.per[0]);
  dy = min_image1(o.y - q.y, g.L[1], g.halfL[1], g.per[1]);
  dz = min_image1(o.z - q.z, g.L[2], g.halfL[2], g.per[2]);
  fpj = __ldg(fp + j);
}

// Force pass on pair coefficients.  Geo: GeoQ over the gather records
// (mixed) or GeoD4 (FP64, fp from the array).  EV == 1: virial partials.
// KD (mixed): then the next step's kick + drift of the atom.
template <class Geo, int LPA, int U, int EV, bool KD, class F>
__global__ void __launch_bounds__(256) k_eam_force_pc(
    Geo g, NbrView nl, int n, const typename PcPair<typename Geo::T>::type* __restrict__ pc,
    const typename Geo::T* __restrict__ fp, ForceOut<F> out, double* __restrict__ partials,
    KickDrift kd) {
  using T = typename Geo::T;
  using C2 = typename PcPair<T>::type;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = tid / LPA;
  const int sub = tid % LPA;
  const bool active = i < n;
  Acc<T> fx, fy, fz;
  double w[6] = {0, 0, 0, 0, 0, 0};
  if (active) {
    const typename Geo::Own o = g.own(i);
    T fpi;
    if constexpr (Geo::kRecords)
      fpi = __int_as_float(o.w);
    else
      fpi = __ldg(fp + i);
    const long long row = nl.row(i);
    const int c = nl.count(i);
    for (int base = U * sub; base < c; base += U * LPA) {
      int jj[U];
      nbr_batch<true>(nl, row, base, c, jj);
      C2 cf[U];
      pc_load<U>(pc + row + base, cf);
      T dx[U], dy[U], dz[U], fpj[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (jj[u] >= 0 && (cf[u].x != T(0) || cf[u].y != T(0)))
          pc_delta(g, o, jj[u], fp, dx[u], dy[u], dz[u], fpj[u]);
        else
          jj[u] = -1;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (jj[u] >= 0) {
          const T fpair = -(cf[u].x + (fpi + fpj[u]) * cf[u].y);
          fx.add(mul_rn(fpair, dx[u]));
          fy.add(mul_rn(fpair, dy[u]));
          fz.add(mul_rn(fpair, dz[u]));
          if (EV == 1) add_virial(w, fpair, dx[u], dy[u], dz[u]);
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
      static_assert(Geo::kRecords && sizeof(F) == sizeof(float), "fused kick-drift: mixed path");
      kick_drift_atom(kd, i, static_cast<float>(fx.value()), static_cast<float>(fy.value()),
                      static_cast<float>(fz.value()));
    }
  }
  if (KD && kd.step && blockIdx.x == 0 && threadIdx.x == 0) *kd.step += 1;
  if (EV == 1 && partials) write_ev_partials(0.0, w, partials);
}

}  // namespace tdmd_b200
