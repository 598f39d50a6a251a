// fit.cu -- force-matching loss over a set of snapshots and its gradient
// with respect to the potential's parameters, by the adjoint of the force
// expressions (tdmd_fit_* in the C ABI).
//
// No reference counterpart: tdmd_Claude computes no gradients.  The forces
// are the ones of its Morse (src/potentials/morse.hpp:37-55) and EAM
// (src/potentials/eam_alloy.cpp:196-295) paths; the loss is
//   L = 1/(3 M) sum_i |F_i - T_i|^2   over all M atoms of all snapshots.
// With G_i = dL/dF_i = 2 (F_i - T_i) / (3 M) and, for an ordered pair (i, j)
// of the full neighbor list, d = r_i - r_j and q_ij = G_i . d / r:
//   Morse  F_i = sum_j f(r) d,  dL/dtheta = sum_(i,j) (G_i . d) df/dtheta;
//   EAM    f = -(phi'_p + F'_i rho'_tj + F'_j rho'_ti) / r, and
//     phi_p coefficients:   -q_ij * dphi'/dc            at r
//     rho_tj coefficients:  -q_ij F'_i drho'/dc          at r
//     rho_ti coefficients:  -q_ij F'_j drho'/dc          at r
//     F_ti coefficients:    w_i * dF'/dc                 at rho_i
//     rho_tj coefficients:  w_i F''_i * drho/dc          at r
//   with the adjoint density weight
//     w_i = -sum_j rho'_tj(r) (G_i - G_j) . d / r.
// No second derivative in positions is needed: the parameters enter the
// forces directly, and through F'(rho) the embedding's second derivative.
//
// B200 layout: the snapshots are batched replicas of one box (one launch per
// pass over all of them), neighbor lists are built once at creation, and
// every pass works on device arrays only (parameters, coefficients, loss and
// gradients are device pointers), so a fitting loop needs no host round trip
// per step.  Gradients accumulate in FP64 (per-block partials for the three
// Morse parameters; FP64 atomics into the coefficient arrays for EAM).
// Passes: Morse = forces+G, gradient; EAM = density (+F', F''), forces+G,
// adjoint (phi / rho-derivative / F terms and w_i, then the rho-value term
// in a second sweep of the same atom's row).
#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "buffers.cuh"
#include "common.cuh"
#include "forces.cuh"
#include "launch.cuh"
#include "replica_geo.cuh"
#include "replicas.cuh"

namespace tdmd_b200 {
namespace {

constexpr int kThreads = 256;
constexpr int kPart = 4;  // doubles per block partial

// Packed spline coefficients a|b|c|d (SplineTable::build_splines layout,
// eam_alloy.cpp:19-50), one spline of ns intervals at `c`.
struct SplC {
  const double* c;
  int ns;
  double step;
};

__device__ __forceinline__ int spl_seg(double x, double step, int ns, double& dx) {
  int k = static_cast<int>(x / step);
  k = k < 0 ? 0 : (k >= ns ? ns - 1 : k);
  dx = x - static_cast<double>(k) * step;
  return k;
}

template <class T>
__device__ __forceinline__ T spl_value(const SplC& s, int k, T dx) {
  const T a = static_cast<T>(__ldg(s.c + k)), b = static_cast<T>(__ldg(s.c + s.ns + k));
  const T c = static_cast<T>(__ldg(s.c + 2 * s.ns + k)),
          d = static_cast<T>(__ldg(s.c + 3 * s.ns + k));
  return a + dx * (b + dx * (c + dx * d));
}

template <class T>
__device__ __forceinline__ T spl_deriv(const SplC& s, int k, T dx) {
  const T b = static_cast<T>(__ldg(s.c + s.ns + k));
  const T c = static_cast<T>(__ldg(s.c + 2 * s.ns + k)),
          d = static_cast<T>(__ldg(s.c + 3 * s.ns + k));
  return b + dx * (T(2) * c + T(3) * d * dx);
}

// Gradient scatter into a packed a|b|c|d spline gradient.
__device__ __forceinline__ void add_value_basis(double* g, int ns, int k, double dx, double w) {
  atomicAdd(g + k, w);
  atomicAdd(g + ns + k, w * dx);
  atomicAdd(g + 2 * ns + k, w * dx * dx);
  atomicAdd(g + 3 * ns + k, w * dx * dx * dx);
}
__device__ __forceinline__ void add_deriv_basis(double* g, int ns, int k, double dx, double w) {
  atomicAdd(g + ns + k, w);
  atomicAdd(g + 2 * ns + k, 2.0 * w * dx);
  atomicAdd(g + 3 * ns + k, 3.0 * w * dx * dx);
}

__device__ __forceinline__ int pair_index(int ti, int tj, int nt) {
  if (ti > tj) {
    const int t = ti;
    ti = tj;
    tj = t;
  }
  return ti * nt - ti * (ti + 1) / 2 + tj;
}

// Device view of the EAM coefficient arrays being fitted and their
// gradients (types 0-based here).
struct FitEam {
  const double* F;
  const double* rho;
  const double* phi;
  double* gF;
  double* grho;
  double* gphi;
  int nt, nsf, nsr;
  double drho, dr;
  __device__ __forceinline__ SplC Fs(int t) const { return SplC{F + 4ll * nsf * t, nsf, drho}; }
  __device__ __forceinline__ SplC rhos(int t) const {
    return SplC{rho + 4ll * nsr * t, nsr, dr};
  }
  __device__ __forceinline__ SplC phis(int p) const {
    return SplC{phi + 4ll * nsr * p, nsr, dr};
  }
};

// Block partial sums: lane merge -> warp -> block; thread 0 writes kPart.
template <int NV>
__device__ __forceinline__ void write_partials(double (&v)[NV], double* part) {
  __shared__ double red[32 * NV];
  block_sum<NV>(v, red);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) part[static_cast<long long>(blockIdx.x) * kPart + k] = v[k];
  }
}

template <class T, int LPA>
__device__ __forceinline__ T lane_sum(T v) {
#pragma unroll
  for (int s = LPA / 2; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
  return v;
}

// ---------------------------------------------------------------------------
// Morse
// ---------------------------------------------------------------------------
template <class Geo, int LPA>
__global__ void __launch_bounds__(kThreads) k_fm_morse_force(
    Geo g, NbrView nl, int n, const double* __restrict__ prm, double rc_sq,
    const double* __restrict__ target, double c, double* __restrict__ G,
    double* __restrict__ fout, double* __restrict__ part) {
  dependent_launch_prologue();
  using T = typename Geo::T;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = tid / LPA, sub = tid % LPA;
  const bool active = i < n;
  const T D = static_cast<T>(prm[0]), alpha = static_cast<T>(prm[1]);
  const double r0d = prm[2];
  Acc<T> fx, fy, fz;
  if (active) {
    const typename Geo::Own o = g.own(i);
    const long long row = nl.row(i);
    const int cnt = nl.count(i);
    for (int k = sub; k < cnt; k += LPA) {
      typename Geo::Pair pr;
      g.pair(o, __ldg(nl.nbr + row + k), pr);
      if (pr.r2 < static_cast<T>(rc_sq)) {
        T r, rinv;
        double rd;
        g.radius(o, pr, r, rinv, rd);
        const T ex = exp(-alpha * static_cast<T>(rd - r0d));
        const T fpair = -over_r(T(2) * D * alpha * (T(1) - ex) * ex, r, rinv);
        fx.add(mul_rn(fpair, pr.dx));
        fy.add(mul_rn(fpair, pr.dy));
        fz.add(mul_rn(fpair, pr.dz));
      }
    }
  }
#pragma unroll
  for (int s = LPA / 2; s > 0; s >>= 1) {
    fx.shfl_merge(s);
    fy.shfl_merge(s);
    fz.shfl_merge(s);
  }
  double v[1] = {0.0};
  if (active && sub == 0) {
    const double f[3] = {fx.value(), fy.value(), fz.value()};
    for (int a = 0; a < 3; ++a) {
      const double e = f[a] - target[3ll * i + a];
      v[0] += c * e * e;
      G[3ll * i + a] = 2.0 * c * e;
      if (fout) fout[3ll * i + a] = f[a];
    }
  }
  write_partials<1>(v, part);
}

template <class Geo, int LPA>
__global__ void __launch_bounds__(kThreads) k_fm_morse_grad(Geo g, NbrView nl, int n,
                                                            const double* __restrict__ prm,
                                                            double rc_sq,
                                                            const double* __restrict__ G,
                                                            double* __restrict__ part) {
  dependent_launch_prologue();
  using T = typename Geo::T;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = tid / LPA, sub = tid % LPA;
  const double D = prm[0], alpha = prm[1], r0 = prm[2];
  const T Dt = static_cast<T>(D), at = static_cast<T>(alpha);
  double v[3] = {0.0, 0.0, 0.0};
  if (i < n) {
    const typename Geo::Own o = g.own(i);
    const double gx = G[3ll * i], gy = G[3ll * i + 1], gz = G[3ll * i + 2];
    const long long row = nl.row(i);
    const int cnt = nl.count(i);
    for (int k = sub; k < cnt; k += LPA) {
      typename Geo::Pair pr;
      g.pair(o, __ldg(nl.nbr + row + k), pr);
      if (pr.r2 < static_cast<T>(rc_sq)) {
        T r, rinv;
        double rd;
        g.radius(o, pr, r, rinv, rd);
        const T ex = exp(-at * static_cast<T>(rd - r0));
        const T ome = T(1) - ex;
        const double gd = (gx * static_cast<double>(pr.dx) + gy * static_cast<double>(pr.dy) +
                           gz * static_cast<double>(pr.dz)) / static_cast<double>(r);
        // df/dtheta * r (the 1/r is folded into gd)
        const T dD = -T(2) * at * ome * ex;
        const T da = -T(2) * Dt * (ome * ex - at * (T(1) - T(2) * ex) *
                                               static_cast<T>(rd - r0) * ex);
        const T dr0 = -T(2) * Dt * at * at * (T(1) - T(2) * ex) * ex;
        v[0] += gd * static_cast<double>(dD);
        v[1] += gd * static_cast<double>(da);
        v[2] += gd * static_cast<double>(dr0);
      }
    }
  }
  write_partials<3>(v, part);
}

// Sums nblk block partials (kPart doubles each) in block order:
// out[0..nv) = column sums.
__global__ void k_fm_sum(const double* __restrict__ part, int nblk, int nv,
                         double* __restrict__ out) {
  dependent_launch_prologue();
  __shared__ double red[32 * kPart];
  double v[kPart] = {0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x)
    for (int k = 0; k < nv; ++k) v[k] += part[static_cast<long long>(b) * kPart + k];
  block_sum<kPart>(v, red);
  if (threadIdx.x == 0)
    for (int k = 0; k < nv; ++k) out[k] = v[k];
}

// ---------------------------------------------------------------------------
// EAM
// ---------------------------------------------------------------------------
template <class Geo, int LPA>
__global__ void __launch_bounds__(kThreads) k_fm_eam_density(
    Geo g, NbrView nl, int n, const int* __restrict__ types, FitEam e, double rc_sq,
    double* __restrict__ rho_out, double* __restrict__ fp_out, double* __restrict__ fpp_out) {
  dependent_launch_prologue();
  using T = typename Geo::T;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = tid / LPA, sub = tid % LPA;
  const bool active = i < n;
  Acc<T> rho;
  if (active) {
    const typename Geo::Own o = g.own(i);
    const long long row = nl.row(i);
    const int cnt = nl.count(i);
    for (int k = sub; k < cnt; k += LPA) {
      const int j = __ldg(nl.nbr + row + k);
      typename Geo::Pair pr;
      g.pair(o, j, pr);
      if (pr.r2 < static_cast<T>(rc_sq)) {
        T r, rinv;
        double rd;
        g.radius(o, pr, r, rinv, rd);
        double dx;
        const int kk = spl_seg(rd, e.dr, e.nsr, dx);
        rho.add(spl_value<T>(e.rhos(__ldg(types + j) - 1), kk, static_cast<T>(dx)));
      }
    }
  }
#pragma unroll
  for (int s = LPA / 2; s > 0; s >>= 1) rho.shfl_merge(s);
  if (active && sub == 0) {
    const double rh = rho.value();
    const SplC F = e.Fs(__ldg(types + i) - 1);
    double dx;
    const int kk = spl_seg(rh, e.drho, e.nsf, dx);
    rho_out[i] = rh;
    fp_out[i] = spl_deriv<double>(F, kk, dx);
    fpp_out[i] = 2.0 * __ldg(F.c + 2 * F.ns + kk) + 6.0 * __ldg(F.c + 3 * F.ns + kk) * dx;
  }
}

template <class Geo, int LPA>
__global__ void __launch_bounds__(kThreads) k_fm_eam_force(
    Geo g, NbrView nl, int n, const int* __restrict__ types, FitEam e, double rc_sq,
    const double* __restrict__ fp, const double* __restrict__ target, double c,
    double* __restrict__ G, double* __restrict__ fout, double* __restrict__ part) {
  dependent_launch_prologue();
  using T = typename Geo::T;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = tid / LPA, sub = tid % LPA;
  const bool active = i < n;
  Acc<T> fx, fy, fz;
  if (active) {
    const typename Geo::Own o = g.own(i);
    const int ti = __ldg(types + i) - 1;
    const T fpi = static_cast<T>(fp[i]);
    const long long row = nl.row(i);
    const int cnt = nl.count(i);
    for (int k = sub; k < cnt; k += LPA) {
      const int j = __ldg(nl.nbr + row + k);
      typename Geo::Pair pr;
      g.pair(o, j, pr);
      if (pr.r2 < static_cast<T>(rc_sq)) {
        T r, rinv;
        double rd;
        g.radius(o, pr, r, rinv, rd);
        const int tj = __ldg(types + j) - 1;
        double dxd;
        const int kk = spl_seg(rd, e.dr, e.nsr, dxd);
        const T dx = static_cast<T>(dxd);
        const T dphi = spl_deriv<T>(e.phis(pair_index(ti, tj, e.nt)), kk, dx);
        const T drj = spl_deriv<T>(e.rhos(tj), kk, dx);
        const T dri = ti == tj ? drj : spl_deriv<T>(e.rhos(ti), kk, dx);
        const T fpair = -over_r(dphi + fpi * drj + static_cast<T>(fp[j]) * dri, r, rinv);
        fx.add(mul_rn(fpair, pr.dx));
        fy.add(mul_rn(fpair, pr.dy));
        fz.add(mul_rn(fpair, pr.dz));
      }
    }
  }
#pragma unroll
  for (int s = LPA / 2; s > 0; s >>= 1) {
    fx.shfl_merge(s);
    fy.shfl_merge(s);
    fz.shfl_merge(s);
  }
  double v[1] = {0.0};
  if (active && sub == 0) {
    const double f[3] = {fx.value(), fy.value(), fz.value()};
    for (int a = 0; a < 3; ++a) {
      const double d = f[a] - target[3ll * i + a];
      v[0] += c * d * d;
      G[3ll * i + a] = 2.0 * c * d;
      if (fout) fout[3ll * i + a] = f[a];
    }
  }
  write_partials<1>(v, part);
}

template <class Geo, int LPA>
__global__ void __launch_bounds__(kThreads) k_fm_eam_adjoint(
    Geo g, NbrView nl, int n, const int* __restrict__ types, FitEam e, double rc_sq,
    const double* __restrict__ rho, const double* __restrict__ fp,
    const double* __restrict__ fpp, const double* __restrict__ G) {
  dependent_launch_prologue();
  using T = typename Geo::T;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = tid / LPA, sub = tid % LPA;
  const bool active = i < n;
  double w = 0.0;
  typename Geo::Own o{};
  int ti = 0, cnt = 0;
  long long row = 0;
  if (active) {
    o = g.own(i);
    ti = __ldg(types + i) - 1;
    row = nl.row(i);
    cnt = nl.count(i);
    const double gix = G[3ll * i], giy = G[3ll * i + 1], giz = G[3ll * i + 2];
    const double fpi = fp[i];
    for (int k = sub; k < cnt; k += LPA) {
      const int j = __ldg(nl.nbr + row + k);
      typename Geo::Pair pr;
      g.pair(o, j, pr);
      if (pr.r2 < static_cast<T>(rc_sq)) {
        T r, rinv;
        double rd;
        g.radius(o, pr, r, rinv, rd);
        const int tj = __ldg(types + j) - 1;
        double dx;
        const int kk = spl_seg(rd, e.dr, e.nsr, dx);
        const double ddx = pr.dx, ddy = pr.dy, ddz = pr.dz, rr = static_cast<double>(r);
        const double q = (gix * ddx + giy * ddy + giz * ddz) / rr;
        const double fpj = fp[j];
        add_deriv_basis(e.gphi + 4ll * e.nsr * pair_index(ti, tj, e.nt), e.nsr, kk, dx, -q);
        if (ti == tj) {
          add_deriv_basis(e.grho + 4ll * e.nsr * tj, e.nsr, kk, dx, -q * (fpi + fpj));
        } else {
          add_deriv_basis(e.grho + 4ll * e.nsr * tj, e.nsr, kk, dx, -q * fpi);
          add_deriv_basis(e.grho + 4ll * e.nsr * ti, e.nsr, kk, dx, -q * fpj);
        }
        const double drj = spl_deriv<double>(e.rhos(tj), kk, dx);
        const double gdiff = (gix - G[3ll * j]) * ddx + (giy - G[3ll * j + 1]) * ddy +
                             (giz - G[3ll * j + 2]) * ddz;
        w -= drj * gdiff / rr;
      }
    }
  }
  w = lane_sum<double, LPA>(w);
  if (!active) return;
  if (sub == 0) {
    double dx;
    const int kk = spl_seg(rho[i], e.drho, e.nsf, dx);
    add_deriv_basis(e.gF + 4ll * e.nsf * ti, e.nsf, kk, dx, w);
  }
  const double wf = w * fpp[i];
  // rho values through rho_i: w_i F''_i * drho_tj/dc at r_ij.
  for (int k = sub; k < cnt; k += LPA) {
    const int j = __ldg(nl.nbr + row + k);
    typename Geo::Pair pr;
    g.pair(o, j, pr);
    if (pr.r2 < static_cast<T>(rc_sq)) {
      T r, rinv;
      double rd;
      g.radius(o, pr, r, rinv, rd);
      const int tj = __ldg(types + j) - 1;
      double dx;
      const int kk = spl_seg(rd, e.dr, e.nsr, dx);
      add_value_basis(e.grho + 4ll * e.nsr * tj, e.nsr, kk, dx, wf);
    }
  }
}

// Single-element alloys: the same adjoint with the r-spline gradients
// (phi, rho) of intervals [k0, k0 + W) accumulated in shared memory by each
// block of a persistent grid and added to the global arrays once per block
// at the end; intervals below k0 (pairs closer than k0 * dr) go straight to
// global memory.  Shared layout: [phi, rho][coefficient 0..3][W].
__device__ __forceinline__ void add_r(double* gl, double* sh, int ns, int k, int k0, int W,
                                      int coef, double v) {
  if (k >= k0) atomicAdd(sh + coef * W + (k - k0), v);
  else atomicAdd(gl + coef * ns + k, v);
}

template <class Geo, int LPA>
__global__ void __launch_bounds__(kThreads) k_fm_eam_adjoint_w(
    Geo g, NbrView nl, int n, FitEam e, double rc_sq, const double* __restrict__ rho,
    const double* __restrict__ fp, const double* __restrict__ fpp,
    const double* __restrict__ G, int k0, int W) {
  dependent_launch_prologue();
  using T = typename Geo::T;
  extern __shared__ double sg[];
  double* const sphi = sg;
  double* const srho = sg + 4 * W;
  for (int k = threadIdx.x; k < 8 * W; k += blockDim.x) sg[k] = 0.0;
  __syncthreads();
  const int ns = e.nsr;
  const int per_block = blockDim.x / LPA;
  const int sub = threadIdx.x % LPA;
  for (long long first = static_cast<long long>(blockIdx.x) * per_block; first < n;
       first += static_cast<long long>(gridDim.x) * per_block) {
    const long long ii = first + threadIdx.x / LPA;
    const bool active = ii < n;
    const int i = active ? static_cast<int>(ii) : 0;
    double w = 0.0;
    typename Geo::Own o{};
    int cnt = 0;
    long long row = 0;
    if (active) {
      o = g.own(i);
      row = nl.row(i);
      cnt = nl.count(i);
      const double gix = G[3ll * i], giy = G[3ll * i + 1], giz = G[3ll * i + 2];
      const double fpi = fp[i];
      for (int k = sub; k < cnt; k += LPA) {
        const int j = __ldg(nl.nbr + row + k);
        typename Geo::Pair pr;
        g.pair(o, j, pr);
        if (pr.r2 < static_cast<T>(rc_sq)) {
          T r, rinv;
          double rd;
          g.radius(o, pr, r, rinv, rd);
          double dx;
          const int kk = spl_seg(rd, e.dr, ns, dx);
          const double ddx = pr.dx, ddy = pr.dy, ddz = pr.dz, rr = static_cast<double>(r);
          const double q = (gix * ddx + giy * ddy + giz * ddz) / rr;
          const double fpj = fp[j];
          // phi' and rho' terms: d/dc of the derivative basis (b, 2c x, 3d x^2)
          const double wp = -q, wr = -q * (fpi + fpj);
          add_r(e.gphi, sphi, ns, kk, k0, W, 1, wp);
          add_r(e.gphi, sphi, ns, kk, k0, W, 2, 2.0 * wp * dx);
          add_r(e.gphi, sphi, ns, kk, k0, W, 3, 3.0 * wp * dx * dx);
          add_r(e.grho, srho, ns, kk, k0, W, 1, wr);
          add_r(e.grho, srho, ns, kk, k0, W, 2, 2.0 * wr * dx);
          add_r(e.grho, srho, ns, kk, k0, W, 3, 3.0 * wr * dx * dx);
          const double drj = spl_deriv<double>(e.rhos(0), kk, dx);
          const double gdiff = (gix - G[3ll * j]) * ddx + (giy - G[3ll * j + 1]) * ddy +
                               (giz - G[3ll * j + 2]) * ddz;
          w -= drj * gdiff / rr;
        }
      }
    }
    w = lane_sum<double, LPA>(w);
    if (active) {
      if (sub == 0) {
        double dx;
        const int kk = spl_seg(rho[i], e.drho, e.nsf, dx);
        add_deriv_basis(e.gF, e.nsf, kk, dx, w);
      }
      const double wf = w * fpp[i];
      // rho values through rho_i: w_i F''_i * drho/dc at r_ij
      for (int k = sub; k < cnt; k += LPA) {
        const int j = __ldg(nl.nbr + row + k);
        typename Geo::Pair pr;
        g.pair(o, j, pr);
        if (pr.r2 < static_cast<T>(rc_sq)) {
          T r, rinv;
          double rd;
          g.radius(o, pr, r, rinv, rd);
          double dx;
          const int kk = spl_seg(rd, e.dr, ns, dx);
          add_r(e.grho, srho, ns, kk, k0, W, 0, wf);
          add_r(e.grho, srho, ns, kk, k0, W, 1, wf * dx);
          add_r(e.grho, srho, ns, kk, k0, W, 2, wf * dx * dx);
          add_r(e.grho, srho, ns, kk, k0, W, 3, wf * dx * dx * dx);
        }
      }
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < 8 * W; k += blockDim.x) {
    const double v = sg[k];
    if (v != 0.0) {
      const int sp = k / (4 * W), coef = (k / W) % 4, b = k % W;
      atomicAdd((sp == 0 ? e.gphi : e.grho) + coef * ns + k0 + b, v);
    }
  }
}

}  // namespace

// Intervals of the r splines whose gradients a block keeps in shared memory
// (8 doubles each: 4 coefficients of phi and of rho): 1280 x 64 B = 80 KiB,
// two blocks per SM.
constexpr int kAdjointWindow = 1280;

class Fit {
 public:
  Fit(int nsnap, int natoms, const tdmd_box& box, const double* pos, const int* types,
      double cutoff, int precision);
  ~Fit();
  Fit(const Fit&) = delete;
  Fit& operator=(const Fit&) = delete;
  void set_targets(const double* t);
  void morse(const double* d_prm, double* d_loss, double* d_grad, double* d_forces,
             cudaStream_t s);
  void eam(int ntypes, int nrho, double drho, int nr, double dr, const double* F,
           const double* rho, const double* phi, double* d_loss, double* gF, double* grho,
           double* gphi, double* d_forces, cudaStream_t s);
  long long natoms() const { return m_; }
  int lanes() const { return lpa_; }

 private:
  template <class Fn>
  void with_geo(Fn&& fn) const;
  NbrView view() const { return NbrView{nbr_.data(), nullptr, cnt_.data(), cap_}; }

  int nsnap_, n_;
  long long m_;
  bool mixed_;
  double rc_, rc_sq_;
  int lpa_ = 4;
  int cap_ = 0;
  int ncells_ = 0;
  bool has_targets_ = false;
  int max_type_ = 0;
  DevArray<RepDesc> reps_;
  DevArray<RepScale> scales_;
  DevArray<RepImg> imgs_;
  DevArray<int> cell_rep_, rep_;
  DevArray<double4> pos4_;
  DevArray<int4> q_;
  DevArray<int> types_;
  DevArray<int> nbr_, cnt_, status_;
  DevArray<double> target_, G_, rho_, fp_, fpp_, part_;
  CellListDev cl_;
};

Fit::Fit(int nsnap, int natoms, const tdmd_box& box, const double* pos, const int* types,
         double cutoff, int precision)
    : nsnap_(nsnap), n_(natoms), mixed_(precision == TDMD_MIXED), rc_(cutoff),
      rc_sq_(cutoff * cutoff) {
  TDMD_REQUIRE(nsnap >= 1 && natoms >= 1, "need at least one snapshot and one atom");
  TDMD_REQUIRE(pos && types, "null positions or types");
  TDMD_REQUIRE(cutoff > 0.0, "cutoff must be positive");
  TDMD_REQUIRE(precision == TDMD_FP64 || precision == TDMD_MIXED, "unknown precision");
  m_ = static_cast<long long>(nsnap) * natoms;
  TDMD_REQUIRE(m_ < INT_MAX / 4, "too many atoms");
  const DevBox b = make_devbox(box, cutoff);
  for (int a = 0; a < 3; ++a)
    TDMD_REQUIRE(!b.periodic[a] || b.L[a] > 2.0 * cutoff,
                 "periodic box edge must exceed twice the cutoff");
  for (long long i = 0; i < m_; ++i) {
    TDMD_REQUIRE(types[i] >= 1, "types are 1-based");
    max_type_ = std::max(max_type_, types[i]);
  }
  std::vector<RepDesc> d(static_cast<size_t>(nsnap));
  const int ncell1 = b.nc[0] * b.nc[1] * b.nc[2];
  for (int s = 0; s < nsnap; ++s) {
    RepDesc& r = d[static_cast<size_t>(s)];
    r = RepDesc{};
    r.box = b;
    r.atom0 = s * natoms;
    r.natoms = natoms;
    r.cell0 = s * ncell1;
    r.ncells = ncell1;
    row_filter_band(b, rc_sq_, &r.lo_f, &r.hi_f, &r.wrap);
  }
  ncells_ = nsnap * ncell1;
  const size_t m = static_cast<size_t>(m_);
  std::vector<int> crep(static_cast<size_t>(ncells_)), arep(m);
  for (int s = 0; s < nsnap; ++s) {
    std::fill(crep.begin() + static_cast<long>(s) * ncell1,
              crep.begin() + static_cast<long>(s + 1) * ncell1, s);
    std::fill(arep.begin() + static_cast<long>(s) * natoms,
              arep.begin() + static_cast<long>(s + 1) * natoms, s);
  }
  std::vector<double4> p4(m);
  std::vector<int4> q(m);
  for (size_t i = 0; i < m; ++i) {
    p4[i] = make_double4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], static_cast<double>(types[i]));
  }
  const RepScale sc = rep_scale(b);
  const RepImg im = rep_img(b);
  std::vector<RepScale> scv(static_cast<size_t>(nsnap), sc);
  std::vector<RepImg> imv(static_cast<size_t>(nsnap), im);
  cudaStream_t s = nullptr;
  TDMD_CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  try {
    reps_.reserve(d.size());
    scales_.reserve(scv.size());
    imgs_.reserve(imv.size());
    cell_rep_.reserve(crep.size());
    rep_.reserve(m);
    pos4_.reserve(m);
    types_.reserve(m);
    cnt_.reserve(m);
    status_.reserve(4);
    target_.reserve(3 * m);
    G_.reserve(3 * m);
    rho_.reserve(m);
    fp_.reserve(m);
    fpp_.reserve(m);
    TDMD_CU(cudaMemcpyAsync(reps_.data(), d.data(), sizeof(RepDesc) * d.size(),
                            cudaMemcpyHostToDevice, s));
    TDMD_CU(cudaMemcpyAsync(scales_.data(), scv.data(), sizeof(RepScale) * scv.size(),
                            cudaMemcpyHostToDevice, s));
    TDMD_CU(cudaMemcpyAsync(imgs_.data(), imv.data(), sizeof(RepImg) * imv.size(),
                            cudaMemcpyHostToDevice, s));
    TDMD_CU(cudaMemcpyAsync(cell_rep_.data(), crep.data(), sizeof(int) * crep.size(),
                            cudaMemcpyHostToDevice, s));
    TDMD_CU(cudaMemcpyAsync(rep_.data(), arep.data(), sizeof(int) * m, cudaMemcpyHostToDevice, s));
    TDMD_CU(cudaMemcpyAsync(pos4_.data(), p4.data(), sizeof(double4) * m, cudaMemcpyHostToDevice,
                            s));
    TDMD_CU(cudaMemcpyAsync(types_.data(), types, sizeof(int) * m, cudaMemcpyHostToDevice, s));
    if (mixed_) {
      for (size_t i = 0; i < m; ++i) {
        q[i].x = static_cast<int>(static_cast<uint32_t>(static_cast<unsigned long long>(
            std::llrint((pos[3 * i] - b.qlo[0]) * b.qinv[0]))));
        q[i].y = static_cast<int>(static_cast<uint32_t>(static_cast<unsigned long long>(
            std::llrint((pos[3 * i + 1] - b.qlo[1]) * b.qinv[1]))));
        q[i].z = static_cast<int>(static_cast<uint32_t>(static_cast<unsigned long long>(
            std::llrint((pos[3 * i + 2] - b.qlo[2]) * b.qinv[2]))));
        q[i].w = types[i];
      }
      q_.reserve(m);
      TDMD_CU(cudaMemcpyAsync(q_.data(), q.data(), sizeof(int4) * m, cudaMemcpyHostToDevice, s));
    }
    // Neighbor rows (r_list = cutoff, no skin: positions never move).
    TDMD_CU(cudaMemsetAsync(status_.data(), 0, sizeof(int) * 4, s));
    build_cell_list_batch(cl_, pos4_.data(), rep_.data(), reps_.data(), m_, ncells_, s);
    build_neighbor_rows_batch(cl_, pos4_.data(), reps_.data(), cell_rep_.data(), rc_sq_, nullptr,
                              0, cnt_.data(), status_.data(), s);
    int st[4];
    TDMD_CU(cudaMemcpyAsync(st, status_.data(), sizeof(st), cudaMemcpyDeviceToHost, s));
    TDMD_CU(cudaStreamSynchronize(s));
    cap_ = std::max(8, (st[1] + 7) / 8 * 8);
    nbr_.reserve(static_cast<size_t>(cap_) * m);
    build_neighbor_rows_batch(cl_, pos4_.data(), reps_.data(), cell_rep_.data(), rc_sq_,
                              nbr_.data(), cap_, cnt_.data(), nullptr, s);
    lpa_ = default_lpa(m_);
    part_.reserve(static_cast<size_t>(force_blocks(m_, 32)) * kPart + kPart);
    TDMD_CU(cudaStreamSynchronize(s));
  } catch (...) {
    cudaStreamDestroy(s);
    throw;
  }
  cudaStreamDestroy(s);
}

Fit::~Fit() = default;

void Fit::set_targets(const double* t) {
  TDMD_REQUIRE(t, "null targets");
  TDMD_CU(cudaMemcpy(target_.data(), t, sizeof(double) * 3 * static_cast<size_t>(m_),
                     cudaMemcpyHostToDevice));
  has_targets_ = true;
}

template <class Fn>
void Fit::with_geo(Fn&& fn) const {
  if (mixed_)
    fn(GeoQB{q_.data(), rep_.data(), scales_.data()});
  else
    fn(GeoD4B{pos4_.data(), rep_.data(), imgs_.data()});
}

void Fit::morse(const double* d_prm, double* d_loss, double* d_grad, double* d_forces,
                cudaStream_t s) {
  TDMD_REQUIRE(has_targets_, "targets not set");
  TDMD_REQUIRE(d_prm && d_loss, "null parameter or loss pointer");
  const NbrView nl = view();
  const int m = static_cast<int>(m_);
  const int nblk = force_blocks(m_, lpa_);
  const double c = 1.0 / (3.0 * static_cast<double>(m_));
  with_geo([&](auto g) {
    using Geo = decltype(g);
    TDMD_LPA_DISPATCH(lpa_, {
      launch(k_fm_morse_force<Geo, L>, nblk, kThreads, 0, s, g, nl, m, d_prm, rc_sq_,
             target_.data(), c, G_.data(), d_forces, part_.data());
    });
  });
  TDMD_LAUNCH_CHECK();
  launch(k_fm_sum, 1, kThreads, 0, s, part_.data(), nblk, 1, d_loss);
  TDMD_LAUNCH_CHECK();
  if (!d_grad) return;
  with_geo([&](auto g) {
    using Geo = decltype(g);
    TDMD_LPA_DISPATCH(lpa_, {
      launch(k_fm_morse_grad<Geo, L>, nblk, kThreads, 0, s, g, nl, m, d_prm, rc_sq_, G_.data(),
             part_.data());
    });
  });
  TDMD_LAUNCH_CHECK();
  launch(k_fm_sum, 1, kThreads, 0, s, part_.data(), nblk, 3, d_grad);
  TDMD_LAUNCH_CHECK();
}

void Fit::eam(int ntypes, int nrho, double drho, int nr, double dr, const double* F,
              const double* rho, const double* phi, double* d_loss, double* gF, double* grho,
              double* gphi, double* d_forces, cudaStream_t s) {
  TDMD_REQUIRE(has_targets_, "targets not set");
  TDMD_REQUIRE(ntypes >= 1 && ntypes <= 64, "ntypes out of range");
  TDMD_REQUIRE(max_type_ <= ntypes, "an atom type exceeds the table's element count");
  // Pairs up to the fit's cutoff evaluate the r tables: past their last knot
  // the cubic of the last interval would be extrapolated.
  TDMD_REQUIRE(rc_ <= static_cast<double>(nr - 1) * dr * (1.0 + 1e-12),
               "the fit's cutoff exceeds the range of the EAM r tables");
  TDMD_REQUIRE(nrho >= 2 && nr >= 2 && drho > 0.0 && dr > 0.0, "bad spline grid");
  TDMD_REQUIRE(F && rho && phi && d_loss, "null coefficient or loss pointer");
  const bool grad = gF || grho || gphi;
  TDMD_REQUIRE(!grad || (gF && grho && gphi), "give all three gradient arrays or none");
  const int npairs = ntypes * (ntypes + 1) / 2;
  FitEam e{F, rho, phi, gF, grho, gphi, ntypes, nrho - 1, nr - 1, drho, dr};
  if (grad) {
    TDMD_CU(cudaMemsetAsync(gF, 0, sizeof(double) * 4 * (nrho - 1) * ntypes, s));
    TDMD_CU(cudaMemsetAsync(grho, 0, sizeof(double) * 4 * (nr - 1) * ntypes, s));
    TDMD_CU(cudaMemsetAsync(gphi, 0, sizeof(double) * 4 * (nr - 1) * npairs, s));
  }
  const NbrView nl = view();
  const int m = static_cast<int>(m_);
  const int nblk = force_blocks(m_, lpa_);
  const double c = 1.0 / (3.0 * static_cast<double>(m_));
  with_geo([&](auto g) {
    using Geo = decltype(g);
    TDMD_LPA_DISPATCH(lpa_, {
      launch(k_fm_eam_density<Geo, L>, nblk, kThreads, 0, s, g, nl, m, types_.data(), e, rc_sq_,
             rho_.data(), fp_.data(), fpp_.data());
      launch(k_fm_eam_force<Geo, L>, nblk, kThreads, 0, s, g, nl, m, types_.data(), e, rc_sq_,
             fp_.data(), target_.data(), c, G_.data(), d_forces, part_.data());
      if (grad && ntypes == 1) {
        // one element: shared-memory window of the r-spline gradients over
        // the top W intervals, a persistent grid of two blocks per SM
        const int W = std::min(nr - 1, kAdjointWindow);
        const size_t smem = sizeof(double) * 8 * static_cast<size_t>(W);
        auto kern = k_fm_eam_adjoint_w<Geo, L>;
        TDMD_CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
        const int grid = std::min(2 * sm_count(), nblk);
        launch(kern, grid, kThreads, smem, s, g, nl, m, e, rc_sq_, rho_.data(), fp_.data(),
               fpp_.data(), G_.data(), (nr - 1) - W, W);
      } else if (grad) {
        launch(k_fm_eam_adjoint<Geo, L>, nblk, kThreads, 0, s, g, nl, m, types_.data(), e, rc_sq_,
               rho_.data(), fp_.data(), fpp_.data(), G_.data());
      }
    });
  });
  TDMD_LAUNCH_CHECK();
  launch(k_fm_sum, 1, kThreads, 0, s, part_.data(), nblk, 1, d_loss);
  TDMD_LAUNCH_CHECK();
}

}  // namespace tdmd_b200

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace tdmd_b200;

struct tdmd_fit {
  Fit f;
  tdmd_fit(int nsnap, int natoms, const tdmd_box& box, const double* pos, const int* types,
           double cutoff, int precision)
      : f(nsnap, natoms, box, pos, types, cutoff, precision) {}
};

extern "C" {

int32_t tdmd_fit_create(int32_t nsnap, int32_t natoms, const tdmd_box* box,
                        const double* positions, const int32_t* types, double cutoff,
                        int32_t precision, tdmd_fit** out) {
  return guarded([&] {
    TDMD_REQUIRE(out && box, "null argument");
    *out = new tdmd_fit(nsnap, natoms, *box, positions, types, cutoff, precision);
  });
}

int32_t tdmd_fit_destroy(tdmd_fit* f) {
  delete f;
  return TDMD_OK;
}

int32_t tdmd_fit_set_targets(tdmd_fit* f, const double* targets) {
  return guarded([&] {
    TDMD_REQUIRE(f, "null handle");
    f->f.set_targets(targets);
  });
}

int32_t tdmd_fit_morse(tdmd_fit* f, const double* d_params, double* d_loss, double* d_grad,
                       double* d_forces, void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(f, "null handle");
    f->f.morse(d_params, d_loss, d_grad, d_forces, as_stream(stream));
  });
}

int32_t tdmd_fit_eam(tdmd_fit* f, int32_t ntypes, int32_t nrho, double drho, int32_t nr,
                     double dr, const double* d_F, const double* d_rho, const double* d_phi,
                     double* d_loss, double* d_gF, double* d_grho, double* d_gphi,
                     double* d_forces, void* stream) {
  return guarded([&] {
    TDMD_REQUIRE(f, "null handle");
    f->f.eam(ntypes, nrho, drho, nr, dr, d_F, d_rho, d_phi, d_loss, d_gF, d_grho, d_gphi,
             d_forces, as_stream(stream));
  });
}

int32_t tdmd_fit_info(const tdmd_fit* f, int64_t* natoms_total, int32_t* lanes_per_atom) {
  return guarded([&] {
    TDMD_REQUIRE(f, "null handle");
    if (natoms_total) *natoms_total = f->f.natoms();
    if (lanes_per_atom) *lanes_per_atom = f->f.lanes();
  });
}

}  // extern "C"
