// determinism.cu -- the ID-ordered energy mode of the free-function force
// calls (tdmd_set_deterministic_reduce).
//
// The reference has a build-time switch for it (TDMD_DETERMINISTIC_REDUCE,
// src/core/determinism.hpp:20-24, ADR 0010): its force kernels then write
// each atom's energy into a buffer and one thread sums the buffer in atom-ID
// order onto *d_energy (sum_per_atom_kernel, src/potentials/device_morse.cu:
// 16-30; eam_sum_per_atom_kernel, device_eam.cu:20 and :366-418).  Here the
// switch is a process-wide flag read at each call.  With it on, an FP64
// tdmd_morse_compute / tdmd_device_eam_compute that asks for an energy or a
// virial runs the kernels below: one thread per atom walking its row in list
// order with the reference's per-pair arithmetic, operation for operation
// (relative FP64 delta, if/else minimum image, (x*x + y*y) + z*z, the
// division-indexed spline a + x(b + x(c + x d)) and its derivative
// b + x(2c + 3x d), sqrt, exp), so each atom's energy has the reference's
// bits; then one thread adds the atoms' energies in ID order, Morse once and
// EAM twice (the embedding energies, then the pair halves), exactly as the
// reference's deterministic build does.  The virial (no reference symbol) is
// summed per atom and in ID order the same way.  Forces come from the same
// kernels.  The mode is slower than the default path (one thread per atom,
// one-thread sums), like the reference's.
//
// Mixed precision keeps the default kernels with the flag on: their
// fixed-order block reduction is already reproducible run to run, and the
// reference's mixed deterministic build evaluates splines whose
// coefficients it computed in FP32 on the host, so no FP64-built table can
// reproduce its bits.
#include <atomic>

#include "common.cuh"
#include "determinism.cuh"

namespace tdmd_b200 {

namespace {
std::atomic<int> g_deterministic{0};
}

bool deterministic_reduce() { return g_deterministic.load(std::memory_order_relaxed) != 0; }

namespace {

constexpr int kThreads = 256;

// SplineTable::eval / eval_deriv on the device (device_eam.cu:36-66).
__device__ __forceinline__ double id_spline(const RefSpline& s, const double* __restrict__ c,
                                            double r) {
  if (s.n < 2) return 0.0;
  double t = (r - s.rmin) / s.dr;
  int k = static_cast<int>(t);
  if (k < 0) k = 0;
  if (k >= s.n - 1) k = s.n - 2;
  double x = r - (s.rmin + static_cast<double>(k) * s.dr);
  const int m = s.n - 1;
  double a = c[s.offset + k];
  double b = c[s.offset + m + k];
  double cc = c[s.offset + 2 * m + k];
  double d = c[s.offset + 3 * m + k];
  return a + x * (b + x * (cc + x * d));
}

__device__ __forceinline__ double id_spline_deriv(const RefSpline& s,
                                                  const double* __restrict__ c, double r) {
  if (s.n < 2) return 0.0;
  double t = (r - s.rmin) / s.dr;
  int k = static_cast<int>(t);
  if (k < 0) k = 0;
  if (k >= s.n - 1) k = s.n - 2;
  double x = r - (s.rmin + static_cast<double>(k) * s.dr);
  const int m = s.n - 1;
  double b = c[s.offset + m + k];
  double cc = c[s.offset + 2 * m + k];
  double d = c[s.offset + 3 * m + k];
  return b + x * (2.0 * cc + x * 3.0 * d);
}

struct IdBox {
  double bx, by, bz;  // box edges (hi - lo)
  int px, py, pz;
};

// r_i - r_j in FP64 with the if/else minimum image of the reference kernels.
__device__ __forceinline__ void id_delta(const double* __restrict__ pos, double xi, double yi,
                                         double zi, int j, const IdBox& b, double& dx,
                                         double& dy, double& dz) {
  const double hx = 0.5 * b.bx, hy = 0.5 * b.by, hz = 0.5 * b.bz;
  dx = xi - pos[3ll * j];
  dy = yi - pos[3ll * j + 1];
  dz = zi - pos[3ll * j + 2];
  if (b.px) {
    if (dx > hx) dx -= b.bx;
    else if (dx < -hx) dx += b.bx;
  }
  if (b.py) {
    if (dy > hy) dy -= b.by;
    else if (dy < -hy) dy += b.by;
  }
  if (b.pz) {
    if (dz > hz) dz -= b.bz;
    else if (dz < -hz) dz += b.bz;
  }
}

// Per-atom virial of the pairs in the row: W += 1/2 fpair d (x) d.
__device__ __forceinline__ void id_virial(double (&w)[6], double fpair, double dx, double dy,
                                          double dz) {
  const double h = 0.5 * fpair;
  const double hx = h * dx, hy = h * dy;
  w[0] += hx * dx;
  w[1] += hy * dy;
  w[2] += (h * dz) * dz;
  w[3] += hx * dy;
  w[4] += hx * dz;
  w[5] += hy * dz;
}

__device__ __forceinline__ void id_store(double* __restrict__ w_atom, int i, const double (&w)[6]) {
  if (w_atom)
    for (int k = 0; k < 6; ++k) w_atom[6ll * i + k] = w[k];
}

// morse_force_kernel's per-atom arithmetic (device_morse.cu:32-132), FP64.
__global__ void k_morse_idorder(const double* __restrict__ pos, double* __restrict__ f,
                                const int* __restrict__ nbr, const int* __restrict__ off,
                                const int* __restrict__ cnt, int n, IdBox b, double D,
                                double alpha, double r0, double rc_sq,
                                double* __restrict__ e_atom, double* __restrict__ w_atom) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = pos[3ll * i], yi = pos[3ll * i + 1], zi = pos[3ll * i + 2];
  double fx = 0.0, fy = 0.0, fz = 0.0, pe = 0.0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  const int o = off[i], c = cnt[i];
  for (int k = 0; k < c; ++k) {
    const int j = nbr[o + k];
    double dx, dy, dz;
    id_delta(pos, xi, yi, zi, j, b, dx, dy, dz);
    double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 < rc_sq) {
      double r = sqrt(r2);
      double dr = r - r0;
      double ex = exp(-alpha * dr);
      double ome = 1.0 - ex;
      pe += 0.5 * D * (ome * ome - 1.0);
      double dudr = 2.0 * D * alpha * ome * ex;
      double fpair = -dudr / r;
      fx += fpair * dx;
      fy += fpair * dy;
      fz += fpair * dz;
      id_virial(w, fpair, dx, dy, dz);
    }
  }
  f[3ll * i] = fx;
  f[3ll * i + 1] = fy;
  f[3ll * i + 2] = fz;
  e_atom[i] = pe;
  id_store(w_atom, i, w);
}

// eam_density_kernel (device_eam.cu:72-133), FP64.
__global__ void k_eam_density_idorder(const double* __restrict__ pos,
                                      const int* __restrict__ types, const int* __restrict__ nbr,
                                      const int* __restrict__ off, const int* __restrict__ cnt,
                                      int n, IdBox b, double rc_sq,
                                      const RefSpline* __restrict__ dens,
                                      const double* __restrict__ coeff,
                                      double* __restrict__ rho) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = pos[3ll * i], yi = pos[3ll * i + 1], zi = pos[3ll * i + 2];
  const int o = off[i], c = cnt[i];
  double rho_i = 0.0;
  for (int k = 0; k < c; ++k) {
    const int j = nbr[o + k];
    double dx, dy, dz;
    id_delta(pos, xi, yi, zi, j, b, dx, dy, dz);
    double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= rc_sq) continue;
    double r = sqrt(r2);
    const int tj = types[j] - 1;
    rho_i += id_spline(dens[tj], coeff, r);
  }
  rho[i] = rho_i;
}

// eam_embedding_kernel (device_eam.cu:137-162): F'(rho_i) and F(rho_i).
__global__ void k_eam_embed_idorder(const int* __restrict__ types, int n,
                                    const RefSpline* __restrict__ emb,
                                    const double* __restrict__ coeff,
                                    const double* __restrict__ rho, double* __restrict__ fp,
                                    double* __restrict__ e_atom) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int ti = types[i] - 1;
  const double rho_i = rho[i];
  fp[i] = id_spline_deriv(emb[ti], coeff, rho_i);
  e_atom[i] = id_spline(emb[ti], coeff, rho_i);
}

__device__ __forceinline__ int id_phi_index(int ti, int tj, int nt) {
  if (ti > tj) {
    const int t = ti;
    ti = tj;
    tj = t;
  }
  return ti * nt - ti * (ti + 1) / 2 + tj;
}

// eam_force_kernel (device_eam.cu:176-278), FP64.
__global__ void k_eam_force_idorder(const double* __restrict__ pos, double* __restrict__ f,
                                    const int* __restrict__ types, const int* __restrict__ nbr,
                                    const int* __restrict__ off, const int* __restrict__ cnt,
                                    int n, int nt, IdBox b, double rc_sq,
                                    const RefSpline* __restrict__ dens,
                                    const RefSpline* __restrict__ phi,
                                    const double* __restrict__ coeff,
                                    const double* __restrict__ fp, double* __restrict__ e_atom,
                                    double* __restrict__ w_atom) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = pos[3ll * i], yi = pos[3ll * i + 1], zi = pos[3ll * i + 2];
  const int ti = types[i] - 1;
  const int o = off[i], c = cnt[i];
  const double fpi = fp[i];
  double fx = 0.0, fy = 0.0, fz = 0.0, pe = 0.0;
  double w[6] = {0, 0, 0, 0, 0, 0};
  for (int k = 0; k < c; ++k) {
    const int j = nbr[o + k];
    double dx, dy, dz;
    id_delta(pos, xi, yi, zi, j, b, dx, dy, dz);
    double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= rc_sq) continue;
    double r = sqrt(r2);
    const int tj = types[j] - 1;
    const int p = id_phi_index(ti, tj, nt);
    double phi_val = id_spline(phi[p], coeff, r);
    pe += 0.5 * phi_val;
    double dphi = id_spline_deriv(phi[p], coeff, r);
    double drho_j = id_spline_deriv(dens[tj], coeff, r);
    double drho_i = id_spline_deriv(dens[ti], coeff, r);
    double fpair = -(dphi + fpi * drho_j + fp[j] * drho_i) / r;
    fx += fpair * dx;
    fy += fpair * dy;
    fz += fpair * dz;
    id_virial(w, fpair, dx, dy, dz);
  }
  f[3ll * i] = fx;
  f[3ll * i + 1] = fy;
  f[3ll * i + 2] = fz;
  e_atom[i] = pe;
  id_store(w_atom, i, w);
}

// One thread: *out += v[0] + v[1] + ... in index order (sum_per_atom_kernel,
// device_morse.cu:16-30); for the virial, each of 6 components over
// v[6i + k].
__global__ void k_sum_in_id_order(const double* __restrict__ v, int n, int stride,
                                  double* __restrict__ out) {
  dependent_launch_prologue();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  for (int k = 0; k < stride; ++k) {
    double s = out[k];
    for (int i = 0; i < n; ++i) s += v[static_cast<long long>(i) * stride + k];
    out[k] = s;
  }
}

IdBox id_box(const tdmd_box& b) {
  return IdBox{b.hi[0] - b.lo[0], b.hi[1] - b.lo[1], b.hi[2] - b.lo[2],
               b.periodic[0] ? 1 : 0, b.periodic[1] ? 1 : 0, b.periodic[2] ? 1 : 0};
}

// Per-call scratch from the stream-ordered pool.
struct Scratch {
  double* p = nullptr;
  cudaStream_t s;
  Scratch(size_t count, cudaStream_t st) : s(st) {
    TDMD_CU(cudaMallocAsync(reinterpret_cast<void**>(&p), sizeof(double) * (count ? count : 1),
                            st));
  }
  ~Scratch() {
    if (p) cudaFreeAsync(p, s);
  }
};

}  // namespace

void RefEamTables::upload(const tdmd_eam& e) {
  const int nt = e.ntypes;
  const int npairs = nt * (nt + 1) / 2;
  const int nsf = 4 * (e.nrho - 1), nsr = 4 * (e.nr - 1);
  std::vector<double> flat;
  flat.reserve(e.Fc.size() + e.rhoc.size() + e.phic.size());
  flat.insert(flat.end(), e.Fc.begin(), e.Fc.end());
  flat.insert(flat.end(), e.rhoc.begin(), e.rhoc.end());
  flat.insert(flat.end(), e.phic.begin(), e.phic.end());
  std::vector<RefSpline> meta(static_cast<size_t>(2 * nt + npairs));
  for (int t = 0; t < nt; ++t) meta[t] = RefSpline{e.drho, 0.0, e.nrho, t * nsf};
  for (int t = 0; t < nt; ++t) meta[nt + t] = RefSpline{e.dr, 0.0, e.nr, nt * nsf + t * nsr};
  for (int p = 0; p < npairs; ++p)
    meta[2 * nt + p] = RefSpline{e.dr, 0.0, e.nr, nt * nsf + nt * nsr + p * nsr};
  coeff.reserve(flat.size());
  splines.reserve(meta.size());
  TDMD_CU(cudaMemcpy(coeff.data(), flat.data(), flat.size() * sizeof(double),
                     cudaMemcpyHostToDevice));
  TDMD_CU(cudaMemcpy(splines.data(), meta.data(), meta.size() * sizeof(RefSpline),
                     cudaMemcpyHostToDevice));
  ntypes = nt;
  cutoff = e.cutoff;
}

void morse_id_ordered(const double* pos, double* forces, const int* nbr, const int* off,
                      const int* cnt, int n, const tdmd_box& box, const tdmd_morse_params& p,
                      double* energy, double* virial, cudaStream_t s) {
  Scratch e_atom(static_cast<size_t>(n), s);
  Scratch w_atom(virial ? 6 * static_cast<size_t>(n) : 0, s);
  launch(k_morse_idorder, ceil_div(n, kThreads), kThreads, 0, s, pos, forces, nbr, off, cnt, n,
         id_box(box), p.d, p.alpha, p.r0, p.rc_sq, e_atom.p, virial ? w_atom.p : nullptr);
  TDMD_LAUNCH_CHECK();
  if (energy) {
    launch(k_sum_in_id_order, 1, 1, 0, s, e_atom.p, n, 1, energy);
    TDMD_LAUNCH_CHECK();
  }
  if (virial) {
    launch(k_sum_in_id_order, 1, 1, 0, s, w_atom.p, n, 6, virial);
    TDMD_LAUNCH_CHECK();
  }
}

void eam_id_ordered(const RefEamTables& t, const double* pos, double* forces, const int* types,
                    const int* nbr, const int* off, const int* cnt, int n, const tdmd_box& box,
                    double* energy, double* virial, double* rho_out, double* fp_out,
                    cudaStream_t s) {
  Scratch rho(static_cast<size_t>(n), s), fp(static_cast<size_t>(n), s);
  Scratch e_atom(static_cast<size_t>(n), s);
  Scratch w_atom(virial ? 6 * static_cast<size_t>(n) : 0, s);
  const IdBox b = id_box(box);
  const double rc_sq = t.cutoff * t.cutoff;  // DeviceEam::compute, device_eam.cu:348
  const int nt = t.ntypes;
  const RefSpline* emb = t.splines.data();
  const RefSpline* dens = emb + nt;
  const RefSpline* phi = emb + 2 * nt;
  const int nb = ceil_div(n, kThreads);
  launch(k_eam_density_idorder, nb, kThreads, 0, s, pos, types, nbr, off, cnt, n, b, rc_sq, dens,
         t.coeff.data(), rho.p);
  TDMD_LAUNCH_CHECK();
  launch(k_eam_embed_idorder, nb, kThreads, 0, s, types, n, emb, t.coeff.data(), rho.p, fp.p,
         e_atom.p);
  TDMD_LAUNCH_CHECK();
  if (energy) {
    launch(k_sum_in_id_order, 1, 1, 0, s, e_atom.p, n, 1, energy);
    TDMD_LAUNCH_CHECK();
  }
  launch(k_eam_force_idorder, nb, kThreads, 0, s, pos, forces, types, nbr, off, cnt, n, nt, b,
         rc_sq, dens, phi, t.coeff.data(), fp.p, e_atom.p, virial ? w_atom.p : nullptr);
  TDMD_LAUNCH_CHECK();
  if (energy) {
    launch(k_sum_in_id_order, 1, 1, 0, s, e_atom.p, n, 1, energy);
    TDMD_LAUNCH_CHECK();
  }
  if (virial) {
    launch(k_sum_in_id_order, 1, 1, 0, s, w_atom.p, n, 6, virial);
    TDMD_LAUNCH_CHECK();
  }
  if (rho_out)
    TDMD_CU(cudaMemcpyAsync(rho_out, rho.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  if (fp_out)
    TDMD_CU(cudaMemcpyAsync(fp_out, fp.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
}

}  // namespace tdmd_b200

extern "C" {

int32_t tdmd_set_deterministic_reduce(int32_t on) {
  tdmd_b200::g_deterministic.store(on ? 1 : 0, std::memory_order_relaxed);
  return TDMD_OK;
}

int32_t tdmd_get_deterministic_reduce(int32_t* on) {
  if (!on) return tdmd_b200::fail(TDMD_ERR_INVALID_ARGUMENT, "null argument");
  *on = tdmd_b200::deterministic_reduce() ? 1 : 0;
  return TDMD_OK;
}

}  // extern "C"
