// scheduler.cu -- FastPipelineScheduler for sm_100a.
//
// Reference: src/scheduler/fast_pipeline_scheduler.{cuh,cu} (ctor :15-40,
// upload :49-73, download :75-85, step/run_until :87-223,
// maybe_rebuild_nlist :225-232) plus the NVT/adaptive-dt wiring of
// PipelineScheduler::run_until (src/scheduler/pipeline_scheduler.cu:
// 235-276), which the reference has only on its zone path.
//
// Per step (NVE): fused kick+drift (half dt on the first step of a
// run_until window, full dt after: OPT-FUSE-1c) -> neighbor rebuild every
// rebuild_every steps -> force (Morse: 1 kernel; EAM: density with the
// embedding fused into its epilogue, then force); one closing half kick per
// window.  With NVT or adaptive dt: kick+drift (scale by the pending NHC
// factor first) -> rebuild -> force -> half kick + FP64 KE/v_max partials
// -> one-block control kernel (fixed-order reduction, NHC half steps,
// next dt).  Nothing returns to the host inside a window.
//
// B200 specifics: state lives in device layouts made for the gathers
// (double4 {x,y,z,type} positions; fixed-point int4 copies for the mixed
// path), each window is split into segments that are captured once as CUDA
// graphs and replayed, the neighbor list is built in one pass into padded
// rows with a device overflow flag (checked at the window's single sync; on
// overflow the window is re-run from a device snapshot with a larger
// capacity), and all energy/virial sums are fixed-order FP64 reductions.
#include <algorithm>
#include <type_traits>
#include <climits>
#include <cmath>
#include <list>
#include <map>
#include <memory>
#include <vector>

#include "buffers.cuh"
#include "common.cuh"
#include "eam_tables.cuh"
#include "forces.cuh"
#include "integrate.cuh"
#include "launch.cuh"
#include "sched.cuh"

namespace tdmd_b200 {

namespace {

constexpr int kThreads = 256;

// --------------------------------------------------------------------------
// Kernels
// --------------------------------------------------------------------------

// positions (double[3n]) -> pos4 {x,y,z,type} (+ fixed-point q)
__global__ void k_pack_positions(const double* __restrict__ x, const int* __restrict__ types,
                                 int n, DevBox b, double4* __restrict__ pos4,
                                 int4* __restrict__ q) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double px = x[3ll * i], py = x[3ll * i + 1], pz = x[3ll * i + 2];
  const int t = types[i];
  pos4[i] = make_double4(px, py, pz, static_cast<double>(t));
  if (q)
    q[i] = make_int4(encode_q(px, b.qlo[0], b.qinv[0]), encode_q(py, b.qlo[1], b.qinv[1]),
                     encode_q(pz, b.qlo[2], b.qinv[2]), t);
}


struct D3 {
  double x, y, z;
};
struct F3 {
  float x, y, z;
};

// The whole per-atom state into the cell order in one pass: dst[i] =
// src[idx[i]] for positions, velocities, types, ids, fixed-point records
// (nullable) and forces.
template <class F>
__global__ void k_gather_state(const int* __restrict__ idx, int n,
                               const double4* __restrict__ p, double4* __restrict__ p_o,
                               const D3* __restrict__ v, D3* __restrict__ v_o,
                               const int* __restrict__ t, int* __restrict__ t_o,
                               const int* __restrict__ id, int* __restrict__ id_o,
                               const int4* __restrict__ q, int4* __restrict__ q_o,
                               const F* __restrict__ f, F* __restrict__ f_o) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int j = idx[i];
  p_o[i] = p[j];
  v_o[i] = v[j];
  t_o[i] = t[j];
  id_o[i] = id[j];
  if (q) q_o[i] = q[j];
  f_o[i] = f[j];
}

__global__ void k_iota(int* __restrict__ a, int n) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

// dst[idx[i]] = src[i]
template <class T>
__global__ void k_scatter(const T* __restrict__ src, const int* __restrict__ idx, int n,
                          T* __restrict__ dst) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[idx[i]] = src[i];
}

__global__ void k_scatter_positions(const double4* __restrict__ pos4, const int* __restrict__ idx,
                                    int n, double* __restrict__ x) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = pos4[i];
  const long long k = idx[i];
  x[3 * k] = p.x;
  x[3 * k + 1] = p.y;
  x[3 * k + 2] = p.z;
}

// A window's prologue in one launch: the state an overflow retry rewinds to
// (positions, fixed-point records when q is non-null, velocities, the
// control block) copied aside, then -- with reset -- the overflow flags of
// the live control block zeroed (after the copy, by the same thread).
__global__ void __launch_bounds__(kThreads) k_window_prologue(
    const double4* __restrict__ pos4, double4* __restrict__ snap_pos4,
    const int4* __restrict__ q, int4* __restrict__ snap_q, const double* __restrict__ vel,
    double* __restrict__ snap_vel, int n, SchedCtl* __restrict__ ctl,
    SchedCtl* __restrict__ snap_ctl, int reset) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    snap_pos4[i] = pos4[i];
    if (q) snap_q[i] = q[i];
    const long long k = 3ll * i;
    snap_vel[k] = vel[k];
    snap_vel[k + 1] = vel[k + 1];
    snap_vel[k + 2] = vel[k + 2];
  }
  if (i == 0) {
    *snap_ctl = *ctl;
    if (reset) {
      for (int c = 0; c < 4; ++c) ctl->status[c] = 0;
    }
  }
}

// Kick (half or full dt, optionally after the pending NHC scale) + drift +
// single-image wrap + fixed-point refresh.  fused_kick_drift_kernel,
// device_velocity_verlet.cu:88-130.  dt comes from the control block when
// `ctl_dt` (adaptive dt), else from the argument.
template <class F, bool FULL, bool SCALE>
__global__ void __launch_bounds__(kThreads) k_kick_drift(double4* __restrict__ pos4,
                                                         int4* __restrict__ q,
                                                         double* __restrict__ v,
                                                         const F* __restrict__ f,
                                                         const int* __restrict__ types,
                                                         const double* __restrict__ inv_mm, int n,
                                                         double dt_arg, SchedCtl* __restrict__ ctl,
                                                         int ctl_dt, DevBox b) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) ctl->step += 1;
  if (i >= n) return;
  const double dt = ctl_dt ? ctl->dt : dt_arg;
  const double kick_dt = FULL ? dt : 0.5 * dt;
  const int t = types[i];
  const double factor = kick_dt * inv_mm[t];
  const double s = SCALE ? ctl->scale : 1.0;
  double4 p = pos4[i];
  double vx = v[3ll * i], vy = v[3ll * i + 1], vz = v[3ll * i + 2];
  if (SCALE) {
    vx *= s;
    vy *= s;
    vz *= s;
  }
  vx += factor * static_cast<double>(f[3ll * i]);
  vy += factor * static_cast<double>(f[3ll * i + 1]);
  vz += factor * static_cast<double>(f[3ll * i + 2]);
  p.x = wrap_single(p.x + dt * vx, b.lo[0], b.L[0], b.periodic[0]);
  p.y = wrap_single(p.y + dt * vy, b.lo[1], b.L[1], b.periodic[1]);
  p.z = wrap_single(p.z + dt * vz, b.lo[2], b.L[2], b.periodic[2]);
  v[3ll * i] = vx;
  v[3ll * i + 1] = vy;
  v[3ll * i + 2] = vz;
  pos4[i] = p;
  if (q)
    q[i] = make_int4(encode_q(p.x, b.qlo[0], b.qinv[0]), encode_q(p.y, b.qlo[1], b.qinv[1]),
                     encode_q(p.z, b.qlo[2], b.qinv[2]), t);
}

// Half kick; with KE, per-block (KE, max|v|^2) partials of the kicked
// velocities (k_ke_vmax_partials layout).
template <class F, bool KE>
__global__ void __launch_bounds__(kThreads) k_half_kick_s(double* __restrict__ v,
                                                          const F* __restrict__ f,
                                                          const int* __restrict__ types,
                                                          const double* __restrict__ masses,
                                                          const double* __restrict__ inv_mm,
                                                          int n, double dt_arg,
                                                          const SchedCtl* __restrict__ ctl,
                                                          int ctl_dt,
                                                          double* __restrict__ partials) {
  dependent_launch_prologue();
  __shared__ double red[32 * 2];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double ke = 0.0, v2 = 0.0;
  if (i < n) {
    const double dt = ctl_dt ? ctl->dt : dt_arg;
    const double m = masses[types[i]];
    const double factor = 0.5 * dt * inv_mm[types[i]];
    const double vx = v[3ll * i] + factor * static_cast<double>(f[3ll * i]);
    const double vy = v[3ll * i + 1] + factor * static_cast<double>(f[3ll * i + 1]);
    const double vz = v[3ll * i + 2] + factor * static_cast<double>(f[3ll * i + 2]);
    v[3ll * i] = vx;
    v[3ll * i + 1] = vy;
    v[3ll * i + 2] = vz;
    if (KE) {
      v2 = vx * vx + vy * vy + vz * vz;
      ke = 0.5 * m * kMvv2e * v2;
    }
  }
  if (KE) {
    ke = warp_sum(ke);
    v2 = warp_max(v2);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
      red[2 * warp] = ke;
      red[2 * warp + 1] = v2;
    }
    __syncthreads();
    if (warp == 0) {
      const int nw = blockDim.x >> 5;
      ke = lane < nw ? red[2 * lane] : 0.0;
      v2 = lane < nw ? red[2 * lane + 1] : 0.0;
      ke = warp_sum(ke);
      v2 = warp_max(v2);
      if (lane == 0) {
        partials[2ll * blockIdx.x] = ke;
        partials[2ll * blockIdx.x + 1] = v2;
      }
    }
  }
}

// KE at integer time while velocities sit half a step behind (NVE windows):
// sum 1/2 m mvv2e |v + dt/2 F/(m mvv2e)|^2, per-block partials.
template <class F>
__global__ void __launch_bounds__(kThreads) k_ke_integer(const double* __restrict__ v,
                                                         const F* __restrict__ f,
                                                         const int* __restrict__ types,
                                                         const double* __restrict__ masses,
                                                         const double* __restrict__ inv_mm,
                                                         int n, double dt,
                                                         double* __restrict__ partials) {
  dependent_launch_prologue();
  __shared__ double red[32 * 2];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double ke = 0.0, v2 = 0.0;
  if (i < n) {
    const double m = masses[types[i]];
    const double factor = 0.5 * dt * inv_mm[types[i]];
    const double vx = v[3ll * i] + factor * static_cast<double>(f[3ll * i]);
    const double vy = v[3ll * i + 1] + factor * static_cast<double>(f[3ll * i + 1]);
    const double vz = v[3ll * i + 2] + factor * static_cast<double>(f[3ll * i + 2]);
    v2 = vx * vx + vy * vy + vz * vz;
    ke = 0.5 * m * kMvv2e * v2;
  }
  ke = warp_sum(ke);
  v2 = warp_max(v2);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[2 * warp] = ke;
    red[2 * warp + 1] = v2;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    ke = lane < nw ? red[2 * lane] : 0.0;
    v2 = lane < nw ? red[2 * lane + 1] : 0.0;
    ke = warp_sum(ke);
    v2 = warp_max(v2);
    if (lane == 0) {
      partials[2ll * blockIdx.x] = ke;
      partials[2ll * blockIdx.x + 1] = v2;
    }
  }
}

enum CtlMode : int {
  kCtlPre = 1,    // window start: thermostat/adaptive-dt from the current velocities
  kCtlPost = 2,   // after the closing half kick of a step
  kCtlNext = 4,   // ...and prepare the next step of the same window
  kCtlLog = 8,    // append an energy-log record
};

// Threads of the single-block reducers below: 1024 above 4096 records (4 M
// atoms: 15 625), else 256 (the extra warps cost more than they hide).
constexpr int kCtlThreads = 1024;
inline int ctl_threads(int nblk) { return nblk > 4096 ? kCtlThreads : 256; }

// Sum of partials[2b] and max of partials[2b + 1] over b < nblk, for thread
// 0 of one block: each thread keeps four independent (sum, max) pairs so
// four loads are in flight (a 15 625-record reduction at 4 M atoms is
// latency-bound otherwise), then the warp tree and the warps in order.  The
// order depends only on nblk and the block size: bit-reproducible.
__device__ __forceinline__ void reduce_ke_v2(const double* __restrict__ partials, int nblk,
                                             double& ke, double& v2) {
  __shared__ double red[32 * 2];
  const int nt = blockDim.x;
  double k4[4] = {0.0, 0.0, 0.0, 0.0}, m4[4] = {0.0, 0.0, 0.0, 0.0};
  const double2* p2 = reinterpret_cast<const double2*>(partials);
  int b = threadIdx.x;
  for (; b + 3 * nt < nblk; b += 4 * nt) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double2 v = p2[b + u * nt];
      k4[u] += v.x;
      m4[u] = fmax(m4[u], v.y);
    }
  }
  for (; b < nblk; b += nt) {
    const double2 v = p2[b];
    k4[0] += v.x;
    m4[0] = fmax(m4[0], v.y);
  }
  ke = warp_sum((k4[0] + k4[1]) + (k4[2] + k4[3]));
  v2 = warp_max(fmax(fmax(m4[0], m4[1]), fmax(m4[2], m4[3])));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[2 * warp] = ke;
    red[2 * warp + 1] = v2;
  }
  __syncthreads();
  ke = 0.0;
  v2 = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < (nt >> 5); ++w) {
      ke += red[2 * w];
      v2 = fmax(v2, red[2 * w + 1]);
    }
  }
}

// One block: reduce (KE, v2max) partials in block order, run the chain and
// the adaptive-dt rule, write the pending scale / next dt, optionally log.
__global__ void __launch_bounds__(kCtlThreads) k_control(SchedCtl* __restrict__ ctl,
                                                         const double* __restrict__ partials,
                                                         int nblk, CtlParams p, int mode,
                                                         double* __restrict__ log, int log_cap) {
  dependent_launch_prologue();
  double ke, v2;
  reduce_ke_v2(partials, nblk, ke, v2);
  if (threadIdx.x != 0) return;
  auto adapt = [&](double vmax2) {
    if (!p.adaptive) return;
    const double vmax = sqrt(vmax2);
    if (vmax > 0.0) {
      double dt = fmin(p.dt_max, p.c2 * p.rc / vmax);
      ctl->dt = fmax(dt, p.dt_min);
    }
  };
  auto chain = [&](double k) {
    return p.nvt ? nhc_half_step(ctl->eta, ctl->eta_v, ctl->eta_m, p.M, p.t_target, p.t_period,
                                 p.n_dof, p.dt_nhc, k)
                 : 1.0;
  };
  if (mode & kCtlPre) {
    adapt(v2);
    ctl->scale = chain(ke);
    ctl->ke = ke;
    return;
  }
  // Post-step half step of the chain on the kicked velocities.
  const double s_post = chain(ke);
  const double ke_post = ke * s_post * s_post;
  ctl->ke = ke_post;
  if (mode & kCtlLog) {
    const int slot = ctl->log_count % (log_cap > 0 ? log_cap : 1);
    double* r = log + 9ll * slot;
    r[0] = static_cast<double>(ctl->step);
    r[1] = ctl->ev[0];
    r[2] = ke_post;
    for (int k = 0; k < 6; ++k) r[3 + k] = ctl->ev[1 + k];
    ctl->log_count += 1;
  }
  if (mode & kCtlNext) {
    adapt(v2 * s_post * s_post);
    const double s_pre = chain(ke_post);
    ctl->scale = s_post * s_pre;
  } else {
    ctl->scale = s_post;
  }
}

// NVE energy-log record: KE partials at integer time + the step's EV sums.
__global__ void __launch_bounds__(kCtlThreads) k_log_nve(SchedCtl* __restrict__ ctl,
                                                         const double* __restrict__ partials,
                                                         int nblk, double* __restrict__ log,
                                                         int log_cap) {
  dependent_launch_prologue();
  double ke, v2;
  reduce_ke_v2(partials, nblk, ke, v2);
  if (threadIdx.x != 0) return;
  const int slot = ctl->log_count % (log_cap > 0 ? log_cap : 1);
  double* r = log + 9ll * slot;
  r[0] = static_cast<double>(ctl->step);
  r[1] = ctl->ev[0];
  r[2] = ke;
  for (int k = 0; k < 6; ++k) r[3 + k] = ctl->ev[1 + k];
  ctl->log_count += 1;
}

__global__ void k_apply_scale(double* __restrict__ v, long long m, const SchedCtl* __restrict__ ctl) {
  dependent_launch_prologue();
  const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < m) v[i] *= ctl->scale;
}

}  // namespace

// ==========================================================================
// Scheduler implementation
// ==========================================================================
Scheduler::Scheduler(const tdmd_box& box, int natoms, const tdmd_fast_pipeline_config& cfg)
    : hbox_(box), n_(natoms), cfg_(cfg) {
  TDMD_REQUIRE(natoms >= 0, "natoms must be non-negative");
  TDMD_REQUIRE(cfg.dt > 0.0, "dt must be positive");
  TDMD_REQUIRE(cfg.r_skin >= 0.0, "r_skin must be non-negative");
  TDMD_REQUIRE(cfg.rebuild_every >= 1, "rebuild_every must be >= 1");
  TDMD_REQUIRE(cfg.precision == TDMD_FP64 || cfg.precision == TDMD_MIXED, "unknown precision");
  TDMD_REQUIRE(cfg.nhc_length >= 0 && cfg.nhc_length <= kMaxChain, "nhc_length out of range");
  mixed_ = cfg.precision == TDMD_MIXED;
  nvt_ = cfg.t_target > 0.0 && cfg.nhc_length > 0;
  thermo_ = nvt_ || cfg.adaptive_dt != 0;
  TDMD_CU(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  TDMD_CU(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
  TDMD_CU(cudaEventCreate(&win_ev_[0]));
  TDMD_CU(cudaEventCreate(&win_ev_[1]));
  TDMD_CU(cudaEventCreateWithFlags(&up_ev_[0], cudaEventDisableTiming));
  TDMD_CU(cudaEventCreateWithFlags(&up_ev_[1], cudaEventDisableTiming));
  ctl_.reserve(1);
  snap_ctl_.reserve(1);
}

Scheduler::~Scheduler() {
  clear_graphs();
  if (stream_) cudaStreamSynchronize(stream_);
  for (const ProfEvents& pe : prof_retired_) {
    cudaEventDestroy(pe.a);
    cudaEventDestroy(pe.b);
  }
  if (h_cellmax_) cudaFreeHost(h_cellmax_);
  if (side_) {
    cudaStreamSynchronize(side_);
    cudaStreamDestroy(side_);
  }
  if (h_stage_) cudaFreeHost(h_stage_);
  for (auto e : up_ev_)
    if (e) cudaEventDestroy(e);
  for (auto& pe : prof_pending_) {
    cudaEventDestroy(pe.second.first);
    cudaEventDestroy(pe.second.second);
  }
  for (auto e : prof_pool_) cudaEventDestroy(e);
  for (auto e : win_ev_)
    if (e) cudaEventDestroy(e);
  if (stream_) {
    cudaStreamSynchronize(stream_);
    cudaStreamDestroy(stream_);
  }
}

void Scheduler::set_morse(const tdmd_morse_params& p) {
  kind_ = TDMD_POT_MORSE;
  cutoff_ = p.rc;
  const double rc_sq = p.rc_sq > 0.0 ? p.rc_sq : p.rc * p.rc;
  m64_ = MorseP<double>{p.d, p.alpha, p.r0, rc_sq, p.r0};
  m32_ = MorseP<float>{static_cast<float>(p.d), static_cast<float>(p.alpha),
                       static_cast<float>(p.r0), static_cast<float>(rc_sq), p.r0};
  finish_setup();
}

void Scheduler::set_eam(const tdmd_eam& e) {
  kind_ = TDMD_POT_EAM;
  cutoff_ = e.cutoff;
  eam_ = std::make_unique<EamDevTables>();
  eam_->upload(e, stream_);
  finish_setup();
}

void Scheduler::finish_setup() {
  TDMD_REQUIRE(cutoff_ > 0.0, "cutoff must be positive");
  box_ = make_devbox(hbox_, cutoff_ + cfg_.r_skin);
  lpa_ = cfg_.lanes_per_atom > 0 ? cfg_.lanes_per_atom : default_lpa(n_ > 0 ? n_ : 1);
  TDMD_REQUIRE(lpa_ == 1 || lpa_ == 2 || lpa_ == 4 || lpa_ == 8 || lpa_ == 16 || lpa_ == 32,
               "lanes_per_atom must be 1,2,4,8,16 or 32");
  TDMD_REQUIRE(cfg_.nbr_batch == 0 || cfg_.nbr_batch == 2 || cfg_.nbr_batch == 4,
               "nbr_batch must be 0 (tuned), 2 or 4");
  nu_ = cfg_.nbr_batch > 0 ? cfg_.nbr_batch : kU;
  lpa_d_ = lpa_;
  nu_d_ = nu_;
}

void Scheduler::upload(const double* x, const double* v, const void* f, const int* types,
                       const int* ids, const double* masses, int n_types) {
  TDMD_REQUIRE(kind_ >= 0, "scheduler has no potential");
  TDMD_REQUIRE(n_types >= 2, "n_types is masses.size() = ntypes + 1 (>= 2)");
  TDMD_REQUIRE(n_ == 0 || (x && v && types && masses), "null host array");
  const size_t n = static_cast<size_t>(n_);
  clear_graphs();
  cudaStream_t s = stream_;
  pos4_.reserve(n);
  vel_.reserve(3 * n);
  types_.reserve(n);
  ids_.reserve(n);
  stage_.reserve(3 * n);
  masses_.reserve(static_cast<size_t>(n_types));
  if (mixed_) {
    q_.reserve(n);
    f32_.reserve(3 * n);
  } else {
    f64_.reserve(3 * n);
  }
  n_types_ = n_types;
  uploaded_ = false;
  cells_from_upload_ = false;
  // Masses, kick factors and the control block through the pinned block
  // (the previous upload's copies from it finished at its synchronisation).
  const size_t stage_bytes = 2 * sizeof(double) * static_cast<size_t>(n_types) + sizeof(SchedCtl);
  if (h_stage_cap_ < stage_bytes) {
    if (h_stage_) cudaFreeHost(h_stage_);
    h_stage_ = nullptr;
    h_stage_cap_ = 0;
    TDMD_CU(cudaMallocHost(reinterpret_cast<void**>(&h_stage_), stage_bytes));
    h_stage_cap_ = stage_bytes;
  }
  double* h_masses = reinterpret_cast<double*>(h_stage_);
  double* h_inv = h_masses + n_types;
  SchedCtl* h_ctl = reinterpret_cast<SchedCtl*>(h_inv + n_types);
  if (n_ > 0) {
    // stream_: types and positions, then packing and the cell list; side_
    // (after stream_'s earlier work and those two copies, so that the
    // positions do not share the bus with the rest): velocities, ids,
    // forces, while the positions are binned.
    TDMD_CU(cudaMemcpyAsync(types_.data(), types, n * sizeof(int), cudaMemcpyHostToDevice, s));
    TDMD_CU(cudaMemcpyAsync(stage_.data(), x, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    TDMD_CU(cudaEventRecord(up_ev_[0], s));
    TDMD_CU(cudaStreamWaitEvent(side_, up_ev_[0], 0));
    TDMD_CU(cudaMemcpyAsync(vel_.data(), v, 3 * n * sizeof(double), cudaMemcpyHostToDevice,
                            side_));
    if (ids)
      TDMD_CU(cudaMemcpyAsync(ids_.data(), ids, n * sizeof(int), cudaMemcpyHostToDevice, side_));
    else
      TDMD_CU(cudaMemsetAsync(ids_.data(), 0, n * sizeof(int), side_));
    const size_t fb = 3 * n * (mixed_ ? sizeof(float) : sizeof(double));
    void* fd = mixed_ ? static_cast<void*>(f32_.data()) : static_cast<void*>(f64_.data());
    if (f)
      TDMD_CU(cudaMemcpyAsync(fd, f, fb, cudaMemcpyHostToDevice, side_));
    else
      TDMD_CU(cudaMemsetAsync(fd, 0, fb, side_));
    TDMD_CU(cudaEventRecord(up_ev_[1], side_));
    launch(k_pack_positions, ceil_div(n_, kThreads), kThreads, 0, s, stage_.data(), types_.data(),
           n_, box_, pos4_.data(), mixed_ ? q_.data() : nullptr);
    TDMD_LAUNCH_CHECK();
    reorder_by_cell(up_ev_[1]);
  }
  std::copy(masses, masses + n_types, h_masses);
  TDMD_CU(cudaMemcpyAsync(masses_.data(), h_masses, sizeof(double) * n_types,
                          cudaMemcpyHostToDevice, s));
  // Kick factor per unit dt, 1/(m mvv2e) -- the reference divides per atom
  // (device_velocity_verlet.cu:100-102); one host division per type here.
  for (int t = 0; t < n_types; ++t) h_inv[t] = masses[t] > 0.0 ? 1.0 / (masses[t] * kMvv2e) : 0.0;
  inv_mm_.reserve(static_cast<size_t>(n_types));
  TDMD_CU(cudaMemcpyAsync(inv_mm_.data(), h_inv, sizeof(double) * n_types,
                          cudaMemcpyHostToDevice, s));
  // Control block: dt, unit scale, fresh chain.
  *h_ctl = SchedCtl{};
  h_ctl->dt = cfg_.dt;
  h_ctl->scale = 1.0;
  if (nvt_)
    nhc_init(h_ctl->eta, h_ctl->eta_v, h_ctl->eta_m, cfg_.nhc_length, cfg_.t_target,
             cfg_.t_period, 3 * n_ - 3);
  TDMD_CU(cudaMemcpyAsync(ctl_.data(), h_ctl, sizeof(SchedCtl), cudaMemcpyHostToDevice, s));
  // Scratch sized for the chosen lanes-per-atom.
  // Energy partials sized for the widest lanes-per-atom the autotuner tries.
  const int nblk_force = force_blocks(n_ > 0 ? n_ : 1, 32);
  ev_part_.reserve(static_cast<size_t>(2 * nblk_force) * kEvStride);
  // (KE, v2max) per block plus the 2-double result of k_ke_vmax_finish.
  ke_part_.reserve(static_cast<size_t>(2 * ceil_div(n_ > 0 ? n_ : 1, kThreads) + 8));
  if (kind_ == TDMD_POT_EAM) {
    if (mixed_)
      fp32_.reserve(n), g_.reserve(n);
    else
      fp64_.reserve(n), g64_.reserve(n);
  }
  if (cfg_.energy_every > 0) {
    log_cap_ = cfg_.energy_log_capacity > 0 ? cfg_.energy_log_capacity : 1024;
    log_.reserve(static_cast<size_t>(log_cap_) * 9);
  }
  // Host types are checked (the kernels index masses[type] directly) while
  // the copies and the reordering run; nothing that indexes by type has
  // been enqueued yet.
  bool types_ok = true, types_in_eam = true;
  for (size_t i = 0; i < n; ++i) types_ok &= types[i] >= 1 && types[i] < n_types;
  if (kind_ == TDMD_POT_EAM)
    for (size_t i = 0; i < n; ++i) types_in_eam &= types[i] <= eam_->ntypes;
  TDMD_CU(cudaStreamSynchronize(s));
  max_cell_ = (n_ > 0 && h_cellmax_) ? *h_cellmax_ : 0;
  TDMD_REQUIRE(types_ok, "atom type out of range of masses");
  TDMD_REQUIRE(types_in_eam, "atom type beyond the EAM element count");
  uploaded_ = true;
  initialized_ = false;
  step_ = 0;
  since_rebuild_ = 0;
}

// Permutes the uploaded state into the cell order of its positions:
// order_ = the cell list's atoms (index order within each cell).  side_done
// (nullable): the event after which the rest of the state is on the device.
void Scheduler::reorder_by_cell(cudaEvent_t side_done) {
  cudaStream_t s = stream_;
  const size_t n = static_cast<size_t>(n_);
  build_cell_list(cl_, pos4_.data(), PosLayout::D4, n_, box_, s);
  cellmax_.reserve(1);
  if (!h_cellmax_) TDMD_CU(cudaMallocHost(reinterpret_cast<void**>(&h_cellmax_), sizeof(int)));
  *h_cellmax_ = 0;
  cell_count_max(cl_, cellmax_.data(), s);
  TDMD_CU(cudaMemcpyAsync(h_cellmax_, cellmax_.data(), sizeof(int), cudaMemcpyDeviceToHost, s));
  order_.reserve(n);
  TDMD_CU(cudaMemcpyAsync(order_.data(), cl_.cell_atoms.data(), n * sizeof(int),
                          cudaMemcpyDeviceToDevice, s));
  // Gather into the second set of buffers, then swap them in.
  if (side_done) TDMD_CU(cudaStreamWaitEvent(s, side_done, 0));
  pos4_alt_.reserve(n);
  vel_alt_.reserve(3 * n);
  types_alt_.reserve(n);
  ids_alt_.reserve(n);
  const int nb = ceil_div(n_, kThreads);
  if (mixed_) {
    q_alt_.reserve(n);
    f32_alt_.reserve(3 * n);
    launch(k_gather_state<F3>, nb, kThreads, 0, s, order_.data(), n_, pos4_.data(),
           pos4_alt_.data(), reinterpret_cast<const D3*>(vel_.data()),
           reinterpret_cast<D3*>(vel_alt_.data()), types_.data(), types_alt_.data(), ids_.data(),
           ids_alt_.data(), q_.data(), q_alt_.data(), reinterpret_cast<const F3*>(f32_.data()),
           reinterpret_cast<F3*>(f32_alt_.data()));
    std::swap(q_, q_alt_);
    std::swap(f32_, f32_alt_);
  } else {
    f64_alt_.reserve(3 * n);
    launch(k_gather_state<D3>, nb, kThreads, 0, s, order_.data(), n_, pos4_.data(),
           pos4_alt_.data(), reinterpret_cast<const D3*>(vel_.data()),
           reinterpret_cast<D3*>(vel_alt_.data()), types_.data(), types_alt_.data(), ids_.data(),
           ids_alt_.data(), nullptr, nullptr, reinterpret_cast<const D3*>(f64_.data()),
           reinterpret_cast<D3*>(f64_alt_.data()));
    std::swap(f64_, f64_alt_);
  }
  TDMD_LAUNCH_CHECK();
  std::swap(pos4_, pos4_alt_);
  std::swap(vel_, vel_alt_);
  std::swap(types_, types_alt_);
  std::swap(ids_, ids_alt_);
  // The cells of the reordered atoms: same counts and starts, and each
  // cell's members are consecutive indices in ID order -- the next
  // build_cells only has to write the identity.
  cells_from_upload_ = true;
}

void Scheduler::neighbor_list(int* counts, int* neighbors, long long capacity,
                              long long* total) const {
  TDMD_REQUIRE(initialized_, "no neighbor list yet: call run_until first");
  TDMD_REQUIRE(counts, "counts is null");
  const size_t n = static_cast<size_t>(n_);
  std::vector<int> cnt(n), ord(n), rows(n * static_cast<size_t>(cap_));
  TDMD_CU(cudaMemcpyAsync(cnt.data(), cnt_.data(), n * sizeof(int), cudaMemcpyDeviceToHost,
                          stream_));
  TDMD_CU(cudaMemcpyAsync(ord.data(), order_.data(), n * sizeof(int), cudaMemcpyDeviceToHost,
                          stream_));
  if (neighbors && !rows.empty())
    TDMD_CU(cudaMemcpyAsync(rows.data(), nbr_.data(), rows.size() * sizeof(int),
                            cudaMemcpyDeviceToHost, stream_));
  TDMD_CU(cudaStreamSynchronize(stream_));
  // internal atom k is the caller's atom ord[k]; its row holds internal indices
  std::vector<long long> off(n + 1, 0);
  for (size_t k = 0; k < n; ++k) {
    TDMD_REQUIRE(cnt[k] <= cap_, "neighbor rows overflowed their capacity");
    counts[ord[k]] = cnt[k];
  }
  for (size_t i = 0; i < n; ++i) off[i + 1] = off[i] + counts[i];
  if (total) *total = off[n];
  if (!neighbors) return;
  TDMD_REQUIRE(capacity >= off[n], "neighbor capacity too small");
  for (size_t k = 0; k < n; ++k) {
    const int* row = rows.data() + k * static_cast<size_t>(cap_);
    int* out = neighbors + off[static_cast<size_t>(ord[k])];
    for (int t = 0; t < cnt[k]; ++t) out[t] = ord[static_cast<size_t>(row[t])];
  }
}

void Scheduler::download(double* x, double* v, void* f, int* types, int* ids, int natoms) const {
  TDMD_REQUIRE(uploaded_, "download before upload");
  TDMD_REQUIRE(natoms >= 0 && natoms <= n_, "natoms out of range");
  const size_t n = static_cast<size_t>(natoms);
  if (n == 0) return;
  cudaStream_t s = stream_;
  // Every array goes back to the caller's order through the staging
  // buffer (stream order serializes its reuse), then the first natoms.
  const int nb = ceil_div(n_, kThreads);
  const int* ord = order_.data();
  if (x) {
    launch(k_scatter_positions, nb, kThreads, 0, s, pos4_.data(), ord, n_, stage_.data());
    TDMD_LAUNCH_CHECK();
    TDMD_CU(cudaMemcpyAsync(x, stage_.data(), 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  auto unpermute = [&](const auto* arr, void* out) {
    using T = std::remove_const_t<std::remove_pointer_t<decltype(arr)>>;
    T* tmp = reinterpret_cast<T*>(stage_.data());
    launch(k_scatter<T>, nb, kThreads, 0, s, arr, ord, n_, tmp);
    TDMD_LAUNCH_CHECK();
    TDMD_CU(cudaMemcpyAsync(out, tmp, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  };
  if (v) unpermute(reinterpret_cast<const D3*>(vel_.data()), v);
  if (f) {
    if (mixed_)
      unpermute(reinterpret_cast<const F3*>(f32_.data()), f);
    else
      unpermute(reinterpret_cast<const D3*>(f64_.data()), f);
  }
  if (types) unpermute(static_cast<const int*>(types_.data()), types);
  if (ids) unpermute(static_cast<const int*>(ids_.data()), ids);
  TDMD_CU(cudaStreamSynchronize(s));
}

// ----- neighbor list ------------------------------------------------------
int Scheduler::build_cells() {
  if (cells_from_upload_) {
    cells_from_upload_ = false;
    launch(k_iota, ceil_div(n_, kThreads), kThreads, 0, stream_, cl_.cell_atoms.data(), n_);
    TDMD_LAUNCH_CHECK();
    return 1;
  }
  build_cell_list(cl_, pos4_.data(), PosLayout::D4, n_, box_, stream_, order_.data());
  return cell_list_kernels();
}

int Scheduler::size_neighbor_list() {
  cudaStream_t s = stream_;
  const int kernels = build_cells();
  cnt_.reserve(static_cast<size_t>(n_));
  const double rl = cutoff_ + cfg_.r_skin;
  TDMD_CU(cudaMemsetAsync(ctl_status(), 0, sizeof(int) * 4, s));
  build_neighbor_rows(cl_, pos4_.data(), PosLayout::D4, n_, box_, rl * rl, nullptr, nullptr, 0,
                      cnt_.data(), ctl_status(), s, max_cell_);
  int st[4];
  TDMD_CU(cudaMemcpyAsync(st, ctl_status(), sizeof(st), cudaMemcpyDeviceToHost, s));
  TDMD_CU(cudaStreamSynchronize(s));
  grow_capacity(st[1]);
  return kernels;
}

void Scheduler::grow_capacity(int max_count) {
  // 25% + 16 slots of headroom, rounded to 8 ints (32 B rows).
  long long want = static_cast<long long>(max_count) + max_count / 4 + 16;
  want = (want + 7) / 8 * 8;
  TDMD_REQUIRE(want * std::max(n_, 1) < (1ll << 40), "neighbor list too large");
  if (want > cap_) {
    cap_ = static_cast<int>(want);
    nbr_.reserve(static_cast<size_t>(cap_) * static_cast<size_t>(std::max(n_, 1)));
    clear_graphs();
  }
}

void Scheduler::enqueue_rebuild() {
  cudaStream_t s = stream_;
  prof_begin(kProfRebuild);
  const int cell_kernels = build_cells();
  const double rl = cutoff_ + cfg_.r_skin;
  build_neighbor_rows(cl_, pos4_.data(), PosLayout::D4, n_, box_, rl * rl, nbr_.data(), nullptr,
                      cap_, cnt_.data(), ctl_status(), s, max_cell_);
  prof_end(kProfRebuild);
  launches_ += cell_kernels + 1;  // cell list + row build
  ++rebuilds_;
}

// ----- forces ---------------------------------------------------------------
void Scheduler::enqueue_force(bool ev, bool kd, int parts) {
  TDMD_REQUIRE(!kd || can_fuse_kick(), "fused kick-drift needs the EAM NVE path");
  cudaStream_t s = stream_;
  const NbrView nl{nbr_.data(), nullptr, cnt_.data(), cap_};
  const int nblk = force_blocks(n_, lpa_);       // pair-force pass records
  const int nblk_d = force_blocks(n_, lpa_d_);   // EAM density pass records
  const Tune td{lpa_d_, nu_d_}, tf{lpa_, nu_};
  double* part = ev ? ev_part_.data() : nullptr;
  if (kind_ == TDMD_POT_MORSE) {
    prof_begin(kProfForce);
    if (mixed_) {
      const GeoQ g = make_geoq(q_.data(), box_);
      launch_morse(g, nl, n_, m32_, f32_.data(), ev, part, tf, s);
    } else {
      GeoD4 g{pos4_.data(), {box_.L[0], box_.L[1], box_.L[2]},
              {box_.halfL[0], box_.halfL[1], box_.halfL[2]},
              {box_.periodic[0], box_.periodic[1], box_.periodic[2]}};
      launch_morse(g, nl, n_, m64_, f64_.data(), ev, part, tf, s);
    }
    prof_end(kProfForce);
    launches_ += 1;
  } else {
    const int* types = eam_->ntypes > 1 ? types_.data() : nullptr;
    double* part2 = ev ? part + static_cast<long long>(nblk_d) * kEvStride : nullptr;
    if (mixed_) {
      // Density reads the position records and writes {q, F'} gather
      // records; the force pass gathers those.
      const GeoQ g = make_geoq(q_.data(), box_);
      const GeoQ gg = make_geoq(g_.data(), box_);
      if (parts & kPassDensity) {
        prof_begin(kProfDensity);
        launch_eam_density<GeoQ, float>(g, nl, n_, eam_->d32, types, fp32_.data(), nullptr,
                                        nullptr, g_.data(), ev, part, td, s);
        prof_end(kProfDensity);
      }
      const KickDrift kdr{pos4_.data(), q_.data(), vel_.data(), types_.data(), inv_mm_.data(),
                          cfg_.dt,
                          reinterpret_cast<long long*>(reinterpret_cast<char*>(ctl_.data()) +
                                                       offsetof(SchedCtl, step)),
                          box_, nullptr, nullptr};
      if (parts & kPassForce) {
        prof_begin(kProfForce);
        launch_eam_force<GeoQ, true, float, float>(gg, nl, n_, eam_->d32, types, fp32_.data(),
                                                   f32_.data(), ev, part2, tf, s,
                                                   kd ? &kdr : nullptr);
        prof_end(kProfForce);
      }
    } else {
      // Density reads the position records and writes {x, y, z, F'} gather
      // records; the force pass gathers those.
      GeoD4 g{pos4_.data(), {box_.L[0], box_.L[1], box_.L[2]},
              {box_.halfL[0], box_.halfL[1], box_.halfL[2]},
              {box_.periodic[0], box_.periodic[1], box_.periodic[2]}};
      GeoD4F gg{g64_.data(), {box_.L[0], box_.L[1], box_.L[2]},
                {box_.halfL[0], box_.halfL[1], box_.halfL[2]},
                {box_.periodic[0], box_.periodic[1], box_.periodic[2]}};
      if (parts & kPassDensity) {
        prof_begin(kProfDensity);
        launch_eam_density<GeoD4, double>(g, nl, n_, eam_->d64, types, fp64_.data(), nullptr,
                                          nullptr, nullptr, ev, part, td, s, nullptr,
                                          g64_.data());
        prof_end(kProfDensity);
      }
      const KickDrift kdr{pos4_.data(), nullptr, vel_.data(), types_.data(), inv_mm_.data(),
                          cfg_.dt,
                          reinterpret_cast<long long*>(reinterpret_cast<char*>(ctl_.data()) +
                                                       offsetof(SchedCtl, step)),
                          box_, nullptr, nullptr};
      if (parts & kPassForce) {
        prof_begin(kProfForce);
        launch_eam_force<GeoD4F, true, double, double>(gg, nl, n_, eam_->d64, types,
                                                       fp64_.data(), f64_.data(), ev, part2, tf,
                                                       s, kd ? &kdr : nullptr);
        prof_end(kProfForce);
      }
    }
    launches_ += ((parts & kPassDensity) ? 1 : 0) + ((parts & kPassForce) ? 1 : 0);
  }
  if (ev) {
    TDMD_REQUIRE(parts == kPassBoth, "energy/virial needs both passes");
    const int nrec = kind_ == TDMD_POT_EAM ? nblk_d + nblk : nblk;
    TDMD_CU(cudaMemsetAsync(ctl_ev(), 0, sizeof(double) * 7, s));
    launch(k_reduce_partials, 1, 256, 0, s, ev_part_.data(), nrec, ctl_ev(), ctl_ev() + 1);
    TDMD_LAUNCH_CHECK();
    launches_ += 1;
  }
}

// ----- integration ----------------------------------------------------------
template <class F>
void Scheduler::enqueue_kick_drift_t(F* f, bool full, bool scale) {
  cudaStream_t s = stream_;
  const int nb = ceil_div(n_, kThreads);
  int4* q = mixed_ ? q_.data() : nullptr;
  const int ctl_dt = thermo_ ? 1 : 0;
  if (scale)
    launch(k_kick_drift<F, false, true>, nb, kThreads, 0, s, pos4_.data(), q, vel_.data(), f,
           types_.data(), inv_mm_.data(), n_, cfg_.dt, ctl_.data(), ctl_dt, box_);
  else if (full)
    launch(k_kick_drift<F, true, false>, nb, kThreads, 0, s, pos4_.data(), q, vel_.data(), f,
           types_.data(), inv_mm_.data(), n_, cfg_.dt, ctl_.data(), ctl_dt, box_);
  else
    launch(k_kick_drift<F, false, false>, nb, kThreads, 0, s, pos4_.data(), q, vel_.data(), f,
           types_.data(), inv_mm_.data(), n_, cfg_.dt, ctl_.data(), ctl_dt, box_);
  TDMD_LAUNCH_CHECK();
  launches_ += 1;
}

void Scheduler::enqueue_kick_drift(bool full, bool scale) {
  prof_begin(kProfKickDrift);
  if (mixed_)
    enqueue_kick_drift_t(f32_.data(), full, scale);
  else
    enqueue_kick_drift_t(f64_.data(), full, scale);
  prof_end(kProfKickDrift);
}

template <class F>
void Scheduler::enqueue_half_kick_t(F* f, bool ke) {
  cudaStream_t s = stream_;
  const int nb = ceil_div(n_, kThreads);
  const int ctl_dt = thermo_ ? 1 : 0;
  if (ke)
    launch(k_half_kick_s<F, true>, nb, kThreads, 0, s, vel_.data(), f, types_.data(),
           masses_.data(), inv_mm_.data(), n_, cfg_.dt, ctl_.data(), ctl_dt, ke_part_.data());
  else
    launch(k_half_kick_s<F, false>, nb, kThreads, 0, s, vel_.data(), f, types_.data(),
           masses_.data(), inv_mm_.data(), n_, cfg_.dt, ctl_.data(), ctl_dt, nullptr);
  TDMD_LAUNCH_CHECK();
  launches_ += 1;
}

void Scheduler::enqueue_half_kick(bool ke) {
  prof_begin(kProfOther);
  if (mixed_)
    enqueue_half_kick_t(f32_.data(), ke);
  else
    enqueue_half_kick_t(f64_.data(), ke);
  prof_end(kProfOther);
}

CtlParams Scheduler::ctl_params() const {
  CtlParams p{};
  p.M = nvt_ ? cfg_.nhc_length : 0;
  p.n_dof = 3 * n_ - 3;
  p.t_target = cfg_.t_target;
  p.t_period = cfg_.t_period;
  p.dt_nhc = cfg_.dt;
  p.adaptive = cfg_.adaptive_dt;
  p.c2 = cfg_.c2;
  p.rc = cutoff_;
  p.dt_min = cfg_.dt_min;
  p.dt_max = cfg_.dt_max;
  p.nvt = nvt_ ? 1 : 0;
  return p;
}

void Scheduler::enqueue_control(int mode) {
  const CtlParams p = ctl_params();
  const int nb = ceil_div(n_, kThreads);
  launch(k_control, 1, ctl_threads(nb), 0, stream_, ctl_.data(), ke_part_.data(), nb, p, mode,
         log_.data(), log_cap_);
  TDMD_LAUNCH_CHECK();
  launches_ += 1;
}

void Scheduler::enqueue_ke_pre() {
  cudaStream_t s = stream_;
  const int nb = ceil_div(n_, kThreads);
  launch(k_ke_vmax_partials, nb, kThreads, 0, s, vel_.data(), types_.data(), masses_.data(), n_,
         ke_part_.data());
  TDMD_LAUNCH_CHECK();
  launches_ += 1;
}

void Scheduler::enqueue_log_nve() {
  cudaStream_t s = stream_;
  const int nb = ceil_div(n_, kThreads);
  if (mixed_)
    launch(k_ke_integer<float>, nb, kThreads, 0, s, vel_.data(), f32_.data(), types_.data(),
           masses_.data(), inv_mm_.data(), n_, cfg_.dt, ke_part_.data());
  else
    launch(k_ke_integer<double>, nb, kThreads, 0, s, vel_.data(), f64_.data(), types_.data(),
           masses_.data(), inv_mm_.data(), n_, cfg_.dt, ke_part_.data());
  TDMD_LAUNCH_CHECK();
  launch(k_log_nve, 1, ctl_threads(nb), 0, s, ctl_.data(), ke_part_.data(), nb, log_.data(),
         log_cap_);
  TDMD_LAUNCH_CHECK();
  launches_ += 2;
}

void Scheduler::enqueue_apply_scale() {
  const long long m = 3ll * n_;
  launch(k_apply_scale, ceil_div(m, kThreads), kThreads, 0, stream_, vel_.data(), m, ctl_.data());
  TDMD_LAUNCH_CHECK();
  launches_ += 1;
}

// One step as planned (see plan_steps): the kernels of the step.
void Scheduler::enqueue_step(const StepPlan& st) {
  if (!thermo_) {
    if (!st.kd_fused) enqueue_kick_drift(/*full=*/!st.first, /*scale=*/false);
    if (st.rebuild) enqueue_rebuild();
    enqueue_force(st.ev, st.fuse_next);
    if (st.ev) enqueue_log_nve();
  } else {
    if (st.first) {
      enqueue_ke_pre();
      enqueue_control(kCtlPre);
    }
    enqueue_kick_drift(/*full=*/false, /*scale=*/true);
    if (st.rebuild) enqueue_rebuild();
    enqueue_force(st.ev);
    enqueue_half_kick(/*ke=*/true);
    enqueue_control(kCtlPost | (st.last ? 0 : kCtlNext) | (st.ev ? kCtlLog : 0));
  }
}

void Scheduler::enqueue_finalize() {
  if (!thermo_)
    enqueue_half_kick(false);
  else
    enqueue_apply_scale();
}

// ----- graphs ---------------------------------------------------------------
void Scheduler::clear_graphs() {
  for (auto& kv : graphs_) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    for (const ProfEvents& pe : kv.second.prof) prof_retired_.push_back(pe);
  }
  graphs_.clear();
  graph_lru_.clear();
}

void Scheduler::run_segment(const std::vector<StepPlan>& seg, bool finalize, int prologue) {
  std::vector<int> key;
  key.reserve(seg.size() + 2);
  for (const auto& st : seg)
    key.push_back((st.first ? 1 : 0) | (st.rebuild ? 2 : 0) | (st.ev ? 4 : 0) | (st.last ? 8 : 0) |
                  (st.kd_fused ? 16 : 0) | (st.fuse_next ? 32 : 0));
  key.push_back(finalize ? 1 : 0);
  key.push_back(prologue);
  key.push_back(profiling_ ? 1 : 0);
  const long long l0 = launches_;
  if (!cfg_.use_graphs) {
    enqueue_prologue(prologue);
    for (const auto& st : seg) enqueue_step(st);
    if (finalize) enqueue_finalize();
    return;
  }
  auto it = graphs_.find(key);
  if (it == graphs_.end()) {
    if (graphs_.size() >= 16) {  // bounded cache, least recently used out
      auto old = graphs_.find(graph_lru_.back());
      if (old != graphs_.end()) {
        cudaGraphExecDestroy(old->second.exec);
        for (const ProfEvents& pe : old->second.prof) prof_retired_.push_back(pe);
        graphs_.erase(old);
      }
      graph_lru_.pop_back();
    }
    cudaGraph_t g = nullptr;
    GraphEntry ge{};
    // Profiling graphs carry event-record nodes around each phase and plain
    // edges between kernels (no programmatic launch inside them).
    if (profiling_) {
      prof_sink_ = &ge.prof;
      suppress_programmatic_launch(true);
    }
    TDMD_CU(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue_prologue(prologue);
      for (const auto& st : seg) enqueue_step(st);
      if (finalize) enqueue_finalize();
    } catch (...) {
      prof_sink_ = nullptr;
      suppress_programmatic_launch(false);
      cudaStreamEndCapture(stream_, &g);
      if (g) cudaGraphDestroy(g);
      for (const ProfEvents& pe : ge.prof) prof_retired_.push_back(pe);
      throw;
    }
    prof_sink_ = nullptr;
    suppress_programmatic_launch(false);
    TDMD_CU(cudaStreamEndCapture(stream_, &g));
    ge.kernels = launches_ - l0;
    const cudaError_t ie = cudaGraphInstantiate(&ge.exec, g, 0);
    cudaGraphDestroy(g);
    TDMD_CU(ie);
    launches_ = l0;  // capture enqueued nothing
    it = graphs_.emplace(key, ge).first;
    graph_lru_.push_front(key);
  } else {
    graph_lru_.remove(key);
    graph_lru_.push_front(key);
  }
  TDMD_CU(cudaGraphLaunch(it->second.exec, stream_));
  launches_ += it->second.kernels;
  ++graph_launches_;
  for (const ProfEvents& pe : it->second.prof) prof_graph_pending_.push_back(pe);
}

// ----- run_until --------------------------------------------------------------
std::vector<StepPlan> Scheduler::plan_steps(int target, int* since_out) const {
  std::vector<StepPlan> plan;
  int since = since_rebuild_;
  for (int s = step_; s < target; ++s) {
    StepPlan st{};
    st.first = s == step_;
    st.last = s + 1 == target;
    // maybe_rebuild_nlist (fast_pipeline_scheduler.cu:225-232): after the
    // kick-drift, when steps since the last build reach rebuild_every.
    st.rebuild = since >= cfg_.rebuild_every;
    if (st.rebuild) since = 0;
    ++since;
    st.ev = cfg_.energy_every > 0 && ((s + 1) % cfg_.energy_every == 0);
    // Mixed EAM NVE: a force pass that logs no energy and is followed by
    // another step of the window also kicks and drifts for that step.
    st.fuse_next = can_fuse_kick() && !st.ev && !st.last;
    st.kd_fused = !plan.empty() && plan.back().fuse_next;
    plan.push_back(st);
  }
  *since_out = since;
  return plan;
}

void Scheduler::initial_forces(bool defer_check) {
  const bool prof = profiling_;
  profiling_ = false;  // timing covers the steps of run_until windows only
  cudaStream_t s = stream_;
  const double rl2 = (cutoff_ + cfg_.r_skin) * (cutoff_ + cfg_.r_skin);
  // The first upload sizes the rows with a count pass; later uploads reuse
  // the capacity and fill directly, counting a second fill only when a row
  // did not fit.
  int passes = 1, cell_kernels = 0;
  const bool reuse = cap_ > 0;
  if (reuse) {
    cell_kernels = build_cells();
    cnt_.reserve(static_cast<size_t>(n_));
  } else {
    cell_kernels = size_neighbor_list();
    ++passes;
  }
  TDMD_CU(cudaMemsetAsync(ctl_status(), 0, sizeof(int) * 4, s));
  build_neighbor_rows(cl_, pos4_.data(), PosLayout::D4, n_, box_, rl2, nbr_.data(), nullptr,
                      cap_, cnt_.data(), ctl_status(), s, max_cell_);
  if (reuse && defer_check) {
    init_check_pending_ = true;
  } else if (reuse) {
    int st[4];
    TDMD_CU(cudaMemcpyAsync(st, ctl_status(), sizeof(st), cudaMemcpyDeviceToHost, s));
    TDMD_CU(cudaStreamSynchronize(s));
    if (st[0]) {
      grow_capacity(st[1]);
      TDMD_CU(cudaMemsetAsync(ctl_status(), 0, sizeof(int) * 4, s));
      build_neighbor_rows(cl_, pos4_.data(), PosLayout::D4, n_, box_, rl2, nbr_.data(), nullptr,
                          cap_, cnt_.data(), ctl_status(), s, max_cell_);
      ++passes;
    }
  }
  launches_ += cell_kernels + passes;  // cell list + (count pass) + fill pass(es)
  ++rebuilds_;
  since_rebuild_ = 0;
  enqueue_force(false);
  initialized_ = true;
  profiling_ = prof;
}

// State a window may have to rewind to (neighbor capacity overflow):
// positions, their fixed-point records, velocities and the control block.
// The forces are not kept: a retry recomputes them from the restored
// positions.  Sized outside any stream capture (allocation is not capturable).
void Scheduler::reserve_snapshot() {
  const size_t n = static_cast<size_t>(n_);
  snap_pos4_.reserve(n);
  snap_vel_.reserve(3 * n);
  if (mixed_) snap_q_.reserve(n);
}

void Scheduler::enqueue_prologue(int prologue) {
  if (prologue & kPrologueSnapshot) {
    launch(k_window_prologue, ceil_div(n_, kThreads), kThreads, 0, stream_, pos4_.data(),
           snap_pos4_.data(), mixed_ ? q_.data() : nullptr, mixed_ ? snap_q_.data() : nullptr,
           vel_.data(), snap_vel_.data(), n_, ctl_.data(), snap_ctl_.data(),
           (prologue & kPrologueResetStatus) ? 1 : 0);
    TDMD_LAUNCH_CHECK();
    launches_ += 1;
  } else if (prologue & kPrologueResetStatus) {
    TDMD_CU(cudaMemsetAsync(ctl_status(), 0, sizeof(int) * 4, stream_));
  }
}

void Scheduler::restore() {
  cudaStream_t s = stream_;
  const size_t n = static_cast<size_t>(n_);
  TDMD_CU(cudaMemcpyAsync(pos4_.data(), snap_pos4_.data(), n * sizeof(double4),
                          cudaMemcpyDeviceToDevice, s));
  TDMD_CU(cudaMemcpyAsync(vel_.data(), snap_vel_.data(), 3 * n * sizeof(double),
                          cudaMemcpyDeviceToDevice, s));
  if (mixed_)
    TDMD_CU(cudaMemcpyAsync(q_.data(), snap_q_.data(), n * sizeof(int4), cudaMemcpyDeviceToDevice, s));
  TDMD_CU(cudaMemcpyAsync(ctl_.data(), snap_ctl_.data(), sizeof(SchedCtl),
                          cudaMemcpyDeviceToDevice, s));
}

void Scheduler::run_until(int target) {
  TDMD_REQUIRE(uploaded_, "run_until before upload");
  if (n_ == 0) {
    step_ = std::max(step_, target);
    return;
  }
  // With a window to run, the first list's overflow check is left to it:
  // no host round trip between the upload and the window.
  if (!initialized_) initial_forces(/*defer_check=*/step_ < target);
  // lanes_per_atom = 0: measure the candidates once on the first window of
  // a system large enough for the choice to matter.
  if (!tuned_ && cfg_.lanes_per_atom == 0 && n_ >= 2048) autotune(nullptr, nullptr, nullptr);
  if (step_ >= target) {
    TDMD_CU(cudaStreamSynchronize(stream_));
    return;
  }
  const int step0 = step_, since0 = since_rebuild_;
  reserve_snapshot();
  for (int attempt = 0;; ++attempt) {
    TDMD_CU(cudaEventRecord(win_ev_[0], stream_));
    // The snapshot and the flag reset go into the first segment's graph: one
    // submission per window.  A pending first-list overflow flag stays set
    // for this window's check.
    const int prologue = kPrologueSnapshot |
                         ((attempt > 0 || !init_check_pending_) ? kPrologueResetStatus : 0);
    int since_end = 0;
    const std::vector<StepPlan> plan = plan_steps(target, &since_end);
    // Segments start at each rebuild step; at most 64 steps each.
    size_t a = 0;
    while (a < plan.size()) {
      size_t b = a + 1;
      while (b < plan.size() && !plan[b].rebuild && b - a < 64) ++b;
      const std::vector<StepPlan> seg(plan.begin() + static_cast<long>(a),
                                      plan.begin() + static_cast<long>(b));
      run_segment(seg, b == plan.size(), a == 0 ? prologue : 0);
      a = b;
    }
    ticks_ += static_cast<long long>(plan.size());
    TDMD_CU(cudaEventRecord(win_ev_[1], stream_));
    int st[4];
    TDMD_CU(cudaMemcpyAsync(st, ctl_status(), sizeof(st), cudaMemcpyDeviceToHost, stream_));
    TDMD_CU(cudaStreamSynchronize(stream_));
    {
      float ms = 0.f;
      TDMD_CU(cudaEventElapsedTime(&ms, win_ev_[0], win_ev_[1]));
      last_window_ms_ = ms;
    }
    prof_collect();
    init_check_pending_ = false;
    if (!st[0]) {
      step_ = target;
      since_rebuild_ = since_end;
      return;
    }
    // Neighbor capacity exceeded during the window: grow, rewind, redo.
    if (attempt >= 3)
      throw Error{TDMD_ERR_NLIST_OVERFLOW, "neighbor list overflow persisted after retries"};
    ++retries_;
    grow_capacity(st[1]);
    restore();
    step_ = step0;
    since_rebuild_ = since0;
    // The restored positions need a list built into the new capacity, and
    // their forces again (those of the snapshot came from an overflowed
    // list when the overflow was the first list's; otherwise the same bits).
    build_cells();
    build_neighbor_rows(cl_, pos4_.data(), PosLayout::D4, n_, box_,
                        (cutoff_ + cfg_.r_skin) * (cutoff_ + cfg_.r_skin), nbr_.data(), nullptr,
                        cap_, cnt_.data(), nullptr, stream_, max_cell_);
    enqueue_force(false);
  }
}

void Scheduler::energies(double* pe, double* ke, double* virial6) {
  TDMD_REQUIRE(uploaded_, "energies before upload");
  if (n_ == 0) {
    if (pe) *pe = 0.0;
    if (ke) *ke = 0.0;
    if (virial6)
      for (int k = 0; k < 6; ++k) virial6[k] = 0.0;
    return;
  }
  if (!initialized_) initial_forces();
  const bool prof = profiling_;
  profiling_ = false;
  enqueue_force(true);
  profiling_ = prof;
  enqueue_ke_pre();
  launch(k_ke_vmax_finish, 1, 256, 0, stream_, ke_part_.data(), ceil_div(n_, kThreads),
         ke_part_.data() + 2ll * ceil_div(n_, kThreads));
  TDMD_LAUNCH_CHECK();
  double ev[7], k2[2];
  TDMD_CU(cudaMemcpyAsync(ev, ctl_ev(), sizeof(ev), cudaMemcpyDeviceToHost, stream_));
  TDMD_CU(cudaMemcpyAsync(k2, ke_part_.data() + 2ll * ceil_div(n_, kThreads), sizeof(k2),
                          cudaMemcpyDeviceToHost, stream_));
  TDMD_CU(cudaStreamSynchronize(stream_));
  if (pe) *pe = ev[0];
  if (ke) *ke = k2[0];
  if (virial6)
    for (int k = 0; k < 6; ++k) virial6[k] = ev[1 + k];
}

void Scheduler::energy_log(double* rec, int cap, int* count) const {
  TDMD_REQUIRE(uploaded_, "energy_log before upload");
  SchedCtl h{};
  TDMD_CU(cudaMemcpy(&h, ctl_.data(), sizeof(h), cudaMemcpyDeviceToHost));
  *count = h.log_count;
  if (!rec || cap <= 0 || log_cap_ <= 0 || h.log_count == 0) return;
  // Oldest first.
  const int have = std::min(h.log_count, log_cap_);
  std::vector<double> all(static_cast<size_t>(log_cap_) * 9);
  TDMD_CU(cudaMemcpy(all.data(), log_.data(), all.size() * sizeof(double), cudaMemcpyDeviceToHost));
  const int start = h.log_count - have;
  for (int k = 0; k < std::min(have, cap); ++k) {
    const int slot = (start + k) % log_cap_;
    for (int c = 0; c < 9; ++c) rec[9ll * k + c] = all[9ull * slot + c];
  }
}

void Scheduler::thermostat_state(double* dt, double* eta, double* eta_v) const {
  SchedCtl h{};
  TDMD_CU(cudaMemcpy(&h, ctl_.data(), sizeof(h), cudaMemcpyDeviceToHost));
  if (dt) *dt = h.dt;
  for (int k = 0; k < cfg_.nhc_length && k < kMaxChain; ++k) {
    if (eta) eta[k] = h.eta[k];
    if (eta_v) eta_v[k] = h.eta_v[k];
  }
}

// ----- per-kernel timing -------------------------------------------------------
// ----- autotuner ---------------------------------------------------------------
// Sweeps the launch shape of each gather pass on its own -- lanes per atom
// {1, ..., 32} x neighbors per lane sweep {2, 4} (only cfg.nbr_batch when
// that is fixed): the EAM density pass first, then the pair-force pass on
// that density.  lanes2 / batch2 = {density, force} (density 0 for Morse);
// ms24[12 * pass + 6 * (batch == 4) + k] = time of lanes 2^k, -1 where not
// measured.
void Scheduler::autotune(int* lanes2, int* batch2, double* ms24) {
  TDMD_REQUIRE(uploaded_, "autotune before upload");
  if (n_ == 0) return;
  if (!initialized_) initial_forces();
  const bool prof = profiling_;
  profiling_ = false;
  const long long l0 = launches_;
  cudaEvent_t e0, e1;
  TDMD_CU(cudaEventCreate(&e0));
  TDMD_CU(cudaEventCreate(&e1));
  const bool eam = kind_ == TDMD_POT_EAM;
  const int cand[6] = {1, 2, 4, 8, 16, 32};
  const int batches[2] = {2, 4};
  if (ms24)
    for (int k = 0; k < 24; ++k) ms24[k] = -1.0;
  auto sweep = [&](int pass) {
    int& lanes = pass == 0 ? lpa_d_ : lpa_;
    int& batch = pass == 0 ? nu_d_ : nu_;
    const int parts = pass == 0 ? kPassDensity : kPassForce;
    double best_ms = 1e300;
    int best_l = lanes, best_u = batch;
    for (int b = 0; b < 2; ++b) {
      if (cfg_.nbr_batch > 0 && batches[b] != cfg_.nbr_batch) continue;
      for (int k = 0; k < 6; ++k) {
        lanes = cand[k];
        batch = batches[b];
        enqueue_force(false, false, parts);  // warm
        double m = 1e300;
        for (int rep = 0; rep < 3; ++rep) {
          TDMD_CU(cudaEventRecord(e0, stream_));
          enqueue_force(false, false, parts);
          TDMD_CU(cudaEventRecord(e1, stream_));
          TDMD_CU(cudaEventSynchronize(e1));
          float ms = 0.f;
          TDMD_CU(cudaEventElapsedTime(&ms, e0, e1));
          m = std::min(m, static_cast<double>(ms));
        }
        if (ms24) ms24[12 * pass + 6 * b + k] = m;
        if (m < best_ms) {
          best_ms = m;
          best_l = cand[k];
          best_u = batches[b];
        }
      }
    }
    lanes = best_l;
    batch = best_u;
  };
  if (eam) {
    sweep(0);
    enqueue_force(false, false, kPassDensity);  // the chosen density pass's output
  }
  sweep(1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // The forces of the current state, summed in the chosen shapes' order.
  enqueue_force(false);
  TDMD_CU(cudaStreamSynchronize(stream_));
  launches_ = l0;  // tuning passes are not part of the run's kernel count
  clear_graphs();
  tuned_ = true;
  profiling_ = prof;
  if (lanes2) {
    lanes2[0] = eam ? lpa_d_ : 0;
    lanes2[1] = lpa_;
  }
  if (batch2) {
    batch2[0] = eam ? nu_d_ : 0;
    batch2[1] = nu_;
  }
}

void Scheduler::set_profiling(bool on) {
  profiling_ = on;
  for (int k = 0; k < kProfCount; ++k) {
    prof_ms_[k] = 0.0;
    prof_n_[k] = 0;
  }
}

void Scheduler::prof_begin(int /*cat*/) {
  if (!profiling_) return;
  if (prof_sink_) {  // capturing: an event-record node the graph owns
    TDMD_CU(cudaEventCreate(&prof_open_));
    TDMD_CU(cudaEventRecordWithFlags(prof_open_, stream_, cudaEventRecordExternal));
    return;
  }
  if (prof_pool_.empty()) {
    cudaEvent_t e;
    TDMD_CU(cudaEventCreate(&e));
    prof_pool_.push_back(e);
  }
  prof_open_ = prof_pool_.back();
  prof_pool_.pop_back();
  TDMD_CU(cudaEventRecord(prof_open_, stream_));
}

void Scheduler::prof_end(int cat) {
  if (!profiling_ || !prof_open_) return;
  if (prof_sink_) {
    cudaEvent_t e;
    TDMD_CU(cudaEventCreate(&e));
    TDMD_CU(cudaEventRecordWithFlags(e, stream_, cudaEventRecordExternal));
    prof_sink_->push_back({cat, prof_open_, e});
    prof_open_ = nullptr;
    return;
  }
  cudaEvent_t e;
  if (prof_pool_.empty()) {
    TDMD_CU(cudaEventCreate(&e));
  } else {
    e = prof_pool_.back();
    prof_pool_.pop_back();
  }
  TDMD_CU(cudaEventRecord(e, stream_));
  prof_pending_.push_back({cat, {prof_open_, e}});
  prof_open_ = nullptr;
}

void Scheduler::prof_collect() {
  for (auto& pe : prof_pending_) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, pe.second.first, pe.second.second) == cudaSuccess) {
      prof_ms_[pe.first] += ms;
      prof_n_[pe.first] += 1;
    }
    prof_pool_.push_back(pe.second.first);
    prof_pool_.push_back(pe.second.second);
  }
  prof_pending_.clear();
  for (const ProfEvents& pe : prof_graph_pending_) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, pe.a, pe.b) == cudaSuccess) {
      prof_ms_[pe.cat] += ms;
      prof_n_[pe.cat] += 1;
    }
  }
  prof_graph_pending_.clear();
  for (const ProfEvents& pe : prof_retired_) {
    cudaEventDestroy(pe.a);
    cudaEventDestroy(pe.b);
  }
  prof_retired_.clear();
}

void Scheduler::kernel_times(double* avg_ms, long long* counts, int ncat) const {
  for (int k = 0; k < ncat && k < kProfCount; ++k) {
    if (avg_ms) avg_ms[k] = prof_n_[k] ? prof_ms_[k] / prof_n_[k] : 0.0;
    if (counts) counts[k] = prof_n_[k];
  }
}

void Scheduler::stats(tdmd_fast_pipeline_stats* o) const {
  o->ticks = ticks_;
  o->kernel_launches = launches_;
  o->rebuilds = rebuilds_;
  o->graph_launches = graph_launches_;
  o->nlist_retries = retries_;
  o->nlist_capacity = cap_;
  o->lanes_per_atom = lpa_;
  o->nbr_batch = nu_;
  o->density_lanes_per_atom = kind_ == TDMD_POT_EAM ? lpa_d_ : 0;
  o->density_nbr_batch = kind_ == TDMD_POT_EAM ? nu_d_ : 0;
}

}  // namespace tdmd_b200

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace tdmd_b200;

struct tdmd_sched {
  std::unique_ptr<Scheduler> s;
};

extern "C" {

int32_t tdmd_sched_create_morse(const tdmd_box* box, int32_t natoms,
                                const tdmd_morse_params* params,
                                const tdmd_fast_pipeline_config* cfg, tdmd_sched** out) {
  return guarded([&] {
    TDMD_REQUIRE(box && params && cfg && out, "null argument");
    TDMD_REQUIRE(params->rc > 0.0, "Morse cutoff must be positive");
    auto h = std::make_unique<tdmd_sched>();
    h->s = std::make_unique<Scheduler>(*box, natoms, *cfg);
    h->s->set_morse(*params);
    *out = h.release();
  });
}

int32_t tdmd_sched_create_eam(const tdmd_box* box, int32_t natoms, const tdmd_eam* eam,
                              const tdmd_fast_pipeline_config* cfg, tdmd_sched** out) {
  return guarded([&] {
    TDMD_REQUIRE(box && eam && cfg && out, "null argument");
    auto h = std::make_unique<tdmd_sched>();
    h->s = std::make_unique<Scheduler>(*box, natoms, *cfg);
    h->s->set_eam(*eam);
    *out = h.release();
  });
}

int32_t tdmd_sched_destroy(tdmd_sched* s) {
  delete s;
  return TDMD_OK;
}

int32_t tdmd_sched_upload(tdmd_sched* s, const double* positions, const double* velocities,
                          const void* forces, const int32_t* types, const int32_t* ids,
                          const double* masses, int32_t n_types) {
  return guarded([&] {
    TDMD_REQUIRE(s, "null handle");
    s->s->upload(positions, velocities, forces, types, ids, masses, n_types);
  });
}

int32_t tdmd_sched_run_until(tdmd_sched* s, int32_t target_step) {
  return guarded([&] {
    TDMD_REQUIRE(s, "null handle");
    s->s->run_until(target_step);
  });
}

int32_t tdmd_sched_download(const tdmd_sched* s, double* positions, double* velocities,
                            void* forces, int32_t* types, int32_t* ids, int32_t natoms) {
  return guarded([&] {
    TDMD_REQUIRE(s, "null handle");
    s->s->download(positions, velocities, forces, types, ids, natoms);
  });
}

int32_t tdmd_sched_stats(const tdmd_sched* s, tdmd_fast_pipeline_stats* out) {
  return guarded([&] {
    TDMD_REQUIRE(s && out, "null argument");
    s->s->stats(out);
  });
}

int32_t tdmd_sched_current_step(const tdmd_sched* s, int32_t* step) {
  return guarded([&] {
    TDMD_REQUIRE(s && step, "null argument");
    *step = s->s->current_step();
  });
}

int32_t tdmd_sched_potential_kind(const tdmd_sched* s, int32_t* kind) {
  return guarded([&] {
    TDMD_REQUIRE(s && kind, "null argument");
    *kind = s->s->potential_kind();
  });
}

int32_t tdmd_sched_interaction_cutoff(const tdmd_sched* s, double* cutoff) {
  return guarded([&] {
    TDMD_REQUIRE(s && cutoff, "null argument");
    *cutoff = s->s->interaction_cutoff();
  });
}

int32_t tdmd_sched_energies(tdmd_sched* s, double* pe, double* ke, double* virial6) {
  return guarded([&] {
    TDMD_REQUIRE(s, "null handle");
    s->s->energies(pe, ke, virial6);
  });
}

int32_t tdmd_sched_energy_log(const tdmd_sched* s, double* records, int32_t cap, int32_t* count) {
  return guarded([&] {
    TDMD_REQUIRE(s && count, "null argument");
    s->s->energy_log(records, cap, count);
  });
}

int32_t tdmd_sched_thermostat_state(const tdmd_sched* s, double* dt, double* eta,
                                    double* eta_v) {
  return guarded([&] {
    TDMD_REQUIRE(s, "null handle");
    s->s->thermostat_state(dt, eta, eta_v);
  });
}

int32_t tdmd_sched_atom_order(const tdmd_sched* s, const int32_t** d_order) {
  return guarded([&] {
    TDMD_REQUIRE(s && d_order, "null argument");
    *d_order = s->s->atom_order();
  });
}

int32_t tdmd_sched_neighbor_list(const tdmd_sched* s, int32_t* counts, int32_t* neighbors,
                                 int64_t capacity, int64_t* total) {
  return guarded([&] {
    TDMD_REQUIRE(s, "null handle");
    long long t = 0;
    s->s->neighbor_list(counts, neighbors, capacity, &t);
    if (total) *total = t;
  });
}

int32_t tdmd_sched_device_state(tdmd_sched* s, void** d_pos4, double** d_vel, void** d_forces) {
  return guarded([&] {
    TDMD_REQUIRE(s, "null handle");
    s->s->device_state(d_pos4, d_vel, d_forces);
  });
}

int32_t tdmd_sched_set_profiling(tdmd_sched* s, int32_t on) {
  return guarded([&] {
    TDMD_REQUIRE(s, "null handle");
    s->s->set_profiling(on != 0);
  });
}

int32_t tdmd_sched_kernel_times(const tdmd_sched* s, double* avg_ms, int64_t* counts,
                                int32_t ncat) {
  return guarded([&] {
    TDMD_REQUIRE(s, "null handle");
    std::vector<long long> c(static_cast<size_t>(ncat > 0 ? ncat : 0));
    s->s->kernel_times(avg_ms, c.data(), ncat);
    if (counts)
      for (int k = 0; k < ncat; ++k) counts[k] = c[static_cast<size_t>(k)];
  });
}

int32_t tdmd_sched_last_window_ms(const tdmd_sched* s, double* ms) {
  return guarded([&] {
    TDMD_REQUIRE(s && ms, "null argument");
    *ms = s->s->last_window_ms();
  });
}

int32_t tdmd_sched_stream(const tdmd_sched* s, void** stream) {
  return guarded([&] {
    TDMD_REQUIRE(s && stream, "null argument");
    *stream = reinterpret_cast<void*>(s->s->stream());
  });
}

}  // extern "C"

extern "C" int32_t tdmd_sched_autotune(tdmd_sched* s, int32_t* lanes2, int32_t* batch2,
                                       double* ms24) {
  return guarded([&] {
    TDMD_REQUIRE(s, "null handle");
    int l[2] = {0, 0}, u[2] = {0, 0};
    s->s->autotune(l, u, ms24);
    for (int k = 0; k < 2; ++k) {
      if (lanes2) lanes2[k] = l[k];
      if (batch2) batch2[k] = u[k];
    }
  });
}
