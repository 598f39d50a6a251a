// batch.cu -- many independent Morse systems ("replicas") of uneven sizes
// advanced together, NVE velocity-Verlet, behind tdmd_batch_* (C ABI).
//
// No reference counterpart: tdmd_Claude runs one system per
// FastPipelineScheduler (src/scheduler/fast_pipeline_scheduler.cu:15-233)
// and only plans multi-step fusion.  Each replica here follows that
// scheduler's semantics exactly -- same step order, same rebuild rule, same
// per-atom arithmetic -- so a replica's trajectory equals the one a single
// scheduler with the same lanes-per-atom produces, bit for bit.
//
// B200 layout: all replicas' atoms are concatenated (replica r owns atoms
// [atom0, atom0 + natoms)), all cells too, and every phase is ONE launch
// over the whole batch: binning, scan, scatter, cell sort, row build (one
// CTA per cell of any replica), Morse forces (LPA lanes per atom), the fused
// kick-drift.  Per-replica constants (box, cell grid, fixed-point scales)
// sit in small descriptor tables that stay in L1/L2; each atom finds its
// replica through rep[i].  A window of K steps (one run_until) is captured
// once as a CUDA graph and replayed, so uneven replicas cost no extra
// launches and the GPU is filled by the batch as a whole.
#include <algorithm>
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
#include "replica_geo.cuh"
#include "replicas.cuh"

namespace tdmd_b200 {
namespace {

constexpr int kThreads = 256;

// Per-atom Morse energy (1/2 U per listed pair), the same expression as the
// force kernel's energy term; only on energy-log windows.
template <class Geo, int LPA, int U, bool VEC>
__global__ void __launch_bounds__(kThreads) k_morse_atom_pe(Geo g, NbrView nl, int n,
                                                            MorseP<typename Geo::T> mp,
                                                            double* __restrict__ pe_atom) {
  dependent_launch_prologue();
  using T = typename Geo::T;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = tid / LPA;
  const int sub = tid % LPA;
  double pe = 0.0;
  if (i < n) {
    const typename Geo::Own o = g.own(i);
    const long long row = nl.row(i);
    const int c = nl.count(i);
    for (int base = U * sub; base < c; base += U * LPA) {
      int jj[U];
      nbr_batch<VEC>(nl, row, base, c, jj);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (jj[u] < 0) continue;
        typename Geo::Pair pr;
        g.pair(o, jj[u], pr);
        if (pr.r2 < mp.rc_sq) {
          T r, rinv;
          double rd;
          g.radius(o, pr, r, rinv, rd);
          const T ex = exp(-mp.alpha * static_cast<T>(rd - mp.r0d));
          const T ome = T(1) - ex;
          pe += 0.5 * static_cast<double>(mp.d * (ome * ome - T(1)));
        }
      }
    }
  }
#pragma unroll
  for (int s = LPA / 2; s > 0; s >>= 1) pe += __shfl_xor_sync(0xffffffffu, pe, s);
  if (i < n && sub == 0) pe_atom[i] = pe;
}

// Per-atom EAM energy F_ti(rho_i) + 1/2 sum_j phi(r_ij), with the force
// pass's spline rows and offsets; only on energy-log windows.
template <class Geo, int LPA, int U, bool VEC, bool MULTI>
__global__ void __launch_bounds__(kThreads) k_eam_atom_pe(Geo g, NbrView nl, int n,
                                                          EamDev<typename Geo::T> e,
                                                          const int* __restrict__ types,
                                                          const double* __restrict__ rho,
                                                          double* __restrict__ pe_atom) {
  dependent_launch_prologue();
  using T = typename Geo::T;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = tid / LPA;
  const int sub = tid % LPA;
  double pe = 0.0;
  if (i < n) {
    const typename Geo::Own o = g.own(i);
    const int ti = MULTI ? __ldg(types + i) - 1 : 0;
    const long long row = nl.row(i);
    const int c = nl.count(i);
    for (int base = U * sub; base < c; base += U * LPA) {
      int jj[U];
      nbr_batch<VEC>(nl, row, base, c, jj);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (jj[u] < 0) continue;
        typename Geo::Pair pr;
        g.pair(o, jj[u], pr);
        if (pr.r2 < e.rc_sq) {
          T r, rinv, sx;
          double rd;
          g.radius(o, pr, r, rinv, rd);
          const int idx = spline_at(r, rd, e.dr, e.inv_dr, e.nr, e.dr_d, sx);
          const int tj = MULTI ? __ldg(types + jj[u]) - 1 : 0;
          const auto cphi = ldv4<T>(e.rtab + static_cast<long long>(idx) * e.S +
                                    (MULTI ? phi_slot(ti, tj, e.ntypes) : 1));
          pe += 0.5 * static_cast<double>(dspl_val(cphi, sx));
        }
      }
    }
  }
#pragma unroll
  for (int s = LPA / 2; s > 0; s >>= 1) pe += __shfl_xor_sync(0xffffffffu, pe, s);
  if (i < n && sub == 0) {
    const int ti = MULTI ? __ldg(types + i) - 1 : 0;
    double Fi, dF;
    embed_eval(e.ftab, e.nrho, e.drho, ti, rho[i], Fi, dF);
    pe_atom[i] = pe + Fi;
  }
}

// Per-replica (PE, KE) in a fixed order: one CTA per replica.
__global__ void __launch_bounds__(kThreads) k_rep_energy(const double* __restrict__ pe_atom,
                                                         const double* __restrict__ v,
                                                         const int* __restrict__ types,
                                                         const double* __restrict__ masses,
                                                         const RepDesc* __restrict__ reps,
                                                         double* __restrict__ out) {
  dependent_launch_prologue();
  __shared__ double red[32 * 2];
  const int r = blockIdx.x;
  const int a0 = reps[r].atom0, na = reps[r].natoms;
  double v2[2] = {0.0, 0.0};
  for (int k = threadIdx.x; k < na; k += blockDim.x) {
    const int i = a0 + k;
    const double vx = v[3ll * i], vy = v[3ll * i + 1], vz = v[3ll * i + 2];
    v2[0] += pe_atom[i];
    v2[1] += 0.5 * masses[types[i]] * kMvv2e * (vx * vx + vy * vy + vz * vz);
  }
  block_sum<2>(v2, red);
  if (threadIdx.x == 0) {
    out[2 * r] = v2[0];
    out[2 * r + 1] = v2[1];
  }
}

__global__ void k_pack_batch(const double* __restrict__ x, const int* __restrict__ types,
                             const int* __restrict__ rep, const RepDesc* __restrict__ reps,
                             int n, double4* __restrict__ pos4, int4* __restrict__ q) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double px = x[3ll * i], py = x[3ll * i + 1], pz = x[3ll * i + 2];
  const int t = types[i];
  pos4[i] = make_double4(px, py, pz, static_cast<double>(t));
  if (q) {
    const DevBox& b = reps[rep[i]].box;
    q[i] = make_int4(encode_q(px, b.qlo[0], b.qinv[0]), encode_q(py, b.qlo[1], b.qinv[1]),
                     encode_q(pz, b.qlo[2], b.qinv[2]), t);
  }
}

__global__ void k_unpack_batch(const double4* __restrict__ pos4, int n, double* __restrict__ x) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = pos4[i];
  x[3ll * i] = p.x;
  x[3ll * i + 1] = p.y;
  x[3ll * i + 2] = p.z;
}

// Kick (half or full dt) + drift + single-image wrap in the atom's replica
// box + fixed-point refresh; fused_kick_drift_kernel,
// device_velocity_verlet.cu:88-130, per replica.
template <class F, bool FULL>
__global__ void __launch_bounds__(kThreads) k_kick_drift_batch(
    double4* __restrict__ pos4, int4* __restrict__ q, double* __restrict__ v,
    const F* __restrict__ f, const int* __restrict__ types, const int* __restrict__ rep,
    const RepDesc* __restrict__ reps, const double* __restrict__ inv_mm, int n, double dt) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double kick_dt = FULL ? dt : 0.5 * dt;
  const int t = types[i];
  const double factor = kick_dt * inv_mm[t];
  const DevBox& b = reps[__ldg(rep + i)].box;
  double4 p = pos4[i];
  double vx = v[3ll * i], vy = v[3ll * i + 1], vz = v[3ll * i + 2];
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

template <class F>
__global__ void __launch_bounds__(kThreads) k_half_kick_batch(double* __restrict__ v,
                                                              const F* __restrict__ f,
                                                              const int* __restrict__ types,
                                                              const double* __restrict__ inv_mm,
                                                              int n, double dt) {
  dependent_launch_prologue();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double factor = 0.5 * dt * inv_mm[types[i]];
  v[3ll * i] += factor * static_cast<double>(f[3ll * i]);
  v[3ll * i + 1] += factor * static_cast<double>(f[3ll * i + 1]);
  v[3ll * i + 2] += factor * static_cast<double>(f[3ll * i + 2]);
}

struct BatchStep {
  bool first, rebuild;
  bool kd_fused;   // kick + drift done by the previous step's force pass
  bool fuse_next;  // this force pass also kicks and drifts for the next step
  bool log_e;      // window end of a logged window: the force pass also writes
                   // per-atom energies, reduced per replica after the half kick
};

}  // namespace

class Batch {
 public:
  // Exactly one of morse / eam is given.
  Batch(int nrep, const tdmd_box* boxes, const int* natoms, const tdmd_morse_params* morse,
        const tdmd_eam* eam, const tdmd_fast_pipeline_config& cfg);
  ~Batch();
  Batch(const Batch&) = delete;
  Batch& operator=(const Batch&) = delete;

  void upload(const double* x, const double* v, const int* types, const double* masses,
              int n_types);
  void download(double* x, double* v, void* f) const;
  void run_until(int target);
  void energies(double* pe, double* ke);
  void energy_log(double* steps, double* pe_ke, int cap, int* count) const;
  void autotune(int* lanes2, int* batch2, double* ms24);
  void stats(tdmd_fast_pipeline_stats* o) const {
    *o = tdmd_fast_pipeline_stats{};
    o->ticks = ticks_;
    o->kernel_launches = launches_;
    o->rebuilds = rebuilds_;
    o->graph_launches = graph_launches_;
    o->nlist_retries = retries_;
    o->nlist_capacity = cap_;
    o->lanes_per_atom = lpa_;
    o->nbr_batch = nu_;
    o->density_lanes_per_atom = eam_ ? lpa_d_ : 0;
    o->density_nbr_batch = eam_ ? nu_d_ : 0;
  }
  int nreplicas() const { return nrep_; }
  long long natoms() const { return n_; }
  int lanes() const { return lpa_; }
  int nbr_batch() const { return nu_; }
  int step() const { return step_; }
  double last_window_ms() const { return last_window_ms_; }
  cudaStream_t stream() const { return stream_; }

 private:
  void rebuild(int* status);
  // parts: which EAM passes (density, pair force); Morse has one pass.
  static constexpr int kPassDensity = 1, kPassForce = 2, kPassBoth = 3;
  void force(bool kd = false, bool pe_atom = false, int parts = kPassBoth);
  void rep_energy();
  void kick_drift(bool full);
  void half_kick();
  void enqueue_step(const BatchStep& st);
  void run_segment(const std::vector<BatchStep>& seg, bool finalize, bool prologue);
  void enqueue_prologue();
  void initial_forces();
  void grow_capacity(int max_count);
  void reduce_energies(double* out);
  void clear_graphs();
  NbrView view() const { return NbrView{nbr_.data(), nullptr, cnt_.data(), cap_}; }

  int nrep_;
  long long n_ = 0;
  tdmd_fast_pipeline_config cfg_;
  bool mixed_;
  double rc_, rl2_;
  MorseP<double> m64_;
  MorseP<float> m32_;
  std::unique_ptr<EamDevTables> eam_;  // EAM replicas (same tables for all)
  DevArray<float> fp32_;
  DevArray<double> fp64_, rho_;
  DevArray<int4> g_;                   // mixed EAM gather records {q, bits(F')}
  DevArray<double4> g64_;              // FP64 EAM gather records {x, y, z, F'}
  std::vector<RepDesc> hreps_;
  int ncells_ = 0;
  int lpa_ = 0;
  int nu_ = kU;  // neighbors per lane per sweep (2 or 4)
  // launch shape of the EAM density pass (lpa_ / nu_: the pair-force pass)
  int lpa_d_ = 0;
  int nu_d_ = kU;
  int cap_ = 0;
  int n_types_ = 0;
  bool uploaded_ = false, initialized_ = false, tuned_ = false;
  int step_ = 0, since_rebuild_ = 0;
  long long ticks_ = 0, launches_ = 0, rebuilds_ = 0, graph_launches_ = 0, retries_ = 0;
  double last_window_ms_ = 0.0;
  cudaStream_t stream_ = nullptr;
  cudaEvent_t win_ev_[2] = {nullptr, nullptr};
  std::map<std::vector<int>, std::pair<cudaGraphExec_t, long long>> graphs_;
  std::list<std::vector<int>> graph_lru_;
  // device state
  DevArray<RepDesc> reps_;
  DevArray<RepScale> scales_;
  DevArray<RepImg> imgs_;
  DevArray<int> cell_rep_;
  DevArray<int> rep_;
  DevArray<double4> pos4_;
  DevArray<int4> q_;
  DevArray<double> vel_;
  DevArray<float> f32_;
  DevArray<double> f64_;
  DevArray<int> types_;
  DevArray<double> masses_, inv_mm_;
  DevArray<double> stage_;
  DevArray<int> nbr_, cnt_, status_;
  DevArray<double> pe_atom_, eout_;
  CellListDev cl_;
  // window snapshot (overflow retry)
  DevArray<double4> snap_pos4_;
  DevArray<int4> snap_q_;
  DevArray<double> snap_vel_;
  // energy log
  std::vector<double> log_steps_;
  std::vector<double> log_;
};

Batch::Batch(int nrep, const tdmd_box* boxes, const int* natoms, const tdmd_morse_params* morse,
             const tdmd_eam* eam, const tdmd_fast_pipeline_config& cfg)
    : nrep_(nrep), cfg_(cfg), mixed_(cfg.precision == TDMD_MIXED) {
  TDMD_REQUIRE((morse != nullptr) != (eam != nullptr), "give a Morse or an EAM potential");
  TDMD_REQUIRE(nrep >= 1, "need at least one replica");
  TDMD_REQUIRE(boxes && natoms, "null boxes or natoms");
  TDMD_REQUIRE(cfg.dt > 0.0, "dt must be positive");
  TDMD_REQUIRE(cfg.r_skin >= 0.0, "r_skin must be non-negative");
  TDMD_REQUIRE(cfg.rebuild_every >= 1, "rebuild_every must be >= 1");
  TDMD_REQUIRE(cfg.precision == TDMD_FP64 || cfg.precision == TDMD_MIXED, "unknown precision");
  if (cfg.t_target > 0.0 || cfg.adaptive_dt)
    throw Error{TDMD_ERR_UNSUPPORTED, "batched replicas run NVE with a fixed dt"};
  if (morse) {
    const tdmd_morse_params& p = *morse;
    TDMD_REQUIRE(p.rc > 0.0, "cutoff must be positive");
    rc_ = p.rc;
    const double rc_sq = p.rc_sq > 0.0 ? p.rc_sq : p.rc * p.rc;
    m64_ = MorseP<double>{p.d, p.alpha, p.r0, rc_sq, p.r0};
    m32_ = MorseP<float>{static_cast<float>(p.d), static_cast<float>(p.alpha),
                         static_cast<float>(p.r0), static_cast<float>(rc_sq), p.r0};
  } else {
    TDMD_REQUIRE(eam->cutoff > 0.0, "cutoff must be positive");
    rc_ = eam->cutoff;
  }
  const double rl = rc_ + cfg.r_skin;
  rl2_ = rl * rl;
  hreps_.resize(static_cast<size_t>(nrep));
  std::vector<RepScale> sc(static_cast<size_t>(nrep));
  std::vector<RepImg> img(static_cast<size_t>(nrep));
  long long atoms = 0, cells = 0;
  for (int r = 0; r < nrep; ++r) {
    TDMD_REQUIRE(natoms[r] >= 0, "replica atom count must be non-negative");
    RepDesc& d = hreps_[static_cast<size_t>(r)];
    d = RepDesc{};
    d.box = make_devbox(boxes[r], rl);
    for (int a = 0; a < 3; ++a)
      TDMD_REQUIRE(!d.box.periodic[a] || d.box.L[a] > 2.0 * rl,
                   "periodic box edge must exceed twice cutoff + skin");
    d.atom0 = static_cast<int>(atoms);
    d.natoms = natoms[r];
    d.cell0 = static_cast<int>(cells);
    d.ncells = d.box.nc[0] * d.box.nc[1] * d.box.nc[2];
    row_filter_band(d.box, rl2_, &d.lo_f, &d.hi_f, &d.wrap);
    RepScale& s = sc[static_cast<size_t>(r)];
    s = RepScale{};
    RepImg& m = img[static_cast<size_t>(r)];
    m = RepImg{};
    for (int a = 0; a < 3; ++a) {
      s.s[a] = d.box.qscale[a];
      s.s2[a] = d.box.qstep[a] * d.box.qstep[a];
      m.L[a] = d.box.L[a];
      m.halfL[a] = d.box.halfL[a];
      m.per[a] = d.box.periodic[a];
    }
    s.iso = d.box.qstep[0] == d.box.qstep[1] && d.box.qstep[1] == d.box.qstep[2];
    atoms += natoms[r];
    cells += d.ncells;
    TDMD_REQUIRE(atoms < INT_MAX / 2 && cells < INT_MAX / 2, "batch too large");
  }
  n_ = atoms;
  ncells_ = static_cast<int>(cells);
  lpa_ = cfg.lanes_per_atom > 0 ? cfg.lanes_per_atom : default_lpa(n_ > 0 ? n_ : 1);
  TDMD_REQUIRE(lpa_ == 1 || lpa_ == 2 || lpa_ == 4 || lpa_ == 8 || lpa_ == 16 || lpa_ == 32,
               "lanes_per_atom must be 1,2,4,8,16 or 32");
  TDMD_REQUIRE(cfg.nbr_batch == 0 || cfg.nbr_batch == 2 || cfg.nbr_batch == 4,
               "nbr_batch must be 0 (tuned), 2 or 4");
  nu_ = cfg.nbr_batch > 0 ? cfg.nbr_batch : kU;
  lpa_d_ = lpa_;
  nu_d_ = nu_;
  TDMD_CU(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  TDMD_CU(cudaEventCreate(&win_ev_[0]));
  TDMD_CU(cudaEventCreate(&win_ev_[1]));
  cudaStream_t s = stream_;
  if (eam) {
    eam_ = std::make_unique<EamDevTables>();
    eam_->upload(*eam, s);
  }
  reps_.reserve(hreps_.size());
  scales_.reserve(sc.size());
  imgs_.reserve(img.size());
  TDMD_CU(cudaMemcpyAsync(reps_.data(), hreps_.data(), sizeof(RepDesc) * hreps_.size(),
                          cudaMemcpyHostToDevice, s));
  TDMD_CU(cudaMemcpyAsync(scales_.data(), sc.data(), sizeof(RepScale) * sc.size(),
                          cudaMemcpyHostToDevice, s));
  TDMD_CU(cudaMemcpyAsync(imgs_.data(), img.data(), sizeof(RepImg) * img.size(),
                          cudaMemcpyHostToDevice, s));
  std::vector<int> crep(static_cast<size_t>(std::max(ncells_, 1)), 0);
  std::vector<int> arep(static_cast<size_t>(std::max<long long>(n_, 1)), 0);
  for (int r = 0; r < nrep; ++r) {
    const RepDesc& d = hreps_[static_cast<size_t>(r)];
    std::fill(crep.begin() + d.cell0, crep.begin() + d.cell0 + d.ncells, r);
    std::fill(arep.begin() + d.atom0, arep.begin() + d.atom0 + d.natoms, r);
  }
  cell_rep_.reserve(crep.size());
  rep_.reserve(arep.size());
  TDMD_CU(cudaMemcpyAsync(cell_rep_.data(), crep.data(), sizeof(int) * crep.size(),
                          cudaMemcpyHostToDevice, s));
  TDMD_CU(cudaMemcpyAsync(rep_.data(), arep.data(), sizeof(int) * arep.size(),
                          cudaMemcpyHostToDevice, s));
  TDMD_CU(cudaStreamSynchronize(s));
}

Batch::~Batch() {
  clear_graphs();
  for (auto e : win_ev_)
    if (e) cudaEventDestroy(e);
  if (stream_) {
    cudaStreamSynchronize(stream_);
    cudaStreamDestroy(stream_);
  }
}

void Batch::clear_graphs() {
  for (auto& kv : graphs_)
    if (kv.second.first) cudaGraphExecDestroy(kv.second.first);
  graphs_.clear();
  graph_lru_.clear();
}

void Batch::upload(const double* x, const double* v, const int* types, const double* masses,
                   int n_types) {
  TDMD_REQUIRE(n_types >= 2, "n_types is masses.size() = ntypes + 1 (>= 2)");
  TDMD_REQUIRE(n_ == 0 || (x && v && types && masses), "null host array");
  const size_t n = static_cast<size_t>(n_);
  for (size_t i = 0; i < n; ++i)
    TDMD_REQUIRE(types[i] >= 1 && types[i] < n_types, "atom type out of range of masses");
  if (eam_)
    for (size_t i = 0; i < n; ++i)
      TDMD_REQUIRE(types[i] <= eam_->ntypes, "atom type beyond the EAM element count");
  clear_graphs();
  cudaStream_t s = stream_;
  const size_t nn = std::max<size_t>(n, 1);
  if (eam_) {
    rho_.reserve(nn);
    if (mixed_)
      fp32_.reserve(nn), g_.reserve(nn);
    else
      fp64_.reserve(nn), g64_.reserve(nn);
  }
  pos4_.reserve(nn);
  vel_.reserve(3 * nn);
  types_.reserve(nn);
  stage_.reserve(3 * nn);
  cnt_.reserve(nn);
  pe_atom_.reserve(nn);
  status_.reserve(4);
  eout_.reserve(2 * static_cast<size_t>(nrep_));
  if (mixed_) {
    q_.reserve(nn);
    f32_.reserve(3 * nn);
  } else {
    f64_.reserve(3 * nn);
  }
  if (n > 0) {
    TDMD_CU(cudaMemcpyAsync(stage_.data(), x, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    TDMD_CU(cudaMemcpyAsync(vel_.data(), v, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    TDMD_CU(cudaMemcpyAsync(types_.data(), types, n * sizeof(int), cudaMemcpyHostToDevice, s));
    launch(k_pack_batch, ceil_div(n_, kThreads), kThreads, 0, s, stage_.data(), types_.data(),
           rep_.data(), reps_.data(), static_cast<int>(n_), pos4_.data(),
           mixed_ ? q_.data() : nullptr);
    TDMD_LAUNCH_CHECK();
  }
  masses_.reserve(static_cast<size_t>(n_types));
  inv_mm_.reserve(static_cast<size_t>(n_types));
  std::vector<double> inv(static_cast<size_t>(n_types), 0.0);
  for (int t = 0; t < n_types; ++t)
    inv[static_cast<size_t>(t)] = masses[t] > 0.0 ? 1.0 / (masses[t] * kMvv2e) : 0.0;
  TDMD_CU(cudaMemcpyAsync(masses_.data(), masses, sizeof(double) * n_types,
                          cudaMemcpyHostToDevice, s));
  TDMD_CU(cudaMemcpyAsync(inv_mm_.data(), inv.data(), sizeof(double) * n_types,
                          cudaMemcpyHostToDevice, s));
  TDMD_CU(cudaStreamSynchronize(s));
  n_types_ = n_types;
  uploaded_ = true;
  initialized_ = false;
  step_ = 0;
  since_rebuild_ = 0;
  log_steps_.clear();
  log_.clear();
}

void Batch::download(double* x, double* v, void* f) const {
  TDMD_REQUIRE(uploaded_, "download before upload");
  if (n_ == 0) return;
  cudaStream_t s = stream_;
  const size_t n = static_cast<size_t>(n_);
  if (x) {
    launch(k_unpack_batch, ceil_div(n_, kThreads), kThreads, 0, s, pos4_.data(),
           static_cast<int>(n_), stage_.data());
    TDMD_LAUNCH_CHECK();
    TDMD_CU(cudaMemcpyAsync(x, stage_.data(), 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  if (v)
    TDMD_CU(cudaMemcpyAsync(v, vel_.data(), 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (f) {
    if (mixed_)
      TDMD_CU(cudaMemcpyAsync(f, f32_.data(), 3 * n * sizeof(float), cudaMemcpyDeviceToHost, s));
    else
      TDMD_CU(cudaMemcpyAsync(f, f64_.data(), 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  TDMD_CU(cudaStreamSynchronize(s));
}

void Batch::grow_capacity(int max_count) {
  long long want = static_cast<long long>(max_count) + max_count / 4 + 16;
  want = (want + 7) / 8 * 8;
  TDMD_REQUIRE(want * std::max<long long>(n_, 1) < (1ll << 40), "neighbor list too large");
  if (want > cap_) {
    cap_ = static_cast<int>(want);
    nbr_.reserve(static_cast<size_t>(cap_) * static_cast<size_t>(std::max<long long>(n_, 1)));
    clear_graphs();
  }
}

void Batch::rebuild(int* status) {
  cudaStream_t s = stream_;
  build_cell_list_batch(cl_, pos4_.data(), rep_.data(), reps_.data(), n_, ncells_, s);
  build_neighbor_rows_batch(cl_, pos4_.data(), reps_.data(), cell_rep_.data(), rl2_,
                            nbr_.data(), cap_, cnt_.data(), status, s);
  launches_ += 4 + device_scan_launches(ncells_);
  ++rebuilds_;
}

void Batch::force(bool kd, bool pea, int parts) {
  cudaStream_t s = stream_;
  const NbrView nl = view();
  const int n = static_cast<int>(n_);
  const Tune td{lpa_d_, nu_d_}, tf{lpa_, nu_};
  const bool dens = parts & kPassDensity, pair = parts & kPassForce;
  TDMD_REQUIRE(!kd || eam_, "fused kick-drift needs the EAM batch");
  if (eam_) {
    // Density + embedding, then forces, over all replicas at once (the
    // single scheduler's passes on the batched geometries).
    const int* types = eam_->ntypes > 1 ? types_.data() : nullptr;
    if (mixed_) {
      const GeoQB g{q_.data(), rep_.data(), scales_.data()};
      const GeoQB gg{g_.data(), rep_.data(), scales_.data()};
      if (dens)
        launch_eam_density<GeoQB, float>(g, nl, n, eam_->d32, types, fp32_.data(), nullptr,
                                         nullptr, g_.data(), false, nullptr, td, s,
                                         pea ? pe_atom_.data() : nullptr);
      // kd: the next step's kick + drift in the same pass (the force pass
      // reads gather records only), each atom in its replica's box
      const KickDrift kdr{pos4_.data(), q_.data(), vel_.data(), types_.data(), inv_mm_.data(),
                          cfg_.dt, nullptr, DevBox{}, rep_.data(), reps_.data()};
      if (pair)
        launch_eam_force<GeoQB, true, float, float>(gg, nl, n, eam_->d32, types, fp32_.data(),
                                                    f32_.data(), pea, nullptr, tf, s,
                                                    kd ? &kdr : nullptr,
                                                    pea ? pe_atom_.data() : nullptr);
    } else {
      // FP64: the density pass writes {x, y, z, F'} gather records, which the
      // force pass reads (so it may also kick and drift, like the mixed pass)
      const GeoD4B g{pos4_.data(), rep_.data(), imgs_.data()};
      const GeoD4BF gg{g64_.data(), rep_.data(), imgs_.data()};
      if (dens)
        launch_eam_density<GeoD4B, double>(g, nl, n, eam_->d64, types, fp64_.data(), nullptr,
                                           nullptr, nullptr, false, nullptr, td, s,
                                           pea ? pe_atom_.data() : nullptr, g64_.data());
      const KickDrift kdr{pos4_.data(), nullptr, vel_.data(), types_.data(), inv_mm_.data(),
                          cfg_.dt, nullptr, DevBox{}, rep_.data(), reps_.data()};
      if (pair)
        launch_eam_force<GeoD4BF, true, double, double>(gg, nl, n, eam_->d64, types,
                                                        fp64_.data(), f64_.data(), pea, nullptr,
                                                        tf, s, kd ? &kdr : nullptr,
                                                        pea ? pe_atom_.data() : nullptr);
    }
    launches_ += (dens ? 1 : 0) + (pair ? 1 : 0);
    return;
  }
  if (mixed_) {
    const GeoQB g{q_.data(), rep_.data(), scales_.data()};
    launch_morse(g, nl, n, m32_, f32_.data(), pea, nullptr, tf, s,
                 pea ? pe_atom_.data() : nullptr);
  } else {
    const GeoD4B g{pos4_.data(), rep_.data(), imgs_.data()};
    launch_morse(g, nl, n, m64_, f64_.data(), pea, nullptr, tf, s,
                 pea ? pe_atom_.data() : nullptr);
  }
  ++launches_;
}

void Batch::kick_drift(bool full) {
  cudaStream_t s = stream_;
  const int n = static_cast<int>(n_);
  const int nb = ceil_div(n_, kThreads);
  if (mixed_) {
    if (full)
      launch(k_kick_drift_batch<float, true>, nb, kThreads, 0, s, pos4_.data(), q_.data(),
             vel_.data(), f32_.data(), types_.data(), rep_.data(), reps_.data(), inv_mm_.data(), n,
             cfg_.dt);
    else
      launch(k_kick_drift_batch<float, false>, nb, kThreads, 0, s, pos4_.data(), q_.data(),
             vel_.data(), f32_.data(), types_.data(), rep_.data(), reps_.data(), inv_mm_.data(), n,
             cfg_.dt);
  } else {
    if (full)
      launch(k_kick_drift_batch<double, true>, nb, kThreads, 0, s, pos4_.data(), nullptr,
             vel_.data(), f64_.data(), types_.data(), rep_.data(), reps_.data(), inv_mm_.data(), n,
             cfg_.dt);
    else
      launch(k_kick_drift_batch<double, false>, nb, kThreads, 0, s, pos4_.data(), nullptr,
             vel_.data(), f64_.data(), types_.data(), rep_.data(), reps_.data(), inv_mm_.data(), n,
             cfg_.dt);
  }
  TDMD_LAUNCH_CHECK();
  ++launches_;
}

void Batch::half_kick() {
  cudaStream_t s = stream_;
  const int n = static_cast<int>(n_);
  const int nb = ceil_div(n_, kThreads);
  if (mixed_)
    launch(k_half_kick_batch<float>, nb, kThreads, 0, s, vel_.data(), f32_.data(), types_.data(),
           inv_mm_.data(), n, cfg_.dt);
  else
    launch(k_half_kick_batch<double>, nb, kThreads, 0, s, vel_.data(), f64_.data(), types_.data(),
           inv_mm_.data(), n, cfg_.dt);
  TDMD_LAUNCH_CHECK();
  ++launches_;
}

// Same step sequence as the single-system scheduler's NVE path: fused
// kick-drift (half kick on the first step of a window), rebuild when due,
// forces; the window closes with a half kick.
void Batch::enqueue_step(const BatchStep& st) {
  if (!st.kd_fused) kick_drift(!st.first);
  if (st.rebuild) rebuild(status_.data());
  force(st.fuse_next, st.log_e);
}

// A window's first segment starts with the snapshot for an overflow retry
// (positions, fixed point, velocities; forces are recomputed from the
// restored positions) and the reset of the overflow flags, captured with its
// steps so that a window is one submission.
void Batch::enqueue_prologue() {
  const size_t n = static_cast<size_t>(n_);
  cudaStream_t s = stream_;
  TDMD_CU(cudaMemcpyAsync(snap_pos4_.data(), pos4_.data(), n * sizeof(double4),
                          cudaMemcpyDeviceToDevice, s));
  TDMD_CU(cudaMemcpyAsync(snap_vel_.data(), vel_.data(), 3 * n * sizeof(double),
                          cudaMemcpyDeviceToDevice, s));
  if (mixed_)
    TDMD_CU(cudaMemcpyAsync(snap_q_.data(), q_.data(), n * sizeof(int4),
                            cudaMemcpyDeviceToDevice, s));
  TDMD_CU(cudaMemsetAsync(status_.data(), 0, sizeof(int) * 4, s));
}

void Batch::run_segment(const std::vector<BatchStep>& seg, bool finalize, bool prologue) {
  std::vector<int> key;
  key.reserve(seg.size() + 2);
  for (const auto& st : seg)
    key.push_back((st.first ? 1 : 0) | (st.rebuild ? 2 : 0) | (st.kd_fused ? 4 : 0) |
                  (st.fuse_next ? 8 : 0) | (st.log_e ? 16 : 0));
  key.push_back(finalize ? 1 : 0);
  key.push_back(prologue ? 1 : 0);
  const long long l0 = launches_;
  // the window's closing half kick, then (logged windows) the per-replica
  // energies of the integer-time state
  auto close = [&] {
    if (!finalize) return;
    half_kick();
    if (!seg.empty() && seg.back().log_e) rep_energy();
  };
  if (!cfg_.use_graphs) {
    if (prologue) enqueue_prologue();
    for (const auto& st : seg) enqueue_step(st);
    close();
    return;
  }
  auto it = graphs_.find(key);
  if (it == graphs_.end()) {
    if (graphs_.size() >= 16) {
      auto old = graphs_.find(graph_lru_.back());
      if (old != graphs_.end()) {
        cudaGraphExecDestroy(old->second.first);
        graphs_.erase(old);
      }
      graph_lru_.pop_back();
    }
    cudaGraph_t g = nullptr;
    TDMD_CU(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    try {
      if (prologue) enqueue_prologue();
      for (const auto& st : seg) enqueue_step(st);
      close();
    } catch (...) {
      cudaStreamEndCapture(stream_, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    TDMD_CU(cudaStreamEndCapture(stream_, &g));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    TDMD_CU(ie);
    const long long kernels = launches_ - l0;
    launches_ = l0;
    it = graphs_.emplace(key, std::make_pair(exec, kernels)).first;
    graph_lru_.push_front(key);
  } else {
    graph_lru_.remove(key);
    graph_lru_.push_front(key);
  }
  TDMD_CU(cudaGraphLaunch(it->second.first, stream_));
  launches_ += it->second.second;
  ++graph_launches_;
}

void Batch::initial_forces() {
  cudaStream_t s = stream_;
  TDMD_CU(cudaMemsetAsync(status_.data(), 0, sizeof(int) * 4, s));
  // Count pass sizes the padded rows, then the real build.
  build_cell_list_batch(cl_, pos4_.data(), rep_.data(), reps_.data(), n_, ncells_, s);
  build_neighbor_rows_batch(cl_, pos4_.data(), reps_.data(), cell_rep_.data(), rl2_, nullptr, 0,
                            cnt_.data(), status_.data(), s);
  int st[4];
  TDMD_CU(cudaMemcpyAsync(st, status_.data(), sizeof(st), cudaMemcpyDeviceToHost, s));
  TDMD_CU(cudaStreamSynchronize(s));
  grow_capacity(st[1]);
  TDMD_CU(cudaMemsetAsync(status_.data(), 0, sizeof(int) * 4, s));
  build_neighbor_rows_batch(cl_, pos4_.data(), reps_.data(), cell_rep_.data(), rl2_,
                            nbr_.data(), cap_, cnt_.data(), status_.data(), s);
  launches_ += 4 + device_scan_launches(ncells_) + 1;
  ++rebuilds_;
  since_rebuild_ = 0;
  force();
  initialized_ = true;
}

// Sweeps the launch shape of each gather pass on its own, as
// Scheduler::autotune does: lanes per atom {1, ..., 32} x neighbors per lane
// sweep {2, 4} (only cfg.nbr_batch when that is fixed), the EAM density
// pass first, then the pair-force pass; ms24 laid out as there.
void Batch::autotune(int* lanes2, int* batch2, double* ms24) {
  TDMD_REQUIRE(uploaded_, "autotune before upload");
  if (n_ == 0) return;
  if (!initialized_) initial_forces();
  cudaStream_t s = stream_;
  const int cands[6] = {1, 2, 4, 8, 16, 32};
  const int batches[2] = {2, 4};
  if (ms24)
    for (int k = 0; k < 24; ++k) ms24[k] = -1.0;
  auto sweep = [&](int pass) {
    int& lanes = pass == 0 ? lpa_d_ : lpa_;
    int& batch = pass == 0 ? nu_d_ : nu_;
    const int parts = pass == 0 ? kPassDensity : kPassForce;
    double best = 1e30;
    int best_l = lanes, best_u = batch;
    for (int b = 0; b < 2; ++b) {
      if (cfg_.nbr_batch > 0 && batches[b] != cfg_.nbr_batch) continue;
      for (int k = 0; k < 6; ++k) {
        lanes = cands[k];
        batch = batches[b];
        force(false, false, parts);  // warm
        TDMD_CU(cudaEventRecord(win_ev_[0], s));
        for (int rep = 0; rep < 5; ++rep) force(false, false, parts);
        TDMD_CU(cudaEventRecord(win_ev_[1], s));
        TDMD_CU(cudaEventSynchronize(win_ev_[1]));
        float ms = 0.f;
        TDMD_CU(cudaEventElapsedTime(&ms, win_ev_[0], win_ev_[1]));
        const double per = ms / 5.0;
        if (ms24) ms24[12 * pass + 6 * b + k] = per;
        if (per < best) {
          best = per;
          best_l = cands[k];
          best_u = batches[b];
        }
      }
    }
    lanes = best_l;
    batch = best_u;
  };
  if (eam_) {
    sweep(0);
    force(false, false, kPassDensity);  // the chosen density pass's output
  }
  sweep(1);
  clear_graphs();
  force();  // forces of the current state with the chosen shapes
  TDMD_CU(cudaStreamSynchronize(s));
  tuned_ = true;
  if (lanes2) {
    lanes2[0] = eam_ ? lpa_d_ : 0;
    lanes2[1] = lpa_;
  }
  if (batch2) {
    batch2[0] = eam_ ? nu_d_ : 0;
    batch2[1] = nu_;
  }
}

void Batch::run_until(int target) {
  TDMD_REQUIRE(uploaded_, "run_until before upload");
  if (n_ == 0) {
    step_ = std::max(step_, target);
    return;
  }
  if (!initialized_) initial_forces();
  if (!tuned_ && cfg_.lanes_per_atom == 0 && n_ >= 2048) autotune(nullptr, nullptr, nullptr);
  if (step_ >= target) {
    TDMD_CU(cudaStreamSynchronize(stream_));
    return;
  }
  const size_t n = static_cast<size_t>(n_);
  cudaStream_t s = stream_;
  const int step0 = step_, since0 = since_rebuild_;
  // snapshot buffers sized outside any stream capture
  snap_pos4_.reserve(n);
  snap_vel_.reserve(3 * n);
  if (mixed_) snap_q_.reserve(n);
  for (int attempt = 0;; ++attempt) {
    TDMD_CU(cudaEventRecord(win_ev_[0], s));
    std::vector<BatchStep> plan;
    int since = since_rebuild_;
    // energy log of windows whose last step is a multiple of energy_every
    // (velocities at integer time), computed inside the window
    const int log_cap = cfg_.energy_log_capacity > 0 ? cfg_.energy_log_capacity : 1024;
    const bool log_now = cfg_.energy_every > 0 && target % cfg_.energy_every == 0 &&
                         static_cast<int>(log_steps_.size()) < log_cap;
    for (int st = step_; st < target; ++st) {
      BatchStep b{};
      b.first = st == step_;
      b.rebuild = since >= cfg_.rebuild_every;
      if (b.rebuild) since = 0;
      ++since;
      // EAM (both precisions): every force pass but the window's last also
      // kicks and drifts for the next step (energies are logged after the
      // window)
      b.fuse_next = eam_ && st + 1 < target;
      b.kd_fused = !plan.empty() && plan.back().fuse_next;
      b.log_e = log_now && st + 1 == target;
      plan.push_back(b);
    }
    size_t a = 0;
    while (a < plan.size()) {
      size_t b = a + 1;
      while (b < plan.size() && !plan[b].rebuild && b - a < 64) ++b;
      run_segment(std::vector<BatchStep>(plan.begin() + static_cast<long>(a),
                                         plan.begin() + static_cast<long>(b)),
                  b == plan.size(), a == 0);
      a = b;
    }
    ticks_ += static_cast<long long>(plan.size());
    TDMD_CU(cudaEventRecord(win_ev_[1], s));
    int st[4];
    TDMD_CU(cudaMemcpyAsync(st, status_.data(), sizeof(st), cudaMemcpyDeviceToHost, s));
    TDMD_CU(cudaStreamSynchronize(s));
    float ms = 0.f;
    TDMD_CU(cudaEventElapsedTime(&ms, win_ev_[0], win_ev_[1]));
    last_window_ms_ = ms;
    if (!st[0]) {
      step_ = target;
      since_rebuild_ = since;
      if (log_now) {
        std::vector<double> e(2 * static_cast<size_t>(nrep_));
        TDMD_CU(cudaMemcpyAsync(e.data(), eout_.data(), sizeof(double) * e.size(),
                                cudaMemcpyDeviceToHost, s));
        TDMD_CU(cudaStreamSynchronize(s));
        log_steps_.push_back(static_cast<double>(step_));
        log_.insert(log_.end(), e.begin(), e.end());
      }
      break;
    }
    if (attempt >= 3)
      throw Error{TDMD_ERR_NLIST_OVERFLOW, "neighbor list overflow persisted after retries"};
    ++retries_;
    grow_capacity(st[1]);
    TDMD_CU(cudaMemcpyAsync(pos4_.data(), snap_pos4_.data(), n * sizeof(double4),
                            cudaMemcpyDeviceToDevice, s));
    TDMD_CU(cudaMemcpyAsync(vel_.data(), snap_vel_.data(), 3 * n * sizeof(double),
                            cudaMemcpyDeviceToDevice, s));
    if (mixed_)
      TDMD_CU(cudaMemcpyAsync(q_.data(), snap_q_.data(), n * sizeof(int4),
                              cudaMemcpyDeviceToDevice, s));
    step_ = step0;
    since_rebuild_ = since0;
    // Rebuild into the new capacity and recompute the forces of the
    // restored state (the window start).
    rebuild(nullptr);
    force();
  }
}

void Batch::reduce_energies(double* out) {
  cudaStream_t s = stream_;
  const NbrView nl = view();
  const int n = static_cast<int>(n_);
  const int nblk = force_blocks(n_, lpa_);
  const Tune tn{lpa_, nu_};
  if (eam_) {
    // rho_i of the current positions, then F(rho_i) + 1/2 sum_j phi(r_ij)
    const int* types = eam_->ntypes > 1 ? types_.data() : nullptr;
    if (mixed_) {
      const GeoQB g{q_.data(), rep_.data(), scales_.data()};
      launch_eam_density<GeoQB, float>(g, nl, n, eam_->d32, types, fp32_.data(), rho_.data(),
                                       nullptr, g_.data(), false, nullptr, Tune{lpa_d_, nu_d_}, s);
      TDMD_MULTI_DISPATCH(types != nullptr, TDMD_VEC_DISPATCH(vec_rows(nl), TDMD_TUNE_DISPATCH(
          tn, {
            launch(k_eam_atom_pe<GeoQB, L, U, V, M>, nblk, kThreads, 0, s, g, nl, n,
                   eam_->d32, types, rho_.data(), pe_atom_.data());
          })));
    } else {
      const GeoD4B g{pos4_.data(), rep_.data(), imgs_.data()};
      launch_eam_density<GeoD4B, double>(g, nl, n, eam_->d64, types, fp64_.data(), rho_.data(),
                                         nullptr, nullptr, false, nullptr, Tune{lpa_d_, nu_d_}, s);
      TDMD_MULTI_DISPATCH(types != nullptr, TDMD_VEC_DISPATCH(vec_rows(nl), TDMD_TUNE_DISPATCH(
          tn, {
            launch(k_eam_atom_pe<GeoD4B, L, U, V, M>, nblk, kThreads, 0, s, g, nl, n,
                   eam_->d64, types, rho_.data(), pe_atom_.data());
          })));
    }
    TDMD_LAUNCH_CHECK();
    launches_ += 1;
  } else {
    TDMD_VEC_DISPATCH(vec_rows(nl), TDMD_TUNE_DISPATCH(tn, {
      if (mixed_)
        launch(k_morse_atom_pe<GeoQB, L, U, V>, nblk, kThreads, 0, s,
               GeoQB{q_.data(), rep_.data(), scales_.data()}, nl, n, m32_, pe_atom_.data());
      else
        launch(k_morse_atom_pe<GeoD4B, L, U, V>, nblk, kThreads, 0, s,
               GeoD4B{pos4_.data(), rep_.data(), imgs_.data()}, nl, n, m64_, pe_atom_.data());
    }));
    TDMD_LAUNCH_CHECK();
  }
  launches_ += 1;
  rep_energy();
  TDMD_CU(cudaMemcpyAsync(out, eout_.data(), sizeof(double) * 2 * nrep_, cudaMemcpyDeviceToHost,
                          s));
  TDMD_CU(cudaStreamSynchronize(s));
}

// Per-replica (PE, KE) from pe_atom_ and the velocities, into eout_.
void Batch::rep_energy() {
  launch(k_rep_energy, nrep_, kThreads, 0, stream_, pe_atom_.data(), vel_.data(), types_.data(),
         masses_.data(), reps_.data(), eout_.data());
  TDMD_LAUNCH_CHECK();
  ++launches_;
}

void Batch::energies(double* pe, double* ke) {
  TDMD_REQUIRE(uploaded_, "energies before upload");
  std::vector<double> e(2 * static_cast<size_t>(nrep_), 0.0);
  if (n_ > 0) {
    if (!initialized_) initial_forces();
    reduce_energies(e.data());
  }
  for (int r = 0; r < nrep_; ++r) {
    if (pe) pe[r] = e[2 * static_cast<size_t>(r)];
    if (ke) ke[r] = e[2 * static_cast<size_t>(r) + 1];
  }
}

void Batch::energy_log(double* steps, double* pe_ke, int cap, int* count) const {
  const int m = static_cast<int>(log_steps_.size());
  if (count) *count = m;
  const int k = std::min(m, std::max(cap, 0));
  for (int i = 0; i < k; ++i) {
    if (steps) steps[i] = log_steps_[static_cast<size_t>(i)];
    if (pe_ke)
      std::copy(log_.begin() + static_cast<long>(2 * nrep_) * i,
                log_.begin() + static_cast<long>(2 * nrep_) * (i + 1),
                pe_ke + static_cast<long>(2 * nrep_) * i);
  }
}

}  // namespace tdmd_b200

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace tdmd_b200;

struct tdmd_batch {
  Batch b;
  tdmd_batch(int nrep, const tdmd_box* boxes, const int* natoms, const tdmd_morse_params* p,
             const tdmd_eam* e, const tdmd_fast_pipeline_config& cfg)
      : b(nrep, boxes, natoms, p, e, cfg) {}
};

extern "C" {

int32_t tdmd_batch_create_morse(int32_t nreplicas, const tdmd_box* boxes, const int32_t* natoms,
                                const tdmd_morse_params* params,
                                const tdmd_fast_pipeline_config* cfg, tdmd_batch** out) {
  return guarded([&] {
    TDMD_REQUIRE(out && params && cfg, "null argument");
    *out = new tdmd_batch(nreplicas, boxes, natoms, params, nullptr, *cfg);
  });
}

int32_t tdmd_batch_create_eam(int32_t nreplicas, const tdmd_box* boxes, const int32_t* natoms,
                              const tdmd_eam* eam, const tdmd_fast_pipeline_config* cfg,
                              tdmd_batch** out) {
  return guarded([&] {
    TDMD_REQUIRE(out && eam && cfg, "null argument");
    *out = new tdmd_batch(nreplicas, boxes, natoms, nullptr, eam, *cfg);
  });
}

int32_t tdmd_batch_destroy(tdmd_batch* b) {
  delete b;
  return TDMD_OK;
}

int32_t tdmd_batch_upload(tdmd_batch* b, const double* positions, const double* velocities,
                          const int32_t* types, const double* masses, int32_t n_types) {
  return guarded([&] {
    TDMD_REQUIRE(b, "null handle");
    b->b.upload(positions, velocities, types, masses, n_types);
  });
}

int32_t tdmd_batch_run_until(tdmd_batch* b, int32_t target_step) {
  return guarded([&] {
    TDMD_REQUIRE(b, "null handle");
    b->b.run_until(target_step);
  });
}

int32_t tdmd_batch_download(const tdmd_batch* b, double* positions, double* velocities,
                            void* forces) {
  return guarded([&] {
    TDMD_REQUIRE(b, "null handle");
    b->b.download(positions, velocities, forces);
  });
}

int32_t tdmd_batch_energies(tdmd_batch* b, double* pe, double* ke) {
  return guarded([&] {
    TDMD_REQUIRE(b, "null handle");
    b->b.energies(pe, ke);
  });
}

int32_t tdmd_batch_energy_log(const tdmd_batch* b, double* steps, double* pe_ke, int32_t cap,
                              int32_t* count) {
  return guarded([&] {
    TDMD_REQUIRE(b, "null handle");
    b->b.energy_log(steps, pe_ke, cap, count);
  });
}

int32_t tdmd_batch_stats(const tdmd_batch* b, tdmd_fast_pipeline_stats* out) {
  return guarded([&] {
    TDMD_REQUIRE(b && out, "null argument");
    b->b.stats(out);
  });
}

int32_t tdmd_batch_info(const tdmd_batch* b, int32_t* nreplicas, int64_t* natoms_total,
                        int32_t* lanes_per_atom, int32_t* current_step) {
  return guarded([&] {
    TDMD_REQUIRE(b, "null handle");
    if (nreplicas) *nreplicas = b->b.nreplicas();
    if (natoms_total) *natoms_total = b->b.natoms();
    if (lanes_per_atom) *lanes_per_atom = b->b.lanes();
    if (current_step) *current_step = b->b.step();
  });
}

int32_t tdmd_batch_autotune(tdmd_batch* b, int32_t* lanes2, int32_t* batch2, double* ms24) {
  return guarded([&] {
    TDMD_REQUIRE(b, "null handle");
    int l[2] = {0, 0}, u[2] = {0, 0};
    b->b.autotune(l, u, ms24);
    for (int k = 0; k < 2; ++k) {
      if (lanes2) lanes2[k] = l[k];
      if (batch2) batch2[k] = u[k];
    }
  });
}

int32_t tdmd_batch_last_window_ms(const tdmd_batch* b, double* ms) {
  return guarded([&] {
    TDMD_REQUIRE(b && ms, "null argument");
    *ms = b->b.last_window_ms();
  });
}

int32_t tdmd_batch_stream(const tdmd_batch* b, void** stream) {
  return guarded([&] {
    TDMD_REQUIRE(b && stream, "null argument");
    *stream = reinterpret_cast<void*>(b->b.stream());
  });
}

}  // extern "C"
