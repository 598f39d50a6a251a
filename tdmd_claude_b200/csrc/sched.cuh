// sched.cuh -- the scheduler object behind tdmd_sched (scheduler.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <list>
#include <map>
#include <memory>
#include <vector>

#include "buffers.cuh"
#include "common.cuh"
#include "eam_tables.cuh"
#include "forces.cuh"
#include "integrate.cuh"

namespace tdmd_b200 {

// Device control block: everything the step kernels decide on the device.
struct SchedCtl {
  double dt;      // current time step (adaptive dt writes it)
  double scale;   // pending NHC velocity scale, applied by the next kick
  double ke;      // last reduced kinetic energy (after the thermostat)
  double ev[8];   // energy pass sums: pe, virial xx,yy,zz,xy,xz,yz
  double eta[kMaxChain], eta_v[kMaxChain], eta_m[kMaxChain];
  long long step;  // device step counter (kick-drift increments it)
  int status[4];   // [0] neighbor overflow flag, [1] max neighbor count
  int log_count;
  int pad;
};

struct CtlParams {
  int M;
  int n_dof;
  double t_target, t_period, dt_nhc;
  int adaptive;
  double c2, rc, dt_min, dt_max;
  int nvt;
};

struct StepPlan {
  bool first;      // first step of the run_until window
  bool last;       // last step of the window
  bool rebuild;    // neighbor rebuild after this step's drift
  bool ev;         // energy-log step
  bool kd_fused;   // this step's kick + drift ran inside the previous force pass
  bool fuse_next;  // this step's force pass also kicks and drifts for the next step
};

enum ProfCat : int {
  kProfKickDrift = 0,
  kProfRebuild = 1,
  kProfDensity = 2,  // EAM density + embedding
  kProfForce = 3,    // Morse or EAM force pass
  kProfOther = 4,    // closing kicks, reductions, control
  kProfCount = 5
};

// A phase's timing events: category, start, end.
struct ProfEvents {
  int cat;
  cudaEvent_t a, b;
};

struct GraphEntry {
  cudaGraphExec_t exec = nullptr;
  long long kernels = 0;
  // profiling graphs: the event-record nodes captured around each phase,
  // recorded again by every replay (owned by the entry)
  std::vector<ProfEvents> prof;
};

class Scheduler {
 public:
  Scheduler(const tdmd_box& box, int natoms, const tdmd_fast_pipeline_config& cfg);
  ~Scheduler();
  Scheduler(const Scheduler&) = delete;
  Scheduler& operator=(const Scheduler&) = delete;

  void set_morse(const tdmd_morse_params& p);
  void set_eam(const tdmd_eam& e);
  void upload(const double* x, const double* v, const void* f, const int* types, const int* ids,
              const double* masses, int n_types);
  void download(double* x, double* v, void* f, int* types, int* ids, int natoms) const;
  void run_until(int target);
  void energies(double* pe, double* ke, double* virial6);
  void energy_log(double* rec, int cap, int* count) const;
  void thermostat_state(double* dt, double* eta, double* eta_v) const;
  void stats(tdmd_fast_pipeline_stats* o) const;
  int current_step() const { return step_; }
  int potential_kind() const { return kind_; }
  double interaction_cutoff() const { return cutoff_; }
  cudaStream_t stream() const { return stream_; }
  // Per-kernel timing with CUDA events on the scheduler's stream (disables
  // graph replay while on).  Categories: see ProfCat.
  void set_profiling(bool on);
  // Times the force passes for lanes-per-atom in {1,2,4,8,16,32} on the
  // current state, keeps the fastest, recomputes the forces with it.
  // ms6[k] = ms of candidate 2^k (nullable).
  void autotune(int* lanes2, int* batch2, double* ms24);
  int lanes_per_atom() const { return lpa_; }
  // Device time of the last run_until window (events on the stream around
  // its enqueued work), ms.
  double last_window_ms() const { return last_window_ms_; }
  void kernel_times(double* avg_ms, long long* counts, int ncat) const;
  const int* atom_order() const { return order_.data(); }
  // The current neighbor list in the caller's atom order, as dense CSR on
  // the host (inspection; synchronises the stream).  counts[n] always;
  // neighbors (capacity entries, nullable) the rows back to back.
  void neighbor_list(int* counts, int* neighbors, long long capacity, long long* total) const;
  void device_state(void** pos4, double** vel, void** forces) {
    if (pos4) *pos4 = pos4_.data();
    if (vel) *vel = vel_.data();
    if (forces)
      *forces = mixed_ ? static_cast<void*>(f32_.data()) : static_cast<void*>(f64_.data());
  }

 private:
  void finish_setup();
  int size_neighbor_list();  // returns the cell-list kernels launched
  void grow_capacity(int max_count);
  // defer_check: leave the list build's overflow flag for the window that
  // follows (it keeps the flag, and its retry rebuilds and recomputes)
  void initial_forces(bool defer_check = false);
  void enqueue_rebuild();
  // kd: the force pass also applies the next step's full kick + drift
  // (mixed EAM, NVE; the force pass reads gather records, not positions).
  // parts: which EAM passes (density, pair force); Morse has one pass.
  static constexpr int kPassDensity = 1, kPassForce = 2, kPassBoth = 3;
  void enqueue_force(bool ev, bool kd = false, int parts = kPassBoth);
  // The EAM force passes of both precisions read gather records, never the
  // positions, so they can carry the next step's kick + drift (NVE only).
  bool can_fuse_kick() const { return kind_ == TDMD_POT_EAM && !thermo_; }
  template <class F>
  void enqueue_kick_drift_t(F* f, bool full, bool scale);
  void enqueue_kick_drift(bool full, bool scale);
  template <class F>
  void enqueue_half_kick_t(F* f, bool ke);
  void enqueue_half_kick(bool ke);
  CtlParams ctl_params() const;
  void enqueue_control(int mode);
  void enqueue_ke_pre();
  void enqueue_log_nve();
  void enqueue_apply_scale();
  void enqueue_step(const StepPlan& st);
  void enqueue_finalize();
  // prologue bits of a window's first segment (captured with its steps)
  static constexpr int kPrologueSnapshot = 1;     // state copy for an overflow retry
  static constexpr int kPrologueResetStatus = 2;  // zero the overflow flags
  void run_segment(const std::vector<StepPlan>& seg, bool finalize, int prologue);
  void enqueue_prologue(int prologue);
  std::vector<StepPlan> plan_steps(int target, int* since_out) const;
  void reserve_snapshot();
  void restore();
  void clear_graphs();
  void prof_begin(int cat);
  void prof_end(int cat);
  void prof_collect();
  // bin + scan + scatter + sort
  int cell_list_kernels() const { return 3 + device_scan_launches(cl_.ncells); }
  void reorder_by_cell(cudaEvent_t side_done = nullptr);
  // Keyed cell list of the current positions; returns the kernels launched.
  int build_cells();
  int* ctl_status() const {
    return reinterpret_cast<int*>(reinterpret_cast<char*>(ctl_.data()) +
                                  offsetof(SchedCtl, status));
  }
  double* ctl_ev() const {
    return reinterpret_cast<double*>(reinterpret_cast<char*>(ctl_.data()) +
                                     offsetof(SchedCtl, ev));
  }

  tdmd_box hbox_;
  DevBox box_{};
  int n_;
  tdmd_fast_pipeline_config cfg_;
  int kind_ = -1;
  double cutoff_ = 0.0;
  bool mixed_ = false, nvt_ = false, thermo_ = false;
  int lpa_ = 8;
  int nu_ = kU;  // neighbors per lane per sweep (2 or 4)
  // launch shape of the EAM density pass (lpa_ / nu_: the pair-force pass)
  int lpa_d_ = 8;
  int nu_d_ = kU;
  MorseP<double> m64_{};
  MorseP<float> m32_{};
  std::unique_ptr<EamDevTables> eam_;

  // State (device layouts).
  DevArray<double4> pos4_;
  DevArray<int4> q_;
  DevArray<double> vel_;
  DevArray<double> f64_;
  DevArray<float> f32_;
  DevArray<int> types_, ids_;
  // second buffers of the per-atom state: upload gathers into them and swaps
  DevArray<double4> pos4_alt_;
  DevArray<int4> q_alt_;
  DevArray<double> vel_alt_, f64_alt_;
  DevArray<float> f32_alt_;
  DevArray<int> types_alt_, ids_alt_;
  bool cells_from_upload_ = false;  // cl_ holds the cells of the reordered upload
  DevArray<double> masses_;
  DevArray<double> inv_mm_;  // 1 / (m mvv2e) per type: the kick factor per unit dt
  DevArray<int4> g_;         // mixed EAM: {qx, qy, qz, bits(F'(rho))} per atom
  DevArray<double4> g64_;    // FP64 EAM: {x, y, z, F'(rho)} per atom
  mutable DevArray<double> stage_;
  // Atoms are held in the cell order of the uploaded positions (neighbors of
  // an atom then sit at nearby indices, whatever order the caller used);
  // order_[k] is the caller's index of internal atom k.  Cell lists sort
  // their members by that index, so every neighbor row lists the same atoms
  // in the same order as without the reordering.
  DevArray<int> order_;
  int n_types_ = 0;
  // Largest cell occupancy of the upload (sizes the list build's stage):
  // written by the device into pinned host memory, read after the upload's
  // stream synchronisation.
  DevArray<int> cellmax_;
  int* h_cellmax_ = nullptr;
  int max_cell_ = 0;
  // Upload: velocities, ids and forces come in on a side stream while the
  // positions are binned on stream_ (joined before the cell-order gather);
  // the small per-type and control copies go from a pinned block, so they
  // never hold the host back behind the stream.
  cudaStream_t side_ = nullptr;
  cudaEvent_t up_ev_[2] = {nullptr, nullptr};
  unsigned char* h_stage_ = nullptr;
  size_t h_stage_cap_ = 0;

  // Neighbor list: padded rows of cap_ entries.
  CellListDev cl_;
  DevArray<int> nbr_, cnt_;
  int cap_ = 0;

  // Scratch.
  DevArray<float> fp32_;
  DevArray<double> fp64_;
  DevArray<double> ev_part_, ke_part_;
  DevArray<SchedCtl> ctl_, snap_ctl_;
  DevArray<double> log_;
  int log_cap_ = 0;

  // Snapshot for the overflow retry.
  DevArray<double4> snap_pos4_;
  DevArray<int4> snap_q_;
  DevArray<double> snap_vel_;

  cudaStream_t stream_ = nullptr;
  std::map<std::vector<int>, GraphEntry> graphs_;
  std::list<std::vector<int>> graph_lru_;

  cudaEvent_t win_ev_[2] = {nullptr, nullptr};
  double last_window_ms_ = 0.0;
  bool profiling_ = false;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_pending_;
  // events of replayed profiling graphs awaiting this window's collection,
  // the capture in progress (nullable), and events of evicted graphs freed at
  // the next collection
  std::vector<ProfEvents> prof_graph_pending_;
  std::vector<ProfEvents>* prof_sink_ = nullptr;
  std::vector<ProfEvents> prof_retired_;
  std::vector<cudaEvent_t> prof_pool_;
  cudaEvent_t prof_open_ = nullptr;
  double prof_ms_[kProfCount] = {0, 0, 0, 0, 0};
  long long prof_n_[kProfCount] = {0, 0, 0, 0, 0};

  bool uploaded_ = false, initialized_ = false, tuned_ = false;
  bool init_check_pending_ = false;  // the first list's overflow flag awaits the window
  int step_ = 0, since_rebuild_ = 0;
  long long ticks_ = 0, launches_ = 0, rebuilds_ = 0, graph_launches_ = 0, retries_ = 0;
};

}  // namespace tdmd_b200
