// scheduler/pipeline_scheduler.cuh -- include-path shim for compiling
// reference callers unchanged.  The TD zone pipeline (PipelineScheduler,
// src/scheduler/pipeline_scheduler.cuh) is outside this library's path: the
// declarations below let a caller that names it compile, and constructing
// one throws tdmd::Error with TDMD_ERR_UNSUPPORTED.  Test infrastructure
// only; not part of the library.
#pragma once
#include "tdmd_b200.hpp"

namespace tdmd {
namespace domain {
struct ZonePartition {
  i32 n_zones() const noexcept { return 0; }
};
}  // namespace domain

namespace scheduler {
struct PipelineConfig {
  real dt{real{0.001}};
  real r_skin{real{1.0}};
  i32 n_zones{0};
  i32 n_streams{4};
  i32 rebuild_every{10};
  bool deterministic{false};
  real t_target{0};
  real t_period{real{0.1}};
  i32 nhc_length{3};
  bool adaptive_dt{false};
  real dt_max{real{0.002}};
  real dt_min{real{0.0001}};
  real c2{real{0.05}};
};

struct PipelineStats {
  i64 kernel_launches{0};
  i64 dep_check_calls{0};
  i64 dep_check_failures{0};
  i64 ticks{0};
};

class PipelineScheduler {
 public:
  PipelineScheduler(const Box&, i32, const potentials::MorseParams&, const PipelineConfig&) {
    throw StatusError(TDMD_ERR_UNSUPPORTED, "the TD zone PipelineScheduler is not part of this library");
  }
  void upload(const PositionVec*, const VelocityVec*, const ForceVec*, const i32*, const i32*,
              const real*, i32) {}
  void run_until(i32) {}
  void download(PositionVec*, VelocityVec*, ForceVec*, i32*, i32*, i32) const {}
  const PipelineStats& stats() const noexcept { return stats_; }
  const domain::ZonePartition& partition() const noexcept { return zones_; }

 private:
  PipelineStats stats_{};
  domain::ZonePartition zones_{};
};
}  // namespace scheduler
}  // namespace tdmd
