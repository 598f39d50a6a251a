// tdmd_standalone on the GPU, native: the command line, thermo lines and
// dump files of the reference's driver (src/drivers/tdmd_main.cpp:46-270),
// with the run on FastPipelineScheduler through the C++ layer
// (include/tdmd_b200.hpp) and so through the library's C ABI.
//
// Precision is fixed when the binary is built, as the reference's is:
// -DTDMD_PRECISION_MIXED=1 gives the mixed build, the default is FP64.
//
// Deliberate differences from the reference driver:
//   * the neighbor list is rebuilt every --rebuild-every steps (default 10)
//     on the device instead of on the skin criterion; at the default skin
//     of 1.0 A no pair within the cutoff is missed either way;
//   * PE and KE of a thermo line come from the device energy pass at that
//     integer step (the reference prints the PE of the last force call and
//     the KE of the host velocities, the same quantities).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "tdmd_b200.hpp"

namespace {

constexpr const char* kVersion = "0.7.0-dev (tdmd_claude_b200, native)";

struct RunConfig {
  std::string data_file;
  int nsteps = 1000;
  double dt = 0.001;
  double morse_d = 0.3429, morse_alpha = 1.3588, morse_r0 = 2.866, morse_rc = 9.5;
  std::string eam_file;
  double skin = 1.0;
  int thermo_every = 100;
  std::string dump_forces_file;
  std::string dump_final_file;
  int rebuild_every = 10;
};

void print_usage() {
  std::printf(
      "Usage: tdmd_standalone [options]\n"
      "  --data <file>          LAMMPS data file (required)\n"
      "  --nsteps <N>           Number of steps (default 1000)\n"
      "  --dt <ps>              Time step in ps (default 0.001)\n"
      "  --morse D,alpha,r0,rc  Morse parameters (default 0.3429,1.3588,2.866,9.5)\n"
      "  --eam <setfl-file>     EAM/alloy potential (overrides --morse)\n"
      "  --skin <A>             Neighbor list skin (default 1.0)\n"
      "  --thermo <N>           Print thermo every N steps (default 100)\n"
      "  --dump-forces <file>   Write step-0 forces in LAMMPS dump format\n"
      "  --dump-final <file>    Write final-state dump after main loop\n"
      "  --rebuild-every <R>    Neighbor rebuild interval in steps (default 10)\n"
      "  --version, -v          Print version\n"
      "  --help, -h             Print this help\n");
}

// Thermo line of tdmd_main.cpp:110-123: T = 2 KE / (3 N kB).
void print_thermo(long long step, double pe, double ke, long long natoms) {
  const double te = pe + ke;
  const double temp =
      natoms > 0 ? 2.0 * ke / (3.0 * static_cast<double>(natoms) * tdmd::kBoltzmann) : 0.0;
  std::printf("Step %8lld  PE %20.14f  KE %20.14f  TE %20.14f  T %10.4f\n", step, pe, ke, te,
              temp);
  std::fflush(stdout);
}

// Device PE and KE of the scheduler's current state.
void energies(const tdmd::scheduler::FastPipelineScheduler& s, double& pe, double& ke) {
  tdmd::detail::check(tdmd_sched_energies(s.handle(), &pe, &ke, nullptr));
}

// Positions and forces of the scheduler, in the caller's atom order, into
// `state`, then the reference's dump (id type x y z fx fy fz).
void dump_state(const tdmd::scheduler::FastPipelineScheduler& s, tdmd::SystemState& state,
                long long step, const std::string& path) {
  s.download(state.positions.data(), state.velocities.data(), state.forces.data(), nullptr,
             nullptr, static_cast<tdmd::i32>(state.natoms));
  state.step = step;
  tdmd::io::write_lammps_force_dump(state, path);
}

int run(int argc, char** argv) {
  RunConfig cfg;
  for (int i = 1; i < argc; ++i) {
    const std::string arg{argv[i]};
    if (arg == "--version" || arg == "-v") {
      std::printf("tdmd v%s\n", kVersion);
      return 0;
    }
    if (arg == "--help" || arg == "-h") {
      print_usage();
      return 0;
    }
    const bool has_value = i + 1 < argc;
    if (arg == "--data" && has_value) {
      cfg.data_file = argv[++i];
    } else if (arg == "--nsteps" && has_value) {
      cfg.nsteps = std::atoi(argv[++i]);
    } else if (arg == "--dt" && has_value) {
      cfg.dt = std::atof(argv[++i]);
    } else if (arg == "--skin" && has_value) {
      cfg.skin = std::atof(argv[++i]);
    } else if (arg == "--thermo" && has_value) {
      cfg.thermo_every = std::atoi(argv[++i]);
    } else if (arg == "--dump-forces" && has_value) {
      cfg.dump_forces_file = argv[++i];
    } else if (arg == "--dump-final" && has_value) {
      cfg.dump_final_file = argv[++i];
    } else if (arg == "--morse" && has_value) {
      if (std::sscanf(argv[++i], "%lf,%lf,%lf,%lf", &cfg.morse_d, &cfg.morse_alpha,
                      &cfg.morse_r0, &cfg.morse_rc) != 4) {
        std::fprintf(stderr, "Error: --morse expects D,alpha,r0,rc\n");
        return 1;
      }
    } else if (arg == "--eam" && has_value) {
      cfg.eam_file = argv[++i];
    } else if (arg == "--rebuild-every" && has_value) {
      cfg.rebuild_every = std::atoi(argv[++i]);
    }
  }

  if (cfg.data_file.empty()) {
    std::printf("tdmd v%s\n", kVersion);
    std::printf("  Time-Decomposition Molecular Dynamics engine\n");
    std::printf("  Use --data <file> to run a simulation. --help for options.\n");
    return 0;
  }

  std::printf("tdmd v%s\n", kVersion);
  std::printf("Reading: %s\n", cfg.data_file.c_str());
  tdmd::SystemState state = tdmd::io::read_lammps_data(cfg.data_file);
  const tdmd::Vec3D L = state.box.size();
  std::printf("Atoms: %lld  Types: %zu  Box: %.3f x %.3f x %.3f\n",
              static_cast<long long>(state.natoms), state.masses.size() - 1, L.x, L.y, L.z);

  const bool use_eam = !cfg.eam_file.empty();
  tdmd::potentials::EamAlloy eam;
  if (use_eam) eam.read_setfl(cfg.eam_file);
  const tdmd::real rc = static_cast<tdmd::real>(cfg.morse_rc);
  const tdmd::potentials::MorseParams morse{static_cast<tdmd::real>(cfg.morse_d),
                                            static_cast<tdmd::real>(cfg.morse_alpha),
                                            static_cast<tdmd::real>(cfg.morse_r0), rc, rc * rc};
  tdmd::scheduler::FastPipelineConfig pc{};
  pc.dt = static_cast<tdmd::real>(cfg.dt);
  pc.r_skin = static_cast<tdmd::real>(cfg.skin);
  pc.rebuild_every = cfg.rebuild_every;

  const tdmd::i32 n = static_cast<tdmd::i32>(state.natoms);
  auto sched = use_eam ? std::make_unique<tdmd::scheduler::FastPipelineScheduler>(
                             state.box, n, eam, pc)
                       : std::make_unique<tdmd::scheduler::FastPipelineScheduler>(
                             state.box, n, morse, pc);
  sched->upload(state.positions.data(), state.velocities.data(), nullptr, state.types.data(),
                state.ids.data(), state.masses.data(),
                static_cast<tdmd::i32>(state.masses.size()));
  sched->run_until(0);  // neighbor list and step-0 forces

  if (use_eam)
    std::printf("\nEAM/alloy: %s  cutoff=%.3f A\n", cfg.eam_file.c_str(),
                static_cast<double>(eam.cutoff()));
  else
    std::printf("\nMorse: D=%.4f alpha=%.4f r0=%.3f rc=%.1f\n", cfg.morse_d, cfg.morse_alpha,
                cfg.morse_r0, cfg.morse_rc);
  std::printf("dt=%.4f ps  nsteps=%d  skin=%.1f A\n\n", cfg.dt, cfg.nsteps, cfg.skin);

  double pe = 0.0, ke = 0.0;
  energies(*sched, pe, ke);
  print_thermo(0, pe, ke, state.natoms);
  if (!cfg.dump_forces_file.empty()) {
    dump_state(*sched, state, 0, cfg.dump_forces_file);
    std::printf("Wrote step-0 force dump to %s\n", cfg.dump_forces_file.c_str());
  }

  // Advance to each thermo step in one run_until (one graph-replayed
  // window per rebuild interval inside).
  int step = 0;
  while (step < cfg.nsteps) {
    const int next = cfg.thermo_every > 0
                         ? std::min(cfg.nsteps, (step / cfg.thermo_every + 1) * cfg.thermo_every)
                         : cfg.nsteps;
    sched->run_until(next);
    step = next;
    if (cfg.thermo_every > 0 && step % cfg.thermo_every == 0) {
      energies(*sched, pe, ke);
      print_thermo(step, pe, ke, state.natoms);
    }
  }
  if (cfg.nsteps > 0) {
    energies(*sched, pe, ke);
    std::printf("\nFinal:\n");
    print_thermo(cfg.nsteps, pe, ke, state.natoms);
    // loop rebuilds, as the reference counts them (the initial build excluded)
    std::printf("Neighbor list rebuilds: %lld\n",
                static_cast<long long>(sched->stats().rebuilds - 1));
  }
  if (!cfg.dump_final_file.empty()) {
    dump_state(*sched, state, cfg.nsteps, cfg.dump_final_file);
    std::printf("Wrote final-state dump to %s\n", cfg.dump_final_file.c_str());
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    return run(argc, argv);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "Error: %s\n", e.what());
    return 1;
  }
}
