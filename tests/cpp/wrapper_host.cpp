// Compiles against include/tdmd_b200.hpp the way reference code would (same
// class names and signatures) and exercises the parts that need no GPU:
// config defaults, setfl parsing, the host Nose-Hoover chain, the io
// readers and writers, and error translation.  Prints one "key value" pair per line for the Python test.
#include <cstdio>
#include <string>

#include "tdmd_b200.hpp"

int main(int argc, char** argv) {
  if (argc < 2) return 2;
  using namespace tdmd;
  scheduler::FastPipelineConfig cfg{real(0.001), real(0.3), 10};
  const tdmd_fast_pipeline_config c = cfg.to_c();
  std::printf("dt %.17g\nskin %.17g\nrebuild %d\nprecision %d\n", c.dt, c.r_skin,
              c.rebuild_every, c.precision);

  potentials::EamAlloy eam;
  eam.read_setfl(argv[1]);
  std::printf("ntypes %d\ncutoff %.17g\n", eam.ntypes(), static_cast<double>(eam.cutoff()));

  integrator::NoseHooverChain nhc(integrator::NHCConfig{real(300.0), real(0.1), 3}, real(0.001),
                                  765);
  std::printf("scale0 %.17g\n", static_cast<double>(nhc.half_step(12.0)));
  nhc.set_t_target(real(400.0));
  std::printf("t_target %.17g\n", static_cast<double>(nhc.t_target()));

  // tdmd::io: data file in, out and back; force dump; setfl written back
  if (argc >= 4) {
    SystemState s = io::read_lammps_data(argv[2]);
    std::printf("natoms %lld\nmass1 %.17g\nx0 %.17g\n", static_cast<long long>(s.natoms),
                static_cast<double>(s.masses[1]), s.positions[0].x);
    const std::string out = argv[3];
    io::write_lammps_data(s, out + ".data");
    const SystemState r = io::read_lammps_data(out + ".data");
    bool same = r.natoms == s.natoms && r.masses == s.masses;
    for (size_t i = 0; same && i < s.positions.size(); ++i)
      same = r.positions[i].x == s.positions[i].x && r.positions[i].y == s.positions[i].y &&
             r.positions[i].z == s.positions[i].z && r.velocities[i].x == s.velocities[i].x &&
             r.types[i] == s.types[i] && r.ids[i] == s.ids[i];
    std::printf("data_roundtrip %d\n", same ? 1 : 0);
    for (auto& f : s.forces) f = ForceVec{force_t(1.5), force_t(-2.25), force_t(0.125)};
    s.step = 7;
    io::write_lammps_force_dump(s, out + ".dump");
    const std::vector<io::DumpAtom> d = io::read_lammps_dump(out + ".dump");
    std::printf("dump_n %zu\ndump_fx0 %.17g\ndump_id0 %d\n", d.size(),
                static_cast<double>(d[0].force.x), d[0].id);
    io::write_setfl(eam, out + ".eam.alloy");
    potentials::EamAlloy again;
    again.read_setfl(out + ".eam.alloy");
    std::printf("setfl_cutoff %.17g\n", static_cast<double>(again.cutoff()));
  }

  try {
    potentials::EamAlloy bad;
    bad.read_setfl(std::string(argv[1]) + ".missing");
    std::printf("error none\n");
  } catch (const Error& e) {
    std::printf("error %d\n", e.status());
  }
  return 0;
}
