// Compiles against include/tdmd_b200.hpp the way reference code would (same
// class names and signatures) and exercises the parts that need no GPU:
// config defaults, setfl parsing, the host Nose-Hoover chain and error
// translation.  Prints one "key value" pair per line for the Python test.
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

  try {
    potentials::EamAlloy bad;
    bad.read_setfl(std::string(argv[1]) + ".missing");
    std::printf("error none\n");
  } catch (const Error& e) {
    std::printf("error %d\n", e.status());
  }
  return 0;
}
