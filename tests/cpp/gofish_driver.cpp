// Runs a scenario of scenarios.h through this library's drop-in GO_Fish / Spectrum headers and
// writes the binary dump that tests/gfdump.py reads.  Built with plain g++ (no CUDA compiler):
//   gofish_driver <scenario> <out.bin> key=value ...
#include <chrono>
#include <cstdio>
#include <string>

#include "scenarios.h"

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: gofish_driver <scenario> <out.bin> key=value ...\n");
    return 2;
  }
  scn::Args args(argc, argv, 3);
  if (std::string(argv[1]) == "dadi") {  // replicate table of the two-population validation model
    const auto t0 = std::chrono::steady_clock::now();
    scn::dadi_table(args, argv[2]);
    const auto t1 = std::chrono::steady_clock::now();
    std::printf("sim_ms %.3f\n", std::chrono::duration<double, std::milli>(t1 - t0).count());
    return 0;
  }
  GO_Fish::allele_trajectories a;
  const auto t0 = std::chrono::steady_clock::now();
  if (!scn::run_scenario(argv[1], a, args)) {
    std::fprintf(stderr, "unknown scenario %s\n", argv[1]);
    return 2;
  }
  const auto t1 = std::chrono::steady_clock::now();
  std::printf("sim_ms %.3f\n", std::chrono::duration<double, std::milli>(t1 - t0).count());
  scn::dump_results(a, args, argv[2]);
  return 0;
}
