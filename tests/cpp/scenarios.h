// Simulation scenarios written only against the public GO_Fish / Sim_Model / Spectrum API.
//
// The same source is compiled twice: against the reference's own headers (oracle/ref_driver.cu,
// nvcc, for the bit-exact oracle run on the GPU) and against this library's drop-in headers
// (tests/cpp/gofish_driver.cpp, plain g++), so the two programs differ only in the library behind
// the API.  Each scenario takes key=value parameters and the driver writes every time sample, the
// mutation IDs and the requested spectra to one binary dump (format in dump_results below; reader in
// tests/gfdump.py).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

// Test harness only: both libraries keep the arrays of a time sample private, and the only public way
// to start a run from a given state is prev_sim.  To start the reference and the drop-in from one
// identical stored state (save_state / load_state below), the harness opens the private members of
// allele_trajectories, whose names are the same in both header sets.  Nothing else depends on this.
#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif
#define private public
#include "go_fish.cuh"
#include "spectrum.h"
#undef private

#ifdef __CUDACC__
#define SCN_HD __host__ __device__
#define SCN_D __device__
#else
#define SCN_HD
#define SCN_D
#endif

namespace scn {

struct Args {
  std::map<std::string, std::string> kv;
  Args(int argc, char** argv, int first) {
    for (int i = first; i < argc; ++i) {
      std::string s(argv[i]);
      const size_t eq = s.find('=');
      if (eq != std::string::npos) kv[s.substr(0, eq)] = s.substr(eq + 1);
    }
  }
  double num(const char* k, double def) const {
    auto it = kv.find(k);
    return it == kv.end() ? def : std::strtod(it->second.c_str(), nullptr);
  }
  long long integer(const char* k, long long def) const {
    auto it = kv.find(k);
    return it == kv.end() ? def : std::strtoll(it->second.c_str(), nullptr, 0);
  }
  std::string str(const char* k, const char* def) const {
    auto it = kv.find(k);
    return it == kv.end() ? std::string(def) : it->second;
  }
};

// take a time sample every `k` generations after `start` (and never at `start` itself)
struct every_k {
  int k;
  int start;
  every_k(int k = 0, int start = 0) : k(k), start(start) {}
  bool operator()(const int g) const { return k > 0 && g > start && ((g - start) % k) == 0; }
};

// Three populations: pop 0 is the ancestor (N0 individuals), pop 1 splits off at split1 and pop 2 at
// split2, each founded by N0 individuals drawn from pop 0 and growing logistically at `rate` to its
// own carrying capacity.
struct split_demography {
  int N0;
  float rate;
  int split1, split2;
  int K0, K1, K2;
  SCN_HD int logistic(int K, int t) const {
    const float term = expf(rate * t);
    return (int)roundf(static_cast<float>(K) * N0 * term / (K + N0 * (term - 1)));
  }
  SCN_HD int operator()(const int pop, const int gen) const {
    if (pop == 0) return logistic(K0, gen);
    if (pop == 1) return gen >= split1 ? logistic(K1, gen - split1) : 0;
    return gen >= split2 ? logistic(K2, gen - split2) : 0;
  }
};

// At a population's split generation all of its chromosomes come from pop 0; otherwise existing
// populations exchange migrants symmetrically at rate m.
struct split_migration {
  float m;
  int split1, split2;
  SCN_HD bool exists(int pop, int gen) const { return pop == 0 || (pop == 1 ? gen >= split1 : gen >= split2); }
  SCN_HD bool founding(int pop, int gen) const { return (pop == 1 && gen == split1) || (pop == 2 && gen == split2); }
  SCN_HD float operator()(const int from, const int to, const int gen) const {
    if (!exists(to, gen)) return from == to ? 1.f : 0.f;
    if (founding(to, gen)) return from == 0 ? 1.f : 0.f;
    if (!exists(from, gen) || founding(from, gen)) return 0.f;
    int live = 0;
    for (int p = 0; p < 3; ++p) live += (exists(p, gen) && !founding(p, gen)) ? 1 : 0;
    if (from == to) return 1.f - (live - 1) * m;
    return m;
  }
};

// ---------------------------------------------------------------------------------------------
// scenario "wf": one population (or several identical ones), constant size, constant selection
// ---------------------------------------------------------------------------------------------
template <typename Selection>
inline void run_wf(GO_Fish::allele_trajectories& a, const Args& args, const GO_Fish::allele_trajectories* prev,
                   const Sim_Model::F_mu_h_constant& mutation, const Sim_Model::demography_constant& demography,
                   const Sim_Model::migration_constant_equal& migration, const Selection& selection,
                   const Sim_Model::F_mu_h_constant& inbreeding, const Sim_Model::F_mu_h_constant& dominance) {
  every_k sample(static_cast<int>(args.integer("sample_every", 0)), 0);
  if (prev) {  // continue from sample 0 of a stored state (see load_state)
    a.sim_input_constants.init_mse = false;
    a.sim_input_constants.prev_sim_sample = 0;
    GO_Fish::run_sim(a, mutation, demography, migration, selection, inbreeding, dominance, Sim_Model::bool_off(),
                     sample, *prev);
  } else {
    GO_Fish::run_sim(a, mutation, demography, migration, selection, inbreeding, dominance, Sim_Model::bool_off(),
                     sample);
  }
}

// A user selection model that is not affine in frequency, s(x) = a x^2 + b, written against the
// reference's functor contract (a __device__ call operator, template_inline_simulation_functors.cuh:36-38).
struct quadratic_selection {
  float a, b;
  SCN_D float operator()(const int population, const int generation, const float freq) const {
    return a * freq * freq + b;
  }
};

// Selection is selection_constant(gamma); with sine_A != 0 the seasonal model
// selection_sine_wave(sine_A, sine_pi, gamma, rho = sine_rho); with quad_a != 0 the user model
// quadratic_selection(quad_a / 2N, gamma / 2N) -- all scaled by the population size.
inline void scenario_wf(GO_Fish::allele_trajectories& a, const Args& args,
                        const GO_Fish::allele_trajectories* prev = NULL) {
  using namespace Sim_Model;
  a.sim_input_constants.seed1 = static_cast<int>(args.integer("seed1", 0xbeef));
  a.sim_input_constants.seed2 = static_cast<int>(args.integer("seed2", 0xdecaf));
  a.sim_input_constants.num_generations = static_cast<int>(args.integer("gens", 1000));
  a.sim_input_constants.num_sites = static_cast<float>(args.num("L", 2e7));
  a.sim_input_constants.num_populations = static_cast<int>(args.integer("pops", 1));
  a.sim_input_constants.init_mse = args.integer("mse", 1) != 0;
  a.sim_input_constants.compact_interval = static_cast<int>(args.integer("compact", 35));
  const int P = a.sim_input_constants.num_populations;
  F_mu_h_constant mutation(static_cast<float>(args.num("mu", 1e-9)));
  F_mu_h_constant inbreeding(static_cast<float>(args.num("F", 0.0)));
  demography_constant demography(static_cast<int>(args.integer("N", 10000)));
  migration_constant_equal migration(static_cast<float>(args.num("m", 0.0)), P);
  F_mu_h_constant dominance(static_cast<float>(args.num("h", 0.5)));
  const float gamma = static_cast<float>(args.num("gamma", 0.0));
  const float sine_A = static_cast<float>(args.num("sine_A", 0.0));
  const float quad_a = static_cast<float>(args.num("quad_a", 0.0));
  if (quad_a != 0.f) {
    const float twoN = 2.f * static_cast<float>(args.integer("N", 10000));
    quadratic_selection selection = {quad_a / twoN, gamma / twoN};
    run_wf(a, args, prev, mutation, demography, migration, selection, inbreeding, dominance);
  } else if (sine_A != 0.f) {
    selection_sine_wave selection(sine_A, static_cast<float>(args.num("sine_pi", 0.05)), gamma, demography, inbreeding,
                                  static_cast<float>(args.num("sine_rho", 0.0)));
    const int sine_pop = static_cast<int>(args.integer("sine_pop", -1));
    if (sine_pop >= 0) {  // seasonal selection in one population, constant in the others
      selection_population_specific<selection_constant, selection_sine_wave> specific(
          selection_constant(gamma, demography, inbreeding), selection, sine_pop);
      run_wf(a, args, prev, mutation, demography, migration, specific, inbreeding, dominance);
    } else {
      run_wf(a, args, prev, mutation, demography, migration, selection, inbreeding, dominance);
    }
  } else {
    selection_constant selection(gamma, demography, inbreeding);
    run_wf(a, args, prev, mutation, demography, migration, selection, inbreeding, dominance);
  }
}

// ---------------------------------------------------------------------------------------------
// scenario "compilation": two inbred populations (N = 1000, F = 1) with migration 0.005 start
// blank, run a burn-in with weakly deleterious mutations (s = -1/1000), then continue for `gens2`
// generations from the burn-in's final sample with beneficial selection (s = +20/1000) in
// population 1, sampling the starting generation.
// ---------------------------------------------------------------------------------------------
inline void scenario_compilation(GO_Fish::allele_trajectories& a, const Args& args) {
  using namespace Sim_Model;
  a.sim_input_constants.seed1 = static_cast<int>(args.integer("seed1", 0xbeeff00d));
  a.sim_input_constants.seed2 = static_cast<int>(args.integer("seed2", 0xdecafbad));
  a.sim_input_constants.num_sites = static_cast<float>(args.num("L", 2e8));
  a.sim_input_constants.num_populations = 2;
  a.sim_input_constants.init_mse = false;
  F_mu_h_constant mutation(1e-9f);
  F_mu_h_constant inbreeding(1.f);
  demography_constant demography(1000);
  migration_constant_equal migration(static_cast<float>(args.num("m", 0.005)), 2);
  selection_constant deleterious(-1.f / 1000.f);
  F_mu_h_constant dominance(0.f);
  a.sim_input_constants.compact_interval = static_cast<int>(args.integer("compact", 100));
  a.sim_input_constants.num_generations = static_cast<int>(args.integer("gens1", 20000));
  GO_Fish::run_sim(a, mutation, demography, migration, deleterious, inbreeding, dominance, bool_off(), bool_off());
  bool_pulse<bool_off, bool_on> sample_start(bool_off(), bool_on(), 0, a.sim_input_constants.num_generations);
  a.sim_input_constants.num_generations = static_cast<int>(args.integer("gens2", 1000));
  a.sim_input_constants.prev_sim_sample = 0;
  selection_constant beneficial(20.f / 1000.f);
  selection_population_specific<selection_constant, selection_constant> selection(deleterious, beneficial, 1);
  GO_Fish::run_sim(a, mutation, demography, migration, selection, inbreeding, dominance, bool_off(), sample_start, a);
}

// ---------------------------------------------------------------------------------------------
// scenario "split3": three populations split from an ancestor, grow logistically, exchange
// migrants, and switch selection from gamma1 to gamma2 at `switch_gen`; population 2 is inbred.
// ---------------------------------------------------------------------------------------------
inline void scenario_split3(GO_Fish::allele_trajectories& a, const Args& args) {
  using namespace Sim_Model;
  a.sim_input_constants.seed1 = static_cast<int>(args.integer("seed1", 0xbeef));
  a.sim_input_constants.seed2 = static_cast<int>(args.integer("seed2", 0xdecaf));
  a.sim_input_constants.num_generations = static_cast<int>(args.integer("gens", 5000));
  a.sim_input_constants.num_sites = static_cast<float>(args.num("L", 2e8));
  a.sim_input_constants.num_populations = 3;
  a.sim_input_constants.init_mse = args.integer("mse", 1) != 0;
  a.sim_input_constants.compact_interval = static_cast<int>(args.integer("compact", 35));
  split_demography dem;
  dem.N0 = static_cast<int>(args.integer("N0", 10000));
  dem.rate = static_cast<float>(args.num("rate", 0.005));
  dem.split1 = static_cast<int>(args.integer("split1", 1));
  dem.split2 = static_cast<int>(args.integer("split2", 2000));
  dem.K0 = static_cast<int>(args.integer("K0", 100000));
  dem.K1 = static_cast<int>(args.integer("K1", 200000));
  dem.K2 = static_cast<int>(args.integer("K2", 500000));
  split_migration mig;
  mig.m = static_cast<float>(args.num("m", 1e-4));
  mig.split1 = dem.split1;
  mig.split2 = dem.split2;
  F_mu_h_constant mutation(static_cast<float>(args.num("mu", 1e-9)));
  F_mu_h_population_specific<F_mu_h_constant, F_mu_h_constant> inbreeding(
      F_mu_h_constant(0.f), F_mu_h_constant(static_cast<float>(args.num("F2", 0.1))), 2);
  selection_piecewise<selection_constant, selection_constant> selection(
      selection_constant(static_cast<float>(args.num("gamma1", -5.0)), dem, inbreeding),
      selection_constant(static_cast<float>(args.num("gamma2", 2.0)), dem, inbreeding),
      static_cast<int>(args.integer("switch_gen", 3000)));
  F_mu_h_constant dominance(static_cast<float>(args.num("h", 0.3)));
  every_k sample(static_cast<int>(args.integer("sample_every", 500)), 0);
  GO_Fish::run_sim(a, mutation, dem, mig, selection, inbreeding, dominance, bool_off(), sample);
}

// Three populations: pop 0 exists from the start, pop 1 is founded at found1 and pop 2 at found2; each
// starts at N0 individuals and grows exponentially at `rate` per generation until it reaches its cap.
struct capped_growth_demography {
  int N0;
  float rate;
  int found1, found2;
  int cap0, cap1, cap2;
  SCN_HD int operator()(const int pop, const int gen) const {
    const int found = pop == 0 ? 0 : (pop == 1 ? found1 : found2);
    const int cap = pop == 0 ? cap0 : (pop == 1 ? cap1 : cap2);
    if (pop > 0 && gen < found) return 0;
    const float n = static_cast<float>(N0) * expf(rate * static_cast<float>(gen - found));
    return n >= static_cast<float>(cap) ? cap : static_cast<int>(roundf(n));
  }
};

// Pop 1 is founded from pop 0 and pop 2 from pop 1 (all chromosomes of the founding generation come
// from the parent); otherwise existing populations exchange migrants symmetrically at rate m.
struct founder_migration {
  float m;
  int found1, found2;
  SCN_HD bool exists(int pop, int gen) const { return pop == 0 || (pop == 1 ? gen >= found1 : gen >= found2); }
  SCN_HD float operator()(const int from, const int to, const int gen) const {
    if (!exists(to, gen)) return from == to ? 1.f : 0.f;
    if (to == 1 && gen == found1) return from == 0 ? 1.f : 0.f;
    if (to == 2 && gen == found2) return from == 1 ? 1.f : 0.f;
    if (!exists(from, gen)) return 0.f;
    int live = 0;
    for (int p = 0; p < 3; ++p) live += exists(p, gen) ? 1 : 0;
    if (from == to) return 1.f - (live - 1) * m;
    return m;
  }
};

// ---------------------------------------------------------------------------------------------
// scenario "multipop": the three-population benchmark model -- an ancestral population of N0 = 1e4
// at mutation-selection equilibrium, population 1 founded from it at generation 1 and population 2
// from population 1 at generation 2000, each growing at r = 0.005 to a cap (1e5, 2.5e5, 5e5);
// symmetric migration 1e-4, selection gamma -5 switching to +2 at generation 3000 (selection_constant
// scaled by the ancestral size), h = 0.3, F = 0.1 in population 2, mu = 1e-9, L = 2e8, compaction
// every 35 generations and a time sample every 500.  With a stored start (prev) the run continues
// from that state's generation for `gens` more generations.
// ---------------------------------------------------------------------------------------------
inline void scenario_multipop(GO_Fish::allele_trajectories& a, const Args& args,
                              const GO_Fish::allele_trajectories* prev = NULL) {
  using namespace Sim_Model;
  a.sim_input_constants.seed1 = static_cast<int>(args.integer("seed1", 0xbeef));
  a.sim_input_constants.seed2 = static_cast<int>(args.integer("seed2", 0xdecaf));
  a.sim_input_constants.num_generations = static_cast<int>(args.integer("gens", 5000));
  a.sim_input_constants.num_sites = static_cast<float>(args.num("L", 2e8));
  a.sim_input_constants.num_populations = 3;
  a.sim_input_constants.init_mse = true;
  a.sim_input_constants.compact_interval = static_cast<int>(args.integer("compact", 35));
  capped_growth_demography dem;
  dem.N0 = static_cast<int>(args.integer("N0", 10000));
  dem.rate = static_cast<float>(args.num("rate", 0.005));
  dem.found1 = static_cast<int>(args.integer("found1", 1));
  dem.found2 = static_cast<int>(args.integer("found2", 2000));
  dem.cap0 = static_cast<int>(args.integer("cap0", 100000));
  dem.cap1 = static_cast<int>(args.integer("cap1", 250000));
  dem.cap2 = static_cast<int>(args.integer("cap2", 500000));
  founder_migration mig;
  mig.m = static_cast<float>(args.num("m", 1e-4));
  mig.found1 = dem.found1;
  mig.found2 = dem.found2;
  F_mu_h_constant mutation(static_cast<float>(args.num("mu", 1e-9)));
  F_mu_h_population_specific<F_mu_h_constant, F_mu_h_constant> inbreeding(
      F_mu_h_constant(0.f), F_mu_h_constant(static_cast<float>(args.num("F2", 0.1))), 2);
  selection_piecewise<selection_constant, selection_constant> selection(
      selection_constant(static_cast<float>(args.num("gamma1", -5.0)), dem, inbreeding),
      selection_constant(static_cast<float>(args.num("gamma2", 2.0)), dem, inbreeding),
      static_cast<int>(args.integer("switch_gen", 3000)));
  F_mu_h_constant dominance(static_cast<float>(args.num("h", 0.3)));
  every_k sample(static_cast<int>(args.integer("sample_every", 500)), 0);
  const float quad_a = static_cast<float>(args.num("quad_a", 0.0));
  if (quad_a != 0.f) {
    // the user model s(x) = quad_a / 2N0 x^2 + gamma1 / 2N0 in every population (continuations only:
    // the equilibrium start integrates affine models)
    const float twoN = 2.f * static_cast<float>(dem.N0);
    quadratic_selection user = {quad_a / twoN, static_cast<float>(args.num("gamma1", -5.0)) / twoN};
    if (prev) {
      a.sim_input_constants.init_mse = false;
      a.sim_input_constants.prev_sim_sample = 0;
      GO_Fish::run_sim(a, mutation, dem, mig, user, inbreeding, dominance, bool_off(), sample, *prev);
    } else {
      GO_Fish::run_sim(a, mutation, dem, mig, user, inbreeding, dominance, bool_off(), sample);
    }
    return;
  }
  if (prev) {
    a.sim_input_constants.init_mse = false;
    a.sim_input_constants.prev_sim_sample = 0;
    GO_Fish::run_sim(a, mutation, dem, mig, selection, inbreeding, dominance, bool_off(), sample, *prev);
  } else {
    GO_Fish::run_sim(a, mutation, dem, mig, selection, inbreeding, dominance, bool_off(), sample);
  }
}

// ---------------------------------------------------------------------------------------------
// scenario "dadi": the two-population model the reference validates against a diffusion solution
// (examples/example_dadi/run.cu): population 0 starts at mutation-selection equilibrium with N
// individuals and doubles at generation 1; population 1 splits off at generation 100 with 0.05 N
// individuals drawn from population 0 and grows exponentially to 5 N by generation 1000; migration
// 1/(2N) between them from generation 101; gamma = -4, h = 0.5, F = 0, mu = 1e-9, L = 2e9,
// compaction every 30.  Replicate j uses seeds (0xbeeff00d + 2j, 0xdecafbad - 2j).  The SFS is
// population 1's, n = 1001, at the final generation.
// ---------------------------------------------------------------------------------------------
inline void scenario_dadi(GO_Fish::allele_trajectories& b, const Args& args, int rep) {
  typedef Sim_Model::demography_constant dem_const;
  typedef Sim_Model::demography_population_specific<dem_const, dem_const> dem_pop_const;
  typedef Sim_Model::demography_piecewise<dem_pop_const, dem_pop_const> init_expansion;
  typedef Sim_Model::demography_exponential_growth exp_growth;
  typedef Sim_Model::demography_population_specific<dem_const, exp_growth> dem_pop_const_exp;
  typedef Sim_Model::migration_constant_equal mig_const;
  typedef Sim_Model::migration_constant_directional<mig_const> mig_dir;
  typedef Sim_Model::migration_constant_directional<mig_dir> mig_split;
  typedef Sim_Model::migration_piecewise<mig_const, mig_split> split_pop0;
  b.sim_input_constants.num_populations = 2;
  b.sim_input_constants.num_generations = 1001;
  Sim_Model::F_mu_h_constant codominant(0.5f);
  Sim_Model::F_mu_h_constant outbred(0.f);
  Sim_Model::F_mu_h_constant mutation(1e-9f);
  const int N = static_cast<int>(args.integer("N", 10000));
  dem_const pop0(N), pop1(0), pop0_final(2 * N);
  dem_pop_const gen0(pop0, pop1, 1), gen1(pop0_final, pop1, 1);
  init_expansion gen_0_1(gen0, gen1, 1);
  exp_growth pop1_growth(std::log(100.f) / 900.f, static_cast<int>(0.05 * N), 100);
  dem_pop_const_exp gen100(pop0_final, pop1_growth, 1);
  Sim_Model::demography_piecewise<init_expansion, dem_pop_const_exp> demography(gen_0_1, gen100, 100);
  mig_const none;
  mig_dir no_pop1(0.f, 1, 1, none);
  mig_split found_pop1(1.f, 0, 1, no_pop1);
  split_pop0 split(none, found_pop1, 100);
  mig_const equal(1.f / (2.f * N), 2);
  Sim_Model::migration_piecewise<split_pop0, mig_const> migration(split, equal, 101);
  Sim_Model::selection_constant weak_del(-4.f, demography, outbred);
  b.sim_input_constants.compact_interval = static_cast<int>(args.integer("compact", 30));
  b.sim_input_constants.num_sites = static_cast<float>(args.num("L", 2e9));
  b.sim_input_constants.seed1 = static_cast<int>(0xbeeff00d + 2 * rep);
  b.sim_input_constants.seed2 = static_cast<int>(0xdecafbad - 2 * rep);
  GO_Fish::run_sim(b, mutation, demography, migration, weak_del, outbred, codominant, Sim_Model::bool_off(),
                   Sim_Model::bool_off());
}

// Runs `reps` replicates of scenario "dadi" and writes, per allele count i = 1 .. n-1, the mean and
// standard deviation over replicates of SFS[i] / (num_sites - SFS[0]) (the reference example's
// table), then one line per replicate with its raw SFS.
inline void dadi_table(const Args& args, const char* path) {
  const int reps = static_cast<int>(args.integer("reps", 50));
  const int n = static_cast<int>(args.integer("sfs_n", 1001));
  std::vector<std::vector<float>> res(reps, std::vector<float>(n));
  GO_Fish::allele_trajectories b;
  Spectrum::SFS sfs;
  for (int j = 0; j < reps; ++j) {
    scenario_dadi(b, args, j);
    Spectrum::site_frequency_spectrum(sfs, b, 0, 1, n);
    for (int i = 0; i < n; ++i) res[j][i] = sfs.frequency_spectrum[i];
  }
  FILE* f = std::fopen(path, "w");
  const double L = static_cast<double>(b.num_sites());
  for (int i = 1; i < n; ++i) {
    double avg = 0, var = 0;
    for (int j = 0; j < reps; ++j) avg += res[j][i] / (reps * (L - res[j][0]));
    for (int j = 0; j < reps; ++j) var += std::pow(res[j][i] / (L - res[j][0]) - avg, 2) / (reps - 1);
    std::fprintf(f, "%d\t%.9g\t%.9g\n", i, avg, std::sqrt(var));
  }
  for (int j = 0; j < reps; ++j) {
    std::fprintf(f, "rep%d", j);
    for (int i = 0; i < n; ++i) std::fprintf(f, "\t%.9g", res[j][i]);
    std::fprintf(f, "\n");
  }
  std::fclose(f);
}

// ---------------------------------------------------------------------------------------------
// stored states: the final time sample of a run, written so that another run -- of either library --
// can start from exactly that state through prev_sim.  Format (int32 little-endian words, float32
// arrays): 'GFS1' P num_sites(float) generation M Nc[P] extinct[P] freq[P*M] ids[M*4]; the IDs are
// stored raw, with the sign that marks a preserved mutation.
// ---------------------------------------------------------------------------------------------
inline void put(FILE* f, int32_t v);

inline void save_state(GO_Fish::allele_trajectories& a, const char* path) {
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    std::perror(path);
    std::exit(2);
  }
  const int P = a.sim_run_constants.num_populations;
  const int s = a.num_samples - 1;
  const int M = a.time_samples[s]->num_mutations;
  std::fwrite("GFS1", 1, 4, f);
  put(f, P);
  const float L = a.sim_run_constants.num_sites;
  std::fwrite(&L, sizeof(float), 1, f);
  put(f, a.time_samples[s]->sampled_generation);
  put(f, M);
  for (int p = 0; p < P; ++p) put(f, a.time_samples[s]->Nchrom_e[p]);
  for (int p = 0; p < P; ++p) put(f, a.time_samples[s]->extinct[p] ? 1 : 0);
  if (M) std::fwrite(a.time_samples[s]->mutations_freq, sizeof(float), static_cast<size_t>(P) * M, f);
  if (M) std::fwrite(a.mutations_ID, sizeof(GO_Fish::mutID), M, f);
  std::fclose(f);
}

inline void load_state(GO_Fish::allele_trajectories& a, const char* path) {
  FILE* f = std::fopen(path, "rb");
  char magic[4];
  int32_t P, gen, M;
  float L;
  if (!f || std::fread(magic, 1, 4, f) != 4 || std::memcmp(magic, "GFS1", 4) != 0 || std::fread(&P, 4, 1, f) != 1 ||
      std::fread(&L, 4, 1, f) != 1 || std::fread(&gen, 4, 1, f) != 1 || std::fread(&M, 4, 1, f) != 1) {
    std::fprintf(stderr, "load_state: cannot read %s\n", path);
    std::exit(2);
  }
  a.sim_input_constants.num_populations = P;
  a.sim_input_constants.num_sites = L;
  a.initialize_sim_result_vector(1);
  GO_Fish::allele_trajectories::time_sample* t = a.time_samples[0];
  t->sampled_generation = gen;
  t->num_mutations = M;
  t->Nchrom_e = new int[P];
  t->extinct = new bool[P];
  t->mutations_freq = new float[static_cast<size_t>(P) * std::max(M, 1)];
  std::vector<int32_t> w(2 * static_cast<size_t>(P));
  bool ok = std::fread(w.data(), 4, w.size(), f) == w.size();
  for (int p = 0; p < P; ++p) {
    t->Nchrom_e[p] = w[p];
    t->extinct[p] = w[P + p] != 0;
  }
  ok = ok && std::fread(t->mutations_freq, sizeof(float), static_cast<size_t>(P) * M, f) == static_cast<size_t>(P) * M;
  a.mutations_ID = static_cast<GO_Fish::mutID*>(std::malloc(sizeof(GO_Fish::mutID) * std::max(M, 1)));
  ok = ok && std::fread(a.mutations_ID, sizeof(GO_Fish::mutID), M, f) == static_cast<size_t>(M);
  a.all_mutations = M;
  std::fclose(f);
  if (!ok) {
    std::fprintf(stderr, "load_state: %s is truncated\n", path);
    std::exit(2);
  }
}

// Runs a scenario.  key=value options shared by every scenario: state_in=<path> continues from a
// stored state (scenarios wf and multipop), state_out=<path> stores the run's final sample.  The
// stored state is loaded into the result object itself, which is then passed as prev_sim too, as the
// reference's example_compilation does: the reference accepts prev_sim_sample only below the sample
// count of the object receiving the results (go_fish_impl.cuh:602), so a fresh result object could
// not continue from another object's sample there.
inline bool run_scenario(const std::string& name, GO_Fish::allele_trajectories& a, const Args& args) {
  const std::string state_in = args.str("state_in", "");
  if (!state_in.empty()) load_state(a, state_in.c_str());
  const GO_Fish::allele_trajectories* start = state_in.empty() ? NULL : &a;
  if (name == "wf") scenario_wf(a, args, start);
  else if (name == "multipop") scenario_multipop(a, args, start);
  else if (name == "compilation") scenario_compilation(a, args);
  else if (name == "split3") scenario_split3(a, args);
  else return false;
  const std::string state_out = args.str("state_out", "");
  if (!state_out.empty()) save_state(a, state_out.c_str());
  return true;
}

// ---------------------------------------------------------------------------------------------
// binary dump: int32 little-endian words and float32 arrays
//   'GFD1' P S
//   per sample: generation M Nc[P] extinct[P] freq[P*M]
//   A ids[A*4]
//   K, then K spectra: sample pop kind(0 = SFS, 1 = histogram) n len values[len]
// ---------------------------------------------------------------------------------------------
inline void put(FILE* f, int32_t v) { std::fwrite(&v, sizeof(v), 1, f); }

inline void dump_results(GO_Fish::allele_trajectories& a, const Args& args, const char* path) {
  const std::string text = args.str("text", "");
  if (!text.empty()) {  // the library's own text dump, operator<<(ostream&, allele_trajectories&)
    std::ofstream out(text.c_str());
    out << a;
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    std::perror(path);
    std::exit(2);
  }
  const int P = a.num_populations();
  const int S = a.num_time_samples();
  std::fwrite("GFD1", 1, 4, f);
  put(f, P);
  put(f, S);
  for (int s = 0; s < S; ++s) {
    const int M = a.num_mutations_time_sample(s);
    put(f, a.sampled_generation(s));
    put(f, M);
    for (int p = 0; p < P; ++p) put(f, a.effective_number_of_chromosomes(s, p));
    for (int p = 0; p < P; ++p) put(f, a.extinct(s, p) ? 1 : 0);
    std::vector<float> row(static_cast<size_t>(M));
    for (int p = 0; p < P; ++p) {
      for (int i = 0; i < M; ++i) row[i] = a.frequency(s, p, i);
      if (M) std::fwrite(row.data(), sizeof(float), M, f);
    }
  }
  const int A = a.maximal_num_mutations();
  put(f, A);
  for (int i = 0; i < A; ++i) {
    const GO_Fish::mutID id = a.mutation_ID(i);
    put(f, id.origin_generation);
    put(f, id.origin_population);
    put(f, id.origin_threadID);
    put(f, id.reserved);
  }
  const int n = static_cast<int>(args.integer("sfs_n", 0));
  const bool hist = args.integer("hist", 0) != 0;
  std::vector<std::vector<int>> specs;
  for (int s = 0; s < S; ++s)
    for (int p = 0; p < P; ++p) {
      const int Nc = a.effective_number_of_chromosomes(s, p);
      if (Nc <= 1) continue;
      if (n > 0 && n < Nc) specs.push_back({s, p, 0, n});
      if (hist) specs.push_back({s, p, 1, Nc});
    }
  put(f, static_cast<int32_t>(specs.size()));
  for (const auto& sp : specs) {
    Spectrum::SFS sfs;
    if (sp[2] == 0) Spectrum::site_frequency_spectrum(sfs, a, sp[0], sp[1], sp[3]);
    else Spectrum::population_frequency_histogram(sfs, a, sp[0], sp[1]);
    const int len = sfs.sample_size[0];
    put(f, sp[0]);
    put(f, sp[1]);
    put(f, sp[2]);
    put(f, sp[3]);
    put(f, len);
    std::fwrite(sfs.frequency_spectrum, sizeof(float), len, f);
  }
  std::fclose(f);
}

}  // namespace scn
