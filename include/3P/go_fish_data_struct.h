/*
 * go_fish_data_struct.h -- GO_Fish output structures of the B200 engine (host-only C++).
 *
 * Source-compatible with ParallelPopGen 3P's go_fish_data_struct.h (go_fish_data_struct.h:35-161,
 * inline definitions in _internal/inline_go_fish_data_struct.hpp:14-281): the same types, members,
 * defaults, accessors, bounds checks and text dump, so code written against the reference compiles
 * unchanged.  Like the reference header it needs no CUDA and can be included from plain C++.
 */
#ifndef GOFISH_B200_GO_FISH_DATA_STRUCT_H_
#define GOFISH_B200_GO_FISH_DATA_STRUCT_H_

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <utility>

namespace Spectrum {
struct SFS;
}
namespace gofish_detail {
struct trajectory_access;
struct spectrum_access;
}

namespace GO_Fish {

/* Identity of one mutation: generation and population of origin, index among that generation's new
 * mutations of that population (1-based), and a reserved word (0).  A negative origin_threadID
 * inside the engine marks a preserved mutation; the accessors report its absolute value. */
struct mutID {
  int origin_generation;
  int origin_population;
  int origin_threadID;
  int reserved;

  inline mutID() : origin_generation(0), origin_population(0), origin_threadID(0), reserved(0) {}
  inline mutID(int g, int p, int t, int r) : origin_generation(g), origin_population(p), origin_threadID(t), reserved(r) {}
  inline std::string toString() const {
    std::ostringstream os;
    os << "(" << origin_generation << "," << origin_population << "," << std::abs(origin_threadID) << "," << reserved
       << ")";
    return os.str();
  }
  inline std::string toString() { return static_cast<const mutID&>(*this).toString(); }
};

/* Control and output structure of a simulation run: input constants, run constants and the time
 * samples (frequencies of every mutation in every population) plus the mutation IDs. */
struct allele_trajectories {
  struct sim_constants {
    int seed1;             /* default 0xbeeff00d */
    int seed2;             /* default 0xdecafbad */
    int num_generations;   /* default 0 */
    float num_sites;       /* default 1000 */
    int num_populations;   /* default 1 */
    bool init_mse;         /* default true */
    int prev_sim_sample;   /* default -1 */
    int compact_interval;  /* default 35; 0 = never compact */
    int device;            /* default -1 */
    inline sim_constants()
        : seed1(static_cast<int>(0xbeeff00d)),
          seed2(static_cast<int>(0xdecafbad)),
          num_generations(0),
          num_sites(1000),
          num_populations(1),
          init_mse(true),
          prev_sim_sample(-1),
          compact_interval(35),
          device(-1) {}
  };

  sim_constants sim_input_constants;

  inline allele_trajectories() : time_samples(NULL), num_samples(0), mutations_ID(NULL), all_mutations(0) {}
  inline allele_trajectories(const allele_trajectories& in);
  inline allele_trajectories& operator=(allele_trajectories in) {
    swap(*this, in);
    return *this;
  }
  inline ~allele_trajectories() { reset(); }

  inline sim_constants last_run_constants() { return sim_run_constants; }
  inline int num_sites() { return static_cast<int>(sim_run_constants.num_sites); }
  inline int num_populations() { return sim_run_constants.num_populations; }
  inline int num_time_samples() { return num_samples; }
  inline int maximal_num_mutations() { return all_mutations; }
  inline int num_mutations_time_sample(int sample_index);
  inline int final_generation() { return sampled_generation(num_samples - 1); }
  inline int sampled_generation(int sample_index);
  inline bool extinct(int sample_index, int population_index);
  inline int effective_number_of_chromosomes(int sample_index, int population_index);
  inline float frequency(int sample_index, int population_index, int mutation_index);
  inline mutID mutation_ID(int mutation_index);
  inline void delete_time_sample(int sample_index);
  inline void reset();

  friend inline void swap(allele_trajectories& a, allele_trajectories& b) {
    std::swap(a.sim_input_constants, b.sim_input_constants);
    std::swap(a.sim_run_constants, b.sim_run_constants);
    std::swap(a.time_samples, b.time_samples);
    std::swap(a.num_samples, b.num_samples);
    std::swap(a.mutations_ID, b.mutations_ID);
    std::swap(a.all_mutations, b.all_mutations);
  }
  friend inline std::ostream& operator<<(std::ostream& stream, allele_trajectories& A);
  friend struct gofish_detail::trajectory_access;
  friend struct gofish_detail::spectrum_access;

 private:
  struct time_sample {
    float* mutations_freq; /* [num_populations][num_mutations] */
    bool* extinct;         /* [num_populations] */
    int* Nchrom_e;         /* [num_populations] */
    int num_mutations;
    int sampled_generation;
    time_sample() : mutations_freq(NULL), extinct(NULL), Nchrom_e(NULL), num_mutations(0), sampled_generation(0) {}
    ~time_sample() {
      delete[] mutations_freq;
      delete[] extinct;
      delete[] Nchrom_e;
    }
  };

  inline void initialize_sim_result_vector(int new_length) {
    sim_constants keep = sim_input_constants;
    reset();
    num_samples = new_length;
    time_samples = new time_sample*[num_samples];
    for (int i = 0; i < num_samples; ++i) time_samples[i] = new time_sample();
    sim_input_constants = keep;
    sim_run_constants = keep;
  }

  static inline void die(const char* what) {
    std::fprintf(stderr, "%s\n", what);
    std::exit(1);
  }

  sim_constants sim_run_constants;
  time_sample** time_samples;
  int num_samples;
  mutID* mutations_ID;
  int all_mutations;
};

inline allele_trajectories::allele_trajectories(const allele_trajectories& in)
    : sim_input_constants(in.sim_input_constants),
      sim_run_constants(in.sim_run_constants),
      time_samples(NULL),
      num_samples(in.num_samples),
      mutations_ID(NULL),
      all_mutations(in.all_mutations) {
  if (all_mutations > 0) {
    mutations_ID = static_cast<mutID*>(std::malloc(sizeof(mutID) * all_mutations));
    std::memcpy(mutations_ID, in.mutations_ID, sizeof(mutID) * all_mutations);
  }
  if (num_samples > 0) {
    const int P = sim_run_constants.num_populations;
    time_samples = new time_sample*[num_samples];
    for (int i = 0; i < num_samples; ++i) {
      const time_sample* src = in.time_samples[i];
      time_sample* dst = new time_sample();
      dst->num_mutations = src->num_mutations;
      dst->sampled_generation = src->sampled_generation;
      dst->Nchrom_e = new int[P];
      dst->extinct = new bool[P];
      for (int p = 0; p < P; ++p) {
        dst->Nchrom_e[p] = src->Nchrom_e[p];
        dst->extinct[p] = src->extinct[p];
      }
      dst->mutations_freq = new float[static_cast<size_t>(P) * src->num_mutations];
      if (src->num_mutations > 0)
        std::memcpy(dst->mutations_freq, src->mutations_freq, sizeof(float) * static_cast<size_t>(P) * src->num_mutations);
      time_samples[i] = dst;
    }
  }
}

inline int allele_trajectories::num_mutations_time_sample(int sample_index) {
  if (!time_samples || num_samples == 0) die("num_mutations error: empty allele_trajectories");
  if (sample_index < 0 || sample_index >= num_samples) {
    std::fprintf(stderr, "num_mutations error: requested sample index out of bounds: sample %d [0 %d)\n", sample_index,
                 num_samples);
    std::exit(1);
  }
  return time_samples[sample_index]->num_mutations;
}

inline int allele_trajectories::sampled_generation(int sample_index) {
  if (!time_samples || num_samples == 0) die("sampled_generation error: empty allele_trajectories");
  if (sample_index < 0 || sample_index >= num_samples) {
    std::fprintf(stderr, "sampled_generation error: requested sample index out of bounds: sample %d [0 %d)\n",
                 sample_index, num_samples);
    std::exit(1);
  }
  return time_samples[sample_index]->sampled_generation;
}

inline bool allele_trajectories::extinct(int sample_index, int population_index) {
  if (!time_samples || num_samples == 0) die("extinct error: empty allele_trajectories");
  const int P = sim_run_constants.num_populations;
  if (sample_index < 0 || sample_index >= num_samples || population_index < 0 || population_index >= P) {
    std::fprintf(stderr, "extinct error: index out of bounds: sample %d [0 %d), population %d [0 %d)\n", sample_index,
                 num_samples, population_index, P);
    std::exit(1);
  }
  return time_samples[sample_index]->extinct[population_index];
}

inline int allele_trajectories::effective_number_of_chromosomes(int sample_index, int population_index) {
  if (!time_samples || num_samples == 0) die("effective_number_of_chromosomes error: empty allele_trajectories");
  const int P = sim_run_constants.num_populations;
  if (sample_index < 0 || sample_index >= num_samples || population_index < 0 || population_index >= P) {
    std::fprintf(stderr,
                 "effective_number_of_chromosomes error: index out of bounds: sample %d [0 %d), population %d [0 %d)\n",
                 sample_index, num_samples, population_index, P);
    std::exit(1);
  }
  return time_samples[sample_index]->Nchrom_e[population_index];
}

/* A mutation that had not arisen by `sample_index` reports frequency 0. */
inline float allele_trajectories::frequency(int sample_index, int population_index, int mutation_index) {
  if (!time_samples || num_samples == 0) die("frequency error: empty allele_trajectories");
  const int P = sim_run_constants.num_populations;
  const int M_final = time_samples[num_samples - 1]->num_mutations;
  if (sample_index < 0 || sample_index >= num_samples || population_index < 0 || population_index >= P ||
      mutation_index < 0 || mutation_index >= M_final) {
    std::fprintf(stderr,
                 "frequency error: index out of bounds: sample %d [0 %d), population %d [0 %d), mutation %d [0 %d)\n",
                 sample_index, num_samples, population_index, P, mutation_index, M_final);
    std::exit(1);
  }
  const time_sample* s = time_samples[sample_index];
  if (mutation_index >= s->num_mutations) return 0;
  return s->mutations_freq[static_cast<size_t>(population_index) * s->num_mutations + mutation_index];
}

inline mutID allele_trajectories::mutation_ID(int mutation_index) {
  if (num_samples <= 0 || !time_samples) die("mutation_ID error: empty allele_trajectories");
  if (mutation_index < 0 || mutation_index >= all_mutations) {
    std::fprintf(stderr, "mutation_ID error: requested mutation index out of bounds: mutation %d [0 %d)\n",
                 mutation_index, all_mutations);
    std::exit(1);
  }
  const mutID& m = mutations_ID[mutation_index];
  return mutID(m.origin_generation, m.origin_population, std::abs(m.origin_threadID), m.reserved);
}

/* Deleting the final sample keeps the ID array but moves maximal_num_mutations() to the new last
 * sample; deleting the only sample resets the object. */
inline void allele_trajectories::delete_time_sample(int sample_index) {
  if (!time_samples || num_samples == 0) die("delete_time_sample error: empty allele_trajectories");
  if (sample_index < 0 || sample_index >= num_samples) {
    std::fprintf(stderr, "delete_time_sample error: requested sample index out of bounds: sample %d [0 %d)\n",
                 sample_index, num_samples);
    std::exit(1);
  }
  if (num_samples == 1) {
    reset();
    return;
  }
  delete time_samples[sample_index];
  time_sample** keep = new time_sample*[num_samples - 1];
  for (int i = 0, j = 0; i < num_samples; ++i)
    if (i != sample_index) keep[j++] = time_samples[i];
  delete[] time_samples;
  time_samples = keep;
  num_samples -= 1;
  all_mutations = time_samples[num_samples - 1]->num_mutations;
}

inline void allele_trajectories::reset() {
  if (time_samples) {
    for (int i = 0; i < num_samples; ++i) delete time_samples[i];
    delete[] time_samples;
  }
  if (mutations_ID) std::free(mutations_ID);
  time_samples = NULL;
  num_samples = 0;
  mutations_ID = NULL;
  all_mutations = 0;
  sim_run_constants = sim_constants();
  sim_input_constants = sim_constants();
}

inline std::ostream& operator<<(std::ostream& stream, const mutID& id) {
  stream << id.toString();
  return stream;
}

/* Text dump: run constants, per-sample features (one major column per sample, one minor column per
 * population), then one row per mutation with its frequency in every sample and population --
 * the layout of the reference's dump (inline_go_fish_data_struct.hpp:208-267). */
inline std::ostream& operator<<(std::ostream& stream, allele_trajectories& A) {
  const allele_trajectories::sim_constants& c = A.sim_run_constants;
  stream << "seed1\t" << c.seed1 << std::endl;
  stream << "seed2\t" << c.seed2 << std::endl;
  stream << "num_generations\t" << c.num_generations << std::endl;
  stream << "num_sites\t" << c.num_sites << std::endl;
  stream << "num_populations\t" << c.num_populations << std::endl;
  stream << "init_mse\t" << c.init_mse << std::endl;
  stream << "prev_sim_sample\t" << c.prev_sim_sample << std::endl;
  stream << "compact_interval\t" << c.compact_interval << std::endl;
  stream << "device\t" << c.device << std::endl << std::endl;
  if (A.num_samples == 0) {
    stream << "no simulation stored" << std::endl;
    return stream;
  }
  const int P = c.num_populations;
  stream << "time sample:";
  for (int j = 0; j < A.num_samples; ++j) {
    stream << "\t" << j;
    for (int k = 0; k < P - 1; ++k) stream << "\t";
  }
  stream << std::endl << "generation:";
  for (int j = 0; j < A.num_samples; ++j) {
    stream << "\t" << A.sampled_generation(j);
    for (int k = 0; k < P - 1; ++k) stream << "\t";
  }
  stream << std::endl << "number of mutations reported:";
  for (int j = 0; j < A.num_samples; ++j) {
    stream << "\t" << A.num_mutations_time_sample(j);
    for (int k = 0; k < P - 1; ++k) stream << "\t";
  }
  stream << std::endl << "population:";
  for (int j = 0; j < A.num_samples; ++j)
    for (int k = 0; k < P; ++k) stream << "\t" << k;
  stream << std::endl << "effective population size (chromosomes):";
  for (int j = 0; j < A.num_samples; ++j)
    for (int k = 0; k < P; ++k) stream << "\t" << A.effective_number_of_chromosomes(j, k);
  stream << std::endl << "population extinct:";
  for (int j = 0; j < A.num_samples; ++j)
    for (int k = 0; k < P; ++k) stream << "\t" << A.extinct(j, k);
  stream << std::endl;
  if (A.all_mutations == 0) {
    stream << std::endl << "no mutations stored" << std::endl;
    return stream;
  }
  stream << "mutation ID (origin_generation,origin_population,origin_threadID,reserved)";
  for (int j = 0; j < A.num_samples; ++j)
    for (int k = 0; k < P; ++k) stream << "\tfrequency";
  stream << std::endl;
  for (int i = 0; i < A.all_mutations; ++i) {
    stream << A.mutation_ID(i) << ":";
    for (int j = 0; j < A.num_samples; ++j)
      for (int k = 0; k < P; ++k) stream << "\t" << A.frequency(j, k, i);
    stream << std::endl;
  }
  return stream;
}

}  // namespace GO_Fish

#endif  // GOFISH_B200_GO_FISH_DATA_STRUCT_H_
