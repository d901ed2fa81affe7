/*
 * spectrum.h -- site frequency spectrum API of the B200 engine (host-only C++).
 *
 * Source-compatible with ParallelPopGen 3P's spectrum.h (spectrum.h:24-43; behaviour of
 * spectrum.cu:149-294).  The functions copy one population row of one time sample to the GPU, run
 * the sm_100a histogram / projection kernels of libgofish_b200.so and fill `mySFS` on the host.
 */
#ifndef GOFISH_B200_SPECTRUM_H_
#define GOFISH_B200_SPECTRUM_H_

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <utility>

#include "../gofish_b200.h"
#include "go_fish_data_struct.h"

namespace gofish_detail {
gf_engine* spectrum_engine(int device);
}

namespace Spectrum {

/* Site frequency spectrum of one population at one time point. */
struct SFS {
  float* frequency_spectrum; /* [sample_size[0]] bins; bin 0 = monomorphic sites */
  int* populations;          /* which populations are in the SFS */
  int* sample_size;          /* sample size per population */
  int num_populations;
  float num_sites;
  float num_mutations;       /* num_sites - frequency_spectrum[0] */
  int sampled_generation;

  SFS()
      : frequency_spectrum(NULL), populations(NULL), sample_size(NULL), num_populations(0), num_sites(0),
        num_mutations(0), sampled_generation(0) {}
  ~SFS() { clear(); }
  /* Copies are deep.  The reference's SFS is copyable too (spectrum.h:24-37, implicit members), but
   * its copies share the arrays that both destructors then delete; here each copy owns its own. */
  SFS(const SFS& in)
      : frequency_spectrum(NULL), populations(NULL), sample_size(NULL), num_populations(in.num_populations),
        num_sites(in.num_sites), num_mutations(in.num_mutations), sampled_generation(in.sampled_generation) {
    if (in.sample_size && in.num_populations > 0) {
      sample_size = new int[in.num_populations];
      std::memcpy(sample_size, in.sample_size, sizeof(int) * in.num_populations);
    }
    if (in.populations && in.num_populations > 0) {
      populations = new int[in.num_populations];
      std::memcpy(populations, in.populations, sizeof(int) * in.num_populations);
    }
    const size_t n = in.bins();
    if (in.frequency_spectrum && n > 0) {
      frequency_spectrum = new float[n];
      std::memcpy(frequency_spectrum, in.frequency_spectrum, sizeof(float) * n);
    }
  }
  SFS& operator=(SFS in) {
    std::swap(frequency_spectrum, in.frequency_spectrum);
    std::swap(populations, in.populations);
    std::swap(sample_size, in.sample_size);
    num_populations = in.num_populations;
    num_sites = in.num_sites;
    num_mutations = in.num_mutations;
    sampled_generation = in.sampled_generation;
    return *this;
  }
  /* frees the arrays (the reference leaks them when an SFS is reused; this version frees first) */
  void clear() {
    delete[] frequency_spectrum;
    delete[] populations;
    delete[] sample_size;
    frequency_spectrum = NULL;
    populations = NULL;
    sample_size = NULL;
  }

 private:
  /* floats in frequency_spectrum: the sample size of a single population's spectrum or histogram,
   * the product of (n + 1) over the populations of a joint spectrum */
  size_t bins() const {
    if (!sample_size || num_populations <= 0) return 0;
    if (num_populations == 1) return static_cast<size_t>(sample_size[0]);
    size_t b = 1;
    for (int i = 0; i < num_populations; ++i) b *= static_cast<size_t>(sample_size[i] + 1);
    return b;
  }
};

}  // namespace Spectrum

namespace gofish_detail {

inline gf_engine* spectrum_engine(int device) {
  static gf_engine* engines[64] = {NULL};
  static gf_engine* current_default = NULL;
  gf_engine** slot = (device >= 0 && device < 64) ? &engines[device] : &current_default;
  if (!*slot) {
    const gf_status st = gf_engine_create(device, NULL, slot);
    if (st != GF_OK) {
      std::fprintf(stderr, "error creating the Spectrum engine on device %d: %s\n", device, gf_status_string(st));
      std::exit(1);
    }
  }
  return *slot;
}

struct spectrum_access {
  typedef GO_Fish::allele_trajectories AT;
  /* one population row of one time sample, with the reference's bounds check (spectrum.cu:163-165) */
  static void row(AT& a, int sample_index, int population_index, const float** freq, int* M, int* Nc, int* generation,
                  float* num_sites) {
    const int S = a.num_time_samples();
    const int P = a.num_populations();
    if (S == 0) {
      std::fprintf(stderr, "error transferring allele_trajectories to spectrum: empty allele_trajectories\n");
      std::exit(1);
    }
    if (!(sample_index >= 0 && sample_index < S) || !(population_index >= 0 && population_index < P)) {
      std::fprintf(stderr,
                   "site_frequency_spectrum error: requested indices out of bounds: sample %d [0 %d), population %d [0 %d)\n",
                   sample_index, S, population_index, P);
      std::exit(1);
    }
    const AT::time_sample* ts = a.time_samples[sample_index];
    *M = ts->num_mutations;
    *Nc = ts->Nchrom_e[population_index];
    *generation = ts->sampled_generation;
    *num_sites = a.sim_run_constants.num_sites;
    *freq = (*M > 0) ? ts->mutations_freq + static_cast<size_t>(population_index) * (*M) : NULL;
  }
};

}  // namespace gofish_detail

namespace Spectrum {

/* Frequency histogram of mutations (allele counts 0 .. Nchrom_e-1) in one population at one time
 * sample; bin 0 also holds fixed mutations and the num_sites - num_mutations monomorphic sites. */
inline void population_frequency_histogram(SFS& mySFS, const GO_Fish::allele_trajectories& all_results,
                                           const int sample_index, const int population_index, int cuda_device = -1) {
  GO_Fish::allele_trajectories& a = const_cast<GO_Fish::allele_trajectories&>(all_results);
  const float* freq;
  int M, Nc, generation;
  float L;
  gofish_detail::spectrum_access::row(a, sample_index, population_index, &freq, &M, &Nc, &generation, &L);
  gf_engine* e = gofish_detail::spectrum_engine(cuda_device);
  float* h = new float[Nc];
  const gf_status st = gf_population_histogram(e, freq, M, Nc, L, h);
  if (st != GF_OK) {
    std::fprintf(stderr, "population_frequency_histogram error: %s\n", gf_engine_last_error(e));
    std::exit(1);
  }
  mySFS.clear();
  mySFS.frequency_spectrum = h;
  mySFS.num_populations = 1;
  mySFS.sample_size = new int[1];
  mySFS.sample_size[0] = Nc;
  mySFS.num_sites = L;
  mySFS.num_mutations = mySFS.num_sites - mySFS.frequency_spectrum[0];
  mySFS.populations = new int[1];
  mySFS.populations[0] = population_index;
  mySFS.sampled_generation = generation;
}

/* Single-population SFS of sample size n, projected binomially from the population frequencies;
 * requires 1 <= n < Nchrom_e. */
inline void site_frequency_spectrum(SFS& mySFS, const GO_Fish::allele_trajectories& all_results, const int sample_index,
                                    const int population_index, const int sample_size, int cuda_device = -1) {
  GO_Fish::allele_trajectories& a = const_cast<GO_Fish::allele_trajectories&>(all_results);
  const float* freq;
  int M, Nc, generation;
  float L;
  gofish_detail::spectrum_access::row(a, sample_index, population_index, &freq, &M, &Nc, &generation, &L);
  if (sample_size <= 0 || sample_size >= Nc) {
    std::fprintf(stderr, "site_frequency_spectrum error: requested sample_size out of range [1,population_size): sample_size %d [1,%d)",
                 sample_size, Nc);
    std::exit(1);
  }
  gf_engine* e = gofish_detail::spectrum_engine(cuda_device);
  float* h = new float[sample_size];
  const gf_status st = gf_site_frequency_spectrum(e, freq, M, Nc, sample_size, L, h);
  if (st != GF_OK) {
    std::fprintf(stderr, "site_frequency_spectrum error: %s\n", gf_engine_last_error(e));
    std::exit(1);
  }
  mySFS.clear();
  mySFS.frequency_spectrum = h;
  mySFS.num_populations = 1;
  mySFS.sample_size = new int[1];
  mySFS.sample_size[0] = sample_size;
  mySFS.num_sites = L;
  mySFS.num_mutations = mySFS.num_sites - mySFS.frequency_spectrum[0];
  mySFS.populations = new int[1];
  mySFS.populations[0] = population_index;
  mySFS.sampled_generation = generation;
}

/* Joint SFS of populations a and b at one time sample (an extension; the reference computes
 * single-population marginals only): frequency_spectrum[i * (n_b + 1) + j] = expected number of sites
 * with i derived copies in a sample of n_a from population a and j in a sample of n_b from b, plus the
 * monomorphic sites at (0, 0).  Requires 1 <= n_a < Nchrom_e(a), 1 <= n_b < Nchrom_e(b), n <= 1023. */
inline void joint_site_frequency_spectrum(SFS& mySFS, const GO_Fish::allele_trajectories& all_results,
                                          const int sample_index, const int population_a, const int population_b,
                                          const int sample_size_a, const int sample_size_b, int cuda_device = -1) {
  GO_Fish::allele_trajectories& a = const_cast<GO_Fish::allele_trajectories&>(all_results);
  const float *fa, *fb;
  int M, Nca, Ncb, generation;
  float L;
  gofish_detail::spectrum_access::row(a, sample_index, population_a, &fa, &M, &Nca, &generation, &L);
  gofish_detail::spectrum_access::row(a, sample_index, population_b, &fb, &M, &Ncb, &generation, &L);
  if (sample_size_a <= 0 || sample_size_a >= Nca || sample_size_b <= 0 || sample_size_b >= Ncb) {
    std::fprintf(stderr,
                 "joint_site_frequency_spectrum error: requested sample sizes out of range: %d [1,%d), %d [1,%d)\n",
                 sample_size_a, Nca, sample_size_b, Ncb);
    std::exit(1);
  }
  gf_engine* e = gofish_detail::spectrum_engine(cuda_device);
  const size_t bins = static_cast<size_t>(sample_size_a + 1) * (sample_size_b + 1);
  float* h = new float[bins];
  const gf_status st = gf_joint_site_frequency_spectrum(e, fa, fb, M, sample_size_a, sample_size_b, L, h);
  if (st != GF_OK) {
    std::fprintf(stderr, "joint_site_frequency_spectrum error: %s\n", gf_engine_last_error(e));
    std::exit(1);
  }
  mySFS.clear();
  mySFS.frequency_spectrum = h;
  mySFS.num_populations = 2;
  mySFS.sample_size = new int[2];
  mySFS.sample_size[0] = sample_size_a;
  mySFS.sample_size[1] = sample_size_b;
  mySFS.num_sites = L;
  mySFS.num_mutations = mySFS.num_sites - mySFS.frequency_spectrum[0];
  mySFS.populations = new int[2];
  mySFS.populations[0] = population_a;
  mySFS.populations[1] = population_b;
  mySFS.sampled_generation = generation;
}

/* Joint SFS of populations a, b and c at one time sample (the same extension):
 * frequency_spectrum[(i * (n_b + 1) + j) * (n_c + 1) + k] = expected number of sites with i, j and k
 * derived copies in samples of n_a, n_b and n_c from populations a, b and c, plus the monomorphic sites
 * at (0, 0, 0).  Requires 1 <= n < Nchrom_e for each population, n <= 1023 and
 * (n_a + 1)(n_b + 1)(n_c + 1) <= 2^24. */
inline void joint_site_frequency_spectrum(SFS& mySFS, const GO_Fish::allele_trajectories& all_results,
                                          const int sample_index, const int population_a, const int population_b,
                                          const int population_c, const int sample_size_a, const int sample_size_b,
                                          const int sample_size_c, int cuda_device = -1) {
  GO_Fish::allele_trajectories& a = const_cast<GO_Fish::allele_trajectories&>(all_results);
  const float *fa, *fb, *fc;
  int M, Nca, Ncb, Ncc, generation;
  float L;
  gofish_detail::spectrum_access::row(a, sample_index, population_a, &fa, &M, &Nca, &generation, &L);
  gofish_detail::spectrum_access::row(a, sample_index, population_b, &fb, &M, &Ncb, &generation, &L);
  gofish_detail::spectrum_access::row(a, sample_index, population_c, &fc, &M, &Ncc, &generation, &L);
  if (sample_size_a <= 0 || sample_size_a >= Nca || sample_size_b <= 0 || sample_size_b >= Ncb || sample_size_c <= 0 ||
      sample_size_c >= Ncc) {
    std::fprintf(stderr,
                 "joint_site_frequency_spectrum error: requested sample sizes out of range: %d [1,%d), %d [1,%d), "
                 "%d [1,%d)\n",
                 sample_size_a, Nca, sample_size_b, Ncb, sample_size_c, Ncc);
    std::exit(1);
  }
  gf_engine* e = gofish_detail::spectrum_engine(cuda_device);
  const size_t bins = static_cast<size_t>(sample_size_a + 1) * (sample_size_b + 1) * (sample_size_c + 1);
  float* h = new float[bins];
  const gf_status st =
      gf_joint3_site_frequency_spectrum(e, fa, fb, fc, M, sample_size_a, sample_size_b, sample_size_c, L, h);
  if (st != GF_OK) {
    delete[] h;
    std::fprintf(stderr, "joint_site_frequency_spectrum error: %s\n", gf_engine_last_error(e));
    std::exit(1);
  }
  mySFS.clear();
  mySFS.frequency_spectrum = h;
  mySFS.num_populations = 3;
  mySFS.sample_size = new int[3];
  mySFS.sample_size[0] = sample_size_a;
  mySFS.sample_size[1] = sample_size_b;
  mySFS.sample_size[2] = sample_size_c;
  mySFS.num_sites = L;
  mySFS.num_mutations = mySFS.num_sites - mySFS.frequency_spectrum[0];
  mySFS.populations = new int[3];
  mySFS.populations[0] = population_a;
  mySFS.populations[1] = population_b;
  mySFS.populations[2] = population_c;
  mySFS.sampled_generation = generation;
}

}  // namespace Spectrum

#endif  // GOFISH_B200_SPECTRUM_H_
