/*
 * gofish_b200.h -- C ABI of the B200 (sm_100a) GO_Fish forward Wright-Fisher engine and the
 * Spectrum site-frequency-spectrum path.
 *
 * Plain C types only (pointers, sizes, ints, floats): no CUDA or C++ types cross this boundary, so
 * the library can be bound from C, C++ (the header front-end in include/3P/), ctypes or any FFI.
 * Every entry point returns a gf_status; gf_engine_last_error() holds the message of the last
 * failure on that engine.  Nothing in the library calls exit().
 *
 * Each declaration cites the reference interface it replaces, as `file:line` within
 * ParallelPopGen 3P v0.3.2.
 */
#ifndef GOFISH_B200_H_
#define GOFISH_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Largest number of populations one simulation may hold.  The reference has no fixed bound; the
 * per-generation parameter block below is a fixed-size struct so it can be passed by value to the
 * drift kernel. */
#define GF_MAX_POPULATIONS 16

/* Largest generation number the engine accepts: on the device a mutation's origin generation and
 * origin population share one 32-bit word (24 + 7 bits); the origin thread ID keeps its own word. */
#define GF_MAX_GENERATION ((1 << 24) - 1)

typedef enum gf_status {
  GF_OK = 0,
  GF_ERR_INVALID_ARGUMENT = 1, /* a parameter is out of range (check_sim_parameters, go_fish_impl.cuh:431-452) */
  GF_ERR_CUDA = 2,             /* a CUDA runtime call failed (cudaCheckErrors, shared.cuh:24) */
  GF_ERR_OUT_OF_MEMORY = 3,    /* device allocation failed */
  GF_ERR_CAPACITY = 4,         /* a documented size limit was exceeded */
  GF_ERR_STATE = 5,            /* call out of order, e.g. gf_sim_run before a gf_sim_begin_* */
  GF_ERR_DEVICE = 6,           /* a kernel reported a fault through the engine's device status word */
  GF_ERR_NO_DEVICE = 7         /* no CUDA device, or the requested ordinal does not exist */
} gf_status;

typedef struct gf_engine gf_engine;

/* ---------------------------------------------------------------------------------------------
 * Engine lifecycle.  An engine owns one device, one CUDA stream and the device buffers of one
 * simulation at a time.  Replaces set_cuda_device (shared.cuh:27-37) and the stream/event set-up
 * of GO_Fish::run_sim (go_fish_impl.cuh:561-587).
 *   device       CUDA ordinal, or -1 for the current device.
 *   cuda_stream  a cudaStream_t to run on, or NULL to let the engine create its own.
 * ------------------------------------------------------------------------------------------- */
gf_status gf_engine_create(int device, void* cuda_stream, gf_engine** out_engine);
void gf_engine_destroy(gf_engine* engine);
const char* gf_engine_last_error(const gf_engine* engine);
/* CUDA ordinal the engine runs on (set_cuda_device reports it back, shared.cuh:35). */
int32_t gf_engine_device(const gf_engine* engine);
const char* gf_status_string(gf_status status);
/* Library version, "major.minor.patch". */
const char* gf_version(void);

/* Simulation constants (allele_trajectories::sim_constants, go_fish_data_struct.h:57-70). */
typedef struct gf_sim_config {
  int32_t seed1;            /* Philox key word 0 */
  int32_t seed2;            /* Philox key word 1 */
  float num_sites;          /* L */
  int32_t num_populations;  /* P, 1 .. GF_MAX_POPULATIONS */
  int32_t compact_interval; /* 0 = never compact */
  int32_t reserve_mutations;/* initial capacity hint in mutations (0 = automatic) */
} gf_sim_config;

/* Per-population model values at one generation, evaluated by the caller from its model functions
 * (Sim_Model functors).  Selection must be affine in frequency at a fixed population and
 * generation: s(freq) = sel_slope * freq + sel_intercept, which covers every selection model the
 * reference ships (template_inline_simulation_functors.cuh:46-158). */
typedef struct gf_population_params {
  int32_t Nchrom_e;      /* effective chromosomes 2N/(1+F) (go_fish_impl.cuh:659); 0 = not simulated */
  int32_t drift;         /* 1: run migration/selection/drift for this population this generation */
  int32_t alive;         /* demography(pop, generation) > 0, used by the compaction flag (:156) */
  int32_t mutate;        /* 1: draw new mutations for this population (calc_new_mutations_Index :462) */
  float mu;              /* per-site mutation rate */
  float F;               /* inbreeding coefficient */
  float h;               /* dominance coefficient */
  float sel_slope;       /* selection coefficient slope in frequency */
  float sel_intercept;   /* selection coefficient at frequency 0 */
} gf_population_params;

/* One generation (the body of the run_sim loop, go_fish_impl.cuh:645-714). */
typedef struct gf_generation {
  int32_t generation;
  int32_t compact;   /* compact after this generation (:705) */
  int32_t preserve;  /* mark survivors of this compaction as preserved (:686, scatter_arrays) */
  int32_t selection_table; /* 1: the selection coefficient of every drifted (population, mutation) is
                            * read from the table of gf_sim_selection_view, filled by the caller for
                            * this generation (sel_slope / sel_intercept are ignored); such a
                            * generation is passed to gf_sim_run alone */
  gf_population_params pop[GF_MAX_POPULATIONS];
  /* migration[from * GF_MAX_POPULATIONS + to]: proportion of chromosomes in `to` from `from`
   * (Functor_migration, go_fish.cuh:238). */
  float migration[GF_MAX_POPULATIONS * GF_MAX_POPULATIONS];
} gf_generation;

/* Begin a simulation from an empty mutation array at `start_generation`
 * (init_blank_prev_run, blank branch: go_fish_impl.cuh:335-349). */
gf_status gf_sim_begin_blank(gf_engine* engine, const gf_sim_config* config, int32_t start_generation);

/* Begin a simulation from host arrays (init_blank_prev_run, resume branch: go_fish_impl.cuh:339-365).
 *   freq       [num_populations][num_mutations] row-major frequencies
 *   mut_ids    [num_mutations][4] int32 = (origin_generation, origin_population, origin_threadID, reserved);
 *              a negative threadID marks a preserved mutation
 *   extinct    [num_populations] 0/1 (may be NULL)
 *   preserve   1: mark every loaded mutation preserved (preserve_prev_run_mutations, go_fish_impl.cu:191-194) */
gf_status gf_sim_begin_from_state(gf_engine* engine, const gf_sim_config* config, int32_t start_generation,
                                  const float* freq, const int32_t* mut_ids, int32_t num_mutations,
                                  const uint8_t* extinct, int32_t preserve);

/* Per-population inputs of the mutation-selection-equilibrium start (initialize_mse,
 * go_fish_impl.cuh:242-332).  Selection is affine in frequency, as in gf_population_params. */
typedef struct gf_mse_population {
  int32_t N_ind;         /* demography(pop, 0) */
  int32_t Nchrom_e;      /* 2 * N_ind / (1 + F) */
  float mu;
  float F;
  float h;
  float sel_slope;
  float sel_intercept;
} gf_mse_population;

/* Begin at mutation-selection equilibrium at generation 0 (initialize_mse).  Neutral populations
 * use lambda(x) = 2 mu L / x exactly as the reference; selected ones integrate the MSE density with
 * a fixed-order (deterministic) scan.  preserve = preserve(0) | sample(0). */
gf_status gf_sim_begin_mse(gf_engine* engine, const gf_sim_config* config, const gf_mse_population* pops,
                           int32_t preserve);

/* Run `num_generations` consecutive generations (run_sim loop body, go_fish_impl.cuh:645-714:
 * fused migration/selection/drift + new mutations, then compaction where gens[i].compact is set).
 * Asynchronous: returns once the work is queued on the engine's stream. */
gf_status gf_sim_run(gf_engine* engine, const gf_generation* gens, int32_t num_generations);

/* Selection models that are not affine in frequency.  The reference evaluates
 * s = sel_coeff(pop, generation, x_mig) per mutation inside migration_selection_drift
 * (go_fish_impl.cuh:98-105), with x_mig = sum over k of migration(k, pop, generation) * freq[k][i]
 * accumulated in k order with fused multiply-adds.  For such a model the caller evaluates the model on
 * the device before the generation: it computes x_mig the same way from `freq` and the generation's
 * migration matrix and writes s (unclamped; the engine applies max(s, -1)) to
 * selection[pop * selection_stride + i] for every drifted population and every i < *num_mutations,
 * with a kernel launched on `cuda_stream`, then runs the generation with selection_table = 1.  The
 * header front-end (include/3P/go_fish.cuh) does this with a kernel instantiated for the user's
 * functor when the user's translation unit is compiled by nvcc.  The view is valid until the next
 * gf_sim_* call. */
typedef struct gf_selection_view {
  const float* freq;               /* [num_populations][row_stride] frequencies the generation starts from */
  int64_t row_stride;
  const int32_t* num_mutations;    /* device word: mutations the generation starts from */
  float* selection;                /* [num_populations][selection_stride] coefficients to write */
  int64_t selection_stride;
  int32_t num_populations;
  int32_t reserved;
  void* cuda_stream;               /* the engine's cudaStream_t */
} gf_selection_view;

gf_status gf_sim_selection_view(gf_engine* engine, gf_selection_view* out);

/* Current number of mutations in the array (h_mutations_Index).  Synchronizes the stream. */
gf_status gf_sim_num_mutations(gf_engine* engine, int32_t* out_num_mutations);

/* Copy the current state to host memory (store_time_sample, go_fish_impl.cuh:477-501).
 *   freq_out   [num_populations][num_mutations] (may be NULL)
 *   ids_out    [num_mutations][4] int32 mutID layout (may be NULL)
 *   max_mutations  capacity of the caller's arrays, in mutations
 * Synchronizes the stream. */
gf_status gf_sim_read_state(gf_engine* engine, float* freq_out, int32_t* ids_out, int32_t max_mutations,
                            int32_t* out_num_mutations);

/* The same copy without stopping the run (the time-sample pipeline: store_time_sample's copy into
 * the trajectory, go_fish_impl.cuh:477-501).  gf_sim_sample_begin packs the state on the device at this
 * point of the engine's stream into engine-owned scratch and returns; the caller may enqueue more
 * generations.  gf_sim_sample_wait copies the packed rows into freq_out ([num_populations][M]) and the
 * IDs into ids_out ([M][4]) on a second stream, exactly M of them, while the engine's stream runs what
 * was enqueued after the begin, and returns M (and, out_bytes_copied may be NULL, the bytes moved).
 * Page-locked arrays (cudaMallocHost / cudaHostRegister) keep the copies direct.  max_mutations must
 * cover the count at the begin (checked against the engine's upper bound on it, read exactly if that
 * bound is larger; GF_ERR_CAPACITY otherwise).  One sample may be in flight per engine, and the
 * caller's arrays must stay untouched until its wait returns.  With freq_out and ids_out both NULL the
 * wait copies the rows (not the IDs) into page-locked staging the engine owns, readable through
 * gf_sim_sample_staged until the next begin. */
gf_status gf_sim_sample_begin(gf_engine* engine, float* freq_out, int32_t* ids_out, int32_t max_mutations);
gf_status gf_sim_sample_wait(gf_engine* engine, int32_t* out_num_mutations, int64_t* out_bytes_copied);
gf_status gf_sim_sample_staged(gf_engine* engine, const float** out_freq);

/* Device pointer to the current frequency rows ([P][stride] floats) and their row stride, for
 * device-side consumers (valid until the next gf_sim_* call). */
gf_status gf_sim_device_state(gf_engine* engine, const float** out_freq, int32_t* out_row_stride,
                              int32_t* out_num_mutations);

/* Host-side new-mutation count of one population in one generation, exactly as the reference draws
 * it on the host (calc_new_mutations_Index, go_fish_impl.cuh:454-467, ApproxRandPois1
 * shared.cuh:251-256): max(Poisson~(mu * Nchrom_e * L), 0) with counter (1, generation, pop, 0). */
int32_t gf_new_mutation_count(int32_t seed1, int32_t seed2, float mu, int32_t Nchrom_e, float num_sites,
                              int32_t generation, int32_t population);

/* Selection coefficients of Sim_Model::selection_sine_wave, s = A sin(pi t + rho) + D for
 * t = t0 .. t0 + count - 1 (t = generation - generation_shift), into host out[count].  The reference
 * evaluates this expression inside its drift kernel under --use_fast_math
 * (template_inline_simulation_functors.cuh:92), where the sine is the hardware approximation; this
 * call evaluates it on the engine's device with the same expression and flags, so the per-generation
 * intercept the caller passes in gf_population_params is the float the reference's kernel uses.
 * Synchronizes the engine's stream. */
gf_status gf_selection_sine_values(gf_engine* engine, float A, float pi, float rho, float D, int32_t t0, int32_t count,
                                   float* out);

/* ---------------------------------------------------------------------------------------------
 * Batched replicates (no reference counterpart: the reference runs one simulation per run_sim call,
 * go_fish_impl.cuh:553-730).  Thousands of independent single-population simulations with their own
 * sizes, demographies, selection, seeds and run lengths advance together: each super-step runs one
 * compaction window of every unfinished replicate in one launch of the window kernel, followed by a
 * segmented compaction.  Replicate r's result is bit-identical to a plain gf_sim_* run with the same
 * seeds, model and compaction schedule (MSE start, compaction every compact_interval generations and
 * at the final one).
 * ------------------------------------------------------------------------------------------- */
typedef struct gf_replicate {
  int32_t seed1, seed2;
  float num_sites;          /* L */
  float mu;                 /* per-site mutation rate */
  float F, h;               /* inbreeding, dominance */
  float sel_slope, sel_intercept; /* selection s(freq) = slope * freq + intercept */
  int32_t N0;               /* individuals at generation 0 */
  float growth_rate;        /* N(g) = round(N0 * exp(growth_rate * g)), as demography_exponential_growth */
  int32_t N_min, N_max;     /* ... clamped to [N_min, N_max] (N_min >= 1) */
  int32_t num_generations;  /* generations to run after the MSE start */
  int32_t compact_interval; /* >= 1 */
} gf_replicate;

/* Population size of replicate `rep` at `generation` (the clamped exponential above, evaluated on the
 * host in float like Sim_Model::demography_exponential_growth), for building the equivalent plain run. */
int32_t gf_replicate_population(const gf_replicate* rep, int32_t generation);
/* The same for generations first .. first+count-1 into out[count]. */
void gf_replicate_population_table(const gf_replicate* rep, int32_t first, int32_t count, int32_t* out);

/* Begin R replicates at mutation-selection equilibrium (initialize_mse for each). */
gf_status gf_batch_begin(gf_engine* engine, const gf_replicate* reps, int32_t num_replicates);
/* Run super-steps until every replicate has finished (max_super_steps <= 0) or for at most
 * max_super_steps; *out_active (may be NULL) receives the number of unfinished replicates. */
gf_status gf_batch_run(gf_engine* engine, int32_t max_super_steps, int32_t* out_active);
/* Current state of replicate r (frequencies [M], IDs [M][4]), its count and generation. */
gf_status gf_batch_read_state(gf_engine* engine, int32_t r, float* freq_out, int32_t* ids_out, int32_t max_mutations,
                              int32_t* out_num_mutations, int32_t* out_generation);
/* Projected SFS of sample size n of every replicate's current state, host out[r * n + k]. */
gf_status gf_batch_sfs(gf_engine* engine, int32_t n, float* out);
typedef struct gf_batch_stats {
  double mutation_generations; /* all replicates, all generations */
  int64_t generations;         /* sum over replicates */
  int64_t super_steps;
  int32_t replicates;
  int32_t active;
  int64_t arena_slots;         /* device slots reserved for all replicates */
  double record_wait_ms;       /* host time spent waiting for generation records to be drawn */
  int32_t record_producers;    /* host threads drawing the records (0: none) */
  int32_t reserved;
} gf_batch_stats;
gf_status gf_batch_stats_read(gf_engine* engine, gf_batch_stats* out);
/* Generation records (one per replicate per generation, 36 bytes, page-locked on the host and on
 * the device) the batched engine keeps resident.  Host threads draw them region by region (about 512
 * generations of every replicate per region) while the super-steps run: a batch within the budget
 * (default 67,108,864) keeps every region resident; a larger one cycles its regions through as many
 * slots as fit the budget (at least two); 0 builds each super-step's records on the host and reads
 * the counts back per super-step.  Results are identical in every case.  Takes effect at the next
 * gf_batch_begin. */
gf_status gf_batch_set_record_budget(gf_engine* engine, int64_t records);

/* ---------------------------------------------------------------------------------------------
 * Spectrum (spectrum.h:24-43, spectrum.cu:153-294).  Inputs are one population row of a host time
 * sample, as the reference's functions take it; outputs are host arrays.
 * ------------------------------------------------------------------------------------------- */

/* Population frequency histogram (Spectrum::population_frequency_histogram, spectrum.cu:153-210):
 * out[k] = number of mutations with round(Nchrom_e * freq) == k (k == Nchrom_e folds into 0),
 * plus (num_sites - num_mutations) in out[0].  out has Nchrom_e floats. */
gf_status gf_population_histogram(gf_engine* engine, const float* freq, int32_t num_mutations, int32_t Nchrom_e,
                                  float num_sites, float* out);

/* Binomially projected SFS of sample size n (Spectrum::site_frequency_spectrum, spectrum.cu:213-294):
 * out[k] = sum over mutations segregating in this population (0 < p < 1) of C(n,k) p^k (1-p)^(n-k)
 * for k = 1 .. n-1; out[0] collects k = 0 and k = n, every non-segregating mutation and
 * (num_sites - num_mutations).  Requires 1 <= n < Nchrom_e.  out has n floats. */
gf_status gf_site_frequency_spectrum(gf_engine* engine, const float* freq, int32_t num_mutations,
                                     int32_t Nchrom_e, int32_t n, float num_sites, float* out);

/* The same two functions on a device-resident frequency row (no host copies). */
gf_status gf_population_histogram_device(gf_engine* engine, const float* d_freq, int32_t num_mutations,
                                         int32_t Nchrom_e, float num_sites, float* d_out);
gf_status gf_site_frequency_spectrum_device(gf_engine* engine, const float* d_freq, int32_t num_mutations,
                                            int32_t Nchrom_e, int32_t n, float num_sites, float* d_out);

/* Projected SFS that allocates no device memory (no counterpart in the reference).
 *
 * Same result as gf_site_frequency_spectrum_device, for callers that cannot call cudaMalloc: code
 * embedded in a framework that owns the GPU's memory budget (a caching allocator or a pre-reserved
 * pool that a library's own cudaMalloc would bypass, and that can fail mid-run), and code on a
 * latency-critical path, where cudaMalloc / cudaFree would synchronize the device.  It needs no
 * gf_engine: inputs and output are the caller's device buffers, work goes on `cuda_stream` (NULL: the
 * legacy default stream) of the current device, and the only scratch is one file-scope device array
 * of GF_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until the process exits.
 *   Limits: Nchrom_e <= GF_NOALLOC_MAX_NCHROM, 1 <= n < Nchrom_e, n <= GF_NOALLOC_MAX_SAMPLE; larger
 *   sizes return GF_ERR_CAPACITY.
 *   The first call on a device does that device's set-up: it looks the scratch array's address up
 *   (cudaGetSymbolAddress) and sets the histogram kernel's shared-memory limit; make it before any
 *   stream capture begins.  Under lazy module loading (the CUDA default) that first call may also load
 *   the module, which is when the array takes its device memory; later calls take none.  The set-up
 *   is kept for the life of the process and does not survive cudaDeviceReset: do not call this entry
 *   point on a device after resetting it.
 *   All calls on a device share the scratch array, which keeps the last call's contents: calls whose
 *   GPU work overlaps (two streams, two host threads) race; serialize them.  Each call clears what it
 *   accumulates into before using it.
 *   Every call synchronizes `cuda_stream` once: it reads back whether every frequency lies on the
 *   1/Nchrom_e grid to choose the projection.  Status codes only: there is no engine to hold a
 *   message. */
#define GF_NOALLOC_MAX_NCHROM (1 << 20)
#define GF_NOALLOC_MAX_SAMPLE 1023
#define GF_NOALLOC_SCRATCH_BYTES (4194560 + 256 + 8192 + 2097152)
gf_status gf_site_frequency_spectrum_noalloc(const float* d_freq, int32_t num_mutations, int32_t Nchrom_e, int32_t n,
                                             float num_sites, float* d_out, void* cuda_stream);

/* Synchronize the engine's stream and report any pending device-side fault. */
gf_status gf_engine_synchronize(gf_engine* engine);

/* ---------------------------------------------------------------------------------------------
 * Measurement (no reference counterpart: the reference's examples time whole run_sim calls with
 * cudaEvents, examples/example_speed/run.cu:29-45).
 * ------------------------------------------------------------------------------------------- */
typedef struct gf_sim_stats {
  double mutation_generations; /* sum over generations of the slots the drift pass updated */
  int64_t generations;         /* generations run since the simulation began */
  int64_t compactions;
  int64_t kernel_launches;     /* kernels this engine launched since it was created */
} gf_sim_stats;

/* Counters of the current simulation.  Synchronizes the stream. */
gf_status gf_sim_stats_read(gf_engine* engine, gf_sim_stats* out);

/* Joint SFS of two populations (an extension: the reference computes single-population marginals,
 * Spectrum::site_frequency_spectrum, spectrum.cu:213-294).  out[i * (n_b + 1) + j] = expected number of
 * sites whose sample of n_a chromosomes from population a holds i derived copies and whose sample of
 * n_b from population b holds j: every one of the M mutations contributes the product of its two
 * binomial projections (spectrum.cu:90-139), and the num_sites - M monomorphic sites go to (0, 0).
 * For 1 <= i <= n_a - 1 the row sums equal population a's single-population SFS.  1 <= n_a, n_b <= 1023.
 * freq_a / freq_b are the two populations' rows of the same M mutations.  Computed in double,
 * deterministic.  The _device variant takes device pointers and runs asynchronously. */
gf_status gf_joint_site_frequency_spectrum(gf_engine* engine, const float* freq_a, const float* freq_b,
                                           int32_t num_mutations, int32_t n_a, int32_t n_b, float num_sites,
                                           float* out);
gf_status gf_joint_site_frequency_spectrum_device(gf_engine* engine, const float* d_freq_a, const float* d_freq_b,
                                                  int32_t num_mutations, int32_t n_a, int32_t n_b,
                                                  float num_sites, float* d_out);

/* Joint SFS of three populations (the same extension): out[(i * (n_b + 1) + j) * (n_c + 1) + k] =
 * expected number of sites whose samples of n_a, n_b and n_c chromosomes from populations a, b and c
 * hold i, j and k derived copies, each mutation contributing the product of its three binomial
 * projections; the num_sites - M monomorphic sites go to (0, 0, 0).  Summed over k it is the joint SFS
 * of a and b.  1 <= n_a, n_b, n_c <= 1023 and (n_a + 1)(n_b + 1)(n_c + 1) <= 2^24 bins (larger:
 * GF_ERR_CAPACITY).  Computed in double, deterministic; the _device variant takes device pointers and
 * runs asynchronously. */
gf_status gf_joint3_site_frequency_spectrum(gf_engine* engine, const float* freq_a, const float* freq_b,
                                            const float* freq_c, int32_t num_mutations, int32_t n_a, int32_t n_b,
                                            int32_t n_c, float num_sites, float* out);
gf_status gf_joint3_site_frequency_spectrum_device(gf_engine* engine, const float* d_freq_a, const float* d_freq_b,
                                                   const float* d_freq_c, int32_t num_mutations, int32_t n_a,
                                                   int32_t n_b, int32_t n_c, float num_sites, float* d_out);

/* Launch choices of the drift pass (results do not depend on them). */
typedef struct gf_tuning {
  int32_t draw_strategy; /* 0: each thread draws its own four lanes in order; 1: warp-cooperative draws,
                            pooled in shared memory by sampler branch; 2: each thread draws its lanes
                            grouped by sampler branch (normal approximation first, then the searches);
                            3: the normal approximation of all four lanes at once, then the searches;
                            4: the normal approximation of all four lanes in each thread, then the
                            warp's search-branch draws pooled in shared memory and run together */
  int32_t blocks_per_sm; /* resident drift blocks per SM (0: the occupancy maximum) */
  int32_t windows;       /* 1 (default): single-population generations between compactions run as one
                            window launch; 0: one launch per generation */
} gf_tuning;
gf_status gf_engine_set_tuning(gf_engine* engine, const gf_tuning* tuning);
gf_status gf_engine_get_tuning(const gf_engine* engine, gf_tuning* tuning);

/* When enabled, the engine brackets every drift launch and every compaction (scan + scatter) with
 * CUDA events on its stream; gf_engine_read_profile() returns the accumulated device times and
 * resets them.  Disabled by default. */
gf_status gf_engine_set_profiling(gf_engine* engine, int32_t enable);
typedef struct gf_kernel_times {
  double drift_ms;
  int64_t drift_launches;
  double compact_ms;
  int64_t compactions;
} gf_kernel_times;
gf_status gf_engine_read_profile(gf_engine* engine, gf_kernel_times* out);

#ifdef __cplusplus
}
#endif

#endif /* GOFISH_B200_H_ */
