/*
 * go_fish.cuh -- GO_Fish simulation API of the B200 engine: Sim_Model functors and GO_Fish::run_sim.
 *
 * Source-compatible with ParallelPopGen 3P's go_fish.cuh (go_fish.cuh:26-334; functor semantics
 * template_inline_simulation_functors.cuh:46-649; run_sim go_fish_impl.cuh:524-730).  Unlike the
 * reference header it also compiles as plain C++ (g++/clang++): run_sim evaluates every model
 * function on the host, packs one gf_generation record per generation and hands them to the sm_100a
 * engine in libgofish_b200.so through the C ABI declared in gofish_b200.h.  Link with
 * -lgofish_b200.
 *
 * Model-function contract (as in the reference):
 *   selection   float(int population, int generation, float freq)   -- must be affine in freq at a
 *               fixed (population, generation), as every shipped selection model is; shipped types
 *               expose the coefficients exactly through gf_affine(), other functors are sampled
 *   migration   float(int pop_FROM, int pop_TO, int generation)
 *   demography  int(int population, int generation)
 *   F, mu, h    float(int population, int generation)
 *   preserve / sample   bool(int generation)
 * Errors print the reference's message to stderr and exit(1), as the reference does.
 */
#ifndef GOFISH_B200_GO_FISH_CUH_
#define GOFISH_B200_GO_FISH_CUH_

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <utility>
#include <vector>

#include "../gofish_b200.h"
#include "go_fish_data_struct.h"

namespace gofish_detail {
/* selection_sine_wave's coefficient at t = generation - generation_shift, evaluated on the device
 * (defined below) */
inline float sine_selection(float A, float pi, float rho, float D, int t);
}  // namespace gofish_detail

#if defined(__CUDACC__)
#define GF_HD __host__ __device__
#else
#define GF_HD
#endif

namespace Sim_Model {

/* ----- selection models ----- */
/* Selection coefficients: AA 1, Aa 1+hs, aa 1+s; effective selection gamma = 2Ns/(1+F). */

/* constant selection coefficient s */
struct selection_constant {
  float s;
  inline selection_constant() : s(0) {}
  inline selection_constant(float s) : s(s) {}
  /* effective selection: s = gamma / (2 N(0, shift) / (1 + F(0, shift))) (population 0) */
  template <typename Functor_demography, typename Functor_inbreeding>
  inline selection_constant(float gamma, Functor_demography demography, Functor_inbreeding F,
                            int forward_generation_shift = 0) {
    s = gamma / (2 * demography(0, forward_generation_shift) / (1 + F(0, forward_generation_shift)));
  }
  GF_HD inline float operator()(const int population, const int generation, const float freq) const { return s; }
  inline void gf_affine(int, int, float& slope, float& intercept) const {
    slope = 0.f;
    intercept = s;
  }
};

/* s(freq) = slope * freq + intercept */
struct selection_linear_frequency_dependent {
  float slope;
  float intercept;
  inline selection_linear_frequency_dependent() : slope(0), intercept(0) {}
  inline selection_linear_frequency_dependent(float slope, float intercept) : slope(slope), intercept(intercept) {}
  template <typename Functor_demography, typename Functor_inbreeding>
  inline selection_linear_frequency_dependent(float gamma_slope, float gamma_intercept, Functor_demography demography,
                                              Functor_inbreeding F, int forward_generation_shift = 0) {
    slope = gamma_slope / (2 * demography(0, forward_generation_shift) / (1 + F(0, forward_generation_shift)));
    intercept = gamma_intercept / (2 * demography(0, forward_generation_shift) / (1 + F(0, forward_generation_shift)));
  }
  GF_HD inline float operator()(const int population, const int generation, const float freq) const {
    return slope * freq + intercept;
  }
  inline void gf_affine(int, int, float& s, float& i) const {
    s = slope;
    i = intercept;
  }
};

/* s(generation) = A sin(pi (generation - generation_shift) + rho) + D */
struct selection_sine_wave {
  float A;
  float pi;
  float rho;
  float D;
  int generation_shift;
  inline selection_sine_wave() : A(0), pi(0), rho(0), D(0), generation_shift(0) {}
  inline selection_sine_wave(float A, float pi, float D, float rho = 0, int generation_shift = 0)
      : A(A), pi(pi), rho(rho), D(D), generation_shift(generation_shift) {}
  template <typename Functor_demography, typename Functor_inbreeding>
  inline selection_sine_wave(float gamma_A, float pi, float gamma_D, Functor_demography demography,
                             Functor_inbreeding F, float rho = 0, int generation_shift = 0,
                             int forward_generation_shift = 0)
      : pi(pi), rho(rho), generation_shift(generation_shift) {
    A = gamma_A / (2 * demography(0, forward_generation_shift) / (1 + F(0, forward_generation_shift)));
    D = gamma_D / (2 * demography(0, forward_generation_shift) / (1 + F(0, forward_generation_shift)));
  }
  GF_HD inline float operator()(const int population, const int generation, const float freq) const {
    return A * std::sin(pi * (generation - generation_shift) + rho) + D;
  }
  /* The reference evaluates this model inside its drift kernel under --use_fast_math, where sin is the
   * hardware approximation; the engine's device evaluates the same expression for the front-end. */
  inline void gf_affine(int population, int generation, float& s, float& i) const {
    (void)population;
    s = 0.f;
    i = gofish_detail::sine_selection(A, pi, rho, D, generation - generation_shift);
  }
};

/* population `pop` uses s_pop, every other population uses s */
template <typename Functor_sel, typename Functor_sel_pop>
struct selection_population_specific {
  int pop;
  int generation_shift;
  Functor_sel s;
  Functor_sel_pop s_pop;
  inline selection_population_specific() : pop(0), generation_shift(0), s(), s_pop() {}
  inline selection_population_specific(Functor_sel s_in, Functor_sel_pop s_pop_in, int pop, int generation_shift = 0)
      : pop(pop), generation_shift(generation_shift), s(s_in), s_pop(s_pop_in) {}
  GF_HD inline float operator()(const int population, const int generation, const float freq) const {
    if (pop == population) return s_pop(population, generation - generation_shift, freq);
    return s(population, generation - generation_shift, freq);
  }
};

/* s1 before generation inflection_point (+ shift), s2 from then on */
template <typename Functor_sel1, typename Functor_sel2>
struct selection_piecewise {
  int inflection_point;
  int generation_shift;
  Functor_sel1 s1;
  Functor_sel2 s2;
  inline selection_piecewise() : inflection_point(0), generation_shift(0), s1(), s2() {}
  inline selection_piecewise(Functor_sel1 s1_in, Functor_sel2 s2_in, int inflection_point, int generation_shift = 0)
      : inflection_point(inflection_point), generation_shift(generation_shift), s1(s1_in), s2(s2_in) {}
  GF_HD inline float operator()(const int population, const int generation, const float freq) const {
    if (generation >= inflection_point + generation_shift) return s2(population, generation - generation_shift, freq);
    return s1(population, generation - generation_shift, freq);
  }
};

/* ----- inbreeding, mutation and dominance models ----- */
struct F_mu_h_constant {
  float p;
  inline F_mu_h_constant() : p(0) {}
  inline F_mu_h_constant(float p) : p(p) {}
  GF_HD inline float operator()(const int population, const int generation) const { return p; }
};

struct F_mu_h_sine_wave {
  float A;
  float pi;
  float rho;
  float D;
  int generation_shift;
  inline F_mu_h_sine_wave() : A(0), pi(0), rho(0), D(0), generation_shift(0) {}
  inline F_mu_h_sine_wave(float A, float pi, float D, float rho = 0, int generation_shift = 0)
      : A(A), pi(pi), rho(rho), D(D), generation_shift(generation_shift) {}
  GF_HD inline float operator()(const int population, const int generation) const {
    return A * std::sin(pi * (generation - generation_shift) + rho) + D;
  }
};

template <typename Functor_p, typename Functor_p_pop>
struct F_mu_h_population_specific {
  int pop;
  int generation_shift;
  Functor_p p;
  Functor_p_pop p_pop;
  inline F_mu_h_population_specific() : pop(0), generation_shift(0), p(), p_pop() {}
  inline F_mu_h_population_specific(Functor_p p_in, Functor_p_pop p_pop_in, int pop, int generation_shift = 0)
      : pop(pop), generation_shift(generation_shift), p(p_in), p_pop(p_pop_in) {}
  GF_HD inline float operator()(const int population, const int generation) const {
    if (pop == population) return p_pop(population, generation - generation_shift);
    return p(population, generation - generation_shift);
  }
};

template <typename Functor_p1, typename Functor_p2>
struct F_mu_h_piecewise {
  int inflection_point;
  int generation_shift;
  Functor_p1 p1;
  Functor_p2 p2;
  inline F_mu_h_piecewise() : inflection_point(0), generation_shift(0), p1(), p2() {}
  inline F_mu_h_piecewise(Functor_p1 p1_in, Functor_p2 p2_in, int inflection_point, int generation_shift = 0)
      : inflection_point(inflection_point), generation_shift(generation_shift), p1(p1_in), p2(p2_in) {}
  GF_HD inline float operator()(const int population, const int generation) const {
    if (generation >= inflection_point + generation_shift) return p2(population, generation - generation_shift);
    return p1(population, generation - generation_shift);
  }
};

/* ----- demography models (population size in individuals) ----- */
struct demography_constant {
  int N;
  inline demography_constant() : N(0) {}
  inline demography_constant(int p) : N(p) {}
  GF_HD inline int operator()(const int population, const int generation) const { return N; }
};

/* (int)A * sin(pi (generation - shift) + rho) + D -- the cast binds to A, as in the reference */
struct demography_sine_wave {
  float A;
  float pi;
  float rho;
  float D;
  int generation_shift;
  inline demography_sine_wave() : A(0), pi(0), rho(0), D(0), generation_shift(0) {}
  inline demography_sine_wave(float A, float pi, int D, float rho = 0, int generation_shift = 0)
      : A(A), pi(pi), rho(rho), D(D), generation_shift(generation_shift) {}
  GF_HD inline int operator()(const int population, const int generation) const {
    return (int)A * std::sin(pi * (generation - generation_shift) + rho) + D;
  }
};

/* round(N0 exp(rate (generation - shift))) */
struct demography_exponential_growth {
  float rate;
  int initial_population_size;
  int generation_shift;
  inline demography_exponential_growth() : rate(0), initial_population_size(0), generation_shift(0) {}
  inline demography_exponential_growth(float rate, int initial_population_size, int generation_shift = 0)
      : rate(rate), initial_population_size(initial_population_size), generation_shift(generation_shift) {}
  GF_HD inline int operator()(const int population, const int generation) const {
    return (int)std::round(initial_population_size * std::exp(rate * (generation - generation_shift)));
  }
};

/* round(K N0 e^{rt} / (K + N0 (e^{rt} - 1))); the K * N0 product is formed in float so that large
 * capacities do not overflow int (identical to the reference's int product whenever that fits). */
struct demography_logistic_growth {
  float rate;
  int initial_population_size;
  int carrying_capacity;
  int generation_shift;
  inline demography_logistic_growth() : rate(0), initial_population_size(0), carrying_capacity(0), generation_shift(0) {}
  inline demography_logistic_growth(float rate, int initial_population_size, int carrying_capacity,
                                    int generation_shift = 0)
      : rate(rate),
        initial_population_size(initial_population_size),
        carrying_capacity(carrying_capacity),
        generation_shift(generation_shift) {}
  GF_HD inline int operator()(const int population, const int generation) const {
    const float term = std::exp(rate * (generation - generation_shift));
    return (int)std::round(static_cast<float>(carrying_capacity) * initial_population_size * term /
                           (carrying_capacity + initial_population_size * (term - 1)));
  }
};

template <typename Functor_d, typename Functor_d_pop>
struct demography_population_specific {
  int pop;
  int generation_shift;
  Functor_d d;
  Functor_d_pop d_pop;
  inline demography_population_specific() : pop(0), generation_shift(0), d(), d_pop() {}
  inline demography_population_specific(Functor_d d_in, Functor_d_pop d_pop_in, int pop, int generation_shift = 0)
      : pop(pop), generation_shift(generation_shift), d(d_in), d_pop(d_pop_in) {}
  GF_HD inline int operator()(const int population, const int generation) const {
    if (pop == population) return d_pop(population, generation - generation_shift);
    return d(population, generation - generation_shift);
  }
};

template <typename Functor_d1, typename Functor_d2>
struct demography_piecewise {
  int inflection_point;
  int generation_shift;
  Functor_d1 d1;
  Functor_d2 d2;
  inline demography_piecewise() : inflection_point(0), generation_shift(0), d1(), d2() {}
  inline demography_piecewise(Functor_d1 d1_in, Functor_d2 d2_in, int inflection_point, int generation_shift = 0)
      : inflection_point(inflection_point), generation_shift(generation_shift), d1(d1_in), d2(d2_in) {}
  GF_HD inline int operator()(const int population, const int generation) const {
    if (generation >= inflection_point + generation_shift) return d2(population, generation - generation_shift);
    return d1(population, generation - generation_shift);
  }
};

/* ----- migration models: proportion of chromosomes in pop_TO that come from pop_FROM ----- */
struct migration_constant_equal {
  float m;
  int num_pop;
  inline migration_constant_equal() : m(0), num_pop(1) {}
  inline migration_constant_equal(float m, int num_pop) : m(m), num_pop(std::max(num_pop, 1)) {}
  GF_HD inline float operator()(const int pop_FROM, const int pop_TO, const int generation) const {
    if (pop_FROM == pop_TO) return 1 - (num_pop - 1) * m;
    return (num_pop > 1) * m;
  }
};

template <typename Functor_m1>
struct migration_constant_directional {
  float m;
  int pop1;
  int pop2;
  Functor_m1 rest;
  inline migration_constant_directional() : m(0), pop1(0), pop2(0), rest() {}
  inline migration_constant_directional(float m, int pop1, int pop2, Functor_m1 rest_in)
      : m(m), pop1(pop1), pop2(pop2), rest(rest_in) {}
  GF_HD inline float operator()(const int pop_FROM, const int pop_TO, const int generation) const {
    if (pop_FROM == pop1 && pop_TO == pop2) return m;
    return rest(pop_FROM, pop_TO, generation);
  }
};

template <typename Functor_m1, typename Functor_m2>
struct migration_piecewise {
  int inflection_point;
  int generation_shift;
  Functor_m1 m1;
  Functor_m2 m2;
  inline migration_piecewise() : inflection_point(0), generation_shift(0), m1(), m2() {}
  inline migration_piecewise(Functor_m1 m1_in, Functor_m2 m2_in, int inflection_point, int generation_shift = 0)
      : inflection_point(inflection_point), generation_shift(generation_shift), m1(m1_in), m2(m2_in) {}
  GF_HD inline float operator()(const int pop_FROM, const int pop_TO, const int generation) const {
    if (generation >= inflection_point + generation_shift) return m2(pop_FROM, pop_TO, generation - generation_shift);
    return m1(pop_FROM, pop_TO, generation - generation_shift);
  }
};

/* ----- preserving and sampling functions ----- */
struct bool_off {
  GF_HD inline bool operator()(const int generation) const { return false; }
};
struct bool_on {
  GF_HD inline bool operator()(const int generation) const { return true; }
};

template <typename Functor_default, typename Functor_action>
struct bool_pulse {
  int pulse;
  int generation_shift;
  Functor_default f_default;
  Functor_action f_action;
  bool_pulse() : pulse(0), generation_shift(0), f_default(), f_action() {}
  bool_pulse(int pulse, int generation_shift = 0)
      : pulse(pulse), generation_shift(generation_shift), f_default(), f_action() {}
  bool_pulse(Functor_default f_default_in, Functor_action f_action_in, int pulse, int generation_shift = 0)
      : pulse(pulse), generation_shift(generation_shift), f_default(f_default_in), f_action(f_action_in) {}
  GF_HD inline bool operator()(const int generation) const {
    if (generation == pulse + generation_shift) return f_action(generation);
    return f_default(generation);
  }
};

template <typename Functor_first, typename Functor_second>
struct bool_piecewise {
  int inflection_point;
  int generation_shift;
  Functor_first f1;
  Functor_second f2;
  inline bool_piecewise() : inflection_point(0), generation_shift(0), f1(), f2() {}
  inline bool_piecewise(int inflection_point, int generation_shift = 0)
      : inflection_point(inflection_point), generation_shift(generation_shift), f1(), f2() {}
  inline bool_piecewise(Functor_first f1_in, Functor_second f2_in, int inflection_point, int generation_shift = 0)
      : inflection_point(inflection_point), generation_shift(generation_shift), f1(f1_in), f2(f2_in) {}
  GF_HD inline bool operator()(const int generation) const {
    if (generation >= inflection_point + generation_shift) return f2(generation);
    return f1(generation);
  }
};

}  // namespace Sim_Model

namespace gofish_detail {

/* ---- exact affine coefficients of a selection model at (population, generation) ---- */
template <typename T>
struct has_gf_affine {
  template <typename U>
  static auto test(int) -> decltype(std::declval<const U&>().gf_affine(0, 0, std::declval<float&>(), std::declval<float&>()),
                                    std::true_type());
  template <typename>
  static std::false_type test(...);
  static constexpr bool value = decltype(test<T>(0))::value;
};

template <typename Sel>
inline void selection_affine(const Sel& sel, int pop, int gen, float& slope, float& intercept);

template <typename Sel>
struct affine_of {
  static inline void get(const Sel& sel, int pop, int gen, float& slope, float& intercept) {
    if constexpr (has_gf_affine<Sel>::value) {
      sel.gf_affine(pop, gen, slope, intercept);
    } else {
      // user model: sample it and require linearity in frequency
      const float s0 = sel(pop, gen, 0.f), s1 = sel(pop, gen, 1.f), sh = sel(pop, gen, 0.5f);
      const float a = s1 - s0;
      if (std::fabs((s0 + 0.5f * a) - sh) > 1e-6f * (1.f + std::fabs(sh))) {
        std::fprintf(stderr,
                     "run_sim error: selection model is not affine in frequency (population %d, generation %d); the "
                     "engine evaluates s(freq) = slope * freq + intercept\n",
                     pop, gen);
        std::exit(1);
      }
      slope = a;
      intercept = s0;
    }
  }
};

template <typename S, typename SP>
struct affine_of<Sim_Model::selection_population_specific<S, SP>> {
  static inline void get(const Sim_Model::selection_population_specific<S, SP>& sel, int pop, int gen, float& slope,
                         float& intercept) {
    if (sel.pop == pop) affine_of<SP>::get(sel.s_pop, pop, gen - sel.generation_shift, slope, intercept);
    else affine_of<S>::get(sel.s, pop, gen - sel.generation_shift, slope, intercept);
  }
};

template <typename S1, typename S2>
struct affine_of<Sim_Model::selection_piecewise<S1, S2>> {
  static inline void get(const Sim_Model::selection_piecewise<S1, S2>& sel, int pop, int gen, float& slope,
                         float& intercept) {
    if (gen >= sel.inflection_point + sel.generation_shift)
      affine_of<S2>::get(sel.s2, pop, gen - sel.generation_shift, slope, intercept);
    else
      affine_of<S1>::get(sel.s1, pop, gen - sel.generation_shift, slope, intercept);
  }
};

template <typename Sel>
inline void selection_affine(const Sel& sel, int pop, int gen, float& slope, float& intercept) {
  affine_of<Sel>::get(sel, pop, gen, slope, intercept);
}

/* true when every leaf of the selection model exposes its coefficients exactly (gf_affine) */
template <typename Sel>
struct exact_affine : has_gf_affine<Sel> {};
template <typename S, typename SP>
struct exact_affine<Sim_Model::selection_population_specific<S, SP>>
    : std::integral_constant<bool, exact_affine<S>::value && exact_affine<SP>::value> {};
template <typename S1, typename S2>
struct exact_affine<Sim_Model::selection_piecewise<S1, S2>>
    : std::integral_constant<bool, exact_affine<S1>::value && exact_affine<S2>::value> {};


/* ---- one engine per device, created on first use ---- */
inline gf_engine* engine_for(int device) {
  static gf_engine* engines[64] = {NULL};
  static gf_engine* current_default = NULL;
  gf_engine** slot = (device >= 0 && device < 64) ? &engines[device] : &current_default;
  if (!*slot) {
    gf_status st = gf_engine_create(device, NULL, slot);
    if (st != GF_OK) {
      std::fprintf(stderr, "error creating the GO_Fish engine on device %d: %s\n", device, gf_status_string(st));
      std::exit(1);
    }
  }
  return *slot;
}

inline void check(gf_engine* e, gf_status st, const char* what) {
  if (st != GF_OK) {
    std::fprintf(stderr, "%s: %s: %s\n", what, gf_status_string(st), gf_engine_last_error(e));
    std::exit(1);
  }
}

/* engine of the run_sim call in progress on this thread (model functions evaluated on its device) */
inline gf_engine*& model_engine() {
  static thread_local gf_engine* e = NULL;
  return e;
}

/* Coefficients of selection_sine_wave come from gf_selection_sine_values in blocks of consecutive
 * t, cached per thread and per parameter set (compared bit for bit). */
inline float sine_selection(float A, float pi, float rho, float D, int t) {
  struct Block {
    float key[4];
    int t0;
    std::vector<float> v;
  };
  static thread_local std::vector<Block> blocks;
  const float key[4] = {A, pi, rho, D};
  Block* hit = NULL;
  for (size_t b = 0; b < blocks.size(); ++b)
    if (std::memcmp(blocks[b].key, key, sizeof(key)) == 0) {
      hit = &blocks[b];
      if (t >= hit->t0 && t < hit->t0 + static_cast<int>(hit->v.size())) return hit->v[t - hit->t0];
      break;
    }
  if (!hit) {
    if (blocks.size() >= 16) blocks.erase(blocks.begin());
    blocks.push_back(Block());
    hit = &blocks.back();
    std::memcpy(hit->key, key, sizeof(key));
  }
  const int kBlock = 4096;
  hit->t0 = t;
  hit->v.assign(kBlock, 0.f);
  gf_engine* e = model_engine() ? model_engine() : engine_for(-1);
  check(e, gf_selection_sine_values(e, A, pi, rho, D, t, kBlock, hit->v.data()), "selection_sine_wave");
  return hit->v[0];
}

#ifdef __CUDACC__
/* ---- selection models evaluated on the device (translation units compiled by nvcc) ----
 * A selection functor without exact affine coefficients is evaluated per mutation on the device, as
 * the reference evaluates every selection functor inside migration_selection_drift
 * (go_fish_impl.cuh:98-105): before each generation, selection_table_kernel -- instantiated here, in
 * the user's translation unit, for the user's functor -- writes s(pop, generation, x_mig) for every
 * mutation into the engine's selection table (gf_sim_selection_view), and the engine's drift reads it. */
struct migration_matrix {
  float m[GF_MAX_POPULATIONS * GF_MAX_POPULATIONS];
};

template <typename Functor_selection>
__global__ void selection_table_kernel(const Functor_selection sel, const float* __restrict__ freq, long long stride,
                                       const int* __restrict__ num_mutations, int P, unsigned drift_mask,
                                       int generation, const migration_matrix mig, float* __restrict__ out,
                                       long long out_stride) {
  const int M = *num_mutations;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
    for (int p = 0; p < P; ++p) {
      if (!((drift_mask >> p) & 1u)) continue;
      // x_mig in the order and rounding of the engine's drift kernels (k order, fused multiply-add)
      float x = 0.f;
      for (int k = 0; k < P; ++k) x = __fmaf_rn(mig.m[k * GF_MAX_POPULATIONS + p], freq[k * stride + i], x);
      out[p * out_stride + i] = sel(p, generation, x);
    }
  }
}

/* s(pop, gen, x) at x = 0, 1/2 and 1, evaluated on the device */
template <typename Functor_selection>
__global__ void selection_probe_kernel(const Functor_selection sel, int pop, int gen, float* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    out[0] = sel(pop, gen, 0.f);
    out[1] = sel(pop, gen, 0.5f);
    out[2] = sel(pop, gen, 1.f);
  }
}

inline void cuda_check(cudaError_t err, const char* what) {
  if (err != cudaSuccess) {
    std::fprintf(stderr, "%s: CUDA error %s\n", what, cudaGetErrorString(err));
    std::exit(1);
  }
}

/* Fill the engine's selection table for generation G (the caller then runs G alone). */
template <typename Functor_selection>
inline void launch_selection_table(gf_engine* eng, const Functor_selection& sel, const gf_generation& G, int P) {
  gf_selection_view v;
  check(eng, gf_sim_selection_view(eng, &v), "run_sim");
  migration_matrix mig;
  std::memcpy(mig.m, G.migration, sizeof(mig.m));
  unsigned mask = 0;
  for (int p = 0; p < P; ++p)
    if (G.pop[p].drift && G.pop[p].Nchrom_e > 0) mask |= 1u << p;
  selection_table_kernel<Functor_selection><<<148 * 4, 256, 0, static_cast<cudaStream_t>(v.cuda_stream)>>>(
      sel, v.freq, v.row_stride, v.num_mutations, P, mask, G.generation, mig, v.selection, v.selection_stride);
  cuda_check(cudaGetLastError(), "run_sim: selection_table_kernel");
}

/* Affine coefficients of a device-evaluated model at (pop, gen), for the equilibrium start: the
 * model must be affine in frequency at generation 0 there, as the engine's start integrates
 * s(x) = slope x + intercept. */
template <typename Functor_selection>
inline void device_selection_affine(gf_engine* eng, const Functor_selection& sel, int pop, int gen, float& slope,
                                    float& intercept) {
  (void)eng;
  float* d = NULL;
  float h[3];
  cuda_check(cudaMalloc(&d, sizeof(h)), "run_sim");
  selection_probe_kernel<Functor_selection><<<1, 32>>>(sel, pop, gen, d);
  cuda_check(cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost), "run_sim");
  cudaFree(d);
  const float a = h[2] - h[0];
  if (std::fabs((h[0] + 0.5f * a) - h[1]) > 1e-6f * (1.f + std::fabs(h[1]))) {
    std::fprintf(stderr,
                 "run_sim error: the mutation-selection-equilibrium start needs a selection model that is affine in "
                 "frequency at generation 0 (population %d); start from a blank state or from prev_sim instead\n",
                 pop);
    std::exit(1);
  }
  slope = a;
  intercept = h[0];
}
#endif

/* Where the coefficients of a selection model come from: the host (exact affine models, and every
 * model in a translation unit not compiled by nvcc) or the device (other models under nvcc). */
template <typename Sel>
struct uses_device_selection
#ifdef __CUDACC__
    : std::integral_constant<bool, !exact_affine<Sel>::value> {
#else
    : std::false_type {
#endif
};

template <bool DEVICE>
struct selection_dispatch {
  /* coefficients for the equilibrium start at generation 0 */
  template <typename Sel>
  static void start(gf_engine*, const Sel& sel, int pop, float& slope, float& intercept) {
    selection_affine(sel, pop, 0, slope, intercept);
  }
  /* coefficients packed into a generation record */
  template <typename Sel>
  static void generation(const Sel& sel, int pop, int gen, float& slope, float& intercept) {
    selection_affine(sel, pop, gen, slope, intercept);
  }
  /* a generation that needs the device: nothing to do on the host path */
  template <typename Sel>
  static void run_alone(gf_engine*, const Sel&, gf_generation&, int) {}
};

#ifdef __CUDACC__
template <>
struct selection_dispatch<true> {
  template <typename Sel>
  static void start(gf_engine* eng, const Sel& sel, int pop, float& slope, float& intercept) {
    device_selection_affine(eng, sel, pop, 0, slope, intercept);
  }
  template <typename Sel>
  static void generation(const Sel&, int, int, float& slope, float& intercept) {
    slope = 0.f;
    intercept = 0.f;
  }
  /* fill the selection table for G, then run G alone */
  template <typename Sel>
  static void run_alone(gf_engine* eng, const Sel& sel, gf_generation& G, int P) {
    G.selection_table = 1;
    launch_selection_table(eng, sel, G, P);
    check(eng, gf_sim_run(eng, &G, 1), "run_sim");
  }
};
#endif

/* privileged access to allele_trajectories (a friend of it) */
struct trajectory_access {
  typedef GO_Fish::allele_trajectories AT;
  static int& num_samples(AT& a) { return a.num_samples; }
  static AT::sim_constants& run_constants(AT& a) { return a.sim_run_constants; }
  static const AT::sim_constants& run_constants(const AT& a) { return a.sim_run_constants; }
  static int prev_num_samples(const AT& a) { return a.num_samples; }
  static bool has_samples(const AT& a) { return a.time_samples != NULL; }
  static int sample_generation(const AT& a, int s) { return a.time_samples[s]->sampled_generation; }
  static int sample_mutations(const AT& a, int s) { return a.time_samples[s]->num_mutations; }
  static const float* sample_freq(const AT& a, int s) { return a.time_samples[s]->mutations_freq; }
  static const bool* sample_extinct(const AT& a, int s) { return a.time_samples[s]->extinct; }
  static const int* sample_Nchrom(const AT& a, int s) { return a.time_samples[s]->Nchrom_e; }
  static const GO_Fish::mutID* ids(const AT& a) { return a.mutations_ID; }
  static int all_mutations(const AT& a) { return a.all_mutations; }
  static void init_results(AT& a, int n) { a.initialize_sim_result_vector(n); }

  /* store_time_sample (go_fish_impl.cuh:477-501): the engine's current state becomes sample `s` */
  template <typename Dem, typename FI>
  static void store(AT& a, int s, gf_engine* e, int generation, bool final_sample, const bool* extinct, Dem demography,
                    FI FI_) {
    const int P = a.sim_run_constants.num_populations;
    int M = 0;
    check(e, gf_sim_num_mutations(e, &M), "store_time_sample");
    AT::time_sample* ts = a.time_samples[s];
    ts->num_mutations = M;
    ts->sampled_generation = generation;
    ts->mutations_freq = new float[static_cast<size_t>(P) * M];
    int32_t* ids = NULL;
    if (final_sample) ids = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * 4 * std::max(M, 1)));
    int got = 0;
    check(e, gf_sim_read_state(e, ts->mutations_freq, ids, M, &got), "store_time_sample");
    if (final_sample) {
      a.mutations_ID = reinterpret_cast<GO_Fish::mutID*>(ids);
      a.all_mutations = M;
    }
    ts->extinct = new bool[P];
    ts->Nchrom_e = new int[P];
    for (int i = 0; i < P; ++i) {
      ts->extinct[i] = extinct[i];
      ts->Nchrom_e[i] = 2 * demography(i, generation) / (1 + FI_(i, generation));
    }
  }

  /* The same for a sample that is not the last, with its copy overlapped with the generations that
   * follow: store_begin records the sample's generation, extinctions and sizes and has the engine pack
   * its rows at this point of the run; store_finish, called once later generations are enqueued,
   * copies them into the sample while those generations run. */
  template <typename Dem, typename FI>
  static void store_begin(AT& a, int s, gf_engine* e, int generation, const bool* extinct, Dem demography, FI FI_) {
    const int P = a.sim_run_constants.num_populations;
    AT::time_sample* ts = a.time_samples[s];
    ts->sampled_generation = generation;
    ts->extinct = new bool[P];
    ts->Nchrom_e = new int[P];
    for (int i = 0; i < P; ++i) {
      ts->extinct[i] = extinct[i];
      ts->Nchrom_e[i] = 2 * demography(i, generation) / (1 + FI_(i, generation));
    }
    check(e, gf_sim_sample_begin(e, NULL, NULL, 0x7fffffff), "store_time_sample");
  }
  static void store_finish(AT& a, int s, gf_engine* e) {
    const int P = a.sim_run_constants.num_populations;
    int M = 0;
    check(e, gf_sim_sample_wait(e, &M, NULL), "store_time_sample");
    const float* staged = NULL;
    check(e, gf_sim_sample_staged(e, &staged), "store_time_sample");
    AT::time_sample* ts = a.time_samples[s];
    ts->num_mutations = M;
    ts->mutations_freq = new float[static_cast<size_t>(P) * M];
    if (M > 0) std::memcpy(ts->mutations_freq, staged, sizeof(float) * static_cast<size_t>(P) * M);
  }
};

/* check_sim_parameters (go_fish_impl.cuh:431-452), with the reference's messages */
template <typename Mu, typename Dem, typename Mig, typename FI>
inline void check_sim_parameters(const Mu& mu_rate, const Dem& demography, const Mig& mig_prop, const FI& FI_, int P,
                                 const bool* extinct, int generation) {
  for (int pop = 0; pop < P; ++pop) {
    double migration = 0;
    if (mu_rate(pop, generation) < 0) {
      std::fprintf(stderr, "check_sim_parameters: mutation error: mu_rate < 0\tgeneration %d\t population %d\n",
                   generation, pop);
      std::exit(1);
    }
    const int N = demography(pop, generation);
    if (N > 0 && extinct[pop]) {
      std::fprintf(stderr,
                   "check_sim_parameters: demography error: extinct population with population size > 0\tgeneration "
                   "%d\t population %d\n",
                   generation, pop);
      std::exit(1);
    }
    const float fi = FI_(pop, generation);
    if (fi < 0) {
      std::fprintf(stderr, "check_sim_parameters: inbreeding error: inbreeding coefficient < 0\tgeneration %d\t population %d\n",
                   generation, pop);
      std::exit(1);
    }
    if (fi > 1) {
      std::fprintf(stderr, "check_sim_parameters: inbreeding error: inbreeding coefficient > 1\tgeneration %d\t population %d\n",
                   generation, pop);
      std::exit(1);
    }
    for (int pop2 = 0; pop2 < P; ++pop2) {
      const float m_from = mig_prop(pop, pop2, generation);
      if (m_from < 0) {
        std::fprintf(stderr,
                     "check_sim_parameters: migration error: migration rate < 0\tgeneration %d\t population_from %d\t "
                     "population_to %d\n",
                     generation, pop, pop2);
        std::exit(1);
      }
      if (m_from > 0 && ((N <= 0 || extinct[pop]) && !(demography(pop2, generation) <= 0 || extinct[pop2]))) {
        std::fprintf(stderr,
                     "migration error, migration from non-existant population\tgeneration %d\t population_from %d\t "
                     "population_to %d\n",
                     generation, pop, pop2);
        std::exit(1);
      }
      const float m_to = mig_prop(pop2, pop, generation);
      migration += static_cast<double>(m_to);
    }
    if (static_cast<float>(migration) != 1.f && !(N <= 0 || extinct[pop])) {
      std::fprintf(stderr,
                   "check_sim_parameters: migration error: migration rate does not sum to 1\tgeneration %d\t "
                   "population_TO %d\t total_migration_proportion %f\n",
                   generation, pop, migration);
      std::exit(1);
    }
  }
}

}  // namespace gofish_detail

namespace GO_Fish {

/* Runs a single-locus Wright-Fisher simulation (go_fish_impl.cuh:553-730) on the B200 engine and
 * stores the sampled and final generations in all_results.  prev_sim: if
 * all_results.sim_input_constants.init_mse is false and prev_sim_sample is a valid sample index of
 * prev_sim, the run starts from that time sample. */
template <typename Functor_mutation, typename Functor_demography, typename Functor_migration, typename Functor_selection,
          typename Functor_inbreeding, typename Functor_dominance, typename Functor_preserve, typename Functor_timesample>
inline void run_sim(allele_trajectories& all_results, const Functor_mutation mu_rate, const Functor_demography demography,
                    const Functor_migration mig_prop, const Functor_selection sel_coeff, const Functor_inbreeding FI,
                    const Functor_dominance dominance, const Functor_preserve preserve_mutations,
                    const Functor_timesample take_sample, const allele_trajectories& prev_sim) {
  using gofish_detail::check;
  typedef gofish_detail::trajectory_access TA;
  allele_trajectories::sim_constants input = all_results.sim_input_constants;
  const int P = input.num_populations;
  if (P < 1 || P > GF_MAX_POPULATIONS) {
    std::fprintf(stderr, "run_sim error: num_populations %d outside [1, %d]\n", P, GF_MAX_POPULATIONS);
    std::exit(1);
  }
  gf_engine* eng = gofish_detail::engine_for(input.device);
  gofish_detail::model_engine() = eng;
  typedef gofish_detail::selection_dispatch<gofish_detail::uses_device_selection<Functor_selection>::value> sel_path;
  const bool device_selection = gofish_detail::uses_device_selection<Functor_selection>::value;
  all_results.sim_input_constants.device = input.device = gf_engine_device(eng);  // reported back, as set_cuda_device does
  std::vector<char> extinct_v(P, 0);
  bool* extinct = reinterpret_cast<bool*>(extinct_v.data());

  gf_sim_config cfg;
  cfg.seed1 = input.seed1;
  cfg.seed2 = input.seed2;
  cfg.num_sites = input.num_sites;
  cfg.num_populations = P;
  cfg.compact_interval = input.compact_interval;
  cfg.reserve_mutations = 0;

  int generation = 0;
  int final_generation = input.num_generations;
  const int compact_interval = input.compact_interval;

  if (input.init_mse) {
    gofish_detail::check_sim_parameters(mu_rate, demography, mig_prop, FI, P, extinct, generation);
    std::vector<gf_mse_population> pops(P);
    for (int p = 0; p < P; ++p) {
      const int N_ind = demography(p, 0);
      const float F = FI(p, 0);
      pops[p].N_ind = N_ind;
      pops[p].Nchrom_e = 2 * N_ind / (1 + F);
      pops[p].mu = mu_rate(p, 0);
      pops[p].F = F;
      pops[p].h = dominance(p, 0);
      sel_path::start(eng, sel_coeff, p, pops[p].sel_slope, pops[p].sel_intercept);
    }
    check(eng, gf_sim_begin_mse(eng, &cfg, pops.data(), (preserve_mutations(0) | take_sample(0)) ? 1 : 0), "run_sim");
  } else {
    const int sample_index = input.prev_sim_sample;
    if (sample_index >= 0 && sample_index < TA::prev_num_samples(prev_sim) && TA::has_samples(prev_sim)) {
      const float prev_sites = TA::run_constants(prev_sim).num_sites;
      const int prev_P = TA::run_constants(prev_sim).num_populations;
      if (input.num_sites == prev_sites && P == prev_P) {
        generation = TA::sample_generation(prev_sim, sample_index);
        final_generation += generation;
        const bool* prev_ext = TA::sample_extinct(prev_sim, sample_index);
        std::vector<uint8_t> ext8(P);
        for (int p = 0; p < P; ++p) {
          extinct[p] = prev_ext[p];
          ext8[p] = prev_ext[p] ? 1 : 0;
        }
        const int M = TA::sample_mutations(prev_sim, sample_index);
        const int preserve0 = (preserve_mutations(generation) | take_sample(generation)) ? 1 : 0;
        check(eng,
              gf_sim_begin_from_state(eng, &cfg, generation, TA::sample_freq(prev_sim, sample_index),
                                      reinterpret_cast<const int32_t*>(TA::ids(prev_sim)), M, ext8.data(), preserve0),
              "run_sim");
      } else {
        std::fprintf(stderr,
                     "run_sim error: prev_sim parameters do not match current simulation parameters: prev_sim num_sites "
                     "%f\tcurrent_sim num_sites %f,\tprev_sim num_populations %d\tcurrent_sim num_populations %d\n",
                     prev_sites, input.num_sites, prev_P, P);
        std::exit(1);
      }
    } else if (sample_index < 0) {
      check(eng, gf_sim_begin_blank(eng, &cfg, 0), "run_sim");
    } else {
      if (!TA::has_samples(prev_sim)) {
        std::fprintf(stderr, "run_sim error: requested time sample from empty prev_sim\n");
        std::exit(1);
      }
      std::fprintf(stderr, "run_sim error: requested sample index out of bounds for prev_sim: sample %d\t[0\t %d)\n",
                   sample_index, TA::prev_num_samples(prev_sim));
      std::exit(1);
    }
    gofish_detail::check_sim_parameters(mu_rate, demography, mig_prop, FI, P, extinct, generation);
  }

  // result vector (calc_sim_result_vector_length, go_fish_impl.cuh:469-475)
  int new_length = 1;
  for (int g = generation; g < final_generation; ++g)
    if (take_sample(g)) ++new_length;
  TA::init_results(all_results, new_length);

  int sample_index = 0;
  int pending_sample = -1;   // a time sample whose copy overlaps the generations enqueued after it
  auto finish_pending = [&]() {
    if (pending_sample >= 0) {
      TA::store_finish(all_results, pending_sample, eng);
      pending_sample = -1;
    }
  };
  if (take_sample(generation) && generation != final_generation) {
    TA::store_begin(all_results, sample_index, eng, generation, extinct, demography, FI);
    pending_sample = sample_index;
    ++sample_index;
  }

  int next_compact_generation = generation + compact_interval;
  std::vector<gf_generation> batch;
  batch.reserve(256);
  auto flush = [&]() {
    if (!batch.empty()) {
      check(eng, gf_sim_run(eng, batch.data(), static_cast<int32_t>(batch.size())), "run_sim");
      batch.clear();
    }
  };
  // in device-selection mode every generation runs alone, so nothing is ever queued before it
  auto flush_before_last = [&]() {
    if (batch.size() > 1) {
      check(eng, gf_sim_run(eng, batch.data(), static_cast<int32_t>(batch.size() - 1)), "run_sim");
      batch.erase(batch.begin(), batch.end() - 1);
    }
  };
  while (generation + 1 <= final_generation) {
    ++generation;
    gofish_detail::check_sim_parameters(mu_rate, demography, mig_prop, FI, P, extinct, generation);
    batch.emplace_back();
    gf_generation& G = batch.back();
    std::memset(&G, 0, sizeof(G));
    G.generation = generation;
    for (int pop = 0; pop < P; ++pop) {
      gf_population_params& pp = G.pop[pop];
      int N_ind = demography(pop, generation);
      bool drift = !extinct[pop];
      if (drift && N_ind <= 0) {
        if (demography(pop, generation - 1) > 0) {
          N_ind = 0;  // the population goes extinct this generation
          extinct[pop] = true;
        } else {
          drift = false;  // not yet arisen
        }
      }
      const float F = FI(pop, generation);
      pp.drift = drift ? 1 : 0;
      pp.Nchrom_e = drift ? static_cast<int>(2 * N_ind / (1 + F)) : 0;
      pp.alive = demography(pop, generation) > 0 ? 1 : 0;
      pp.mutate = (!extinct[pop] && demography(pop, generation) > 0) ? 1 : 0;
      pp.mu = mu_rate(pop, generation);
      pp.F = F;
      pp.h = dominance(pop, generation);
      sel_path::generation(sel_coeff, pop, generation, pp.sel_slope, pp.sel_intercept);
      for (int to = 0; to < P; ++to) G.migration[pop * GF_MAX_POPULATIONS + to] = mig_prop(pop, to, generation);
    }
    const bool preserve = preserve_mutations(generation) | take_sample(generation);
    const bool compact = (generation == next_compact_generation || generation == final_generation || preserve) &&
                         compact_interval > 0;
    G.compact = compact ? 1 : 0;
    G.preserve = (compact && preserve) ? 1 : 0;
    if (compact) next_compact_generation = generation + compact_interval;
    const bool sample_now = take_sample(generation) && generation != final_generation;
    if (device_selection) {  // the generation reads the selection table filled just before it
      flush_before_last();
      sel_path::run_alone(eng, sel_coeff, G, P);
      batch.clear();
    }
    if (sample_now || batch.size() >= 256) flush();
    if (sample_now) {
      finish_pending();   // the previous sample's copy ran beside the generations just enqueued
      TA::store_begin(all_results, sample_index, eng, generation, extinct, demography, FI);
      pending_sample = sample_index;
      ++sample_index;
    }
  }
  flush();
  finish_pending();
  TA::store(all_results, sample_index, eng, generation, true, extinct, demography, FI);
}

/* run_sim starting from mutation-selection equilibrium or a blank array (no prev_sim). */
template <typename Functor_mutation, typename Functor_demography, typename Functor_migration, typename Functor_selection,
          typename Functor_inbreeding, typename Functor_dominance, typename Functor_preserve, typename Functor_timesample>
inline void run_sim(allele_trajectories& all_results, const Functor_mutation mu_rate, const Functor_demography demography,
                    const Functor_migration mig_prop, const Functor_selection sel_coeff, const Functor_inbreeding FI,
                    const Functor_dominance dominance, const Functor_preserve preserve_mutations,
                    const Functor_timesample take_sample) {
  run_sim(all_results, mu_rate, demography, mig_prop, sel_coeff, FI, dominance, preserve_mutations, take_sample,
          allele_trajectories());
}

}  // namespace GO_Fish

#endif  // GOFISH_B200_GO_FISH_CUH_
