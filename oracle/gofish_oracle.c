/*
 * gofish_oracle.c -- CPU restatement of the GO_Fish hot path.  TEST INFRASTRUCTURE ONLY: used by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arms as the checker and
 * the timed CPU baseline; the product (parallelpopgen_b200/libgofish_b200.so) never calls it.
 *
 * Each function cites the reference code it restates (paths inside ParallelPopGen 3P v0.3.2).
 * Parity pins (tests/test_oracle.py):
 *   - Philox4x32-10 and the host Poisson draw are checked against golden vectors that the reference's
 *     own host code produced (tests/golden/ref_hostrng.bin, made by tests/golden/make_golden.py);
 *   - integer logic (counter layout, quad/tail split, compaction order, histogram binning) is exact;
 *   - drawn values depend on CUDA's fast-math device functions (normcdfinv, __expf, approximate
 *     division), which a CPU cannot reproduce bit for bit; the oracle uses libm and its own inverse
 *     normal CDF, so a small fraction of draws that sit on a rounding boundary differ by one count.
 *     The bit-exact pin for drawn values is the reference itself run on the GPU (oracle/_ref).
 *
 * Build: oracle/Makefile (gcc -O3 -fopenmp -shared).
 */
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_MAXP 16

/* ---------------------------------------------------------------------------------------------
 * Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), as keyed by RNG::Philox (shared.cuh:67-82):
 * key = (seed1, seed2), counter = (k, step, population, round).
 * ------------------------------------------------------------------------------------------- */
void or_philox(uint32_t k0, uint32_t k1, const uint32_t ctr_in[4], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    const uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline void philox_ctr(int seed1, int seed2, int k, int step, int pop, uint32_t out[4]) {
  const uint32_t ctr[4] = {(uint32_t)k, (uint32_t)step, (uint32_t)pop, 0u};
  or_philox((uint32_t)seed1, (uint32_t)seed2, ctr, out);
}

/* bits * 2^-32 + 2^-33 (uint_float_01, shared.cuh:59-64) */
float or_u01(uint32_t bits) { return (float)bits * 0x1p-32f + 0x1p-33f; }

/* ---------------------------------------------------------------------------------------------
 * Inverse standard normal CDF: P. J. Acklam's rational approximation (2003, relative error below
 * 1.2e-9) followed by one Halley step on erfc, in double precision.  Stands in for CUDA's
 * normcdfinv, which the oracle does not reproduce bit for bit.
 * ------------------------------------------------------------------------------------------- */
double or_normcdfinv(double p) {
  static const double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                              1.383577518672690e+02,  -3.066479806614716e+01, 2.506628277459239e+00};
  static const double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                              6.680131188771972e+01,  -1.328068155288572e+01};
  static const double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                              -2.549732539343734e+00, 4.374664141464968e+00,  2.938163982698783e+00};
  static const double d[4] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                              3.754408661907416e+00};
  if (p <= 0.0) return -INFINITY;
  if (p >= 1.0) return INFINITY;
  const double plow = 0.02425, phigh = 1 - plow;
  double x;
  if (p < plow) {
    const double q = sqrt(-2 * log(p));
    x = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
        ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1);
  } else if (p <= phigh) {
    const double q = p - 0.5, r = q * q;
    x = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
        (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1);
  } else {
    const double q = sqrt(-2 * log(1 - p));
    x = -(((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
        ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1);
  }
  /* Halley refinement */
  const double e = 0.5 * erfc(-x / sqrt(2.0)) - p;
  const double u = e * sqrt(2 * M_PI) * exp(x * x / 2);
  x = x - u / (1 + x * u / 2);
  return x;
}

/* float -> int as the GPU converts it: saturating, NaN -> 0 */
static inline int sat_int(float v) {
  if (v != v) return 0;
  if (v >= 2147483648.0f) return INT_MAX;
  if (v <= -2147483648.0f) return INT_MIN;
  return (int)v;
}

/* largest value the sequential searches return for a given mean: the `|| mean <= c` exits of
 * poiscdfinv / binomcdfinv (shared.cuh:105-165, 188-248), indexed by j -> c (0 = none) */
static const int kCapMean[70] = {
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 2, 0, 0, 3, 0, 0, 4, 0, 5, 0, 6, 0, 7, 0, 8, 0, 9, 0, 10, 0, 11,
    0, 12, 0, 13, 0, 14, 15, 0, 16, 0, 17, 18, 0, 19, 0, 20, 21, 0, 22, 0, 23, 24, 0, 25, 26, 0, 27, 28, 0, 29,
    30, 0, 31, 32, 0};

/* Poisson inverse CDF by sequential search (poiscdfinv, shared.cuh:168-249) */
int or_pois_search(float r, float mean) {
  float emu = expf(-1 * mean);
  float cdf = emu;
  if (cdf >= r) return 0;
  for (int j = 1; j < 70; ++j) {
    emu *= mean / (float)j;
    cdf += emu;
    if (cdf >= r || (kCapMean[j] > 0 && mean <= (float)kCapMean[j])) return j;
  }
  return 70;
}

/* Binomial inverse CDF by sequential search (binomcdfinv, shared.cuh:84-166) */
int or_binom_search(float r, float mean, float x, float n) {
  float emu = powf(1 - x, n);
  if (emu == 1) emu = expf(-1 * mean);
  float cdf = emu;
  if (cdf >= r) return 0;
  for (int j = 1; j < 70; ++j) {
    const float jf = (float)j;
    emu *= ((n + 1.f - jf) * x) / (jf * (1 - x));
    cdf += emu;
    if (cdf >= r || (kCapMean[j] > 0 && mean <= (float)kCapMean[j])) return j;
  }
  return 70;
}

static inline float round_normal(float u, float var, float mean) {
  const float z = (float)or_normcdfinv((double)u);
  return roundf(z * sqrtf(var) + mean);
}

/* Approximate Binomial(N, mean/N) from 32 random bits (ApproxRandBinomHelper, shared.cu:10-18) */
int or_binom_draw(uint32_t bits, float mean, float var, float N) {
  const float u = or_u01(bits);
  if (mean <= 6) {
    if (N < 100) return or_binom_search(u, mean, mean / N, N);
    return or_pois_search(u, mean);
  } else if (mean >= N - 6) {
    if (N < 100) return sat_int(N - (float)or_binom_search(u, N - mean, (N - mean) / N, N));
    return sat_int(N - (float)or_pois_search(u, N - mean));
  }
  return sat_int(round_normal(u, var, mean));
}

/* Approximate Poisson draw, counter (id, generation, population, 0) (ApproxRandPois1, shared.cuh:251-256) */
int or_pois_draw(float mean, float var, float N, int seed1, int seed2, int id, int generation, int population) {
  uint32_t r[4];
  philox_ctr(seed1, seed2, id, generation, population, r);
  const float u = or_u01(r[0]);
  if (mean <= 6) return or_pois_search(u, mean);
  if (mean >= N - 6) return sat_int(N - (float)or_pois_search(u, N - mean));
  return sat_int(round_normal(u, var, mean));
}

/* new mutations of one population in one generation (calc_new_mutations_Index, go_fish_impl.cuh:454-467) */
int or_new_mutation_count(int seed1, int seed2, float mu, int Nchrom_e, float num_sites, int generation, int pop) {
  const float lambda = mu * Nchrom_e * num_sites;
  if (Nchrom_e == 0 || lambda == 0) return 0;
  const int c = or_pois_draw(lambda, lambda, Nchrom_e * num_sites, seed1, seed2, 1, generation, pop);
  return c > 0 ? c : 0;
}

/* ---------------------------------------------------------------------------------------------
 * One generation of migration, selection and drift (migration_selection_drift,
 * go_fish_impl.cuh:93-124) for every population p with drift[p] != 0.
 *   prev, next   [P][stride] rows;  M slots are updated
 * Counter layout: slots i < 4*floor(M/4) use Philox(k = i/4 + 2) lane i%4 and a float variance;
 * the scalar tail uses Philox(k = i + 2) lane x and a variance computed in double.
 * ------------------------------------------------------------------------------------------- */
typedef struct or_gen {
  int generation;
  int P;
  int seed1, seed2;
  int drift[OR_MAXP];
  int Nc[OR_MAXP];
  float F[OR_MAXP], h[OR_MAXP];
  float sel_slope[OR_MAXP], sel_intercept[OR_MAXP];
  float mig[OR_MAXP * OR_MAXP]; /* [from * P + to] */
} or_gen;

static inline float selected(float x, float sa, float sb, float F, float h) {
  float s = sa * x + sb;
  if (s < -1.f) s = -1.f;
  return (s * x * x + x + (F + h - h * F) * s * x * (1 - x)) / (x * x * s + (F + 2 * h - 2 * h * F) * s * x * (1 - x) + 1);
}

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

void or_drift(const float* prev, float* next, long stride, int M, const or_gen* g, int threads) {
  const int P = g->P;
  const int nquads = M / 4;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(static) if (threads != 1)
#endif
  for (int q = 0; q < nquads; ++q) {
    for (int p = 0; p < P; ++p) {
      if (!g->drift[p]) continue;
      const int N = g->Nc[p];
      float xs[4];
      for (int j = 0; j < 4; ++j) {
        float xm = 0.f;
        for (int k = 0; k < P; ++k) xm += g->mig[k * P + p] * prev[k * stride + 4 * q + j];
        xs[j] = selected(xm, g->sel_slope[p], g->sel_intercept[p], g->F[p], g->h[p]);
      }
      if (N <= 0) {
        for (int j = 0; j < 4; ++j) next[p * stride + 4 * q + j] = 0.f;
        continue;
      }
      uint32_t r[4];
      philox_ctr(g->seed1, g->seed2, q + 2, g->generation, p, r);
      for (int j = 0; j < 4; ++j) {
        const float mean = xs[j] * N;
        const float var = (1.0f - xs[j]) * mean;
        const int c = clampi(or_binom_draw(r[j], mean, var, (float)N), 0, N);
        next[p * stride + 4 * q + j] = (float)c / (float)N;
      }
    }
  }
  for (int i = 4 * nquads; i < M; ++i) {
    for (int p = 0; p < P; ++p) {
      if (!g->drift[p]) continue;
      const int N = g->Nc[p];
      float xm = 0.f;
      for (int k = 0; k < P; ++k) xm += g->mig[k * P + p] * prev[k * stride + i];
      if (N <= 0) {
        next[p * stride + i] = 0.f;
        continue;
      }
      const float xs = selected(xm, g->sel_slope[p], g->sel_intercept[p], g->F[p], g->h[p]);
      const float mean = xs * N;
      const float var = (float)((1.0 - (double)xs) * (double)mean);
      uint32_t r[4];
      philox_ctr(g->seed1, g->seed2, i + 2, g->generation, p, r);
      const int c = clampi(or_binom_draw(r[0], mean, var, (float)N), 0, N);
      next[p * stride + i] = (float)c / (float)N;
    }
  }
}

/* New mutations of one population (add_new_mutations, go_fish_impl.cu:138-145): slots
 * [first, first + count) get frequency 1/Nc in `pop` and 0 elsewhere; IDs (gen, pop, id + 1, 0). */
void or_add_new(float* freq, long stride, int P, int32_t* ids, int first, int count, float new_freq, int pop, int gen) {
  for (int id = 0; id < count; ++id) {
    for (int k = 0; k < P; ++k) freq[k * stride + first + id] = (k == pop) ? new_freq : 0.f;
    int32_t* m = ids + 4 * (long)(first + id);
    m[0] = gen;
    m[1] = pop;
    m[2] = id + 1;
    m[3] = 0;
  }
}

/* Stable compaction (flag_segregating_mutations + scatter_arrays, go_fish_impl.cuh:137-176,
 * go_fish_impl.cu:147-189): keep slot i iff it is not lost in every alive population and not fixed
 * in every alive population, or it is preserved (threadID < 0); `preserve` marks survivors.
 * Compacts in place; returns the new count. */
int or_compact(float* freq, long stride, int P, int32_t* ids, int M, const int* alive, int preserve) {
  int w = 0;
  for (int i = 0; i < M; ++i) {
    int zero = 1, one = 1;
    for (int p = 0; p < P; ++p) {
      if (!alive[p]) continue;
      const float f = freq[p * stride + i];
      zero = zero && (f <= 0.f);
      one = one && (f >= 1.f);
    }
    const int keep = !(zero || one) || ids[4 * (long)i + 2] < 0;
    if (!keep) continue;
    for (int p = 0; p < P; ++p) freq[p * stride + w] = freq[p * stride + i];
    for (int k = 0; k < 4; ++k) ids[4 * (long)w + k] = ids[4 * (long)i + k];
    if (preserve) ids[4 * (long)w + 2] = -abs(ids[4 * (long)w + 2]);
    ++w;
  }
  return w;
}

/* Population frequency histogram (population_hist + uint_to_float, spectrum.cu:74-88): bin
 * round(Nc * f), Nc folds into 0, plus (num_sites - M) in bin 0, uint32 arithmetic. */
void or_histogram(const float* f, int M, int Nc, float num_sites, float* out) {
  uint32_t* h = (uint32_t*)calloc((size_t)Nc + 1, sizeof(uint32_t));
  for (int i = 0; i < M; ++i) {
    int j = (int)roundf(Nc * f[i]);
    if (j < 0) j = 0;
    if (j > Nc) j = Nc;
    h[j] += 1;
  }
  h[0] += h[Nc];
  h[0] += (uint32_t)((int)num_sites - M);
  for (int k = 0; k < Nc; ++k) out[k] = (float)h[k];
  free(h);
}

/* Binomially projected SFS of sample size n in double precision (binom<1024>, spectrum.cu:111-139):
 * out[k] for k < n; k = n and every non-segregating mutation fold into 0, plus (num_sites - M). */
void or_sfs(const float* f, int M, int n, float num_sites, double* out) {
  double* lgc = (double*)malloc(sizeof(double) * (n + 1));
  const double ln = lgamma(n + 1.0);
  for (int k = 0; k <= n; ++k) lgc[k] = ln - lgamma(k + 1.0) - lgamma(n - k + 1.0);
  double* acc = (double*)calloc((size_t)n + 1, sizeof(double));
  double nonseg = 0;
  for (int i = 0; i < M; ++i) {
    const float p = f[i];
    if (!(p > 0.f && p < 1.f)) {
      nonseg += 1;
      continue;
    }
    const double lp = log((double)p), lq = log1p(-(double)p);
    for (int k = 0; k <= n; ++k) acc[k] += exp(lgc[k] + k * lp + (n - k) * lq);
  }
  for (int k = 0; k < n; ++k) out[k] = acc[k];
  out[0] += acc[n] + nonseg + (double)(num_sites - M);
  free(acc);
  free(lgc);
}

/* ---------------------------------------------------------------------------------------------
 * Whole single-population run from a given state (the run_sim loop, go_fish_impl.cuh:645-714) for
 * a constant model: used as the CPU baseline and for CPU-side statistics.  `freq` and `ids` must
 * have room for `capacity` slots; returns the final count, or -1 if capacity is exceeded.
 * Sum of slots drifted over all generations is written to *mutation_generations.
 * ------------------------------------------------------------------------------------------- */
int or_run_single(float* freq, float* scratch, int32_t* ids, int M, int capacity, int first_gen, int num_gens,
                  int Nc, float F, float h, float sel_slope, float sel_intercept, float mu, float num_sites,
                  int seed1, int seed2, int compact_interval, int threads, double* mutation_generations) {
  or_gen g;
  memset(&g, 0, sizeof(g));
  g.P = 1;
  g.seed1 = seed1;
  g.seed2 = seed2;
  g.drift[0] = 1;
  g.Nc[0] = Nc;
  g.F[0] = F;
  g.h[0] = h;
  g.sel_slope[0] = sel_slope;
  g.sel_intercept[0] = sel_intercept;
  g.mig[0] = 1.f;
  const int alive[1] = {1};
  const float new_freq = 1.f / Nc;
  double mg = 0;
  int next_compact = first_gen + compact_interval;
  const int final_gen = first_gen + num_gens;
  float* cur = freq;
  float* nxt = scratch;
  for (int gen = first_gen + 1; gen <= final_gen; ++gen) {
    g.generation = gen;
    or_drift(cur, nxt, capacity, M, &g, threads);
    mg += M;
    const int c = or_new_mutation_count(seed1, seed2, mu, Nc, num_sites, gen, 0);
    if (M + c > capacity) return -1;
    or_add_new(nxt, capacity, 1, ids, M, c, new_freq, 0, gen);
    M += c;
    float* t = cur;
    cur = nxt;
    nxt = t;
    if ((gen == next_compact || gen == final_gen) && compact_interval > 0) {
      M = or_compact(cur, capacity, 1, ids, M, alive, 0);
      next_compact = gen + compact_interval;
    }
  }
  if (cur != freq) memcpy(freq, cur, sizeof(float) * (size_t)M);
  if (mutation_generations) *mutation_generations = mg;
  return M;
}

int or_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
