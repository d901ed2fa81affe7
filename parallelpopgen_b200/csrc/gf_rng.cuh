// Counter-based random numbers and the approximate binomial / Poisson samplers used by
// every kernel of the engine.
//
// Bit-compatibility contract with ParallelPopGen 3P (the reference):
//   * Philox4x32 with 10 rounds, key = (seed1, seed2), counter = (k, step, population, round),
//     exactly as RNG::Philox (3P/_internal/shared.cuh:67-82).  The bijection is the published
//     Philox4x32 of Salmon, Moraes, Dror and Shaw ("Parallel random numbers: as easy as 1, 2, 3",
//     SC'11): two 32x32->64 multiplies per round and a Weyl-sequence key schedule.
//   * u = bits * 2^-32 + 2^-33 (shared.cuh:59-64), so u lies in (0, 1].
//   * the branch structure of RNG::ApproxRandBinomHelper / ApproxRandBinom1 / ApproxRandPois1
//     (shared.cu:10-18, shared.cuh:251-267): sequential inverse-CDF search when the mean is within
//     6 of either boundary (binomial search below N = 100, Poisson search otherwise), else the
//     normal approximation round(z * sqrt(var) + mean).
//   * the sequential searches stop at the same mean-dependent caps as binomcdfinv / poiscdfinv
//     (shared.cuh:89-249).  The loops below are fully unrolled so that every divisor j is a
//     compile-time constant, as it is in the reference's hand-unrolled code; the compiler then
//     makes the same code for `mean / j`.
// Device code is compiled with --use_fast_math, like the reference, and calls the same CUDA math
// functions (normcdfinv, sqrtf, expf, powf, roundf); none of them is re-derived here.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <math.h>

namespace gf {

// Published Philox4x32 constants (SC'11, Table 2 and section 5.1).
constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;  // golden ratio
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;  // sqrt(3) - 1

// Boundaries of the exact-search branches (shared.cuh:44-45).
constexpr float kMeanBoundary = 6.0f;
constexpr float kBinomNBoundary = 100.0f;

__host__ __device__ __forceinline__ void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
#ifdef __CUDA_ARCH__
  lo = a * b;
  hi = __umulhi(a, b);
#else
  const uint64_t p = static_cast<uint64_t>(a) * b;
  lo = static_cast<uint32_t>(p);
  hi = static_cast<uint32_t>(p >> 32);
#endif
}

// Philox4x32-10: ten rounds; the key is bumped by the Weyl constants before every round but the first.
__host__ __device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += kPhiloxW0;
      k1 += kPhiloxW1;
    }
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(kPhiloxM0, c.x, hi0, lo0);
    mulhilo32(kPhiloxM1, c.z, hi1, lo1);
    c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
  }
  return c;
}

// The ten round keys of one key (seed1, seed2), for kernels whose key is the same for every thread:
// passed by value as a kernel parameter they sit in the constant bank, so a round's key costs no
// instruction.
struct PhiloxKeys {
  uint32_t k0[10];
  uint32_t k1[10];
};

__host__ __device__ __forceinline__ PhiloxKeys philox_round_keys(int seed1, int seed2) {
  PhiloxKeys K;
  uint32_t k0 = static_cast<uint32_t>(seed1), k1 = static_cast<uint32_t>(seed2);
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += kPhiloxW0;
      k1 += kPhiloxW1;
    }
    K.k0[r] = k0;
    K.k1[r] = k1;
  }
  return K;
}

// philox4x32_10 with precomputed round keys (the same bijection).
__host__ __device__ __forceinline__ uint4 philox4x32_10_keys(uint4 c, const PhiloxKeys& K) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(kPhiloxM0, c.x, hi0, lo0);
    mulhilo32(kPhiloxM1, c.z, hi1, lo1);
    c = make_uint4(hi1 ^ c.y ^ K.k0[r], lo1, hi0 ^ c.w ^ K.k1[r], lo0);
  }
  return c;
}

// Counter layout of the reference: (k, step, population, round), key (seed1, seed2).
__host__ __device__ __forceinline__ uint4 philox(int seed1, int seed2, int k, int step, int population,
                                                 int round = 0) {
  return philox4x32_10(make_uint4(static_cast<uint32_t>(k), static_cast<uint32_t>(step),
                                  static_cast<uint32_t>(population), static_cast<uint32_t>(round)),
                       static_cast<uint32_t>(seed1), static_cast<uint32_t>(seed2));
}

// 32 random bits -> (0, 1]: bits * 2^-32 + 2^-33.
__host__ __device__ __forceinline__ float u01(uint32_t bits) {
  const float factor = 0x1p-32f;
  const float half_factor = 0x1p-33f;
  return static_cast<float>(bits) * factor + half_factor;
}

// Largest value the sequential searches may return for a given mean (the `|| mean <= c` exits of
// binomcdfinv / poiscdfinv).  Only means <= 6 reach these searches from the samplers below.
#define GF_SEARCH_STEP(J, CAP_MEAN)                                 \
  {                                                                 \
    GF_ITER(static_cast<float>(J));                                 \
    if (cdf >= r || ((CAP_MEAN) > 0 && mean <= (CAP_MEAN))) return J; \
  }

// Poisson inverse CDF by sequential search (poiscdfinv, shared.cuh:168-249).
__host__ __device__ __forceinline__ int pois_search(float r, float mean) {
  float emu = expf(-1 * mean);
  float cdf = emu;
  if (cdf >= r) return 0;
#define GF_ITER(JF)          \
  {                          \
    emu *= mean / (JF);      \
    cdf += emu;              \
  }
  GF_SEARCH_STEP(1, 0) GF_SEARCH_STEP(2, 0) GF_SEARCH_STEP(3, 0) GF_SEARCH_STEP(4, 0)
  GF_SEARCH_STEP(5, 0) GF_SEARCH_STEP(6, 0) GF_SEARCH_STEP(7, 0) GF_SEARCH_STEP(8, 0)
  GF_SEARCH_STEP(9, 0) GF_SEARCH_STEP(10, 0) GF_SEARCH_STEP(11, 1) GF_SEARCH_STEP(12, 0)
  GF_SEARCH_STEP(13, 0) GF_SEARCH_STEP(14, 2) GF_SEARCH_STEP(15, 0) GF_SEARCH_STEP(16, 0)
  GF_SEARCH_STEP(17, 3) GF_SEARCH_STEP(18, 0) GF_SEARCH_STEP(19, 0) GF_SEARCH_STEP(20, 4)
  GF_SEARCH_STEP(21, 0) GF_SEARCH_STEP(22, 5) GF_SEARCH_STEP(23, 0) GF_SEARCH_STEP(24, 6)
  GF_SEARCH_STEP(25, 0) GF_SEARCH_STEP(26, 7) GF_SEARCH_STEP(27, 0) GF_SEARCH_STEP(28, 8)
  GF_SEARCH_STEP(29, 0) GF_SEARCH_STEP(30, 9) GF_SEARCH_STEP(31, 0) GF_SEARCH_STEP(32, 10)
  GF_SEARCH_STEP(33, 0) GF_SEARCH_STEP(34, 11) GF_SEARCH_STEP(35, 0) GF_SEARCH_STEP(36, 12)
  GF_SEARCH_STEP(37, 0) GF_SEARCH_STEP(38, 13) GF_SEARCH_STEP(39, 0) GF_SEARCH_STEP(40, 14)
  GF_SEARCH_STEP(41, 15) GF_SEARCH_STEP(42, 0) GF_SEARCH_STEP(43, 16) GF_SEARCH_STEP(44, 0)
  GF_SEARCH_STEP(45, 17) GF_SEARCH_STEP(46, 18) GF_SEARCH_STEP(47, 0) GF_SEARCH_STEP(48, 19)
  GF_SEARCH_STEP(49, 0) GF_SEARCH_STEP(50, 20) GF_SEARCH_STEP(51, 21) GF_SEARCH_STEP(52, 0)
  GF_SEARCH_STEP(53, 22) GF_SEARCH_STEP(54, 0) GF_SEARCH_STEP(55, 23) GF_SEARCH_STEP(56, 24)
  GF_SEARCH_STEP(57, 0) GF_SEARCH_STEP(58, 25) GF_SEARCH_STEP(59, 26) GF_SEARCH_STEP(60, 0)
  GF_SEARCH_STEP(61, 27) GF_SEARCH_STEP(62, 28) GF_SEARCH_STEP(63, 0) GF_SEARCH_STEP(64, 29)
  GF_SEARCH_STEP(65, 30) GF_SEARCH_STEP(66, 0) GF_SEARCH_STEP(67, 31) GF_SEARCH_STEP(68, 32)
  GF_SEARCH_STEP(69, 0)
#undef GF_ITER
  return 70;
}

// Binomial inverse CDF by sequential search (binomcdfinv, shared.cuh:84-166); x = p, n = N.
__host__ __device__ __forceinline__ int binom_search(float r, float mean, float x, float n) {
  float emu = powf(1 - x, n);
  if (emu == 1) emu = expf(-1 * mean);
  float cdf = emu;
  if (cdf >= r) return 0;
#define GF_ITER(JF)                                       \
  {                                                       \
    emu *= ((n + 1.f - (JF)) * x) / ((JF) * (1 - x));     \
    cdf += emu;                                           \
  }
  GF_SEARCH_STEP(1, 0) GF_SEARCH_STEP(2, 0) GF_SEARCH_STEP(3, 0) GF_SEARCH_STEP(4, 0)
  GF_SEARCH_STEP(5, 0) GF_SEARCH_STEP(6, 0) GF_SEARCH_STEP(7, 0) GF_SEARCH_STEP(8, 0)
  GF_SEARCH_STEP(9, 0) GF_SEARCH_STEP(10, 0) GF_SEARCH_STEP(11, 1) GF_SEARCH_STEP(12, 0)
  GF_SEARCH_STEP(13, 0) GF_SEARCH_STEP(14, 2) GF_SEARCH_STEP(15, 0) GF_SEARCH_STEP(16, 0)
  GF_SEARCH_STEP(17, 3) GF_SEARCH_STEP(18, 0) GF_SEARCH_STEP(19, 0) GF_SEARCH_STEP(20, 4)
  GF_SEARCH_STEP(21, 0) GF_SEARCH_STEP(22, 5) GF_SEARCH_STEP(23, 0) GF_SEARCH_STEP(24, 6)
  GF_SEARCH_STEP(25, 0) GF_SEARCH_STEP(26, 7) GF_SEARCH_STEP(27, 0) GF_SEARCH_STEP(28, 8)
  GF_SEARCH_STEP(29, 0) GF_SEARCH_STEP(30, 9) GF_SEARCH_STEP(31, 0) GF_SEARCH_STEP(32, 10)
  GF_SEARCH_STEP(33, 0) GF_SEARCH_STEP(34, 11) GF_SEARCH_STEP(35, 0) GF_SEARCH_STEP(36, 12)
  GF_SEARCH_STEP(37, 0) GF_SEARCH_STEP(38, 13) GF_SEARCH_STEP(39, 0) GF_SEARCH_STEP(40, 14)
  GF_SEARCH_STEP(41, 15) GF_SEARCH_STEP(42, 0) GF_SEARCH_STEP(43, 16) GF_SEARCH_STEP(44, 0)
  GF_SEARCH_STEP(45, 17) GF_SEARCH_STEP(46, 18) GF_SEARCH_STEP(47, 0) GF_SEARCH_STEP(48, 19)
  GF_SEARCH_STEP(49, 0) GF_SEARCH_STEP(50, 20) GF_SEARCH_STEP(51, 21) GF_SEARCH_STEP(52, 0)
  GF_SEARCH_STEP(53, 22) GF_SEARCH_STEP(54, 0) GF_SEARCH_STEP(55, 23) GF_SEARCH_STEP(56, 24)
  GF_SEARCH_STEP(57, 0) GF_SEARCH_STEP(58, 25) GF_SEARCH_STEP(59, 26) GF_SEARCH_STEP(60, 0)
  GF_SEARCH_STEP(61, 27) GF_SEARCH_STEP(62, 28) GF_SEARCH_STEP(63, 0) GF_SEARCH_STEP(64, 29)
  GF_SEARCH_STEP(65, 30) GF_SEARCH_STEP(66, 0) GF_SEARCH_STEP(67, 31) GF_SEARCH_STEP(68, 32)
  GF_SEARCH_STEP(69, 0)
#undef GF_ITER
  return 70;
}
#undef GF_SEARCH_STEP

// Approximate Binomial(N, mean/N) draw from 32 random bits, `var` = (1 - p) * mean
// (ApproxRandBinomHelper, shared.cu:10-18).  Inline body shared by the two call shapes below.
__host__ __device__ __forceinline__ int binom_draw_body(uint32_t bits, float mean, float var, float N) {
  if (mean <= kMeanBoundary) {
    if (N < kBinomNBoundary) return binom_search(u01(bits), mean, mean / N, N);
    return pois_search(u01(bits), mean);
  } else if (mean >= N - kMeanBoundary) {
    if (N < kBinomNBoundary) return N - binom_search(u01(bits), N - mean, (N - mean) / N, N);
    return N - pois_search(u01(bits), N - mean);
  }
  return round(normcdfinv(u01(bits)) * sqrtf(var) + mean);
}

// Draw used for the four lanes of a mutation quad.  Kept out of line, as the reference keeps its
// quad-lane helper in a separate translation unit, so the arithmetic inside sees `mean` and `var`
// as already-rounded values in both programs.
static __device__ __noinline__ int binom_draw_lane(uint32_t bits, float mean, float var, float N) {
  return binom_draw_body(bits, mean, var, N);
}

// Draw used for the scalar tail (M % 4 leftover mutations); inlined, as ApproxRandBinom1 is.
__device__ __forceinline__ int binom_draw_tail(uint32_t bits, float mean, float var, float N) {
  return binom_draw_body(bits, mean, var, N);
}

// Poisson draw with the counter (id, generation, population, 0) (ApproxRandPois1, shared.cuh:251-256).
// Host-callable: the per-generation new-mutation count is drawn on the host, as in the reference.
__host__ __device__ __forceinline__ int pois_draw(float mean, float var, float N, int seed1, int seed2, int id,
                                                  int generation, int population) {
  const uint4 i = philox(seed1, seed2, id, generation, population, 0);
  if (mean <= kMeanBoundary) return pois_search(u01(i.x), mean);
  if (mean >= N - kMeanBoundary) return N - pois_search(u01(i.x), N - mean);
  return round(normcdfinv(u01(i.x)) * sqrtf(var) + mean);
}

}  // namespace gf
