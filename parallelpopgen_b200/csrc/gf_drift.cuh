// Per-slot model arithmetic shared by every drift kernel (per-generation and windowed): the
// expressions of migration_selection_drift (go_fish_impl.cuh:93-124) in the reference's order, so
// all kernels produce identical draws for identical (slot, generation) inputs.
#pragma once

#include "gf_rng.cuh"

// Resident drift blocks per SM the register allocation must allow (6: at most 40 registers; the
// drift kernels are latency-bound, and 6 resident blocks beat 4 by ~4% with no spills).
#ifndef GF_DRIFT_MIN_BLOCKS
#define GF_DRIFT_MIN_BLOCKS 6
#endif

namespace gf {


// Frequency after selection (go_fish_impl.cuh:105 / :119).  With s == 0 the expression reduces to
// x exactly, which the NEUTRAL instantiation uses directly.
template <bool NEUTRAL>
__device__ __forceinline__ float selected_freq(float x, float sa, float sb, float F, float h) {
  if (NEUTRAL) return x;
  const float s = fmaxf(sa * x + sb, -1.f);
  return (s * x * x + x + (F + h - h * F) * s * x * (1 - x)) /
         (x * x * s + (F + 2 * h - 2 * h * F) * s * x * (1 - x) + 1);
}

// Drift of one quad lane: returns the new count j in [0, N].  Lost (x == 0) and, for N > 6, fixed
// (x == 1) slots have a certain outcome (0 and N) and skip the sampler.
__device__ __forceinline__ int drift_lane(uint32_t bits, float xs, int N) {
  if (xs == 0.f) return 0;
  if (xs == 1.f && N > 6) return N;
  const float mean = xs * N;
  const float var = (1.0f - xs) * mean;
  return binom_draw_lane(bits, mean, var, static_cast<float>(N));
}

// Drift of one scalar-tail slot: counter (slot + 2, generation, pop, 0), variance evaluated in
// double as the reference's scalar tail does (go_fish_impl.cuh:121).
__device__ __forceinline__ int drift_tail(int seed1, int seed2, int slot, int generation, int pop, float xs, int N) {
  if (xs == 0.f) return 0;
  if (xs == 1.f && N > 6) return N;
  const float mean = xs * N;
  const float var = static_cast<float>((1.0 - static_cast<double>(xs)) * static_cast<double>(mean));
  const uint4 r = philox(seed1, seed2, slot + 2, generation, pop, 0);
  return binom_draw_tail(r.x, mean, var, static_cast<float>(N));
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return max(lo, min(v, hi)); }

// The quad-lane sampler is inlined; the reference compiles its counterpart out of line in another
// translation unit (shared.cu:10-18).  Both forms give bit-identical draws on sm_100a (checked against
// the reference kernel for every sampler branch), and inlining is ~8% faster.  GF_DRAW_OUT_OF_LINE
// restores the out-of-line call.
#ifdef GF_DRAW_OUT_OF_LINE
#define GF_LANE_DRAW binom_draw_lane
#else
#define GF_LANE_DRAW binom_draw_body
#endif


}  // namespace gf
