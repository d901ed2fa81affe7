// Mutation-selection-equilibrium start (initialize_mse and friends, go_fish_impl.cuh:20-71, 201-332):
// per-element and per-block device code shared by the plain engine's start and the batched start, so
// both give identical class counts for identical inputs.
#pragma once

#include "gf_rng.cuh"

namespace gf {

__device__ __forceinline__ float mse_density(float i, int N, float F, float h, float s) {
  return exp(2 * N * s * i * ((2 * h + (1 - 2 * h) * i) * (1 - F) + 2 * F) / (1 + F));
}

// Trapezoid slice `id` of the MSE integrand from frequency 1 down to 0 (calculate_area +
// trapezoidal_upper + mse_integrand, go_fish_impl.cuh:24-53).
__device__ __forceinline__ float mse_area(int id, float step, int N_ind, float F, float h, float sa, float sb) {
  const float a = static_cast<float>(1.0 - id * step);
  const float b = a - step;
  const float s1 = fmaxf(sa * a + sb, -1.f);
  const float s2 = fmaxf(sa * b + sb, -1.f);
  const float f1 = mse_density(a, N_ind, F, h, -1 * s1);
  const float f2 = mse_density(b, N_ind, F, h, -1 * s2);
  return step * (f1 + f2) / 2;
}

// Deterministic inclusive scan of the slices in double precision by one 1024-thread block, stored
// reversed as float: integral[id] = sum_{k <= num_freq-1-id} area[k] (the reference scans in float
// with CUB and then reverses, go_fish_impl.cuh:213-221; its float summation order is not fixed).
__device__ __forceinline__ void mse_integral_block(const float* __restrict__ area, float* __restrict__ integral,
                                                   int num_freq) {
  __shared__ double s_warp[32];
  __shared__ double s_carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = 0.0;
  __syncthreads();
  for (int base = 0; base < num_freq; base += 1024) {
    const int idx = base + threadIdx.x;
    const double v = idx < num_freq ? static_cast<double>(area[idx]) : 0.0;
    double incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const double w = s_warp[lane];
      double wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
        if (lane >= o) wi += y;
      }
      s_warp[lane] = wi - w;
    }
    __syncthreads();
    const double total = s_carry + s_warp[warp] + incl;
    if (idx < num_freq) integral[num_freq - 1 - idx] = static_cast<float>(total);
    __syncthreads();
    if (threadIdx.x == 1023) s_carry = total;
    __syncthreads();
  }
}

// Poisson count of mutations in frequency class `id` (initialize_mse_frequency_array,
// go_fish_impl.cuh:58-71); counter (0, class, pop, 0).
__device__ __forceinline__ unsigned mse_class_count(int id, const float* __restrict__ integral, float mse_total,
                                                    float mu, int N_ind, int Nchrom, float L, float sa, float sb,
                                                    float F, float h, int seed1, int seed2, int pop) {
  const float i = (id + 1.f) / Nchrom;
  const float j = ((Nchrom - id) + 1.f) / Nchrom;
  const float s = sa * i + sb;
  float lambda;
  if (s == 0) {
    lambda = 2 * mu * L / i;
  } else {
    lambda = 2 * mu * L * (mse_density(i, N_ind, F, h, s) * integral[id]) / (mse_total * i * j);
  }
  return static_cast<unsigned>(max(pois_draw(lambda, lambda, L * Nchrom, seed1, seed2, 0, id, pop), 0));
}

}  // namespace gf
