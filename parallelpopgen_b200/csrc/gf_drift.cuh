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
// The bound the window kernel is compiled for (its state lives in registers across a whole window).
// Six resident 256-thread blocks per SM: the batched form (round keys derived per thread) needs the
// bound to stay within 40 registers.  The single-replicate form (round keys from the kernel
// parameters) is compiled for 5, which lets the compiler use 40 registers, with which six blocks still
// fit (40 x 256 x 6 = 61,440 of 65,536): ~1 % faster than asking for 6 (36 registers).  Asking for 8
// fits it in 29 registers without spills but is 3.5 % slower.
#ifndef GF_WINDOW_MIN_BLOCKS
#define GF_WINDOW_MIN_BLOCKS GF_DRIFT_MIN_BLOCKS
#endif
#ifndef GF_WINDOW_MIN_BLOCKS_KEYS
#define GF_WINDOW_MIN_BLOCKS_KEYS 5
#endif
// 1: a single-replicate window launch takes its Philox round keys from the kernel parameters.
#ifndef GF_WINDOW_UNIFORM_KEYS
#define GF_WINDOW_UNIFORM_KEYS 1
#endif
// 1: the lane-order draw schedule walks a quad's lanes in a rolled loop (one inlined copy of the
// sampler instead of four); 0: the loop is unrolled.
#ifndef GF_LANES_ROLLED
#define GF_LANES_ROLLED 0
#endif

namespace gf {


// Frequency after selection (go_fish_impl.cuh:105 / :119).  With s == 0 the expression reduces to
// x exactly, which the NEUTRAL instantiation uses directly.
// The selection step for a given coefficient s (already clamped at -1).
__device__ __forceinline__ float selection_step(float x, float s, float F, float h) {
  return (s * x * x + x + (F + h - h * F) * s * x * (1 - x)) /
         (x * x * s + (F + 2 * h - 2 * h * F) * s * x * (1 - x) + 1);
}

template <bool NEUTRAL>
__device__ __forceinline__ float selected_freq(float x, float sa, float sb, float F, float h) {
  if (NEUTRAL) return x;
  return selection_step(x, fmaxf(sa * x + sb, -1.f), F, h);
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


// How the draws of a warp's quads are scheduled.  All three give identical results: every lane
// calls the same sampler on the same (bits, mean, var, N); only the order of the calls differs.
enum DrawStrategy : int {
  kDrawLanes = 0,    // each thread draws its needed lanes in lane order
  kDrawWarp = 1,     // the warp pools its draws in shared memory and runs them branch by branch
  kDrawGrouped = 2,  // each thread draws its normal-branch lanes first, then its search-branch lanes
  kDrawNormalAll = 3,  // the normal approximation of all four lanes at once, then the search lanes
  kDrawPooledSearch = 4,  // the normal approximation of all four lanes in each thread, then the warp's
                          // search-branch draws pooled in shared memory and run together
};
constexpr int kDrawStrategies = 5;

// Sampler branch of a lane (binom_draw_body): the sequential searches for mean <= 6 or
// mean >= N - 6, the normal approximation otherwise.
__device__ __forceinline__ bool search_branch(float mean, float Nf) {
  return mean <= kMeanBoundary || mean >= Nf - kMeanBoundary;
}

// Work items of one warp for kDrawWarp: the draws of its 128 slots that need the sampler, compacted
// so that every round of 32 lanes runs the same branch of the sampler.  Normal-approximation items
// fill the arrays from the front, sequential-search items from the back.  The results are read
// back four at a time (int4), so the struct is 16-byte aligned wherever it is declared.
struct __align__(16) WarpDraws {
  uint32_t bits[128];
  float mean[128];
  float var[128];
  int res[128];
  unsigned char slot[128];
};
static_assert(alignof(WarpDraws) == 16 && sizeof(WarpDraws) % 16 == 0, "int4 reads of WarpDraws::res");

// Draws of the lanes of one quad whose bit is set in `need` (res[j] keeps its value elsewhere).
// kDrawWarp must be called by all 32 lanes of the warp together; `w` is only used by it.
template <int DRAW>
__device__ __forceinline__ void draw_quad(const float xs[4], const uint4 r, unsigned need, int N, int lane,
                                          WarpDraws* w, int res[4]) {
  const float Nf = static_cast<float>(N);
  const uint32_t rb[4] = {r.x, r.y, r.z, r.w};
  if (DRAW == kDrawLanes) {
#if GF_LANES_ROLLED
#pragma unroll 1
    for (unsigned m = need; m; m &= m - 1u) {
      const int j = __ffs(m) - 1;
      const float x = j == 0 ? xs[0] : j == 1 ? xs[1] : j == 2 ? xs[2] : xs[3];
      const uint32_t b = j == 0 ? rb[0] : j == 1 ? rb[1] : j == 2 ? rb[2] : rb[3];
      const int d = GF_LANE_DRAW(b, x * N, (1.0f - x) * (x * N), Nf);
      res[0] = j == 0 ? d : res[0];
      res[1] = j == 1 ? d : res[1];
      res[2] = j == 2 ? d : res[2];
      res[3] = j == 3 ? d : res[3];
    }
#else
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if ((need >> j) & 1u) res[j] = GF_LANE_DRAW(rb[j], xs[j] * N, (1.0f - xs[j]) * (xs[j] * N), Nf);
#endif
    return;
  }
  if (DRAW == kDrawNormalAll) {
    // The normal-approximation branch of binom_draw_body for the four lanes without branches between
    // them (independent chains the scheduler can interleave); lanes whose mean takes a search branch
    // then replace their value.  Lanes that need no draw compute a value that is discarded.
    if (!need) return;
    float mean[4], var[4];
    int nrm[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      mean[j] = xs[j] * N;
      var[j] = (1.0f - xs[j]) * (xs[j] * N);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) nrm[j] = round(normcdfinv(u01(rb[j])) * sqrtf(var[j]) + mean[j]);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (!((need >> j) & 1u)) continue;
      res[j] = search_branch(mean[j], Nf) ? GF_LANE_DRAW(rb[j], mean[j], var[j], Nf) : nrm[j];
    }
    return;
  }
  if (DRAW == kDrawPooledSearch) {
    // Every lane of the warp calls this together.  The normal approximation of a thread's four lanes
    // runs without branches between them; the draws that take a sequential search (means within 6
    // of 0 or N, about one lane in five) are pooled across the warp and run 32 at a time, so the warp
    // runs the search code about once per quad position set instead of once per lane position.  Each
    // pooled draw calls the same sampler on the same (bits, mean, var, N) as the lane-order schedule.
    float mean[4], var[4];
    unsigned search = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      mean[j] = xs[j] * N;
      var[j] = (1.0f - xs[j]) * (xs[j] * N);
      if (((need >> j) & 1u) && search_branch(mean[j], Nf)) search |= 1u << j;
    }
    if (need & ~search) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int nrm = round(normcdfinv(u01(rb[j])) * sqrtf(var[j]) + mean[j]);
        if (((need & ~search) >> j) & 1u) res[j] = nrm;
      }
    }
    const unsigned lt = (1u << lane) - 1u;
    int nS = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const bool mine = (search >> j) & 1u;
      const unsigned b = __ballot_sync(0xFFFFFFFFu, mine);
      if (mine) {
        const int k = nS + __popc(b & lt);
        w->bits[k] = rb[j];
        w->mean[k] = mean[j];
        w->var[k] = var[j];
        w->slot[k] = static_cast<unsigned char>(4 * lane + j);
      }
      nS += __popc(b);
    }
    if (nS == 0) return;   // warp-uniform
    __syncwarp();
    for (int k = lane; k < nS; k += 32) w->res[w->slot[k]] = GF_LANE_DRAW(w->bits[k], w->mean[k], w->var[k], Nf);
    __syncwarp();
    if (search) {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if ((search >> j) & 1u) res[j] = w->res[4 * lane + j];
    }
    __syncwarp();
    return;
  }
  if (DRAW == kDrawGrouped) {
    // A warp's lanes mix both branches at almost every lane position, so drawing lane j of every
    // thread at once runs both branches four times; grouping a thread's lanes by branch runs the
    // normal branch (at most) four times and the search branch only as often as the thread with
    // the most search lanes needs.  The lane is picked by selects, keeping the quad in registers.
    unsigned search = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (((need >> j) & 1u) && search_branch(xs[j] * N, Nf)) search |= 1u << j;
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
      for (unsigned m = pass ? search : (need & ~search); m; m &= m - 1u) {
        const int j = __ffs(m) - 1;
        const float x = j == 0 ? xs[0] : j == 1 ? xs[1] : j == 2 ? xs[2] : xs[3];
        const uint32_t b = j == 0 ? rb[0] : j == 1 ? rb[1] : j == 2 ? rb[2] : rb[3];
        const int d = GF_LANE_DRAW(b, x * N, (1.0f - x) * (x * N), Nf);
        res[0] = j == 0 ? d : res[0];
        res[1] = j == 1 ? d : res[1];
        res[2] = j == 2 ? d : res[2];
        res[3] = j == 3 ? d : res[3];
      }
    }
    return;
  }
  const unsigned lt = (1u << lane) - 1u;
  int nN = 0, nS = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const bool has = (need >> j) & 1u;
    const float mean = xs[j] * N;
    const float var = (1.0f - xs[j]) * mean;
    const bool search = has && search_branch(mean, Nf);
    const bool normal = has && !search;
    const unsigned bN = __ballot_sync(0xFFFFFFFFu, normal);
    const unsigned bS = __ballot_sync(0xFFFFFFFFu, search);
    int k = -1;
    if (normal) k = nN + __popc(bN & lt);
    if (search) k = 127 - (nS + __popc(bS & lt));
    if (k >= 0) {
      w->bits[k] = rb[j];
      w->mean[k] = mean;
      w->var[k] = var;
      w->slot[k] = static_cast<unsigned char>(4 * lane + j);
    }
    nN += __popc(bN);
    nS += __popc(bS);
  }
  __syncwarp();
  for (int k = lane; k < nN; k += 32) w->res[w->slot[k]] = GF_LANE_DRAW(w->bits[k], w->mean[k], w->var[k], Nf);
  for (int k = lane; k < nS; k += 32) {
    const int kk = 127 - k;
    w->res[w->slot[kk]] = GF_LANE_DRAW(w->bits[kk], w->mean[kk], w->var[kk], Nf);
  }
  __syncwarp();
  if (need) {
    const int4 rr = reinterpret_cast<const int4*>(w->res)[lane];
    if (need & 1u) res[0] = rr.x;
    if (need & 2u) res[1] = rr.y;
    if (need & 4u) res[2] = rr.z;
    if (need & 8u) res[3] = rr.w;
  }
  __syncwarp();
}

}  // namespace gf
