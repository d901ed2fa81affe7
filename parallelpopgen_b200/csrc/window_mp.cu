// Windowed drift for 2 to 4 populations: every generation of a compaction window in one launch.
//
// Migration mixes the frequencies of one mutation across populations and nothing else, so a thread
// can carry the P rows of its quad through all generations of a window in registers, as the
// single-population window kernel (window.cu) does for one row.  Each generation repeats the
// per-generation kernel's arithmetic for every drifted population in order (migration_selection_drift,
// go_fish_impl.cuh:93-124): the migration sum over the rows as they stood at the start of the
// generation, selection, the draw with counter (q + 2, g, p, 0) for whole quads and (slot + 2, g, p, 0)
// for the scalar tail, float(j) / Nc.  Births are appended after the drift (add_new_mutations,
// go_fish_impl.cu:138-145: row p = 1/Nc of the population that drew them, other rows 0, in population
// order), and only the last generation writes the rows and the compaction flags
// (flag_segregating_mutations, go_fish_impl.cuh:137-176).
//
// The per-generation kernel leaves the rows of populations that it does not drift untouched; the engine
// forms a window only while every such row is zero in both state buffers (a population that has not
// been founded yet), so writing those rows back unchanged is the same as not writing them.
#include <cuda_runtime.h>

#include <algorithm>

#include "gf_drift.cuh"
#include "gf_internal.h"

// Resident blocks per SM the register allocation must allow: the P rows and their migration sums
// live in registers across the window.
#ifndef GF_WINDOW_MP_MIN_BLOCKS
#define GF_WINDOW_MP_MIN_BLOCKS 4
#endif

namespace gf {

constexpr int kMpThreads = kDriftThreads;
constexpr int kMpTile = kMpThreads * 4;
static_assert(kMpTile == kTileSlots, "a window tile is a compaction tile");

// The fields of one generation record the window kernel reads, for P populations.
template <int P>
struct MpGen {
  int generation;
  int neutral;  // every drifted population has s(x) == 0 (the per-generation kernel's NEUTRAL case)
  int drift_mask;
  int alive_mask;
  int new_offset[P + 1];  // exclusive prefix of the per-population birth counts
  int Nc[P];
  float new_freq[P];
  float F[P], h[P], sel_a[P], sel_b[P];
  float mig[P * P];  // [from * P + to]
};

// v[p][j] for a (p, j) known only at run time, by selects (the quad stays in registers).
template <int P>
__device__ __forceinline__ float pick(const float (&v)[P][4], int p, int j) {
  float r = v[0][0];
#pragma unroll
  for (int pp = 0; pp < P; ++pp)
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) r = (pp == p && jj == j) ? v[pp][jj] : r;
  return r;
}

template <int P>
__device__ __forceinline__ void put(float (&v)[P][4], int p, int j, float x) {
#pragma unroll
  for (int pp = 0; pp < P; ++pp)
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) v[pp][jj] = (pp == p && jj == j) ? x : v[pp][jj];
}

template <int P>
__global__ void __launch_bounds__(kMpThreads, GF_WINDOW_MP_MIN_BLOCKS)
    window_mp_kernel(const float* __restrict__ A, float* __restrict__ B, long long stride, int* __restrict__ id_gp,
                     int* __restrict__ id_tid, unsigned* __restrict__ flags, unsigned* __restrict__ tile_count,
                     int* __restrict__ d_count, int slot_in, int slot_out, long long capacity,
                     const GenArgs* __restrict__ table, int ngen, long long births, int compact, int check_preserved,
                     int seed1, int seed2, unsigned long long* __restrict__ stats, const PhiloxKeys keys) {
  __shared__ MpGen<P> s_gen[kMaxWindowGenerations];
  __shared__ unsigned s_warp[kMpThreads / 32];
  __shared__ int s_tile;
  int* const sched = d_count + kSchedWord;   // tile scheduler: next tile, blocks finished
  for (int k = threadIdx.x; k < ngen; k += kMpThreads) {
    const GenArgs& a = table[k];
    MpGen<P>& G = s_gen[k];
    G.generation = a.generation;
    G.drift_mask = a.drift_mask;
    int neutral = 1;
#pragma unroll
    for (int p = 0; p < P; ++p)
      if (((a.drift_mask >> p) & 1) && (a.sel_a[p] != 0.f || a.sel_b[p] != 0.f)) neutral = 0;
    G.neutral = neutral;
    G.alive_mask = a.alive_mask;
#pragma unroll
    for (int p = 0; p <= P; ++p) G.new_offset[p] = a.new_offset[p];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      G.Nc[p] = a.Nc[p];
      G.new_freq[p] = a.new_freq[p];
      G.F[p] = a.F[p];
      G.h[p] = a.h[p];
      G.sel_a[p] = a.sel_a[p];
      G.sel_b[p] = a.sel_b[p];
    }
#pragma unroll
    for (int i = 0; i < P * P; ++i) G.mig[i] = a.mig[i];
  }
  __syncthreads();

  const int M0 = d_count[slot_in];
  const long long end = static_cast<long long>(M0) + births;  // slots at the window end
  const int cap = static_cast<int>(capacity);
  const int Mw = static_cast<int>(min(end, capacity));
  const int ntiles = (Mw + kMpTile - 1) / kMpTile;
  const int lane = threadIdx.x & 31;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    d_count[slot_out] = Mw;
    d_count[3] = Mw;
    if (end > capacity) atomicExch(d_count + 2, kFaultCapacity);  // births past the rows are not written
    unsigned long long mg = 0;
    long long m = M0;
    for (int k = 0; k < ngen; ++k) {
      mg += static_cast<unsigned long long>(m);
      m += s_gen[k].new_offset[P];
    }
    stats[0] += mg;
    stats[1] += static_cast<unsigned long long>(ngen);
  }

  // tiles handed out in order by an atomic counter (cheap tiles of late-born slots balance out)
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(sched, 1);
    __syncthreads();
    const int t = s_tile;
    __syncthreads();
    if (t >= ntiles) break;   // block-uniform
    const int q = t * kMpThreads + threadIdx.x;  // quad
    const int s0 = 4 * q;
    float x[P][4];
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const float* row = A + p * stride;
      if (s0 + 3 < M0) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(row + s0));
        x[p][0] = v.x;
        x[p][1] = v.y;
        x[p][2] = v.z;
        x[p][3] = v.w;
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) x[p][j] = (s0 + j < M0) ? row[s0 + j] : 0.f;
      }
    }

    int M = M0;
#pragma unroll 1
    for (int k = 0; k < ngen; ++k) {
      const MpGen<P>& G = s_gen[k];
      const int g = G.generation;
      if (q < (M >> 2)) {
        // whole quad: migration from the rows at the start of the generation, in source order
        float xm[P][4];
#pragma unroll
        for (int p = 0; p < P; ++p) {
#pragma unroll
          for (int j = 0; j < 4; ++j) xm[p][j] = 0.f;
#pragma unroll
          for (int kk = 0; kk < P; ++kk) {
            const float m = G.mig[kk * P + p];
#pragma unroll
            for (int j = 0; j < 4; ++j) xm[p][j] += m * x[kk][j];
          }
        }
#pragma unroll 1
        for (int p = 0; p < P; ++p) {
          if (!((G.drift_mask >> p) & 1)) continue;
          const int N = G.Nc[p];
          float o[4] = {0.f, 0.f, 0.f, 0.f};
          if (N > 0) {  // N == 0: extinction generation, the population's row is cleared
            const bool neutral = G.neutral != 0;
            float xs[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const float v = pick<P>(xm, p, j);
              xs[j] = neutral ? selected_freq<true>(v, 0.f, 0.f, 0.f, 0.f)
                              : selected_freq<false>(v, G.sel_a[p], G.sel_b[p], G.F[p], G.h[p]);
            }
            int res[4];
            unsigned need = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              res[j] = (xs[j] == 1.f && N > 6) ? N : 0;
              if (!(xs[j] == 0.f || (xs[j] == 1.f && N > 6))) need |= 1u << j;
            }
            if (need) {
              // round keys of (seed1, seed2) from the kernel parameters (constant bank)
              const uint4 r = philox4x32_10_keys(
                  make_uint4(static_cast<uint32_t>(q + 2), static_cast<uint32_t>(g), static_cast<uint32_t>(p), 0u), keys);
              draw_quad<kDrawLanes>(xs, r, need, N, lane, nullptr, res);
            }
            const float Nf = static_cast<float>(N);
#pragma unroll
            for (int j = 0; j < 4; ++j) o[j] = static_cast<float>(clampi(res[j], 0, N)) / Nf;
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) put<P>(x, p, j, o[j]);
        }
      } else if (s0 < M) {
        // scalar tail: Philox (slot + 2, g, p, 0) lane x, variance in double
#pragma unroll 1
        for (int j = 0; j < 4; ++j) {
          const int e = s0 + j;
          if (e >= M) break;
          float xo[P];
#pragma unroll
          for (int kk = 0; kk < P; ++kk) xo[kk] = pick<P>(x, kk, j);
#pragma unroll 1
          for (int p = 0; p < P; ++p) {
            if (!((G.drift_mask >> p) & 1)) continue;
            float xm = 0.f;
#pragma unroll
            for (int kk = 0; kk < P; ++kk) xm += G.mig[kk * P + p] * xo[kk];
            const int N = G.Nc[p];
            float o = 0.f;
            if (N > 0) {
              const float xs = G.neutral ? selected_freq<true>(xm, 0.f, 0.f, 0.f, 0.f)
                                         : selected_freq<false>(xm, G.sel_a[p], G.sel_b[p], G.F[p], G.h[p]);
              o = static_cast<float>(clampi(drift_tail(seed1, seed2, e, g, p, xs, N), 0, N)) /
                  static_cast<float>(N);
            }
            put<P>(x, p, j, o);
          }
        }
      }
      // births: slots [M, M + new) in population order, row p = 1/Nc, ID (g, p, slot - offset_p + 1)
      const int Mn = M + G.new_offset[P];
      if (s0 + 3 >= M && s0 < Mn) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int e = s0 + j;
          if (e >= M && e < Mn && e < cap) {
            const int r = e - M;
            int p = 0;
            while (p + 1 < P && r >= G.new_offset[p + 1]) ++p;
            const float f = G.new_freq[p];
#pragma unroll
            for (int pp = 0; pp < P; ++pp) x[pp][j] = (pp == p) ? f : 0.f;
            id_gp[e] = g | (p << 24);
            id_tid[e] = r - G.new_offset[p] + 1;
          }
        }
      }
      M = Mn;
    }

#pragma unroll
    for (int p = 0; p < P; ++p) {
      float* row = B + p * stride;
      if (s0 + 3 < Mw) {
        *reinterpret_cast<float4*>(row + s0) = make_float4(x[p][0], x[p][1], x[p][2], x[p][3]);
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (s0 + j < Mw) row[s0 + j] = x[p][j];
      }
    }

    if (compact) {
      // keep unless lost in every alive population or fixed in every alive population, or preserved
      const int alive = s_gen[ngen - 1].alive_mask;
      unsigned keep = 0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int e = s0 + j;
        if (e >= Mw) continue;
        bool zero = true, one = true;
#pragma unroll
        for (int p = 0; p < P; ++p) {
          if ((alive >> p) & 1) {
            zero = zero && (x[p][j] <= 0.f);
            one = one && (x[p][j] >= 1.f);
          }
        }
        bool k = !(zero || one);
        if (check_preserved && e < M0 && id_tid[e] < 0) k = true;
        if (k) keep |= 1u << j;
      }
      unsigned word = keep << ((lane & 7) * 4);
      word |= __shfl_xor_sync(0xFFFFFFFFu, word, 1);
      word |= __shfl_xor_sync(0xFFFFFFFFu, word, 2);
      word |= __shfl_xor_sync(0xFFFFFFFFu, word, 4);
      if ((lane & 7) == 0) flags[s0 >> 5] = word;
      unsigned c = __popc(keep);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
      if (lane == 0) s_warp[threadIdx.x >> 5] = c;
      __syncthreads();
      if (threadIdx.x == 0) {
        unsigned tot = 0;
#pragma unroll
        for (int w = 0; w < kMpThreads / 32; ++w) tot += s_warp[w];
        tile_count[t] = tot;
      }
      __syncthreads();
    }
  }
  // the last block to finish resets the scheduler for the next launch on this stream
  if (threadIdx.x == 0) {
    __threadfence();
    const int finished = atomicAdd(sched + 1, 1);
    if (finished == static_cast<int>(gridDim.x) - 1) {
      sched[0] = 0;
      sched[1] = 0;
    }
  }
}

template <int P>
static void launch_mp(Engine* e, const WindowMpLaunch& w) {
  // resident blocks per SM, queried once per population count (thread-safe initialisation)
  static const int occupancy = [] {
    int o = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, window_mp_kernel<P>, kMpThreads, 0) != cudaSuccess ||
        o < 1) {
      cudaGetLastError();
      o = 1;
    }
    return o;
  }();
  const int per_sm = e->blocks_per_sm > 0 ? std::min(e->blocks_per_sm, occupancy) : occupancy;
  const int blocks = std::max(1, std::min(w.tiles_bound, e->num_sms * per_sm));
  window_mp_kernel<P><<<blocks, kMpThreads, 0, e->stream>>>(
      w.A, w.B, w.stride, w.id_gp, w.id_tid, w.flags, w.tile_count, w.d_count, w.slot_in, w.slot_out, w.stride,
      w.table, w.ngen, w.births, w.compact, w.check_preserved, w.seed1, w.seed2, w.stats,
      philox_round_keys(w.seed1, w.seed2));
}

gf_status window_mp_run(Engine* e, const WindowMpLaunch& w) {
  if (w.ngen < 1 || w.ngen > kMaxWindowGenerations) return fail(e, GF_ERR_INVALID_ARGUMENT, "window of %d generations", w.ngen);
  switch (w.P) {
    case 2: launch_mp<2>(e, w); break;
    case 3: launch_mp<3>(e, w); break;
    case 4: launch_mp<4>(e, w); break;
    default: return fail(e, GF_ERR_INVALID_ARGUMENT, "multi-population window for %d populations", w.P);
  }
  GF_CUDA(e, cudaGetLastError());
  e->kernel_launches += 1;
  return GF_OK;
}

}  // namespace gf
