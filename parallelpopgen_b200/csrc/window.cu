// Windowed drift: every generation of a compaction window in one launch.
//
// Between two compactions a mutation keeps its slot, and its update in generation g depends only
// on its own frequency, the generation's parameters, the slot index and the mutation count M_g at
// the start of g (which decides the quad / scalar-tail counter layout, go_fish_impl.cuh:97-123).
// M_g = M_start + the host-drawn new-mutation counts of the earlier generations of the window, so
// one thread can carry its quad through all generations in registers: read the row once, drift it
// W times with exactly the per-generation arithmetic (gf_drift.cuh), let slots born inside the
// window start at 1/Nc in their birth generation (add_new_mutations, go_fish_impl.cu:138-145), and
// write the row once with the survival flags of the last generation.  A launch covers any number of
// single-population replicates, each in its own 1024-aligned arena segment with its own window
// length, seeds and parameters: the plain engine uses it with one replicate, the batched engine with
// thousands.  Results are bit-identical to running the per-generation kernel W times.
#include <cuda_runtime.h>

#include <algorithm>

#include "gf_drift.cuh"
#include "gf_internal.h"

namespace gf {

constexpr int kWinThreads = 256;
constexpr int kWinTile = kWinThreads * 4;

__device__ __forceinline__ int list_count(const RepList& L, int nreps) { return L.count ? *L.count : nreps; }
__device__ __forceinline__ int list_rep(const RepList& L, int i) { return L.rep ? L.rep[i] : i; }
__device__ __forceinline__ int list_tile0(const RepList& L, const WinRep* __restrict__ reps, int i) {
  return L.tile0 ? L.tile0[i] : reps[i].tile0;
}

// listed replicate owning launch tile `gt` (the last one whose tile0 <= gt)
__device__ __forceinline__ int find_rep(const RepList& L, const WinRep* __restrict__ reps, int n, int gt) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (list_tile0(L, reps, mid) <= gt) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Shared-memory copy of the listed replicates' first tiles (up to kRepCache of them), so the per-tile
// owner search does not chase global memory.
constexpr int kRepCache = 4096;

__device__ __forceinline__ int find_rep_cached(const int* s_tile0, const RepList& L, const WinRep* __restrict__ reps,
                                               int n, int gt) {
  if (n > kRepCache) return find_rep(L, reps, n, gt);
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (s_tile0[mid] <= gt) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void load_tile0(int* s_tile0, const RepList& L, const WinRep* __restrict__ reps, int n) {
  if (n <= kRepCache)
    for (int j = threadIdx.x; j < n; j += blockDim.x) s_tile0[j] = list_tile0(L, reps, j);
  __syncthreads();
}

// Tiles of one super-step, assigned on the device: replicate j's births over its window are summed
// from its generation records, and it gets ceil((M_in + births) / 1024) tiles (at least one, at most
// its segment), laid out in replicate order.  One block.
__global__ void __launch_bounds__(1024) batch_tiles_kernel(WinRep* __restrict__ reps, int nreps,
                                                           const int* __restrict__ M_in,
                                                           const WinGen* __restrict__ recs, int* __restrict__ total) {
  __shared__ int s_warp[32];
  __shared__ int s_carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int base = 0; base < nreps; base += 1024) {
    const int j = base + threadIdx.x;
    int need = 0;
    if (j < nreps) {
      WinRep& R = reps[j];
      long long births = 0;
      for (int k = 0; k < R.ngen; ++k) births += recs[R.rec + k].new_count;
      R.births = births;
      const long long end = static_cast<long long>(M_in[R.rep]) + births;
      const long long cap_tiles = R.capacity / kWinTile;
      need = static_cast<int>(max(1ll, min(cap_tiles, (end + kWinTile - 1) / kWinTile)));
    }
    int incl = need;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      int w = s_warp[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, w, o);
        if (lane >= o) w += y;
      }
      s_warp[lane] = w;
    }
    __syncthreads();
    const int before = s_carry + (warp > 0 ? s_warp[warp - 1] : 0) + incl - need;
    if (j < nreps) {
      reps[j].tile0 = before;
      reps[j].ntiles = need;
    }
    __syncthreads();
    if (threadIdx.x == 0) s_carry += s_warp[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = s_carry;
}

// Tiles of super-step k = *step of a batch with precomputed records, and every replicate's window
// derived on the device: replicate r (cadence c, G generations) runs generations (k c, min(G, (k+1) c)]
// from record slab j = k / slab_windows at its offset in region j; a finished replicate gets no tiles.
// The others get ceil((M_in + births) / 1024) tiles (at least one, at most their segment), in replicate
// order, and are listed (table index, first tile, count) for the window, scan and scatter kernels, which
// then never visit a finished replicate (its state and counts stay as they are).  One block; thread 0
// advances the counter once every thread has read it.
__global__ void __launch_bounds__(1024) batch_step_kernel(WinRep* __restrict__ reps, int R,
                                                          const int* __restrict__ M_in,
                                                          const WinGen* __restrict__ recs, int* __restrict__ total,
                                                          int* __restrict__ step, const BatchStepPlan plan,
                                                          const int* __restrict__ region_off,
                                                          const long long* __restrict__ region_base,
                                                          const StepRep* __restrict__ steprep, int* __restrict__ fault,
                                                          int* __restrict__ list_rep, int* __restrict__ list_tile0,
                                                          int* __restrict__ list_count) {
  __shared__ int s_tiles[32], s_listed[32];
  __shared__ int s_carry_tiles, s_carry_listed;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int k = *step;
  const int j = k / plan.slab_windows;
  const bool in_plan = j < plan.nregions;
  const long long slot_base = !in_plan              ? 0
                              : plan.ring_slots > 0 ? static_cast<long long>(j % plan.ring_slots) * plan.slot_records
                                                    : region_base[j];
  if (threadIdx.x == 0) {
    s_carry_tiles = 0;
    s_carry_listed = 0;
  }
  __syncthreads();   // every thread has read *step
  for (int base = 0; base < R; base += 1024) {
    const int r = base + threadIdx.x;
    int need = 0;
    if (r < R) {
      const StepRep sr = steprep[r];
      const long long gen = static_cast<long long>(k) * sr.cadence;
      int ngen = 0, rec = 0;
      long long births = 0;
      if (in_plan && gen < sr.gens) {
        const int off = region_off[static_cast<size_t>(r) * plan.nregions + j];
        if (off < 0) {
          atomicExch(fault, kFaultRecords);
        } else {
          ngen = static_cast<int>(min(static_cast<long long>(sr.cadence), sr.gens - gen));
          rec = static_cast<int>(slot_base + off + (gen - static_cast<long long>(j) * sr.chunk));
          // the window's new-mutation counts, eight independent loads at a time
          for (int g0 = 0; g0 < ngen; g0 += 8) {
            int c[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) c[i] = g0 + i < ngen ? recs[rec + g0 + i].new_count : 0;
#pragma unroll
            for (int i = 0; i < 8; ++i) births += c[i];
          }
          const long long end = static_cast<long long>(M_in[r]) + births;
          const long long cap_tiles = reps[r].capacity / kWinTile;
          need = static_cast<int>(max(1ll, min(cap_tiles, (end + kWinTile - 1) / kWinTile)));
        }
      }
      WinRep& W = reps[r];
      W.rec = rec;
      W.ngen = ngen;
      W.births = births;
      W.compact = need > 0 ? 1 : 0;
      W.ntiles = need;
    }
    // exclusive scans of the tiles and of the listed (unfinished) replicates over the block
    const int listed = need > 0 ? 1 : 0;
    int incl_t = need, incl_l = listed;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int yt = __shfl_up_sync(0xFFFFFFFFu, incl_t, o);
      const int yl = __shfl_up_sync(0xFFFFFFFFu, incl_l, o);
      if (lane >= o) {
        incl_t += yt;
        incl_l += yl;
      }
    }
    if (lane == 31) {
      s_tiles[warp] = incl_t;
      s_listed[warp] = incl_l;
    }
    __syncthreads();
    if (warp == 0) {
      int wt = s_tiles[lane], wl = s_listed[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int yt = __shfl_up_sync(0xFFFFFFFFu, wt, o);
        const int yl = __shfl_up_sync(0xFFFFFFFFu, wl, o);
        if (lane >= o) {
          wt += yt;
          wl += yl;
        }
      }
      s_tiles[lane] = wt;
      s_listed[lane] = wl;
    }
    __syncthreads();
    const int tile0 = s_carry_tiles + (warp > 0 ? s_tiles[warp - 1] : 0) + incl_t - need;
    const int pos = s_carry_listed + (warp > 0 ? s_listed[warp - 1] : 0) + incl_l - listed;
    if (r < R) reps[r].tile0 = tile0;
    if (listed) {
      list_rep[pos] = r;
      list_tile0[pos] = tile0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      s_carry_tiles += s_tiles[31];
      s_carry_listed += s_listed[31];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    *total = s_carry_tiles;
    *list_count = s_carry_listed;
    *step = k + 1;
  }
}

// DRAW: how a warp schedules its sampler draws (DrawStrategy).  KEYS: every replicate of the launch
// has the seeds whose round keys `keys` holds (a plain-engine launch), so the quads' Philox blocks take
// their round keys from the kernel parameters instead of deriving them from the replicate's seeds.
template <int DRAW, bool KEYS>
__global__ void __launch_bounds__(kWinThreads, KEYS ? GF_WINDOW_MIN_BLOCKS_KEYS : GF_WINDOW_MIN_BLOCKS)
    window_kernel(const float* __restrict__ A, float* __restrict__ B, int* __restrict__ id_gp,
                  int* __restrict__ id_tid, unsigned* __restrict__ flags, unsigned* __restrict__ tile_count,
                  const int* __restrict__ M_in, int* __restrict__ M_end, int* __restrict__ M_next,
                  const WinRep* __restrict__ reps, int nreps, const WinGen* __restrict__ recs, int total_tiles,
                  const int* __restrict__ total_dev, unsigned long long* __restrict__ stats,
                  int* __restrict__ fault, const PhiloxKeys keys, int* __restrict__ sched, const RepList list) {
  __shared__ int s_rep;
  __shared__ int s_tile;
  __shared__ unsigned s_warp[kWinThreads / 32];
  __shared__ int s_tile0[kRepCache];
  __shared__ WarpDraws s_draws[(DRAW == kDrawWarp || DRAW == kDrawPooledSearch) ? kWinThreads / 32 : 1];
  const int lane = threadIdx.x & 31;
  WarpDraws* wd = &s_draws[(DRAW == kDrawWarp || DRAW == kDrawPooledSearch) ? (threadIdx.x >> 5) : 0];
  const int ntiles_all = total_dev ? *total_dev : total_tiles;
  const int nlist = list_count(list, nreps);
  load_tile0(s_tile0, list, reps, nlist);
  // Tiles are handed out in order by an atomic counter, so a block that drew cheap tiles (slots born
  // late in the window) takes more of them: the launch does not wait on the blocks that a fixed
  // assignment would have given the most expensive tiles.
  for (;;) {
    if (threadIdx.x == 0) {
      const int t = atomicAdd(sched, 1);
      s_tile = t;
      if (t < ntiles_all) s_rep = list_rep(list, find_rep_cached(s_tile0, list, reps, nlist, t));
    }
    __syncthreads();
    const int gt = s_tile;
    if (gt >= ntiles_all) break;   // block-uniform
    const WinRep R = reps[s_rep];
    __syncthreads();
    const int t = gt - R.tile0;
    const int q = t * kWinThreads + threadIdx.x;  // quad within the replicate
    const int s0 = 4 * q;
    const int cap = static_cast<int>(R.capacity);
    const int M0 = M_in[R.rep];
    // a tile past the replicate's end-of-window count has nothing to do (tile 0 keeps the bookkeeping)
    if (t > 0 && static_cast<long long>(t) * kWinTile >= M0 + R.births) continue;   // block-uniform
    float* const rowB = B + R.base;
    const float* const rowA = A + R.base;
    int* const gp = id_gp + R.base;
    int* const tid = id_tid + R.base;

    float x[4];
    if (s0 + 3 < M0) {
      const float4 v = __ldg(reinterpret_cast<const float4*>(rowA + s0));
      x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) x[j] = (s0 + j < M0) ? rowA[s0 + j] : 0.f;
    }

    int M = M0;
    int alive = 1;
#pragma unroll 1
    for (int k = 0; k < R.ngen; ++k) {
      const WinGen G = recs[R.rec + k];
      const int N = G.Nc;
      const int g = G.generation;
      alive = G.alive;
      if (N <= 0) {
        // extinction generation: the population's row is cleared
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (s0 + j < M) x[j] = 0.f;
      } else {
        // whole quad: Philox (q + 2, g, 0, 0), lanes x, y, z, w.  Every lane of the warp reaches the
        // draw (N and the loop are uniform over the block), as the warp-pooled strategy requires.
        const bool quad = q < (M >> 2);
        const bool neutral = (G.sel_a == 0.f && G.sel_b == 0.f);
        float xs[4] = {0.f, 0.f, 0.f, 0.f};
        int res[4] = {0, 0, 0, 0};
        unsigned need = 0;
        if (quad) {
#pragma unroll
          for (int j = 0; j < 4; ++j)
            xs[j] = neutral ? selected_freq<true>(x[j], 0.f, 0.f, 0.f, 0.f)
                            : selected_freq<false>(x[j], G.sel_a, G.sel_b, G.F, G.h);
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            res[j] = (xs[j] == 1.f && N > 6) ? N : 0;
            if (!(xs[j] == 0.f || (xs[j] == 1.f && N > 6))) need |= 1u << j;
          }
        }
        uint4 r = make_uint4(0u, 0u, 0u, 0u);
        if (need) {
          if (KEYS) r = philox4x32_10_keys(make_uint4(static_cast<uint32_t>(q + 2), static_cast<uint32_t>(g), 0u, 0u), keys);
          else r = philox(R.seed1, R.seed2, q + 2, g, 0, 0);
        }
        if (DRAW == kDrawWarp || DRAW == kDrawPooledSearch) {
          draw_quad<DRAW>(xs, r, need, N, lane, wd, res);   // every lane of the warp calls it
        } else if (need) {
          draw_quad<DRAW>(xs, r, need, N, lane, wd, res);
        }
        if (quad) {
          const float Nf = static_cast<float>(N);
#pragma unroll
          for (int j = 0; j < 4; ++j) x[j] = static_cast<float>(clampi(res[j], 0, N)) / Nf;
        } else if (s0 < M) {
          // scalar tail: Philox (slot + 2, g, 0, 0) lane x, variance in double
#pragma unroll 1
          for (int j = 0; j < 4; ++j) {
            const int e = s0 + j;
            if (e >= M) break;
            const float xs1 = neutral ? selected_freq<true>(x[j], 0.f, 0.f, 0.f, 0.f)
                                      : selected_freq<false>(x[j], G.sel_a, G.sel_b, G.F, G.h);
            x[j] = static_cast<float>(clampi(drift_tail(R.seed1, R.seed2, e, g, 0, xs1, N), 0, N)) /
                   static_cast<float>(N);
          }
        }
      }
      // births: slots [M, M + new_count) start at 1/Nc with ID (g, 0, slot - M + 1)
      const int Mn = M + G.new_count;
      if (s0 + 3 >= M && s0 < Mn) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int e = s0 + j;
          if (e >= M && e < Mn && e < cap) {
            x[j] = G.new_freq;
            gp[e] = g;
            tid[e] = e - M + 1;
          }
        }
      }
      M = Mn;
    }
    const int Mw = min(M, cap);
    if (s0 + 3 < Mw) {
      *reinterpret_cast<float4*>(rowB + s0) = make_float4(x[0], x[1], x[2], x[3]);
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (s0 + j < Mw) rowB[s0 + j] = x[j];
    }

    if (R.compact) {
      // flag_segregating_mutations for one population: keep unless lost or fixed (when alive), or
      // if preserved
      unsigned keep = 0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int e = s0 + j;
        if (e >= Mw) continue;
        // lost or fixed in the (only) population -- or the population is not alive -- removes it
        bool k = alive && !(x[j] <= 0.f || x[j] >= 1.f);
        if (R.check_preserved && e < M0 && tid[e] < 0) k = true;
        if (k) keep |= 1u << j;
      }
      unsigned word = keep << ((lane & 7) * 4);
      word |= __shfl_xor_sync(0xFFFFFFFFu, word, 1);
      word |= __shfl_xor_sync(0xFFFFFFFFu, word, 2);
      word |= __shfl_xor_sync(0xFFFFFFFFu, word, 4);
      if ((lane & 7) == 0) flags[(R.base + s0) >> 5] = word;
      unsigned c = __popc(keep);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
      if (lane == 0) s_warp[threadIdx.x >> 5] = c;
      __syncthreads();
      if (threadIdx.x == 0) {
        unsigned tot = 0;
#pragma unroll
        for (int w = 0; w < kWinThreads / 32; ++w) tot += s_warp[w];
        tile_count[R.base / kWinTile + t] = tot;
      }
      __syncthreads();
    }

    if (t == 0 && threadIdx.x == 0) {
      // window bookkeeping, once per replicate
      unsigned long long mg = 0;
      int m = M0;
      for (int k = 0; k < R.ngen; ++k) {
        mg += static_cast<unsigned long long>(m);
        m += recs[R.rec + k].new_count;
      }
      atomicAdd(stats, mg);
      atomicAdd(stats + 1, static_cast<unsigned long long>(R.ngen));
      if (M > cap) atomicExch(fault, kFaultCapacity);
      M_end[R.rep] = Mw;
      if (M_next && !R.compact) M_next[R.rep] = Mw;
    }
  }
  // every block has drawn past the last tile once it gets here; the last one resets the scheduler
  // for the next launch on this stream
  if (threadIdx.x == 0) {
    __threadfence();   // this block's last draw from sched[0] is ordered before its count in sched[1]
    const int finished = atomicAdd(sched + 1, 1);
    if (finished == static_cast<int>(gridDim.x) - 1) {
      sched[0] = 0;
      sched[1] = 0;
    }
  }
}

// One block per replicate: exclusive scan of its tile survivor counts, compacted count.  Each thread
// takes kSegScanItems consecutive tiles, so one pass covers 8,192 tiles (8.4 M slots).
constexpr int kSegScanThreads = 1024;
constexpr int kSegScanItems = 8;
__global__ void __launch_bounds__(kSegScanThreads)
    seg_scan_kernel(const unsigned* __restrict__ tile_count, unsigned* __restrict__ tile_offset,
                    const WinRep* __restrict__ reps, const int* __restrict__ M_end, int* __restrict__ M_out,
                    const RepList list) {
  if (list.count && static_cast<int>(blockIdx.x) >= *list.count) return;
  const WinRep R = reps[list_rep(list, blockIdx.x)];
  if (!R.compact) return;
  __shared__ unsigned s_warp[kSegScanThreads / 32];
  __shared__ unsigned s_carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int n = (M_end[R.rep] + kWinTile - 1) / kWinTile;
  const long long t0 = R.base / kWinTile;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += kSegScanThreads * kSegScanItems) {
    const int first = base + threadIdx.x * kSegScanItems;
    unsigned v[kSegScanItems];
    unsigned sum = 0;
#pragma unroll
    for (int k = 0; k < kSegScanItems; ++k) {
      v[k] = first + k < n ? tile_count[t0 + first + k] : 0u;
      sum += v[k];
    }
    unsigned incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const unsigned wv = s_warp[lane];
      unsigned wi = wv;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
        if (lane >= o) wi += y;
      }
      s_warp[lane] = wi - wv;
    }
    __syncthreads();
    unsigned run = s_carry + s_warp[warp] + incl - sum;
#pragma unroll
    for (int k = 0; k < kSegScanItems; ++k) {
      if (first + k < n) tile_offset[t0 + first + k] = run;
      run += v[k];
    }
    __syncthreads();
    if (threadIdx.x == kSegScanThreads - 1) s_carry = run;
    __syncthreads();
  }
  if (threadIdx.x == 0) M_out[R.rep] = static_cast<int>(s_carry);
}

// Stable scatter of every compacting replicate's survivors (scatter_arrays, go_fish_impl.cu:147-189),
// staged through shared memory into one contiguous run per tile.  FUSED stages the frequency and
// both ID words of a tile together (one barrier, the three loads in flight at once, 12 KB of staging)
// -- faster for one large replicate; otherwise the arrays go one after the other through one 4 KB
// buffer, which keeps more blocks resident for the many small tiles of a batch.
template <bool FUSED>
__global__ void __launch_bounds__(kWinThreads)
    seg_scatter_kernel(const float* __restrict__ src, float* __restrict__ dst, const int* __restrict__ gp_src,
                       const int* __restrict__ tid_src, int* __restrict__ gp_dst, int* __restrict__ tid_dst,
                       const unsigned* __restrict__ flags, const unsigned* __restrict__ tile_offset,
                       const WinRep* __restrict__ reps, int nreps, const int* __restrict__ M_end, int total_tiles,
                       const int* __restrict__ total_dev, const RepList list) {
  __shared__ int s_rep;
  __shared__ int s_tile0[kRepCache];
  const int ntiles_all = total_dev ? *total_dev : total_tiles;
  const int nlist = list_count(list, nreps);
  load_tile0(s_tile0, list, reps, nlist);
  __shared__ unsigned s_words[32];
  __shared__ unsigned s_prefix[32];
  __shared__ float s_stage[FUSED ? 3 * kWinTile : kWinTile];
  const int t = threadIdx.x;
  for (int gt = blockIdx.x; gt < ntiles_all; gt += gridDim.x) {
    if (t == 0) s_rep = list_rep(list, find_rep_cached(s_tile0, list, reps, nlist, gt));
    __syncthreads();
    const WinRep R = reps[s_rep];
    __syncthreads();
    const int tile = gt - R.tile0;
    const int ntiles = (M_end[R.rep] + kWinTile - 1) / kWinTile;
    if (!R.compact || tile >= ntiles) continue;  // block-uniform
    const long long atile = R.base / kWinTile + tile;
    if (t < 32) {
      const unsigned w = flags[atile * 32 + t];
      s_words[t] = w;
      const unsigned c = __popc(w);
      unsigned incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (t >= o) incl += y;
      }
      s_prefix[t] = incl - c;
    }
    __syncthreads();
    const int w = t >> 3, sh = (t & 7) * 4;
    const unsigned word = s_words[w];
    const unsigned nib = (word >> sh) & 0xFu;
    const int local = static_cast<int>(s_prefix[w] + __popc(word & ((1u << sh) - 1u)));
    const int count = static_cast<int>(s_prefix[31] + __popc(s_words[31]));
    const long long out0 = R.base + tile_offset[atile];
    const long long in0 = R.base + static_cast<long long>(tile) * kWinTile + 4 * t;
    if constexpr (FUSED) {
      int* s_gstage = reinterpret_cast<int*>(s_stage + kWinTile);
      int* s_tstage = s_gstage + kWinTile;
      if (nib) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(src + in0));
        const int4 g = __ldg(reinterpret_cast<const int4*>(gp_src + in0));
        const int4 d = __ldg(reinterpret_cast<const int4*>(tid_src + in0));
        const bool mark = R.preserve != 0;
        const float vv[4] = {v.x, v.y, v.z, v.w};
        const int gg[4] = {g.x, g.y, g.z, g.w};
        const int dd[4] = {d.x, d.y, d.z, d.w};
        int k = local;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (!((nib >> j) & 1u)) continue;
          s_stage[k] = vv[j];
          s_gstage[k] = gg[j];
          s_tstage[k++] = mark ? -abs(dd[j]) : dd[j];
        }
      }
      __syncthreads();
      for (int k = t; k < count; k += kWinThreads) {
        dst[out0 + k] = s_stage[k];
        gp_dst[out0 + k] = s_gstage[k];
        tid_dst[out0 + k] = s_tstage[k];
      }
      __syncthreads();
      continue;
    }
    if (nib) {
      const float4 v = __ldg(reinterpret_cast<const float4*>(src + in0));
      int k = local;
      if (nib & 1u) s_stage[k++] = v.x;
      if (nib & 2u) s_stage[k++] = v.y;
      if (nib & 4u) s_stage[k++] = v.z;
      if (nib & 8u) s_stage[k++] = v.w;
    }
    __syncthreads();
    for (int k = t; k < count; k += kWinThreads) dst[out0 + k] = s_stage[k];
    __syncthreads();
    int* s_istage = reinterpret_cast<int*>(s_stage);
    for (int arr = 0; arr < 2; ++arr) {
      const int* s = arr ? tid_src : gp_src;
      int* d = arr ? tid_dst : gp_dst;
      if (nib) {
        const int4 v = __ldg(reinterpret_cast<const int4*>(s + in0));
        int k = local;
        const bool mark = arr && R.preserve;
        if (nib & 1u) s_istage[k++] = mark ? -abs(v.x) : v.x;
        if (nib & 2u) s_istage[k++] = mark ? -abs(v.y) : v.y;
        if (nib & 4u) s_istage[k++] = mark ? -abs(v.z) : v.z;
        if (nib & 8u) s_istage[k++] = mark ? -abs(v.w) : v.w;
      }
      __syncthreads();
      for (int k = t; k < count; k += kWinThreads) d[out0 + k] = s_istage[k];
      __syncthreads();
    }
  }
}

// Tile assignment of a batched super-step (batch_tiles_kernel), on the engine stream.
void assign_batch_tiles(Engine* e, WinRep* d_reps, int nreps, const int* M_in, const WinGen* recs,
                        int* total_out) {
  batch_tiles_kernel<<<1, 1024, 0, e->stream>>>(d_reps, nreps, M_in, recs, total_out);
  e->kernel_launches += 1;
}

void batch_step_tiles(Engine* e, WinRep* d_table, int R, const int* M_in, const WinGen* recs, int* total_out,
                      int* d_step, const BatchStepPlan& plan, const int* region_off, const long long* region_base,
                      const StepRep* steprep, int* fault, int* list_rep, int* list_tile0, int* list_count) {
  batch_step_kernel<<<1, 1024, 0, e->stream>>>(d_table, R, M_in, recs, total_out, d_step, plan, region_off,
                                               region_base, steprep, fault, list_rep, list_tile0, list_count);
  e->kernel_launches += 1;
}

template <int DRAW, bool KEYS>
static void launch_window_kernel(Engine* e, const WindowLaunch& w) {
  // resident blocks per SM, queried once per instantiation (thread-safe initialisation; the same on
  // every B200)
  static const int occupancy = [] {
    int o = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, window_kernel<DRAW, KEYS>, kWinThreads, 0) !=
            cudaSuccess ||
        o < 1) {
      cudaGetLastError();
      o = 1;
    }
    return o;
  }();
  const int per_sm = e->blocks_per_sm > 0 ? std::min(e->blocks_per_sm, occupancy) : occupancy;
  const int blocks = std::max(1, std::min(w.total_tiles, e->num_sms * per_sm));
  const PhiloxKeys keys = philox_round_keys(w.seed1, w.seed2);
  window_kernel<DRAW, KEYS><<<blocks, kWinThreads, 0, e->stream>>>(
      w.A, w.B, w.id_gp_cur, w.id_tid_cur, w.flags, w.tile_count, w.M_in, w.M_end, w.M_next, w.reps, w.nreps,
      w.recs, w.total_tiles, w.total_tiles_dev, w.stats, w.fault, keys, w.sched, w.list);
}

// Launch a window over w.nreps replicates and, for the replicates that compact, the segmented scan
// and scatter into `compact_dst` (the other state buffer).
gf_status window_run(Engine* e, const WindowLaunch& w, float* compact_dst, cudaEvent_t after_window,
                     cudaEvent_t before_compaction) {
  const bool keys = GF_WINDOW_UNIFORM_KEYS && w.uniform_key && w.nreps == 1;
  switch (e->draw_strategy) {
    case kDrawWarp: launch_window_kernel<kDrawWarp, false>(e, w); break;
    case kDrawGrouped: launch_window_kernel<kDrawGrouped, false>(e, w); break;
    case kDrawNormalAll: launch_window_kernel<kDrawNormalAll, false>(e, w); break;
    case kDrawPooledSearch:
      if (keys) launch_window_kernel<kDrawPooledSearch, true>(e, w);
      else launch_window_kernel<kDrawPooledSearch, false>(e, w);
      break;
    default:
      if (keys) launch_window_kernel<kDrawLanes, true>(e, w);
      else launch_window_kernel<kDrawLanes, false>(e, w);
      break;
  }
  GF_CUDA(e, cudaGetLastError());
  e->kernel_launches += 1;
  if (after_window) GF_CUDA(e, cudaEventRecord(after_window, e->stream));
  if (before_compaction) GF_CUDA(e, cudaEventRecord(before_compaction, e->stream));
  if (w.any_compact) {
    seg_scan_kernel<<<w.nreps, kSegScanThreads, 0, e->stream>>>(w.tile_count, w.tile_offset, w.reps, w.M_end,
                                                                w.M_out, w.list);
    GF_CUDA(e, cudaGetLastError());
    const int sblocks = std::max(1, std::min(w.total_tiles, e->num_sms * 8));
    auto scatter = w.nreps == 1 ? seg_scatter_kernel<true> : seg_scatter_kernel<false>;
    scatter<<<sblocks, kWinThreads, 0, e->stream>>>(w.B, compact_dst, w.id_gp_cur, w.id_tid_cur, w.id_gp_next,
                                                    w.id_tid_next, w.flags, w.tile_offset, w.reps, w.nreps,
                                                    w.M_end, w.total_tiles, w.total_tiles_dev, w.list);
    GF_CUDA(e, cudaGetLastError());
    e->kernel_launches += 2;
  }
  return GF_OK;
}

}  // namespace gf
