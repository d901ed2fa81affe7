// GO_Fish plain engine for one B200: device state, the per-generation kernels and the host loop.
//
// Device state (all rows have the same stride `capacity`, a multiple of 1024 slots):
//   freq[2]      [P][capacity] fp32, ping-pong between generations (d_prev_freq / d_mutations_freq,
//                go_fish_impl.cuh:183-199)
//   id_gp[2]     origin generation | origin population << 24       (mutID.x, mutID.y)
//   id_tid[2]    origin threadID, negative = preserved              (mutID.z)
//   flags        1 bit per slot: survives the next compaction
//   tile_count / tile_offset   survivors per 1024-slot tile and their exclusive prefix
//   d_count      [0], [1] mutation count ping-pong (written by the device, never synchronized on
//                except for state reads), [2] device status word
//
// One generation = one fused kernel (migration -> selection -> drift for every population of a
// mutation quad, the new-mutation fill of the appended slots, and -- on compaction generations --
// the survival bitmask and per-tile survivor counts).  A compaction adds a one-block scan of the
// tile counts and a stable scatter.  There is no cudaMalloc and no host synchronization inside the
// generation loop: the host tracks an upper bound on the mutation count and tightens it from
// asynchronous read-backs of each compaction's survivor count.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstring>

#include "gf_internal.h"
#include "gf_rng.cuh"
#include "gf_drift.cuh"
#include "gf_mse.cuh"

namespace gf {

// ------------------------------------------------------------------------------------------------
// error helpers
// ------------------------------------------------------------------------------------------------
gf_status fail(Engine* e, gf_status st, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (e) e->last_error = buf;
  return st;
}

gf_status cuda_fail(Engine* e, cudaError_t err, const char* what) {
  const gf_status st = (err == cudaErrorMemoryAllocation) ? GF_ERR_OUT_OF_MEMORY : GF_ERR_CUDA;
  return fail(e, st, "CUDA error %d (%s) in %s", static_cast<int>(err), cudaGetErrorString(err), what);
}

gf_status pool_alloc(Engine* e, void** ptr, size_t bytes) {
  const cudaError_t err = e->pool ? cudaMallocFromPoolAsync(ptr, bytes, e->pool, e->stream)
                                  : cudaMallocAsync(ptr, bytes, e->stream);
  if (err != cudaSuccess) {
    cudaGetLastError();
    *ptr = nullptr;
    return cuda_fail(e, err, "stream-ordered allocation");
  }
  return GF_OK;
}

gf_status ensure_scratch(Engine* e, void** ptr, size_t* have, size_t need) {
  if (*have >= need && *ptr) return GF_OK;
  if (*ptr) {
    GF_CUDA(e, cudaStreamSynchronize(e->stream));
    GF_CUDA(e, cudaFree(*ptr));
    *ptr = nullptr;
    *have = 0;
  }
  const size_t bytes = std::max<size_t>(need, 256);
  GF_CUDA(e, cudaMalloc(ptr, bytes));
  *have = bytes;
  return GF_OK;
}

// ------------------------------------------------------------------------------------------------
// the fused generation kernel
// ------------------------------------------------------------------------------------------------
constexpr int kDriftMinBlocks = GF_DRIFT_MIN_BLOCKS;

// PT: 1 = single-population specialization, 0 = any P <= kMaxPops.
// NEUTRAL: every drifted population has s(x) == 0.
// FLAG: compaction generation -- also write the survival bitmask and tile counts.
// DRAW: how a warp schedules its sampler draws (DrawStrategy, see draw_quad).
// The grid is sized by occupancy and strides over the 1024-slot tiles of the current generation,
// whose number the kernel derives from the device-side mutation count.
template <int PT, bool NEUTRAL, bool FLAG, int DRAW>
__global__ void __launch_bounds__(kDriftThreads, kDriftMinBlocks)
    drift_kernel(const float* __restrict__ prev, float* __restrict__ next, int* __restrict__ id_gp,
                 int* __restrict__ id_tid, unsigned* __restrict__ flags, unsigned* __restrict__ tile_count,
                 int* __restrict__ d_count, unsigned long long* __restrict__ stats, long long stride, int slot_in,
                 int slot_out, long long capacity, const GenArgs* __restrict__ table) {
  __shared__ GenArgs a;
  __shared__ WarpDraws s_draws[(DRAW == kDrawWarp || DRAW == kDrawPooledSearch) ? kDriftThreads / 32 : 1];
  __shared__ unsigned s_warp[kDriftThreads / 32];
  {
    const int* src = reinterpret_cast<const int*>(table);
    int* dst = reinterpret_cast<int*>(&a);
    for (int i = threadIdx.x; i < static_cast<int>(sizeof(GenArgs) / 4); i += kDriftThreads) dst[i] = src[i];
  }
  __syncthreads();
  const int M_in = d_count[slot_in];
  int total = M_in + a.new_total;
  if (total > capacity) total = static_cast<int>(capacity);  // reported below; never written past the rows
  const int ntiles = (total + kTileSlots - 1) / kTileSlots;
  const int nquads = M_in >> 2;
  const int P = (PT > 0) ? PT : a.num_pops;
  const int g = a.generation;
  const int lane = threadIdx.x & 31;
  WarpDraws* w = &s_draws[(DRAW == kDrawWarp || DRAW == kDrawPooledSearch) ? (threadIdx.x >> 5) : 0];

  if (blockIdx.x == 0 && threadIdx.x == 0) {
    d_count[slot_out] = total;
    d_count[3] = total;
    if (M_in + a.new_total > capacity) atomicExch(d_count + 2, kFaultCapacity);
    stats[0] += static_cast<unsigned long long>(M_in);
    stats[1] += 1ull;
  }

  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int q = tile * kDriftThreads + threadIdx.x;  // quad index
    const int base = q * 4;
    const bool quad = q < nquads;
    unsigned keep = 0;  // bit j: slot base + j survives the compaction

    // ---- whole quads: one Philox block per population, lanes x,y,z,w = slots base .. base+3 ----
    unsigned zero = 0xFu, one = 0xFu;
#pragma unroll 1
    for (int p = 0; p < P; ++p) {
      if (!((a.drift_mask >> p) & 1)) continue;
      const int N = a.Nc[p];
      float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
      if (N > 0) {  // N == 0: extinction generation, the population's row is cleared
        float xs[4] = {0.f, 0.f, 0.f, 0.f};
        if (quad) {
          float4 xm = make_float4(0.f, 0.f, 0.f, 0.f);
          for (int k = 0; k < P; ++k) {
            const float m = a.mig[k * P + p];
            const float4 v = __ldg(reinterpret_cast<const float4*>(prev + k * stride + base));
            xm.x += m * v.x;
            xm.y += m * v.y;
            xm.z += m * v.z;
            xm.w += m * v.w;
          }
          const float F = a.F[p], h = a.h[p], sa = a.sel_a[p], sb = a.sel_b[p];
          if (!NEUTRAL && a.sel_table) {  // s(x_mig) evaluated per slot by the caller's model
            const float4 st = __ldg(reinterpret_cast<const float4*>(a.sel_table + p * a.sel_stride + base));
            xs[0] = selection_step(xm.x, fmaxf(st.x, -1.f), F, h);
            xs[1] = selection_step(xm.y, fmaxf(st.y, -1.f), F, h);
            xs[2] = selection_step(xm.z, fmaxf(st.z, -1.f), F, h);
            xs[3] = selection_step(xm.w, fmaxf(st.w, -1.f), F, h);
          } else {
            xs[0] = selected_freq<NEUTRAL>(xm.x, sa, sb, F, h);
            xs[1] = selected_freq<NEUTRAL>(xm.y, sa, sb, F, h);
            xs[2] = selected_freq<NEUTRAL>(xm.z, sa, sb, F, h);
            xs[3] = selected_freq<NEUTRAL>(xm.w, sa, sb, F, h);
          }
        }
        // lost (x == 0) and, for N > 6, fixed (x == 1) slots have a certain outcome
        int res[4];
        unsigned need = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          res[j] = (xs[j] == 1.f && N > 6) ? N : 0;
          if (quad && !(xs[j] == 0.f || (xs[j] == 1.f && N > 6))) need |= 1u << j;
        }
        uint4 r = make_uint4(0u, 0u, 0u, 0u);
        if (need) r = philox(a.seed1, a.seed2, q + 2, g, p, 0);
        draw_quad<DRAW>(xs, r, need, N, lane, w, res);
        const float Nf = static_cast<float>(N);
        o.x = static_cast<float>(clampi(res[0], 0, N)) / Nf;
        o.y = static_cast<float>(clampi(res[1], 0, N)) / Nf;
        o.z = static_cast<float>(clampi(res[2], 0, N)) / Nf;
        o.w = static_cast<float>(clampi(res[3], 0, N)) / Nf;
      }
      if (quad) {
        *reinterpret_cast<float4*>(next + p * stride + base) = o;
        if (FLAG && ((a.alive_mask >> p) & 1)) {
          zero &= (o.x <= 0.f ? 1u : 0u) | (o.y <= 0.f ? 2u : 0u) | (o.z <= 0.f ? 4u : 0u) | (o.w <= 0.f ? 8u : 0u);
          one &= (o.x >= 1.f ? 1u : 0u) | (o.y >= 1.f ? 2u : 0u) | (o.z >= 1.f ? 4u : 0u) | (o.w >= 1.f ? 8u : 0u);
        }
      }
    }
    if (FLAG && quad) {
      keep = ~(zero | one) & 0xFu;
      if (a.check_preserved) {
        const int4 t = *reinterpret_cast<const int4*>(id_tid + base);
        keep |= (t.x < 0 ? 1u : 0u) | (t.y < 0 ? 2u : 0u) | (t.z < 0 ? 4u : 0u) | (t.w < 0 ? 8u : 0u);
      }
    }

    if (!quad && base < total) {
      // ---- scalar tail (slots past the last whole quad) and the new-mutation fill ----
#pragma unroll 1
      for (int j = 0; j < 4; ++j) {
        const int e = base + j;
        if (e >= total) break;
        unsigned z1 = 1u, o1 = 1u;
        if (e < M_in) {
          for (int p = 0; p < P; ++p) {
            if (!((a.drift_mask >> p) & 1)) continue;
            float xm = 0.f;
            for (int k = 0; k < P; ++k) xm += a.mig[k * P + p] * prev[k * stride + e];
            const int N = a.Nc[p];
            float o = 0.f;
            if (N > 0) {
              const float xs =
                  (!NEUTRAL && a.sel_table)
                      ? selection_step(xm, fmaxf(a.sel_table[p * a.sel_stride + e], -1.f), a.F[p], a.h[p])
                      : selected_freq<NEUTRAL>(xm, a.sel_a[p], a.sel_b[p], a.F[p], a.h[p]);
              o = static_cast<float>(clampi(drift_tail(a.seed1, a.seed2, e, g, p, xs, N), 0, N)) /
                  static_cast<float>(N);
            }
            next[p * stride + e] = o;
            if (FLAG && ((a.alive_mask >> p) & 1)) {
              z1 &= (o <= 0.f);
              o1 &= (o >= 1.f);
            }
          }
          if (FLAG) keep |= ((!(z1 | o1)) || (a.check_preserved && id_tid[e] < 0)) ? (1u << j) : 0u;
        } else {
          // new mutation (add_new_mutations, go_fish_impl.cu:138-145): row p = 1/Nc, others 0
          const int r = e - M_in;
          int p = 0;
          while (p + 1 < P && r >= a.new_offset[p + 1]) ++p;
          const int tid = r - a.new_offset[p] + 1;
          for (int k = 0; k < P; ++k) {
            const float v = (k == p) ? a.new_freq[p] : 0.f;
            next[k * stride + e] = v;
            if (FLAG && ((a.alive_mask >> k) & 1)) {
              z1 &= (v <= 0.f);
              o1 &= (v >= 1.f);
            }
          }
          id_gp[e] = g | (p << 24);
          id_tid[e] = tid;
          if (FLAG) keep |= (!(z1 | o1)) ? (1u << j) : 0u;
        }
      }
    }

    if (FLAG) {
      // 8 consecutive threads own the 32 slots of one flag word.
      unsigned word = (keep & 0xFu) << ((lane & 7) * 4);
      word |= __shfl_xor_sync(0xFFFFFFFFu, word, 1);
      word |= __shfl_xor_sync(0xFFFFFFFFu, word, 2);
      word |= __shfl_xor_sync(0xFFFFFFFFu, word, 4);
      if ((lane & 7) == 0) flags[base >> 5] = word;
      // survivors of the tile
      unsigned c = __popc(keep & 0xFu);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
      if (lane == 0) s_warp[threadIdx.x >> 5] = c;
      __syncthreads();
      if (threadIdx.x == 0) {
        unsigned t = 0;
#pragma unroll
        for (int wi = 0; wi < kDriftThreads / 32; ++wi) t += s_warp[wi];
        tile_count[tile] = t;
      }
      __syncthreads();
    }
  }
}

// ------------------------------------------------------------------------------------------------
// single-block exclusive scan of uint32 counts (replaces cub::DeviceScan, go_fish_impl.cuh:389-391)
// ------------------------------------------------------------------------------------------------
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;

// n_from_slots: if not null, n = ceil(*n_from_slots / 1024) -- the tile count of a generation whose
// slot count only the device knows.
__global__ void __launch_bounds__(kScanThreads)
    scan_exclusive_kernel(const unsigned* __restrict__ in, unsigned* __restrict__ out, int n, int* total_out,
                          const int* __restrict__ n_from_slots) {
  __shared__ unsigned s_warp[kScanThreads / 32];
  __shared__ unsigned s_carry;
  if (n_from_slots) n = (*n_from_slots + kTileSlots - 1) / kTileSlots;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += kScanThreads * kScanItems) {
    unsigned v[kScanItems];
    unsigned tsum = 0;
    const int first = base + threadIdx.x * kScanItems;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      const int idx = first + k;
      v[k] = (idx < n) ? in[idx] : 0u;
      tsum += v[k];
    }
    unsigned incl = tsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      unsigned w = s_warp[lane];
      unsigned wi = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
        if (lane >= o) wi += y;
      }
      s_warp[lane] = wi - w;  // exclusive prefix of warp sums
    }
    __syncthreads();
    unsigned run = s_carry + s_warp[warp] + incl - tsum;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      const int idx = first + k;
      if (idx < n) out[idx] = run;
      run += v[k];
    }
    __syncthreads();
    if (threadIdx.x == kScanThreads - 1) s_carry = run;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total_out) *total_out = static_cast<int>(s_carry);
}

// ------------------------------------------------------------------------------------------------
// stable scatter of surviving slots (scatter_arrays, go_fish_impl.cu:147-189), staged through
// shared memory so that every tile writes its survivors as one contiguous, coalesced run
// ------------------------------------------------------------------------------------------------
template <bool PRESERVE>
__global__ void __launch_bounds__(kDriftThreads)
    scatter_kernel(const float* __restrict__ src, float* __restrict__ dst, const int* __restrict__ gp_src,
                   const int* __restrict__ tid_src, int* __restrict__ gp_dst, int* __restrict__ tid_dst,
                   const unsigned* __restrict__ flags, const unsigned* __restrict__ tile_offset, long long stride,
                   int P, const int* __restrict__ d_slots) {
  __shared__ unsigned s_words[32];
  __shared__ unsigned s_prefix[32];
  __shared__ float s_stage[kTileSlots];
  const int t = threadIdx.x;
  const long long ntiles = (*d_slots + kTileSlots - 1) / kTileSlots;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
  if (t < 32) {
    const unsigned w = flags[tile * 32 + t];
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
  const long long out_base = tile_offset[tile];
  const long long in_base = tile * kTileSlots + 4 * t;

  for (int r = 0; r < P; ++r) {
    if (nib) {
      const float4 v = __ldg(reinterpret_cast<const float4*>(src + r * stride + in_base));
      int k = local;
      if (nib & 1u) s_stage[k++] = v.x;
      if (nib & 2u) s_stage[k++] = v.y;
      if (nib & 4u) s_stage[k++] = v.z;
      if (nib & 8u) s_stage[k++] = v.w;
    }
    __syncthreads();
    for (int k = t; k < count; k += kDriftThreads) dst[r * stride + out_base + k] = s_stage[k];
    __syncthreads();
  }
  int* s_istage = reinterpret_cast<int*>(s_stage);
  for (int arr = 0; arr < 2; ++arr) {
    const int* s = arr ? tid_src : gp_src;
    int* d = arr ? tid_dst : gp_dst;
    if (nib) {
      const int4 v = __ldg(reinterpret_cast<const int4*>(s + in_base));
      int k = local;
      auto mark = [&](int x) { return (arr && PRESERVE) ? -abs(x) : x; };
      if (nib & 1u) s_istage[k++] = mark(v.x);
      if (nib & 2u) s_istage[k++] = mark(v.y);
      if (nib & 4u) s_istage[k++] = mark(v.z);
      if (nib & 8u) s_istage[k++] = mark(v.w);
    }
    __syncthreads();
    for (int k = t; k < count; k += kDriftThreads) d[out_base + k] = s_istage[k];
    __syncthreads();
  }
  }
}

// ------------------------------------------------------------------------------------------------
// state load / read helpers
// ------------------------------------------------------------------------------------------------
__global__ void mark_preserved_kernel(int* __restrict__ tid, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += blockDim.x * gridDim.x) tid[i] = -abs(tid[i]);
}

// ------------------------------------------------------------------------------------------------
// mutation-selection-equilibrium start (initialize_mse and friends, go_fish_impl.cuh:20-71, 201-332)
// ------------------------------------------------------------------------------------------------
__global__ void mse_area_kernel(float* __restrict__ area, int num_freq, float step, int N_ind, float F, float h,
                                float sa, float sb) {
  for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < num_freq; id += blockDim.x * gridDim.x)
    area[id] = mse_area(id, step, N_ind, F, h, sa, sb);
}

__global__ void __launch_bounds__(1024) mse_integral_kernel(const float* __restrict__ area, float* __restrict__ integral,
                                                            int num_freq) {
  mse_integral_block(area, integral, num_freq);
}

__global__ void mse_count_kernel(unsigned* __restrict__ counts, const float* __restrict__ integral, int offset,
                                 float mu, int N_ind, int Nchrom, float L, float sa, float sb, float F, float h,
                                 int seed1, int seed2, int pop, int use_integral) {
  const float mse_total = use_integral ? integral[0] : 0.f;
  for (int id = blockIdx.x * blockDim.x + threadIdx.x; id < Nchrom - 1; id += blockDim.x * gridDim.x)
    counts[offset + id] = mse_class_count(id, integral, mse_total, mu, N_ind, Nchrom, L, sa, sb, F, h, seed1, seed2, pop);
}

struct MseClassRange {
  int first_class[kMaxPops + 1];  // global class index where each population's classes start
  int Nc[kMaxPops];
};

// Expand class counts into mutation slots (initialize_mse_mutation_array + mse_set_mutID,
// go_fish_impl.cu:45-70): slot k of class (pop, id) gets frequency (id + 1) / Nc in row pop,
// 0 in the other rows, and ID (0, pop, +-(k + 1), 0).
__global__ void mse_fill_kernel(float* __restrict__ freq, int* __restrict__ id_gp, int* __restrict__ id_tid,
                                const unsigned* __restrict__ starts, int num_classes, int M0, long long stride,
                                int P, int preserve, const MseClassRange cr) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < M0; k += blockDim.x * gridDim.x) {
    // last class whose start <= k
    int lo = 0, hi = num_classes - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (static_cast<int>(starts[mid]) <= k) lo = mid; else hi = mid - 1;
    }
    int pop = 0;
    while (pop + 1 < P && lo >= cr.first_class[pop + 1]) ++pop;
    const int idy = lo - cr.first_class[pop];
    const float f = (idy + 1.f) / cr.Nc[pop];
    for (int r = 0; r < P; ++r) freq[r * stride + k] = (r == pop) ? f : 0.f;
    id_gp[k] = 0 | (pop << 24);
    id_tid[k] = preserve ? -(k + 1) : (k + 1);
  }
}

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
static long long align_up(long long v, long long a) { return (v + a - 1) / a * a; }

// Packed IDs (generation | population << 24, threadID) -> the reference's int4 layout.
__global__ void expand_ids_kernel(const int* __restrict__ gp, const int* __restrict__ tid, int M,
                                  int4* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
    const int w = gp[i];
    out[i] = make_int4(w & 0xFFFFFF, w >> 24, tid[i], 0);
  }
}

// A time sample packed at this point of the stream: the count M (from the device) and the rows
// [P][M] and int4 IDs of the first M slots, into scratch of `bound` slots (M > bound reports -1).
__global__ void pack_sample_kernel(const float* __restrict__ freq, long long capacity, int P,
                                   const int* __restrict__ gp, const int* __restrict__ tid,
                                   const int* __restrict__ count, int bound, float* __restrict__ out_freq,
                                   int4* __restrict__ out_ids, int* __restrict__ out_count) {
  const int M = *count;
  if (M > bound) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *out_count = -1;
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *out_count = M;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
    for (int p = 0; p < P; ++p) out_freq[static_cast<long long>(p) * M + i] = freq[p * capacity + i];
    const int w = gp[i];
    out_ids[i] = make_int4(w & 0xFFFFFF, w >> 24, tid[i], 0);
  }
}

static void release_sim(Engine* e) {
  // stream-ordered frees: the memory returns to the engine's pool for the next simulation
  for (int b = 0; b < 2; ++b) {
    if (e->freq[b]) cudaFreeAsync(e->freq[b], e->stream);
    if (e->id_gp[b]) cudaFreeAsync(e->id_gp[b], e->stream);
    if (e->id_tid[b]) cudaFreeAsync(e->id_tid[b], e->stream);
    e->freq[b] = nullptr;
    e->id_gp[b] = nullptr;
    e->id_tid[b] = nullptr;
  }
  if (e->sel_table) cudaFreeAsync(e->sel_table, e->stream);
  e->sel_table = nullptr;
  e->sel_table_stride = 0;
  if (e->flags) cudaFreeAsync(e->flags, e->stream);
  if (e->tile_count) cudaFreeAsync(e->tile_count, e->stream);
  if (e->tile_offset) cudaFreeAsync(e->tile_offset, e->stream);
  e->flags = nullptr;
  e->tile_count = nullptr;
  e->tile_offset = nullptr;
  for (auto& pc : e->pending) e->free_events.push_back(pc.event);
  e->pending.clear();
  e->capacity = 0;
  e->active = false;
}

// Allocate (zeroed) arrays of `cap` slots.  When `keep` > 0, the first `keep` slots of the current
// buffers are carried over.
static gf_status set_capacity(Engine* e, long long cap, long long keep) {
  cap = align_up(std::max<long long>(cap, kSlotAlign), kSlotAlign);
  if (cap > (1LL << 31) - kSlotAlign) return fail(e, GF_ERR_CAPACITY, "mutation capacity %lld exceeds 2^31 slots", cap);
  const int P = e->P;
  float* nf[2] = {nullptr, nullptr};
  int* ngp[2] = {nullptr, nullptr};
  int* ntid[2] = {nullptr, nullptr};
  unsigned *nflags = nullptr, *ncount = nullptr, *noffset = nullptr;
  const long long ntiles = cap / kTileSlots;
  cudaError_t err = cudaSuccess;
  auto palloc = [e](void** p, size_t bytes) {
    return e->pool ? cudaMallocFromPoolAsync(p, bytes, e->pool, e->stream) : cudaMallocAsync(p, bytes, e->stream);
  };
  for (int b = 0; b < 2 && err == cudaSuccess; ++b) {
    err = palloc(reinterpret_cast<void**>(&nf[b]), sizeof(float) * P * cap);
    if (err == cudaSuccess) err = palloc(reinterpret_cast<void**>(&ngp[b]), sizeof(int) * cap);
    if (err == cudaSuccess) err = palloc(reinterpret_cast<void**>(&ntid[b]), sizeof(int) * cap);
  }
  if (err == cudaSuccess) err = palloc(reinterpret_cast<void**>(&nflags), sizeof(unsigned) * (cap / 32));
  if (err == cudaSuccess) err = palloc(reinterpret_cast<void**>(&ncount), sizeof(unsigned) * ntiles);
  if (err == cudaSuccess) err = palloc(reinterpret_cast<void**>(&noffset), sizeof(unsigned) * ntiles);
  if (err != cudaSuccess) {
    for (int b = 0; b < 2; ++b) {
      if (nf[b]) cudaFreeAsync(nf[b], e->stream);
      if (ngp[b]) cudaFreeAsync(ngp[b], e->stream);
      if (ntid[b]) cudaFreeAsync(ntid[b], e->stream);
    }
    if (nflags) cudaFreeAsync(nflags, e->stream);
    if (ncount) cudaFreeAsync(ncount, e->stream);
    cudaGetLastError();
    return cuda_fail(e, err, "allocating the mutation arrays");
  }
  for (int b = 0; b < 2; ++b) {
    GF_CUDA(e, cudaMemsetAsync(nf[b], 0, sizeof(float) * P * cap, e->stream));
    GF_CUDA(e, cudaMemsetAsync(ngp[b], 0, sizeof(int) * cap, e->stream));
    GF_CUDA(e, cudaMemsetAsync(ntid[b], 0, sizeof(int) * cap, e->stream));
  }
  if (keep > 0 && e->capacity > 0) {
    GF_CUDA(e, cudaMemcpy2DAsync(nf[e->cur], sizeof(float) * cap, e->freq[e->cur], sizeof(float) * e->capacity,
                                 sizeof(float) * keep, P, cudaMemcpyDeviceToDevice, e->stream));
    GF_CUDA(e, cudaMemcpyAsync(ngp[e->id_cur], e->id_gp[e->id_cur], sizeof(int) * keep, cudaMemcpyDeviceToDevice,
                               e->stream));
    GF_CUDA(e, cudaMemcpyAsync(ntid[e->id_cur], e->id_tid[e->id_cur], sizeof(int) * keep, cudaMemcpyDeviceToDevice,
                               e->stream));
  }
  for (int b = 0; b < 2; ++b) {
    if (e->freq[b]) cudaFreeAsync(e->freq[b], e->stream);
    if (e->id_gp[b]) cudaFreeAsync(e->id_gp[b], e->stream);
    if (e->id_tid[b]) cudaFreeAsync(e->id_tid[b], e->stream);
    e->freq[b] = nf[b];
    e->id_gp[b] = ngp[b];
    e->id_tid[b] = ntid[b];
  }
  if (e->flags) cudaFreeAsync(e->flags, e->stream);
  if (e->tile_count) cudaFreeAsync(e->tile_count, e->stream);
  if (e->tile_offset) cudaFreeAsync(e->tile_offset, e->stream);
  e->flags = nflags;
  e->tile_count = ncount;
  e->tile_offset = noffset;
  e->capacity = cap;
  return GF_OK;
}

static gf_status check_device_fault(Engine* e) {
  int fault = 0;
  GF_CUDA(e, cudaMemcpyAsync(&fault, e->d_count + 2, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  GF_CUDA(e, cudaStreamSynchronize(e->stream));
  if (fault != kFaultNone) {
    return fail(e, GF_ERR_DEVICE, "device status word reports fault %d (%s)", fault,
                fault == kFaultCapacity ? "mutation array capacity exceeded" : "bounded wait expired");
  }
  return GF_OK;
}

static gf_status begin_common(Engine* e, const gf_sim_config* c, long long initial_mutations) {
  if (!c) return fail(e, GF_ERR_INVALID_ARGUMENT, "config is NULL");
  if (c->num_populations < 1 || c->num_populations > kMaxPops)
    return fail(e, GF_ERR_INVALID_ARGUMENT, "num_populations %d outside [1, %d]", c->num_populations, kMaxPops);
  if (!(c->num_sites > 0.f)) return fail(e, GF_ERR_INVALID_ARGUMENT, "num_sites must be > 0");
  if (c->compact_interval < 0) return fail(e, GF_ERR_INVALID_ARGUMENT, "compact_interval must be >= 0");
  GF_CUDA(e, cudaSetDevice(e->device));
  GF_CUDA(e, cudaStreamSynchronize(e->stream));
  release_sim(e);
  e->P = c->num_populations;
  e->seed1 = c->seed1;
  e->seed2 = c->seed2;
  e->num_sites = c->num_sites;
  e->compact_interval = c->compact_interval;
  e->any_preserved = false;
  e->live_rows = 0;
  e->step_index = 0;
  e->count_slot = 0;
  e->cur = 0;
  e->id_cur = 0;
  const long long want = std::max<long long>({static_cast<long long>(c->reserve_mutations),
                                               2 * initial_mutations + 65536, 65536});
  gf_status st = set_capacity(e, want, 0);
  if (st != GF_OK) return st;
  GF_CUDA(e, cudaMemsetAsync(e->d_count, 0, sizeof(int) * kCountWords, e->stream));
  GF_CUDA(e, cudaMemsetAsync(e->d_stats, 0, sizeof(unsigned long long) * 2, e->stream));
  e->compactions = 0;
  e->M_upper = initial_mutations;
  e->M_exact = true;
  e->active = true;
  return GF_OK;
}

// Retire completed survivor-count read-backs, tightening the host's upper bound.
static void poll_pending(Engine* e, bool wait_all) {
  while (!e->pending.empty()) {
    PendingCount& pc = e->pending.front();
    if (wait_all) {
      cudaEventSynchronize(pc.event);
    } else if (cudaEventQuery(pc.event) != cudaSuccess) {
      cudaGetLastError();
      break;
    }
    const long long exact = e->h_pinned[pc.slot] + pc.added;
    if (e->pending.size() == 1 && exact <= e->M_upper) {
      e->M_upper = exact;
      e->M_exact = true;
    }
    e->free_events.push_back(pc.event);
    e->pending.pop_front();
  }
}

static gf_status get_event(Engine* e, cudaEvent_t* ev) {
  if (!e->free_events.empty()) {
    *ev = e->free_events.back();
    e->free_events.pop_back();
    return GF_OK;
  }
  GF_CUDA(e, cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
  return GF_OK;
}

int host_new_mutation_count(int seed1, int seed2, float mu, int Nchrom_e, float num_sites, int generation, int pop) {
  // calc_new_mutations_Index (go_fish_impl.cuh:454-467), evaluated on the host like the reference.
  const float lambda = mu * Nchrom_e * num_sites;
  if (Nchrom_e == 0 || lambda == 0) return 0;
  return std::max(pois_draw(lambda, lambda, Nchrom_e * num_sites, seed1, seed2, 1, generation, pop), 0);
}

template <int PT, bool NEUTRAL, bool FLAG, int DRAW>
static void launch_drift_t(Engine* e, int tiles_bound, int slot_in, int slot_out, const GenArgs* a) {
  auto kernel = drift_kernel<PT, NEUTRAL, FLAG, DRAW>;
  // resident blocks per SM, queried once (thread-safe initialisation; the same on every B200)
  static const int occupancy = [kernel] {
    int o = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kernel, kDriftThreads, 0) != cudaSuccess || o < 1) {
      cudaGetLastError();
      o = 1;
    }
    return o;
  }();
  const int per_sm = e->blocks_per_sm > 0 ? std::min(e->blocks_per_sm, occupancy) : occupancy;
  const int blocks = std::max(1, std::min(tiles_bound, e->num_sms * per_sm));
  kernel<<<blocks, kDriftThreads, 0, e->stream>>>(e->freq[e->cur], e->freq[e->cur ^ 1], e->id_gp[e->id_cur],
                                                  e->id_tid[e->id_cur], e->flags, e->tile_count, e->d_count,
                                                  e->d_stats, e->capacity, slot_in, slot_out, e->capacity, a);
}

template <int PT, bool NEUTRAL, bool FLAG>
static void launch_drift_c(Engine* e, int tiles_bound, int slot_in, int slot_out, const GenArgs* a) {
  switch (e->draw_strategy) {
    case kDrawWarp: launch_drift_t<PT, NEUTRAL, FLAG, kDrawWarp>(e, tiles_bound, slot_in, slot_out, a); break;
    case kDrawGrouped: launch_drift_t<PT, NEUTRAL, FLAG, kDrawGrouped>(e, tiles_bound, slot_in, slot_out, a); break;
    case kDrawNormalAll:
      launch_drift_t<PT, NEUTRAL, FLAG, kDrawNormalAll>(e, tiles_bound, slot_in, slot_out, a);
      break;
    case kDrawPooledSearch:
      launch_drift_t<PT, NEUTRAL, FLAG, kDrawPooledSearch>(e, tiles_bound, slot_in, slot_out, a);
      break;
    default: launch_drift_t<PT, NEUTRAL, FLAG, kDrawLanes>(e, tiles_bound, slot_in, slot_out, a); break;
  }
}

static void launch_drift(Engine* e, int tiles_bound, int slot_in, int slot_out, const GenArgs* a, bool single,
                         bool neutral, bool flag) {
  if (single) {
    if (neutral) {
      flag ? launch_drift_c<1, true, true>(e, tiles_bound, slot_in, slot_out, a)
           : launch_drift_c<1, true, false>(e, tiles_bound, slot_in, slot_out, a);
    } else {
      flag ? launch_drift_c<1, false, true>(e, tiles_bound, slot_in, slot_out, a)
           : launch_drift_c<1, false, false>(e, tiles_bound, slot_in, slot_out, a);
    }
  } else {
    if (neutral) {
      flag ? launch_drift_c<0, true, true>(e, tiles_bound, slot_in, slot_out, a)
           : launch_drift_c<0, true, false>(e, tiles_bound, slot_in, slot_out, a);
    } else {
      flag ? launch_drift_c<0, false, true>(e, tiles_bound, slot_in, slot_out, a)
           : launch_drift_c<0, false, false>(e, tiles_bound, slot_in, slot_out, a);
    }
  }
}

static cudaEvent_t prof_event(Engine* e) {
  if (!e->prof_pool.empty()) {
    cudaEvent_t ev = e->prof_pool.back();
    e->prof_pool.pop_back();
    return ev;
  }
  cudaEvent_t ev = nullptr;
  cudaEventCreate(&ev);
  return ev;
}

// Host evaluation of one generation record into kernel arguments: validation, the host-side
// new-mutation draws (calc_new_mutations_Index) and the per-population parameter arrays.
struct GenHost {
  bool neutral;
  bool preserve;
};

static gf_status build_args(Engine* e, const gf_generation& gen, GenArgs& a, GenHost& gh) {
  const int P = e->P;
  if (gen.generation < 0 || gen.generation > GF_MAX_GENERATION)
    return fail(e, GF_ERR_CAPACITY, "generation %d outside [0, %d]", gen.generation, GF_MAX_GENERATION);
  std::memset(&a, 0, sizeof(a));
  a.generation = gen.generation;
  a.num_pops = P;
  a.seed1 = e->seed1;
  a.seed2 = e->seed2;
  bool neutral = true;
  long long new_total = 0;
  a.new_offset[0] = 0;
  for (int p = 0; p < P; ++p) {
    const gf_population_params& pp = gen.pop[p];
    if (pp.Nchrom_e < 0) return fail(e, GF_ERR_INVALID_ARGUMENT, "generation %d population %d: Nchrom_e < 0", gen.generation, p);
    if (pp.alive && !pp.drift)
      return fail(e, GF_ERR_INVALID_ARGUMENT, "generation %d population %d: alive population must be drifted", gen.generation, p);
    if (pp.drift) a.drift_mask |= 1 << p;
    if (pp.alive) a.alive_mask |= 1 << p;
    a.Nc[p] = pp.Nchrom_e;
    a.F[p] = pp.F;
    a.h[p] = pp.h;
    a.sel_a[p] = pp.sel_slope;
    a.sel_b[p] = pp.sel_intercept;
    if (pp.drift && (pp.sel_slope != 0.f || pp.sel_intercept != 0.f)) neutral = false;
    if (pp.drift && gen.selection_table) neutral = false;
    int count = 0;
    if (pp.mutate && pp.Nchrom_e > 0) {
      count = host_new_mutation_count(e->seed1, e->seed2, pp.mu, pp.Nchrom_e, e->num_sites, gen.generation, p);
      a.new_freq[p] = 1.f / pp.Nchrom_e;
    }
    new_total += count;
    if (new_total > (1LL << 30)) return fail(e, GF_ERR_CAPACITY, "generation %d: %lld new mutations", gen.generation, new_total);
    a.new_offset[p + 1] = static_cast<int>(new_total);
    for (int k = 0; k < P; ++k) a.mig[k * P + p] = gen.migration[k * kMaxPops + p];
  }
  for (int p = P; p <= kMaxPops; ++p) a.new_offset[p] = a.new_offset[P];
  a.new_total = static_cast<int>(new_total);
  a.flag = (gen.compact || gen.preserve) && e->compact_interval > 0;
  if (gen.selection_table) {
    if (!e->sel_table)
      return fail(e, GF_ERR_STATE, "generation %d reads a selection table that gf_sim_selection_view has not set up",
                  gen.generation);
    a.sel_table = e->sel_table;
    a.sel_stride = e->sel_table_stride;
  }
  gh.neutral = neutral;
  gh.preserve = gen.preserve != 0;
  return GF_OK;
}

// Compaction of the state a drift or window launch just wrote into freq[cur ^ 1] with its flags and
// tile counts (d_count[3] = slots): exclusive scan of the tile counts (the survivor total lands in
// d_count[slot_out]), then the stable scatter of all P rows and the IDs back into freq[cur]
// (compact, go_fish_impl.cuh:370-429).
static gf_status launch_compaction(Engine* e, int tiles_bound, int slot_out, bool preserve) {
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (e->profiling) {
    ev0 = prof_event(e);
    ev1 = prof_event(e);
    GF_CUDA(e, cudaEventRecord(ev0, e->stream));
  }
  scan_exclusive_kernel<<<1, kScanThreads, 0, e->stream>>>(e->tile_count, e->tile_offset, 0, e->d_count + slot_out,
                                                            e->d_count + 3);
  const int sblocks = std::max(1, std::min(tiles_bound, e->num_sms * 8));
  GF_CUDA(e, cudaGetLastError());
  const int src = e->cur ^ 1;
  if (preserve) {
    scatter_kernel<true><<<sblocks, kDriftThreads, 0, e->stream>>>(
        e->freq[src], e->freq[e->cur], e->id_gp[e->id_cur], e->id_tid[e->id_cur], e->id_gp[e->id_cur ^ 1],
        e->id_tid[e->id_cur ^ 1], e->flags, e->tile_offset, e->capacity, e->P, e->d_count + 3);
    e->any_preserved = true;
  } else {
    scatter_kernel<false><<<sblocks, kDriftThreads, 0, e->stream>>>(
        e->freq[src], e->freq[e->cur], e->id_gp[e->id_cur], e->id_tid[e->id_cur], e->id_gp[e->id_cur ^ 1],
        e->id_tid[e->id_cur ^ 1], e->flags, e->tile_offset, e->capacity, e->P, e->d_count + 3);
  }
  GF_CUDA(e, cudaGetLastError());
  e->kernel_launches += 2;
  e->compactions += 1;
  if (e->profiling) {
    GF_CUDA(e, cudaEventRecord(ev1, e->stream));
    e->prof_compact.emplace_back(ev0, ev1);
  }
  e->id_cur ^= 1;
  return GF_OK;
}

// Launch one generation whose arguments are `h` on the host and `d` in the device table.
static gf_status launch_generation(Engine* e, GenArgs& h, GenArgs* d_table, int index, const GenHost& gh) {
  const int P = e->P;
  const long long new_total = h.new_total;
  if (!e->pending.empty()) poll_pending(e, false);
  // the preserved check is decided when the generation launches (earlier compactions may set it)
  if (h.flag && e->any_preserved && !h.check_preserved) {
    h.check_preserved = 1;
    GF_CUDA(e, cudaMemcpyAsync(&d_table[index].check_preserved, &h.check_preserved, sizeof(int),
                               cudaMemcpyHostToDevice, e->stream));
  }
  long long need = e->M_upper + new_total;
  if (need > e->capacity) {
    poll_pending(e, true);
    need = e->M_upper + new_total;
    if (need > e->capacity) {
      // exact count, then grow
      int M = 0;
      GF_CUDA(e, cudaMemcpyAsync(&M, e->d_count + e->count_slot, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
      GF_CUDA(e, cudaStreamSynchronize(e->stream));
      e->M_upper = M;
      need = M + new_total;
      if (need > e->capacity) {
        gf_status st = set_capacity(e, std::max<long long>(need + need / 2, e->capacity * 3 / 2), M);
        if (st != GF_OK) return st;
      }
    }
  }
  const int tiles_bound = static_cast<int>(align_up(std::max<long long>(need, 1), kTileSlots) / kTileSlots);
  const int slot_in = e->count_slot;
  const int slot_out = slot_in ^ 1;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (e->profiling) {
    ev0 = prof_event(e);
    ev1 = prof_event(e);
    GF_CUDA(e, cudaEventRecord(ev0, e->stream));
  }
  launch_drift(e, tiles_bound, slot_in, slot_out, d_table + index, P == 1, gh.neutral, h.flag != 0);
  GF_CUDA(e, cudaGetLastError());
  e->kernel_launches += 1;
  e->live_rows |= h.drift_mask;
  if (e->profiling) {
    GF_CUDA(e, cudaEventRecord(ev1, e->stream));
    e->prof_drift.emplace_back(ev0, ev1);
  }
  e->M_upper = need;
  for (auto& pc : e->pending) pc.added += new_total;

  if (h.flag) {
    gf_status cst = launch_compaction(e, tiles_bound, slot_out, gh.preserve);
    if (cst != GF_OK) return cst;
    // asynchronous read-back of the survivor count
    poll_pending(e, false);
    PendingCount pc;
    gf_status st = get_event(e, &pc.event);
    if (st != GF_OK) return st;
    pc.slot = e->next_slot;
    e->next_slot = (e->next_slot + 1) % e->pinned_slots;
    pc.added = 0;
    GF_CUDA(e, cudaMemcpyAsync(e->h_pinned + pc.slot, e->d_count + slot_out, sizeof(int), cudaMemcpyDeviceToHost,
                               e->stream));
    GF_CUDA(e, cudaEventRecord(pc.event, e->stream));
    if (static_cast<int>(e->pending.size()) >= e->pinned_slots - 1) poll_pending(e, true);
    e->pending.push_back(pc);
    e->M_exact = false;
  } else {
    e->cur ^= 1;
  }
  e->step_index++;
  e->count_slot ^= 1;
  return GF_OK;
}

// Make room for `need` slots: tighten the host bound from finished read-backs, then from an exact
// (synchronizing) read of the count, and grow the arrays if still short.
static gf_status ensure_capacity(Engine* e, long long new_slots, long long* need_out) {
  long long need = e->M_upper + new_slots;
  if (need > e->capacity) {
    poll_pending(e, true);
    need = e->M_upper + new_slots;
    if (need > e->capacity) {
      int M = 0;
      GF_CUDA(e, cudaMemcpyAsync(&M, e->d_count + e->count_slot, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
      GF_CUDA(e, cudaStreamSynchronize(e->stream));
      e->M_upper = M;
      need = M + new_slots;
      if (need > e->capacity) {
        gf_status st = set_capacity(e, std::max<long long>(need + need / 2, e->capacity * 3 / 2), M);
        if (st != GF_OK) return st;
      }
    }
  }
  *need_out = need;
  return GF_OK;
}

// Queue the asynchronous read-back of the survivor count in d_count[slot].
static gf_status push_readback(Engine* e, int slot) {
  poll_pending(e, false);
  PendingCount pc;
  gf_status st = get_event(e, &pc.event);
  if (st != GF_OK) return st;
  pc.slot = e->next_slot;
  e->next_slot = (e->next_slot + 1) % e->pinned_slots;
  pc.added = 0;
  GF_CUDA(e, cudaMemcpyAsync(e->h_pinned + pc.slot, e->d_count + slot, sizeof(int), cudaMemcpyDeviceToHost,
                             e->stream));
  GF_CUDA(e, cudaEventRecord(pc.event, e->stream));
  if (static_cast<int>(e->pending.size()) >= e->pinned_slots - 1) poll_pending(e, true);
  e->pending.push_back(pc);
  e->M_exact = false;
  return GF_OK;
}

// Single-population generations a window may hold: drifted, no migration factor other than 1.
static bool window_eligible(const Engine* e, const gf_generation& g) {
  return e->use_windows && e->P == 1 && g.pop[0].drift == 1 && g.migration[0] == 1.0f && !g.selection_table;
}

constexpr int kMaxWindow = kMaxWindowGenerations;

// Generations a multi-population window may hold (2 <= P <= 4): every population is either drifted
// with Nc > 0, or not drifted and its rows are zero in both state buffers (`live`: the populations
// whose rows may hold a nonzero value, given the generations before this one).  Extinction
// generations and every generation after an extinction run one launch each.
static bool window_mp_eligible(const Engine* e, const gf_generation& g, int live) {
  return e->use_windows && !g.selection_table && mp_window_generation_ok(g, e->P, live, kMaxWindowPops);
}

static int drift_bits(const gf_generation& g, int P) { return drifted_populations(g, P); }

// Run generations [first, first + count) of the batch as one window launch.
static gf_status launch_window(Engine* e, int b, int first, int count, const GenHost* gh) {
  WinRep& R = e->h_wrep[b][first];
  long long news = 0;
  for (int k = 0; k < count; ++k) news += e->h_wgen[b][first + k].new_count;
  long long need = 0;
  gf_status st = ensure_capacity(e, news, &need);
  if (st != GF_OK) return st;
  const GenArgs& last = e->h_table[b][first + count - 1];
  R.base = 0;
  R.capacity = e->capacity;
  R.rec = first;
  R.ngen = count;
  R.tile0 = 0;
  R.ntiles = static_cast<int>(align_up(std::max<long long>(need, 1), kTileSlots) / kTileSlots);
  R.seed1 = e->seed1;
  R.seed2 = e->seed2;
  R.check_preserved = e->any_preserved ? 1 : 0;
  R.compact = last.flag ? 1 : 0;
  R.preserve = (last.flag && gh[first + count - 1].preserve) ? 1 : 0;
  R.rep = 0;
  R.births = news;
  GF_CUDA(e, cudaMemcpyAsync(e->d_wrep[b] + first, &R, sizeof(WinRep), cudaMemcpyHostToDevice, e->stream));
  const int slot = e->count_slot;
  WindowLaunch w;
  w.A = e->freq[e->cur];
  w.B = e->freq[e->cur ^ 1];
  w.id_gp_cur = e->id_gp[e->id_cur];
  w.id_tid_cur = e->id_tid[e->id_cur];
  w.id_gp_next = e->id_gp[e->id_cur ^ 1];
  w.id_tid_next = e->id_tid[e->id_cur ^ 1];
  w.flags = e->flags;
  w.tile_count = e->tile_count;
  w.tile_offset = e->tile_offset;
  w.M_in = e->d_count + slot;
  w.M_end = e->d_count + 3;
  w.M_next = e->d_count + (slot ^ 1);
  w.M_out = e->d_count + (slot ^ 1);
  w.reps = e->d_wrep[b] + first;
  w.nreps = 1;
  w.recs = e->d_wgen[b];
  w.total_tiles = R.ntiles;
  w.any_compact = R.compact != 0;
  w.stats = e->d_stats;
  w.fault = e->d_count + 2;
  w.sched = e->d_count + kSchedWord;
  w.uniform_key = true;
  w.seed1 = e->seed1;
  w.seed2 = e->seed2;
  // profiling: the window kernel's time counts as drift, its segmented scan and scatter as compaction
  cudaEvent_t ev0 = nullptr, evw = nullptr, evc = nullptr, ev1 = nullptr;
  if (e->profiling) {
    ev0 = prof_event(e);
    evw = prof_event(e);
    evc = prof_event(e);
    ev1 = prof_event(e);
    GF_CUDA(e, cudaEventRecord(ev0, e->stream));
  }
  st = window_run(e, w, e->freq[e->cur], evw, evc);
  if (st != GF_OK) return st;
  if (e->profiling) {
    GF_CUDA(e, cudaEventRecord(ev1, e->stream));
    e->prof_drift.emplace_back(ev0, evw);
    if (R.compact) {
      e->prof_compact.emplace_back(evc, ev1);
    } else {
      e->prof_pool.push_back(evc);
      e->prof_pool.push_back(ev1);
    }
  }
  e->M_upper = need;
  for (auto& pc : e->pending) pc.added += news;
  e->count_slot ^= 1;
  e->step_index += count;
  if (R.compact) {
    if (R.preserve) e->any_preserved = true;
    e->id_cur ^= 1;
    e->compactions += 1;
    st = push_readback(e, e->count_slot);
    if (st != GF_OK) return st;
  } else {
    e->cur ^= 1;
  }
  return GF_OK;
}

// Run generations [first, first + count) of a multi-population batch as one window launch; the
// kernel reads their records from the device table d_table[b].
static gf_status launch_window_mp(Engine* e, int b, int first, int count, const GenHost* gh) {
  long long news = 0;
  int drifted = 0;
  for (int k = 0; k < count; ++k) {
    news += e->h_table[b][first + k].new_total;
    drifted |= e->h_table[b][first + k].drift_mask;
  }
  long long need = 0;
  gf_status st = ensure_capacity(e, news, &need);
  if (st != GF_OK) return st;
  const GenArgs& last = e->h_table[b][first + count - 1];
  const bool compact = last.flag != 0;
  const bool preserve = compact && gh[first + count - 1].preserve;
  const int tiles_bound = static_cast<int>(align_up(std::max<long long>(need, 1), kTileSlots) / kTileSlots);
  const int slot_in = e->count_slot;
  const int slot_out = slot_in ^ 1;
  WindowMpLaunch w;
  w.P = e->P;
  w.A = e->freq[e->cur];
  w.B = e->freq[e->cur ^ 1];
  w.stride = e->capacity;
  w.id_gp = e->id_gp[e->id_cur];
  w.id_tid = e->id_tid[e->id_cur];
  w.flags = e->flags;
  w.tile_count = e->tile_count;
  w.d_count = e->d_count;
  w.slot_in = slot_in;
  w.slot_out = slot_out;
  w.table = e->d_table[b] + first;
  w.ngen = count;
  w.births = news;
  w.compact = compact ? 1 : 0;
  w.check_preserved = e->any_preserved ? 1 : 0;
  w.seed1 = e->seed1;
  w.seed2 = e->seed2;
  w.stats = e->d_stats;
  w.tiles_bound = tiles_bound;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (e->profiling) {
    ev0 = prof_event(e);
    ev1 = prof_event(e);
    GF_CUDA(e, cudaEventRecord(ev0, e->stream));
  }
  st = window_mp_run(e, w);
  if (st != GF_OK) return st;
  if (e->profiling) {
    GF_CUDA(e, cudaEventRecord(ev1, e->stream));
    e->prof_drift.emplace_back(ev0, ev1);
  }
  e->live_rows |= drifted;
  e->M_upper = need;
  for (auto& pc : e->pending) pc.added += news;
  e->step_index += count;
  if (compact) {
    st = launch_compaction(e, tiles_bound, slot_out, preserve);
    if (st != GF_OK) return st;
    e->count_slot ^= 1;
    return push_readback(e, e->count_slot);
  }
  e->cur ^= 1;
  e->count_slot ^= 1;
  return GF_OK;
}

// Run a batch of generations: evaluate all records on the host, upload them as one table, launch.
static gf_status run_batch(Engine* e, const gf_generation* gens, int n) {
  const int b = e->table_next;
  e->table_next ^= 1;
  if (e->table_done[b]) GF_CUDA(e, cudaEventSynchronize(e->table_done[b]));  // the GPU is done with buffer b
  else GF_CUDA(e, cudaEventCreateWithFlags(&e->table_done[b], cudaEventDisableTiming));
  if (e->table_cap[b] < static_cast<size_t>(n)) {
    const size_t cap = std::max<size_t>(n, 256);
    if (e->d_table[b]) GF_CUDA(e, cudaFree(e->d_table[b]));
    if (e->h_table[b]) GF_CUDA(e, cudaFreeHost(e->h_table[b]));
    e->d_table[b] = nullptr;
    e->h_table[b] = nullptr;
    e->table_cap[b] = 0;
    GF_CUDA(e, cudaMalloc(&e->d_table[b], sizeof(GenArgs) * cap));
    GF_CUDA(e, cudaMallocHost(&e->h_table[b], sizeof(GenArgs) * cap));
    e->table_cap[b] = cap;
  }
  const bool windows = e->use_windows && e->P == 1;
  if (windows && e->wtable_cap[b] < static_cast<size_t>(n)) {
    const size_t cap = std::max<size_t>(n, 256);
    if (e->d_wgen[b]) GF_CUDA(e, cudaFree(e->d_wgen[b]));
    if (e->h_wgen[b]) GF_CUDA(e, cudaFreeHost(e->h_wgen[b]));
    if (e->d_wrep[b]) GF_CUDA(e, cudaFree(e->d_wrep[b]));
    if (e->h_wrep[b]) GF_CUDA(e, cudaFreeHost(e->h_wrep[b]));
    e->d_wgen[b] = nullptr;
    e->h_wgen[b] = nullptr;
    e->d_wrep[b] = nullptr;
    e->h_wrep[b] = nullptr;
    e->wtable_cap[b] = 0;
    GF_CUDA(e, cudaMalloc(&e->d_wgen[b], sizeof(WinGen) * cap));
    GF_CUDA(e, cudaMallocHost(&e->h_wgen[b], sizeof(WinGen) * cap));
    GF_CUDA(e, cudaMalloc(&e->d_wrep[b], sizeof(WinRep) * cap));
    GF_CUDA(e, cudaMallocHost(&e->h_wrep[b], sizeof(WinRep) * cap));
    e->wtable_cap[b] = cap;
  }
  std::vector<GenHost> gh(n);
  for (int i = 0; i < n; ++i) {
    gf_status st = build_args(e, gens[i], e->h_table[b][i], gh[i]);
    if (st != GF_OK) return st;
    e->h_table[b][i].check_preserved = e->any_preserved ? 1 : 0;
    if (windows) {
      const GenArgs& a = e->h_table[b][i];
      WinGen& wg = e->h_wgen[b][i];
      wg.generation = a.generation;
      wg.Nc = a.Nc[0];
      wg.new_count = a.new_total;
      wg.new_freq = a.new_freq[0];
      wg.F = a.F[0];
      wg.h = a.h[0];
      wg.sel_a = a.sel_a[0];
      wg.sel_b = a.sel_b[0];
      wg.alive = a.alive_mask & 1;
    }
  }
  GF_CUDA(e, cudaMemcpyAsync(e->d_table[b], e->h_table[b], sizeof(GenArgs) * n, cudaMemcpyHostToDevice, e->stream));
  if (windows)
    GF_CUDA(e, cudaMemcpyAsync(e->d_wgen[b], e->h_wgen[b], sizeof(WinGen) * n, cudaMemcpyHostToDevice, e->stream));
  const bool windows_mp = e->use_windows && e->P >= 2 && e->P <= kMaxWindowPops;
  int i = 0;
  while (i < n) {
    if (windows_mp && window_mp_eligible(e, gens[i], e->live_rows)) {
      int j = i;
      int live = e->live_rows;
      while (j < n && j - i < kMaxWindow && window_mp_eligible(e, gens[j], live)) {
        live |= drift_bits(gens[j], e->P);
        const bool ends = e->h_table[b][j].flag != 0;
        ++j;
        if (ends) break;
      }
      gf_status st = launch_window_mp(e, b, i, j - i, gh.data());
      if (st != GF_OK) return st;
      i = j;
    } else if (windows && window_eligible(e, gens[i])) {
      int j = i;
      while (j < n && j - i < kMaxWindow && window_eligible(e, gens[j])) {
        const bool ends = e->h_table[b][j].flag != 0;
        ++j;
        if (ends) break;
      }
      gf_status st = launch_window(e, b, i, j - i, gh.data());
      if (st != GF_OK) return st;
      i = j;
    } else {
      gf_status st = launch_generation(e, e->h_table[b][i], e->d_table[b], i, gh[i]);
      if (st != GF_OK) return st;
      ++i;
    }
  }
  GF_CUDA(e, cudaEventRecord(e->table_done[b], e->stream));
  return GF_OK;
}

static gf_status current_count(Engine* e, int* M) {
  GF_CUDA(e, cudaMemcpyAsync(M, e->d_count + e->count_slot, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  gf_status st = check_device_fault(e);
  if (st != GF_OK) return st;
  poll_pending(e, true);
  e->M_upper = *M;
  e->M_exact = true;
  return GF_OK;
}

}  // namespace gf

// ==================================================================================================
// C ABI
// ==================================================================================================
using namespace gf;


extern "C" {

const char* gf_version(void) { return "0.1.0"; }

const char* gf_status_string(gf_status s) {
  switch (s) {
    case GF_OK: return "ok";
    case GF_ERR_INVALID_ARGUMENT: return "invalid argument";
    case GF_ERR_CUDA: return "CUDA error";
    case GF_ERR_OUT_OF_MEMORY: return "out of device memory";
    case GF_ERR_CAPACITY: return "capacity limit exceeded";
    case GF_ERR_STATE: return "invalid call order";
    case GF_ERR_DEVICE: return "device-side fault";
    case GF_ERR_NO_DEVICE: return "no CUDA device";
  }
  return "unknown status";
}

gf_status gf_engine_create(int device, void* cuda_stream, gf_engine** out) {
  if (!out) return GF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return GF_ERR_NO_DEVICE;
  }
  if (device < 0) {
    if (cudaGetDevice(&device) != cudaSuccess) return GF_ERR_NO_DEVICE;
  }
  if (device >= n) return GF_ERR_NO_DEVICE;
  if (cudaSetDevice(device) != cudaSuccess) return GF_ERR_NO_DEVICE;
  gf_engine* g = new (std::nothrow) gf_engine();
  if (!g) return GF_ERR_OUT_OF_MEMORY;
  Engine* e = &g->impl;
  e->device = device;
  if (cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || e->num_sms < 1) {
    cudaGetLastError();
    e->num_sms = 148;
  }
  if (cuda_stream) {
    e->stream = static_cast<cudaStream_t>(cuda_stream);
  } else {
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete g;
      return GF_ERR_CUDA;
    }
    e->own_stream = true;
  }
  if (cudaMalloc(&e->d_count, sizeof(int) * kCountWords) != cudaSuccess ||
      cudaMalloc(&e->d_stats, sizeof(unsigned long long) * 2) != cudaSuccess ||
      cudaMallocHost(&e->h_pinned, sizeof(int) * e->pinned_slots) != cudaSuccess) {
    if (e->d_count) cudaFree(e->d_count);
    if (e->own_stream) cudaStreamDestroy(e->stream);
    delete g;
    return GF_ERR_OUT_OF_MEMORY;
  }
  cudaMemsetAsync(e->d_count, 0, sizeof(int) * kCountWords, e->stream);
  cudaMemsetAsync(e->d_stats, 0, sizeof(unsigned long long) * 2, e->stream);
  {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (cudaMemPoolCreate(&e->pool, &props) == cudaSuccess) {
      uint64_t keep_all = UINT64_MAX;
      cudaMemPoolSetAttribute(e->pool, cudaMemPoolAttrReleaseThreshold, &keep_all);
    } else {
      cudaGetLastError();
      e->pool = nullptr;   // fall back to the device's default pool
    }
  }
  *out = g;
  return GF_OK;
}

void gf_engine_destroy(gf_engine* g) {
  if (!g) return;
  Engine* e = &g->impl;
  cudaSetDevice(e->device);
  cudaStreamSynchronize(e->stream);
  if (e->copy_stream) {
    cudaStreamSynchronize(e->copy_stream);
    cudaStreamDestroy(e->copy_stream);
    cudaEventDestroy(e->sample_packed);
    cudaEventDestroy(e->sample_done);
    cudaFreeHost(e->h_sample_count);
    if (e->sample_scratch) cudaFree(e->sample_scratch);
    if (e->h_sample_stage) cudaFreeHost(e->h_sample_stage);
  }
  release_sim(e);
  release_batch(e);
  cudaStreamSynchronize(e->stream);
  if (e->h_rec_stage) cudaFreeHost(e->h_rec_stage);
  if (e->batch_h_M) cudaFreeHost(e->batch_h_M);
  if (e->batch_arena_mem) cudaFree(e->batch_arena_mem);
  if (e->batch_recs_mem) cudaFree(e->batch_recs_mem);
  if (e->batch_plan_mem) cudaFree(e->batch_plan_mem);
  for (cudaEvent_t ev : e->batch_ahead)
    if (ev) cudaEventDestroy(ev);
  if (e->pool) cudaMemPoolDestroy(e->pool);
  for (auto ev : e->free_events) cudaEventDestroy(ev);
  if (e->spec_scratch) cudaFree(e->spec_scratch);
  if (e->spec_in) cudaFree(e->spec_in);
  if (e->spec_out) cudaFree(e->spec_out);
  if (e->d_count) cudaFree(e->d_count);
  if (e->d_stats) cudaFree(e->d_stats);
  for (int b = 0; b < 2; ++b) {
    if (e->d_table[b]) cudaFree(e->d_table[b]);
    if (e->h_table[b]) cudaFreeHost(e->h_table[b]);
    if (e->table_done[b]) cudaEventDestroy(e->table_done[b]);
    if (e->d_wgen[b]) cudaFree(e->d_wgen[b]);
    if (e->h_wgen[b]) cudaFreeHost(e->h_wgen[b]);
    if (e->d_wrep[b]) cudaFree(e->d_wrep[b]);
    if (e->h_wrep[b]) cudaFreeHost(e->h_wrep[b]);
  }
  for (auto& pr : e->prof_drift) e->prof_pool.insert(e->prof_pool.end(), {pr.first, pr.second});
  for (auto& pr : e->prof_compact) e->prof_pool.insert(e->prof_pool.end(), {pr.first, pr.second});
  for (auto ev : e->prof_pool) cudaEventDestroy(ev);
  if (e->h_pinned) cudaFreeHost(e->h_pinned);
  if (e->own_stream) cudaStreamDestroy(e->stream);
  delete g;
}

const char* gf_engine_last_error(const gf_engine* g) { return g ? g->impl.last_error.c_str() : "engine is NULL"; }

int32_t gf_engine_device(const gf_engine* g) { return g ? g->impl.device : -1; }

gf_status gf_engine_synchronize(gf_engine* g) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    GF_CUDA(e, cudaSetDevice(e->device));
    return check_device_fault(e);
  });
}

int32_t gf_new_mutation_count(int32_t seed1, int32_t seed2, float mu, int32_t Nchrom_e, float num_sites,
                              int32_t generation, int32_t population) {
  return host_new_mutation_count(seed1, seed2, mu, Nchrom_e, num_sites, generation, population);
}

gf_status gf_sim_begin_blank(gf_engine* g, const gf_sim_config* c, int32_t start_generation) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    (void)start_generation;
    return begin_common(e, c, 0);
  });
}

gf_status gf_sim_begin_from_state(gf_engine* g, const gf_sim_config* c, int32_t start_generation, const float* freq,
                                  const int32_t* mut_ids, int32_t num_mutations, const uint8_t* extinct,
                                  int32_t preserve) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    (void)start_generation;
    (void)extinct;
    if (num_mutations < 0) return fail(e, GF_ERR_INVALID_ARGUMENT, "num_mutations < 0");
    if (num_mutations > 0 && (!freq || !mut_ids)) return fail(e, GF_ERR_INVALID_ARGUMENT, "freq / mut_ids is NULL");
    gf_status st = begin_common(e, c, num_mutations);
    if (st != GF_OK) return st;
    if (num_mutations == 0) return GF_OK;
    const int P = e->P;
    GF_CUDA(e, cudaMemcpy2DAsync(e->freq[e->cur], sizeof(float) * e->capacity, freq, sizeof(float) * num_mutations,
                                 sizeof(float) * num_mutations, P, cudaMemcpyHostToDevice, e->stream));
    for (int p = 0; p < P; ++p) {  // rows holding anything but +0.0 (bit pattern 0)
      const uint32_t* row = reinterpret_cast<const uint32_t*>(freq + static_cast<size_t>(p) * num_mutations);
      for (int i = 0; i < num_mutations; ++i)
        if (row[i] != 0u) {
          e->live_rows |= 1 << p;
          break;
        }
    }
    std::vector<int> gp(num_mutations), tid(num_mutations);
    bool any_neg = false;
    for (int i = 0; i < num_mutations; ++i) {
      const int gen0 = mut_ids[4 * i + 0], pop0 = mut_ids[4 * i + 1];
      if (gen0 < 0 || gen0 > GF_MAX_GENERATION || pop0 < 0 || pop0 >= 128)
        return fail(e, GF_ERR_CAPACITY, "mutation %d: origin generation %d / population %d outside the packed ID range", i,
                    gen0, pop0);
      gp[i] = gen0 | (pop0 << 24);
      tid[i] = preserve ? -std::abs(mut_ids[4 * i + 2]) : mut_ids[4 * i + 2];
      any_neg |= tid[i] < 0;
    }
    GF_CUDA(e, cudaMemcpyAsync(e->id_gp[e->id_cur], gp.data(), sizeof(int) * num_mutations, cudaMemcpyHostToDevice, e->stream));
    GF_CUDA(e, cudaMemcpyAsync(e->id_tid[e->id_cur], tid.data(), sizeof(int) * num_mutations, cudaMemcpyHostToDevice, e->stream));
    const int M = num_mutations;
    GF_CUDA(e, cudaMemcpyAsync(e->d_count, &M, sizeof(int), cudaMemcpyHostToDevice, e->stream));
    GF_CUDA(e, cudaStreamSynchronize(e->stream));  // host vectors go out of scope
    e->any_preserved = any_neg;
    return GF_OK;
  });
}

gf_status gf_sim_begin_mse(gf_engine* g, const gf_sim_config* c, const gf_mse_population* pops, int32_t preserve) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (!c || !pops) return fail(e, GF_ERR_INVALID_ARGUMENT, "config / pops is NULL");
    if (c->num_populations < 1 || c->num_populations > kMaxPops)
      return fail(e, GF_ERR_INVALID_ARGUMENT, "num_populations %d outside [1, %d]", c->num_populations, kMaxPops);
    const int P = c->num_populations;
    MseClassRange cr;
    std::memset(&cr, 0, sizeof(cr));
    long long num_classes = 0;
    for (int p = 0; p < P; ++p) {
      cr.first_class[p] = static_cast<int>(num_classes);
      cr.Nc[p] = pops[p].Nchrom_e;
      if (pops[p].Nchrom_e > 1) num_classes += pops[p].Nchrom_e - 1;
    }
    for (int p = P; p <= kMaxPops; ++p) cr.first_class[p] = static_cast<int>(num_classes);
    GF_CUDA(e, cudaSetDevice(e->device));
    // class counts, then their exclusive scan; the total is read back once (as the reference does)
    unsigned* d_counts = nullptr;
    unsigned* d_starts = nullptr;
    float* d_area = nullptr;
    float* d_integral = nullptr;
    int* d_total = nullptr;
    const long long ncls = std::max<long long>(num_classes, 1);
    long long max_nc = 1;
    for (int p = 0; p < P; ++p) max_nc = std::max<long long>(max_nc, pops[p].Nchrom_e);
    {
      gf_status ast = pool_alloc(e, reinterpret_cast<void**>(&d_counts), sizeof(unsigned) * ncls);
      if (ast == GF_OK) ast = pool_alloc(e, reinterpret_cast<void**>(&d_starts), sizeof(unsigned) * ncls);
      if (ast == GF_OK) ast = pool_alloc(e, reinterpret_cast<void**>(&d_area), sizeof(float) * max_nc);
      if (ast == GF_OK) ast = pool_alloc(e, reinterpret_cast<void**>(&d_integral), sizeof(float) * max_nc);
      if (ast == GF_OK) ast = pool_alloc(e, reinterpret_cast<void**>(&d_total), sizeof(int));
      if (ast != GF_OK) {
        for (void* q : {static_cast<void*>(d_counts), static_cast<void*>(d_starts), static_cast<void*>(d_area),
                        static_cast<void*>(d_integral), static_cast<void*>(d_total)})
          if (q) cudaFreeAsync(q, e->stream);
        return ast;
      }
    }
    GF_CUDA(e, cudaMemsetAsync(d_counts, 0, sizeof(unsigned) * ncls, e->stream));
    for (int p = 0; p < P; ++p) {
      const gf_mse_population& mp = pops[p];
      const int Nc = mp.Nchrom_e;
      if (Nc <= 1) continue;
      const bool selected = (mp.sel_slope != 0.f || mp.sel_intercept != 0.f);
      if (selected) {
        mse_area_kernel<<<148, 1024, 0, e->stream>>>(d_area, Nc, 1.0f / Nc, mp.N_ind, mp.F, mp.h, mp.sel_slope,
                                                      mp.sel_intercept);
        mse_integral_kernel<<<1, 1024, 0, e->stream>>>(d_area, d_integral, Nc);
      }
      mse_count_kernel<<<std::max(1, std::min(1184, (Nc + 255) / 256)), 256, 0, e->stream>>>(
          d_counts, d_integral, cr.first_class[p], mp.mu, mp.N_ind, Nc, c->num_sites, mp.sel_slope, mp.sel_intercept,
          mp.F, mp.h, c->seed1, c->seed2, p, selected ? 1 : 0);
      GF_CUDA(e, cudaGetLastError());
      e->kernel_launches += selected ? 3 : 1;
    }
    e->kernel_launches += 2;  // class scan + slot fill
    scan_exclusive_kernel<<<1, kScanThreads, 0, e->stream>>>(d_counts, d_starts, static_cast<int>(num_classes), d_total,
                                                              nullptr);
    GF_CUDA(e, cudaGetLastError());
    int M0 = 0;
    GF_CUDA(e, cudaMemcpyAsync(&M0, d_total, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
    GF_CUDA(e, cudaStreamSynchronize(e->stream));
    gf_status st = begin_common(e, c, M0);
    if (st == GF_OK && M0 > 0) {
      mse_fill_kernel<<<std::max(1, std::min(148 * 8, (M0 + 255) / 256)), 256, 0, e->stream>>>(
          e->freq[e->cur], e->id_gp[e->id_cur], e->id_tid[e->id_cur], d_starts, static_cast<int>(num_classes), M0,
          e->capacity, P, preserve ? 1 : 0, cr);
      cudaError_t err = cudaGetLastError();
      if (err != cudaSuccess) st = cuda_fail(e, err, "mse_fill_kernel");
      if (st == GF_OK) {
        err = cudaMemcpyAsync(e->d_count, &M0, sizeof(int), cudaMemcpyHostToDevice, e->stream);
        if (err != cudaSuccess) st = cuda_fail(e, err, "cudaMemcpyAsync");
      }
      e->any_preserved = preserve != 0;
      for (int p = 0; p < P; ++p)  // populations with equilibrium mutations (the others' rows stay zero)
        if (pops[p].Nchrom_e > 1) e->live_rows |= 1 << p;
    }
    cudaFreeAsync(d_counts, e->stream);
    cudaFreeAsync(d_starts, e->stream);
    cudaFreeAsync(d_area, e->stream);
    cudaFreeAsync(d_integral, e->stream);
    cudaFreeAsync(d_total, e->stream);
    return st;
  });
}

gf_status gf_sim_run(gf_engine* g, const gf_generation* gens, int32_t n) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (!e->active) return fail(e, GF_ERR_STATE, "gf_sim_run before gf_sim_begin_*");
    if (n < 0 || (n > 0 && !gens)) return fail(e, GF_ERR_INVALID_ARGUMENT, "bad generation table");
    for (int i = 0; i < n && n > 1; ++i)
      if (gens[i].selection_table)
        return fail(e, GF_ERR_INVALID_ARGUMENT,
                    "generation %d reads a selection table: such a generation is run alone (one record per call)",
                    gens[i].generation);
    GF_CUDA(e, cudaSetDevice(e->device));
    if (n == 0) return GF_OK;
    return run_batch(e, gens, n);
  });
}

gf_status gf_sim_selection_view(gf_engine* g, gf_selection_view* out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g || !out) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (!e->active) return fail(e, GF_ERR_STATE, "gf_sim_selection_view before gf_sim_begin_*");
    GF_CUDA(e, cudaSetDevice(e->device));
    if (!e->sel_table || e->sel_table_stride < e->capacity) {
      if (e->sel_table) cudaFreeAsync(e->sel_table, e->stream);
      e->sel_table = nullptr;
      e->sel_table_stride = 0;
      gf_status st = pool_alloc(e, reinterpret_cast<void**>(&e->sel_table),
                                sizeof(float) * static_cast<size_t>(e->P) * static_cast<size_t>(e->capacity));
      if (st != GF_OK) return st;
      e->sel_table_stride = e->capacity;
    }
    out->freq = e->freq[e->cur];
    out->row_stride = e->capacity;
    out->num_mutations = e->d_count + e->count_slot;
    out->selection = e->sel_table;
    out->selection_stride = e->sel_table_stride;
    out->num_populations = e->P;
    out->reserved = 0;
    out->cuda_stream = e->stream;
    return GF_OK;
  });
}

gf_status gf_sim_num_mutations(gf_engine* g, int32_t* out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g || !out) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (!e->active) return fail(e, GF_ERR_STATE, "no simulation");
    GF_CUDA(e, cudaSetDevice(e->device));
    int M = 0;
    gf_status st = current_count(e, &M);
    if (st != GF_OK) return st;
    *out = M;
    return GF_OK;
  });
}

gf_status gf_sim_read_state(gf_engine* g, float* freq_out, int32_t* ids_out, int32_t max_mutations,
                            int32_t* out_num) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (!e->active) return fail(e, GF_ERR_STATE, "no simulation");
    GF_CUDA(e, cudaSetDevice(e->device));
    int M = 0;
    gf_status st = current_count(e, &M);
    if (st != GF_OK) return st;
    if (out_num) *out_num = M;
    if (M > max_mutations) return fail(e, GF_ERR_CAPACITY, "state holds %d mutations, caller buffer %d", M, max_mutations);
    if (M == 0) return GF_OK;
    if (freq_out) {
      GF_CUDA(e, cudaMemcpy2DAsync(freq_out, sizeof(float) * M, e->freq[e->cur], sizeof(float) * e->capacity,
                                   sizeof(float) * M, e->P, cudaMemcpyDeviceToHost, e->stream));
    }
    if (ids_out) {
      // the reference's int4 IDs (generation, population, threadID, 0) are assembled on the device from
      // the packed words and copied out in one transfer
      int4* d_ids = nullptr;
      gf_status ast = pool_alloc(e, reinterpret_cast<void**>(&d_ids), sizeof(int4) * static_cast<size_t>(M));
      if (ast != GF_OK) return ast;
      expand_ids_kernel<<<std::min(148 * 8, (M + 255) / 256), 256, 0, e->stream>>>(e->id_gp[e->id_cur],
                                                                                 e->id_tid[e->id_cur], M, d_ids);
      cudaError_t err = cudaGetLastError();
      if (err == cudaSuccess)
        err = cudaMemcpyAsync(ids_out, d_ids, sizeof(int4) * static_cast<size_t>(M), cudaMemcpyDeviceToHost, e->stream);
      cudaFreeAsync(d_ids, e->stream);
      if (err != cudaSuccess) return cuda_fail(e, err, "reading mutation IDs");
    }
    GF_CUDA(e, cudaStreamSynchronize(e->stream));
    return GF_OK;
  });
}

gf_status gf_sim_sample_begin(gf_engine* g, float* freq_out, int32_t* ids_out, int32_t max_mutations) {
  return guard_host(g, [&]() -> gf_status {
    if (!g || max_mutations < 0) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (!e->active) return fail(e, GF_ERR_STATE, "no simulation");
    if (e->sample_in_flight) return fail(e, GF_ERR_STATE, "a time sample is already in flight");
    GF_CUDA(e, cudaSetDevice(e->device));
    poll_pending(e, false);
    long long bound = e->M_upper;
    if (bound > max_mutations) {   // the bound is loose: read the count itself
      int M = 0;
      gf_status st = current_count(e, &M);
      if (st != GF_OK) return st;
      if (M > max_mutations)
        return fail(e, GF_ERR_CAPACITY, "state holds %d mutations, caller buffer %d", M, max_mutations);
      bound = M;
    }
    if (!e->copy_stream) {
      GF_CUDA(e, cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking));
      GF_CUDA(e, cudaEventCreateWithFlags(&e->sample_packed, cudaEventDisableTiming));
      GF_CUDA(e, cudaEventCreateWithFlags(&e->sample_done, cudaEventDisableTiming));
      GF_CUDA(e, cudaMallocHost(&e->h_sample_count, sizeof(int)));
    }
    const int P = e->P;
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t fbytes = sizeof(float) * static_cast<size_t>(P) * static_cast<size_t>(bound);
    const size_t ibytes = sizeof(int4) * static_cast<size_t>(bound);
    const size_t need = al(fbytes) + al(ibytes) + 256;
    if (e->sample_scratch_bytes < need) {   // no sample in flight: the old scratch is free
      GF_CUDA(e, cudaStreamSynchronize(e->copy_stream));
      if (e->sample_scratch) GF_CUDA(e, cudaFree(e->sample_scratch));
      e->sample_scratch = nullptr;
      e->sample_scratch_bytes = 0;
      const size_t bytes = need + need / 4;
      GF_CUDA(e, cudaMalloc(&e->sample_scratch, bytes));
      e->sample_scratch_bytes = bytes;
    }
    char* base = static_cast<char*>(e->sample_scratch);
    float* d_freq = reinterpret_cast<float*>(base);
    int4* d_ids = reinterpret_cast<int4*>(base + al(fbytes));
    int* d_cnt = reinterpret_cast<int*>(base + al(fbytes) + al(ibytes));
    e->sample_bound = bound;
    e->sample_P = P;
    const int blocks = static_cast<int>(std::max<long long>(1, std::min<long long>(148 * 8, (bound + 255) / 256)));
    pack_sample_kernel<<<blocks, 256, 0, e->stream>>>(e->freq[e->cur], e->capacity, P, e->id_gp[e->id_cur],
                                                       e->id_tid[e->id_cur], e->d_count + e->count_slot,
                                                       static_cast<int>(bound), d_freq, d_ids, d_cnt);
    GF_CUDA(e, cudaGetLastError());
    e->kernel_launches += 1;
    GF_CUDA(e, cudaEventRecord(e->sample_packed, e->stream));
    // the count follows on the copy stream; the rows and IDs are copied once it is known (at the
    // wait), exactly M of them, while the engine's stream runs whatever was enqueued after this point
    GF_CUDA(e, cudaStreamWaitEvent(e->copy_stream, e->sample_packed, 0));
    GF_CUDA(e, cudaMemcpyAsync(e->h_sample_count, d_cnt, sizeof(int), cudaMemcpyDeviceToHost, e->copy_stream));
    GF_CUDA(e, cudaEventRecord(e->sample_done, e->copy_stream));
    e->sample_in_flight = true;
    e->sample_freq_out = freq_out;
    e->sample_ids_out = ids_out;
    e->sample_to_stage = !freq_out && !ids_out;
    return GF_OK;
  });
}

gf_status gf_sim_sample_wait(gf_engine* g, int32_t* out_num, int64_t* out_bytes) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (!e->sample_in_flight) return fail(e, GF_ERR_STATE, "no time sample in flight");
    GF_CUDA(e, cudaSetDevice(e->device));
    e->sample_in_flight = false;
    GF_CUDA(e, cudaEventSynchronize(e->sample_done));   // the sample is packed and its count is here
    const int M = *e->h_sample_count;
    if (M < 0) return fail(e, GF_ERR_STATE, "the count exceeded the engine's bound on it when the sample was packed");
    const int P = e->sample_P;
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    // the begin's scratch layout: rows [P][M] packed at the front of a bound-sized area, then the IDs
    char* base = static_cast<char*>(e->sample_scratch);
    const size_t fbytes = sizeof(float) * static_cast<size_t>(P) * static_cast<size_t>(e->sample_bound);
    const int4* d_ids = reinterpret_cast<const int4*>(base + al(fbytes));
    long long bytes = sizeof(int);
    if (e->sample_to_stage) {   // the engine's page-locked staging, grown to the sample with headroom
      const size_t need = static_cast<size_t>(P) * static_cast<size_t>(std::max(M, 1));
      if (e->sample_stage_cap < need) {
        if (e->h_sample_stage) GF_CUDA(e, cudaFreeHost(e->h_sample_stage));
        e->h_sample_stage = nullptr;
        e->sample_stage_cap = 0;
        const size_t cap = need + need / 4;
        GF_CUDA(e, cudaMallocHost(&e->h_sample_stage, sizeof(float) * cap));
        e->sample_stage_cap = cap;
      }
      e->sample_freq_out = e->h_sample_stage;
    }
    if (M > 0 && e->sample_freq_out) {
      GF_CUDA(e, cudaMemcpyAsync(e->sample_freq_out, base, sizeof(float) * static_cast<size_t>(P) * M,
                                 cudaMemcpyDeviceToHost, e->copy_stream));
      bytes += static_cast<long long>(sizeof(float)) * P * M;
    }
    if (M > 0 && e->sample_ids_out) {
      GF_CUDA(e, cudaMemcpyAsync(e->sample_ids_out, d_ids, sizeof(int4) * static_cast<size_t>(M), cudaMemcpyDeviceToHost,
                                 e->copy_stream));
      bytes += static_cast<long long>(sizeof(int4)) * M;
    }
    GF_CUDA(e, cudaStreamSynchronize(e->copy_stream));
    if (out_num) *out_num = M;
    if (out_bytes) *out_bytes = bytes;
    return GF_OK;
  });
}

gf_status gf_sim_sample_staged(gf_engine* g, const float** out_freq) {
  return guard_host(g, [&]() -> gf_status {
    if (!g || !out_freq) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (e->sample_in_flight || !e->sample_to_stage || !e->h_sample_stage)
      return fail(e, GF_ERR_STATE, "no staged time sample (begin with NULL arrays, then wait)");
    *out_freq = e->h_sample_stage;
    return GF_OK;
  });
}

gf_status gf_sim_stats_read(gf_engine* g, gf_sim_stats* out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g || !out) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    GF_CUDA(e, cudaSetDevice(e->device));
    unsigned long long st[2] = {0, 0};
    GF_CUDA(e, cudaMemcpyAsync(st, e->d_stats, sizeof(st), cudaMemcpyDeviceToHost, e->stream));
    GF_CUDA(e, cudaStreamSynchronize(e->stream));
    out->mutation_generations = static_cast<double>(st[0]);
    out->generations = static_cast<int64_t>(st[1]);
    out->compactions = e->compactions;
    out->kernel_launches = e->kernel_launches;
    return GF_OK;
  });
}

gf_status gf_engine_set_tuning(gf_engine* g, const gf_tuning* t) {
  return guard_host(g, [&]() -> gf_status {
    if (!g || !t) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (t->draw_strategy < 0 || t->draw_strategy >= kDrawStrategies || t->blocks_per_sm < 0 || t->windows < 0 ||
        t->windows > 1)
      return fail(e, GF_ERR_INVALID_ARGUMENT, "tuning: draw_strategy in {0, 1, 2, 3, 4}, blocks_per_sm >= 0, windows in {0, 1}");
    e->draw_strategy = t->draw_strategy;
    e->blocks_per_sm = t->blocks_per_sm;
    e->use_windows = t->windows != 0;
    return GF_OK;
  });
}

gf_status gf_engine_get_tuning(const gf_engine* g, gf_tuning* t) {
  if (!g || !t) return GF_ERR_INVALID_ARGUMENT;
  t->draw_strategy = g->impl.draw_strategy;
  t->blocks_per_sm = g->impl.blocks_per_sm;
  t->windows = g->impl.use_windows ? 1 : 0;
  return GF_OK;
}

gf_status gf_engine_set_profiling(gf_engine* g, int32_t enable) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    g->impl.profiling = enable != 0;
    return GF_OK;
  });
}

gf_status gf_engine_read_profile(gf_engine* g, gf_kernel_times* out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g || !out) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    GF_CUDA(e, cudaSetDevice(e->device));
    GF_CUDA(e, cudaStreamSynchronize(e->stream));
    auto sum = [&](std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& v, double* ms, int64_t* n) -> gf_status {
      double t = 0;
      for (auto& pr : v) {
        float x = 0.f;
        GF_CUDA(e, cudaEventElapsedTime(&x, pr.first, pr.second));
        t += x;
        e->prof_pool.push_back(pr.first);
        e->prof_pool.push_back(pr.second);
      }
      *ms = t;
      *n = static_cast<int64_t>(v.size());
      v.clear();
      return GF_OK;
    };
    gf_status st = sum(e->prof_drift, &out->drift_ms, &out->drift_launches);
    if (st != GF_OK) return st;
    return sum(e->prof_compact, &out->compact_ms, &out->compactions);
  });
}

gf_status gf_sim_device_state(gf_engine* g, const float** out_freq, int32_t* out_stride, int32_t* out_num) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (!e->active) return fail(e, GF_ERR_STATE, "no simulation");
    GF_CUDA(e, cudaSetDevice(e->device));
    int M = 0;
    gf_status st = current_count(e, &M);
    if (st != GF_OK) return st;
    if (out_freq) *out_freq = e->freq[e->cur];
    if (out_stride) *out_stride = static_cast<int32_t>(e->capacity);
    if (out_num) *out_num = M;
    return GF_OK;
  });
}

}  // extern "C"
