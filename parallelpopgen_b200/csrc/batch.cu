// Batched ragged replicates: thousands of independent single-population GO_Fish simulations with
// their own sizes, growth, selection, seeds and run lengths, advancing together.
//
// Layout: one arena of slots shared by all replicates; replicate r owns [base_r, base_r + cap_r) of
// every per-slot array (frequency ping-pong, the two ID words, flags), base_r a multiple of 1024 so a
// 1024-slot tile belongs to one replicate.  A super-step runs, for every unfinished replicate, the
// generations up to its next compaction (its own window length) in ONE window-kernel launch over
// all replicates' tiles, then one segmented scan (a block per replicate) and one segmented scatter.
// The host draws the per-generation new-mutation counts (as the reference does on its host,
// calc_new_mutations_Index, go_fish_impl.cuh:454-467) ahead of the GPU, and the survivor counts stay
// on the device until the run returns.  Because every per-slot operation is the plain engine's (same Philox counters relative
// to the replicate's own slots, same compaction schedule, same MSE start code), replicate r's state
// is bit-identical to a plain run with the same inputs.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <thread>
#include <vector>

#include "gf_drift.cuh"
#include "gf_internal.h"
#include "gf_mse.cuh"
#include "gf_plan.h"

#ifdef GF_TRACE
#include <chrono>
#include <cstdio>
// phase timings of batch_begin on stderr (build with -DGF_TRACE): time since the previous point
static double gf_trace_elapsed_ms() {
  static auto last = std::chrono::steady_clock::now();
  const auto now = std::chrono::steady_clock::now();
  const double ms = std::chrono::duration<double, std::milli>(now - last).count();
  last = now;
  return ms;
}
#define GF_TRACE_POINT(e, label)                                                     \
  do {                                                                               \
    cudaStreamSynchronize((e)->stream);                                              \
    std::fprintf(stderr, "[batch] %-28s %9.2f ms\n", label, gf_trace_elapsed_ms()); \
  } while (0)
#else
#define GF_TRACE_POINT(e, label) \
  do {                           \
  } while (0)
#endif

namespace gf {

constexpr int kBatchTile = 1024;

static long long align_tiles(long long v) { return (v + kBatchTile - 1) / kBatchTile * kBatchTile; }

// N(g): round(N0 * exp(rate * g)) in float (demography_exponential_growth), clamped
static int rep_population(const gf_replicate& p, int g) {
  const int n = static_cast<int>(std::round(p.N0 * std::exp(p.growth_rate * static_cast<float>(g))));
  return std::min(std::max(n, p.N_min), p.N_max);
}

static int rep_nchrom(const gf_replicate& p, int g) {
  return static_cast<int>(2 * rep_population(p, g) / (1 + p.F));
}

// ------------------------------------------------------------------------------------------------
// batched MSE start
// ------------------------------------------------------------------------------------------------
struct MseRep {
  long long area_off;   // offset of its Nc0 area / integral slices
  long long class_off;  // offset of its Nc0 - 1 classes
  long long slot_base;  // arena base
  int Nc0, N0, selected;
  float mu, L, F, h, sa, sb;
  int seed1, seed2;
};

template <typename Off>
__device__ __forceinline__ int find_seg(const MseRep* __restrict__ r, int n, long long idx, Off off) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off(r[mid]) <= idx) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void batch_mse_area_kernel(float* __restrict__ area, const MseRep* __restrict__ reps, int R,
                                      long long total) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(blockDim.x) * gridDim.x) {
    const int r = find_seg(reps, R, i, [](const MseRep& m) { return m.area_off; });
    const MseRep m = reps[r];
    if (!m.selected) continue;
    const int id = static_cast<int>(i - m.area_off);
    area[i] = mse_area(id, 1.0f / m.Nc0, m.N0, m.F, m.h, m.sa, m.sb);
  }
}

// one block per replicate: the plain engine's integral code on its slice
__global__ void __launch_bounds__(1024) batch_mse_integral_kernel(const float* __restrict__ area,
                                                                  float* __restrict__ integral,
                                                                  const MseRep* __restrict__ reps) {
  const MseRep m = reps[blockIdx.x];
  if (!m.selected) return;
  mse_integral_block(area + m.area_off, integral + m.area_off, m.Nc0);
}

__global__ void batch_mse_count_kernel(unsigned* __restrict__ counts, const float* __restrict__ integral,
                                       const MseRep* __restrict__ reps, int R, long long total) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(blockDim.x) * gridDim.x) {
    const int r = find_seg(reps, R, i, [](const MseRep& m) { return m.class_off; });
    const MseRep m = reps[r];
    const int id = static_cast<int>(i - m.class_off);
    const float* integ = integral + m.area_off;
    const float mse_total = m.selected ? integ[0] : 0.f;
    counts[i] = mse_class_count(id, integ, mse_total, m.mu, m.N0, m.Nc0, m.L, m.sa, m.sb, m.F, m.h, m.seed1,
                                m.seed2, 0);
  }
}

// one block per replicate: exclusive scan of its class counts, M0
__global__ void __launch_bounds__(1024) batch_class_scan_kernel(const unsigned* __restrict__ counts,
                                                                unsigned* __restrict__ starts,
                                                                const MseRep* __restrict__ reps, int* __restrict__ M0) {
  const MseRep m = reps[blockIdx.x];
  const int n = max(m.Nc0 - 1, 0);
  __shared__ unsigned s_warp[32];
  __shared__ unsigned s_carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += 1024) {
    const int i = base + threadIdx.x;
    const unsigned v = i < n ? counts[m.class_off + i] : 0u;
    unsigned incl = v;
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
    const unsigned excl = s_carry + s_warp[warp] + incl - v;
    if (i < n) starts[m.class_off + i] = excl;
    __syncthreads();
    if (threadIdx.x == 1023) s_carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) M0[blockIdx.x] = static_cast<int>(s_carry);
}

// slot k of replicate r: its class by binary search over the class starts; frequency (id + 1) / Nc0,
// ID (0, 0, k + 1) (initialize_mse_mutation_array + mse_set_mutID, go_fish_impl.cu:45-70)
struct FillRep {
  long long slot_prefix;  // global fill index of the replicate's slot 0
  long long class_off;
  long long base;
  int Nc0, M0;
};

__global__ void batch_mse_fill_kernel(float* __restrict__ freq, int* __restrict__ id_gp, int* __restrict__ id_tid,
                                      const unsigned* __restrict__ starts, const FillRep* __restrict__ reps, int R,
                                      long long total) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(blockDim.x) * gridDim.x) {
    int lo = 0, hi = R - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (reps[mid].slot_prefix <= i) lo = mid;
      else hi = mid - 1;
    }
    const FillRep f = reps[lo];
    const int k = static_cast<int>(i - f.slot_prefix);
    if (k >= f.M0) continue;
    int a = 0, b = f.Nc0 - 2;
    while (a < b) {
      const int mid = (a + b + 1) >> 1;
      if (static_cast<int>(starts[f.class_off + mid]) <= k) a = mid;
      else b = mid - 1;
    }
    freq[f.base + k] = (a + 1.f) / f.Nc0;
    id_gp[f.base + k] = 0;
    id_tid[f.base + k] = k + 1;
  }
}

// ------------------------------------------------------------------------------------------------
// batched SFS: one block per replicate, direct projection of its frequencies in double
// ------------------------------------------------------------------------------------------------
struct SfsRep {
  long long base;
  int M;
  float L;
};

constexpr int kBatchSfsThreads = 128;

__global__ void __launch_bounds__(kBatchSfsThreads)
    batch_sfs_kernel(const float* __restrict__ freq, const SfsRep* __restrict__ reps, int n,
                     const double* __restrict__ lgc, float* __restrict__ out) {
  const SfsRep R = reps[blockIdx.x];
  __shared__ double s_lp[kBatchSfsThreads];
  __shared__ double s_lq[kBatchSfsThreads];
  __shared__ unsigned s_seg[kBatchSfsThreads];
  __shared__ double s_acc0[kBatchSfsThreads];
  const int levels = n + 1;
  double acc[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) acc[u] = 0.0;
  unsigned nonseg = 0;
  for (int c0 = 0; c0 < R.M; c0 += kBatchSfsThreads) {
    const int i = c0 + threadIdx.x;
    double lp = 0.0, lq = 0.0;
    unsigned seg = 0;
    if (i < R.M) {
      const float p = freq[R.base + i];
      if (p > 0.f && p < 1.f) {
        seg = 1;
        lp = log(static_cast<double>(p));
        lq = log1p(-static_cast<double>(p));
      } else {
        ++nonseg;
      }
    }
    s_lp[threadIdx.x] = lp;
    s_lq[threadIdx.x] = lq;
    s_seg[threadIdx.x] = seg;
    __syncthreads();
    const int cend = min(kBatchSfsThreads, R.M - c0);
    for (int t = 0; t < cend; ++t) {
      if (!s_seg[t]) continue;
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int k = threadIdx.x + u * kBatchSfsThreads;
        if (k < levels) acc[u] += exp(lgc[k] + k * s_lp[t] + (n - k) * s_lq[t]);
      }
    }
    __syncthreads();
  }
  // non-segregating count of the block
  s_acc0[threadIdx.x] = static_cast<double>(nonseg);
  __syncthreads();
  if (threadIdx.x == 0) {
    double ns = 0;
    for (int t = 0; t < kBatchSfsThreads; ++t) ns += s_acc0[t];
    s_acc0[0] = ns;
  }
  __syncthreads();
  const double ns = s_acc0[0];
  __syncthreads();
  // bin n folds into bin 0: park it in shared memory
  double top = 0.0;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int k = threadIdx.x + u * kBatchSfsThreads;
    if (k == n) top = acc[u];
  }
  if (threadIdx.x == n % kBatchSfsThreads) s_acc0[1] = top;
  __syncthreads();
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int k = threadIdx.x + u * kBatchSfsThreads;
    if (k < n) {
      double v = acc[u];
      if (k == 0) v += s_acc0[1] + ns + static_cast<double>(R.L - R.M);
      out[static_cast<long long>(blockIdx.x) * n + k] = static_cast<float>(v);
    }
  }
}

// ------------------------------------------------------------------------------------------------
// host
// ------------------------------------------------------------------------------------------------
// Grow an engine-owned device buffer to `need` bytes (with a quarter of headroom); its previous
// contents are not kept.  The stream is idle when this runs (a batch begins after the last one ended).
static gf_status grow_device(Engine* e, void** mem, size_t* have, size_t need) {
  if (*have >= need && *mem) return GF_OK;
  if (*mem) GF_CUDA(e, cudaFree(*mem));
  *mem = nullptr;
  *have = 0;
  const size_t bytes = need + need / 4;
  const cudaError_t err = cudaMalloc(mem, bytes);
  if (err != cudaSuccess) {
    cudaGetLastError();
    *mem = nullptr;
    return cuda_fail(e, err, "batched arena allocation");
  }
  *have = bytes;
  return GF_OK;
}

void release_batch(Engine* e) {
  Batch* b = e->batch;
  if (!b) return;
  b->cancel.store(true);
  for (auto& t : b->producers) t.join();
  b->producers.clear();
  cudaStreamSynchronize(e->stream);
  // the arena buffers and the record buffer are slices of engine-owned allocations (kept)
  cudaStreamSynchronize(e->stream);
  // h_M and the device plan (replicate table, record offsets) belong to the engine (kept for the next batch)
  for (auto& g : b->slab_graph)
    if (g) cudaGraphExecDestroy(g);
  if (b->d_recs) cudaFree(b->d_recs);
  if (b->h_recs) cudaFreeHost(b->h_recs);
  if (b->d_reps) cudaFree(b->d_reps);
  if (b->h_reps) cudaFreeHost(b->h_reps);
  for (cudaEvent_t ev : b->slot_upload)
    if (ev) cudaEventDestroy(ev);
  delete b;
  e->batch = nullptr;
}

// Upper bound on a replicate's slots: the equilibrium count of its largest population plus one window
// of new mutations with 7-sigma margins (set_Index_Length's margin, go_fish_impl.cuh:235), with room
// to spare.  The neutral equilibrium count theta (ln Nc + 0.58) is scaled by how far the replicate's
// own mutation-selection-equilibrium start exceeds it at the initial size: positive selection raises
// the count (up to about twice the neutral one, the high-frequency classes filling up), by a factor
// that to first order does not depend on N, so a beneficial-allele replicate that grows keeps room for
// its larger equilibrium; negative selection only lowers it (factor 1).
static long long replicate_capacity(const gf_replicate& p, int M0) {
  auto neutral_eq = [&](int nc) {
    const double theta = 2.0 * p.mu * p.num_sites * nc;
    return theta * (std::log(std::max(nc, 2)) + 0.58);
  };
  int ncmax = 0;
  for (int g : {0, p.num_generations}) ncmax = std::max(ncmax, rep_nchrom(p, g));
  if (p.growth_rate != 0.f) ncmax = std::max(ncmax, static_cast<int>(2 * p.N_max / (1 + p.F)));
  const double eq0 = neutral_eq(rep_nchrom(p, 0));
  const double factor = eq0 > 0.0 ? std::max(1.0, M0 / eq0) : 1.0;
  const double eq = factor * neutral_eq(ncmax);
  const double lam = static_cast<double>(p.mu) * ncmax * p.num_sites;
  const double window = p.compact_interval * (lam + 7.0 * std::sqrt(lam + 1.0));
  const double want = std::max<double>(M0, 1.5 * eq + 10.0 * std::sqrt(eq + 1.0)) + 2.0 * window + 1024.0;
  return align_tiles(static_cast<long long>(want));
}

template <typename T>
static gf_status grow_pinned(Engine* e, T** d, T** h, size_t* cap, size_t need) {
  if (*cap >= need) return GF_OK;
  const size_t c = std::max<size_t>(need, 1024);
  if (*d) GF_CUDA(e, cudaFree(*d));
  if (*h) GF_CUDA(e, cudaFreeHost(*h));
  *d = nullptr;
  *h = nullptr;
  *cap = 0;
  GF_CUDA(e, cudaMalloc(d, sizeof(T) * c));
  GF_CUDA(e, cudaMallocHost(h, sizeof(T) * c));
  *cap = c;
  return GF_OK;
}

// Generation record of replicate `p` at generation g (what the reference's run_sim evaluates per
// generation: population size, Nchrom_e, the host-drawn new-mutation count, calc_new_mutations_Index
// go_fish_impl.cuh:454-467, and the model scalars).
static void make_record(const gf_replicate& p, int g, WinGen& w) {
  const int N = rep_population(p, g);
  const int Nc = static_cast<int>(2 * N / (1 + p.F));
  w.generation = g;
  w.Nc = Nc;
  w.new_count = (N > 0 && Nc > 0) ? host_new_mutation_count(p.seed1, p.seed2, p.mu, Nc, p.num_sites, g, 0) : 0;
  w.new_freq = Nc > 0 ? 1.f / Nc : 0.f;
  w.F = p.F;
  w.h = p.h;
  w.sel_a = p.sel_slope;
  w.sel_b = p.sel_intercept;
  w.alive = N > 0;
}

// Records depend only on each replicate's seeds and size trajectory, so host threads draw them ahead
// of the GPU into the engine's page-locked staging buffer and they are uploaded in bulk; super-steps
// then need neither host record work nor a count read-back.
//
// Slab j of replicate r is its generations (j * S_r, (j + 1) * S_r] with S_r = W * c_r: W windows
// of its cadence c_r, W chosen so that S is about kStreamSlab generations.  Every replicate advances
// one window per super-step, so all of them enter slab j at super-step j * W, and no window straddles
// two slabs.  Region j holds slab j of every replicate that runs that long; producers draw the
// slabs region-major, the order in which the super-steps need them, and a super-step uploads every
// completed region before its launches (waiting, bounded, only for a region it needs).  A batch within
// the engine's record budget keeps all regions resident, one after another; a larger one cycles
// through a ring of K equal slots (K regions fit the budget, at least two): region j goes into slot
// j % K once the super-steps that read region j - K are enqueued (the upload follows them in stream
// order), and its slabs are drawn once the upload of region j - K has read the staging slot.
constexpr int kStreamSlab = 512;

static void produce_records(Batch* b, WinGen* stage) {
  const long long R = b->R;
  const long long jobs = R * b->plan.nregions;
  for (;;) {
    if (b->cancel.load(std::memory_order_relaxed)) return;
    const long long i = b->next_job.fetch_add(1, std::memory_order_relaxed);
    if (i >= jobs) return;
    const int j = static_cast<int>(i / R), r = static_cast<int>(i % R);
    const int off = b->plan.region_off[static_cast<size_t>(r) * b->plan.nregions + j];
    if (off < 0) continue;
    while (j >= b->producible.load(std::memory_order_acquire)) {   // its staging slot is still being read
      if (b->cancel.load(std::memory_order_relaxed)) return;
      std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    const BatchRep& br = b->reps[r];
    const int g0 = j * br.chunk;
    const int g1 = std::min(br.p.num_generations, g0 + br.chunk);
    WinGen* out = stage + b->plan.slot_base(j) + off;
    for (int g = g0 + 1; g <= g1; ++g) make_record(br.p, g, out[g - g0 - 1]);
    b->region_done[j].fetch_add(1, std::memory_order_release);
  }
}

static gf_status precompute_records(Engine* e, Batch* b) {
  b->precomputed = false;
  long long total = 0;
  for (auto& br : b->reps) total += br.p.num_generations;
  if (e->batch_record_budget <= 0 || total == 0) return GF_OK;
  std::vector<gf_replicate> ps(b->R);
  for (int r = 0; r < b->R; ++r) ps[r] = b->reps[r].p;
  b->plan = plan_records(ps.data(), b->R, e->batch_record_budget, kStreamSlab);
  if (b->plan.region_base[b->plan.nregions] != total)
    return fail(e, GF_ERR_STATE, "record layout holds %lld of %lld records", b->plan.region_base[b->plan.nregions], total);
  for (int r = 0; r < b->R; ++r) b->reps[r].chunk = b->plan.chunk[r];
  const int nreg = b->plan.nregions;
  const long long slots = b->plan.slots;
  if (e->h_rec_stage_cap < static_cast<size_t>(slots)) {
    if (e->h_rec_stage) GF_CUDA(e, cudaFreeHost(e->h_rec_stage));
    e->h_rec_stage = nullptr;
    e->h_rec_stage_cap = 0;
    const size_t cap = static_cast<size_t>(slots) + static_cast<size_t>(slots) / 4;
    GF_CUDA(e, cudaMallocHost(&e->h_rec_stage, sizeof(WinGen) * cap));
    e->h_rec_stage_cap = cap;
  }
  gf_status st = grow_device(e, &e->batch_recs_mem, &e->batch_recs_bytes, sizeof(WinGen) * slots);
  if (st != GF_OK) return st;
  b->d_all_recs = static_cast<WinGen*>(e->batch_recs_mem);
  const int K = b->plan.ring_slots > 0 ? b->plan.ring_slots : nreg;
  b->slot_upload.assign(K, nullptr);
  for (int k = 0; k < K && b->plan.ring_slots > 0; ++k)
    GF_CUDA(e, cudaEventCreateWithFlags(&b->slot_upload[k], cudaEventDisableTiming));
  b->region_done.reset(new std::atomic<long long>[nreg]);
  for (int j = 0; j < nreg; ++j) b->region_done[j].store(0);
  b->next_job.store(0);
  b->cancel.store(false);
  b->uploaded = 0;
  b->upload_done = 0;
  b->producible.store(b->plan.ring_slots > 0 ? b->plan.ring_slots : nreg);
  // A producer draws ~25 M records/s; the super-steps, replayed a slab at a time, consume them faster
  // than six producers drew them at the start of a batch, and the thread that enqueues the super-steps
  // mostly waits on events, so the producers get all but two host threads (at most twelve).
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const long long want = std::max<long long>(1, total / 65536);
  const int workers = static_cast<int>(std::min<long long>(want, std::max(1u, std::min(hw > 2 ? hw - 2 : 1u, 12u))));
  WinGen* stage = e->h_rec_stage;
  try {
    for (int t = 0; t < workers; ++t) b->producers.emplace_back(produce_records, b, stage);
  } catch (const std::exception&) {
    if (b->producers.empty()) return fail(e, GF_ERR_STATE, "could not start a record producer thread");
  }
  b->precomputed = true;
  // lock-step bookkeeping: replicate r's last window is super-step ceil(G_r / c_r) - 1
  b->finish_at = plan_finish_steps(ps.data(), b->R);
  b->active_dirty = true;
  // the device side of the plan: the replicate table (static fields), each replicate's cadence,
  // generations and slab length, the region offsets and bases, and the super-step counter
  {
    const int R = b->R;
    auto sz = [](size_t bytes) { return (bytes + 255) / 256 * 256; };
    const size_t n_off = static_cast<size_t>(R) * nreg;
    const size_t need = sz(sizeof(WinRep) * R) + sz(sizeof(StepRep) * R) + sz(sizeof(int) * n_off) +
                        sz(sizeof(long long) * (nreg + 1)) + sz(sizeof(int)) + 2 * sz(sizeof(int) * R) + sz(sizeof(int));
    st = grow_device(e, &e->batch_plan_mem, &e->batch_plan_bytes, need);
    if (st != GF_OK) return st;
    char* cur = static_cast<char*>(e->batch_plan_mem);
    auto pa = [&](void** q, size_t bytes) {
      *q = cur;
      cur += sz(bytes);
    };
    pa(reinterpret_cast<void**>(&b->d_table), sizeof(WinRep) * R);
    pa(reinterpret_cast<void**>(&b->d_steprep), sizeof(StepRep) * R);
    pa(reinterpret_cast<void**>(&b->d_region_off), sizeof(int) * n_off);
    pa(reinterpret_cast<void**>(&b->d_region_base), sizeof(long long) * (nreg + 1));
    pa(reinterpret_cast<void**>(&b->d_step), sizeof(int));
    pa(reinterpret_cast<void**>(&b->d_list_rep), sizeof(int) * R);
    pa(reinterpret_cast<void**>(&b->d_list_tile0), sizeof(int) * R);
    pa(reinterpret_cast<void**>(&b->d_list_count), sizeof(int));
    std::vector<WinRep> table(R);
    std::vector<StepRep> steprep(R);
    b->all_tiles = 0;
    for (int r = 0; r < R; ++r) {
      const BatchRep& br = b->reps[r];
      WinRep& w = table[r];
      w = WinRep{};
      w.base = br.base;
      w.capacity = br.capacity;
      w.seed1 = br.p.seed1;
      w.seed2 = br.p.seed2;
      w.check_preserved = 0;
      w.compact = 0;
      w.preserve = 0;
      w.rep = r;
      steprep[r] = StepRep{std::max(br.p.compact_interval, 1), std::max(br.p.num_generations, 0), br.chunk, 0};
      b->all_tiles += br.capacity / kBatchTile;
    }
    // pageable sources: each copy returns once its source has been staged
    GF_CUDA(e, cudaMemcpyAsync(b->d_table, table.data(), sizeof(WinRep) * R, cudaMemcpyHostToDevice, e->stream));
    GF_CUDA(e, cudaMemcpyAsync(b->d_steprep, steprep.data(), sizeof(StepRep) * R, cudaMemcpyHostToDevice, e->stream));
    GF_CUDA(e, cudaMemcpyAsync(b->d_region_off, b->plan.region_off.data(), sizeof(int) * n_off, cudaMemcpyHostToDevice,
                               e->stream));
    GF_CUDA(e, cudaMemcpyAsync(b->d_region_base, b->plan.region_base.data(), sizeof(long long) * (nreg + 1),
                               cudaMemcpyHostToDevice, e->stream));
    GF_CUDA(e, cudaMemsetAsync(b->d_step, 0, sizeof(int), e->stream));
    b->step_plan = BatchStepPlan{b->plan.slab_windows, nreg, b->plan.ring_slots, 0, b->plan.slot_records};
  }
  GF_TRACE_POINT(e, "record producers started");
  return GF_OK;
}

// Upload the drawn regions a super-step in region `need` may see: every completed region up to
// need + K - 1 in order (K ring slots; all regions when resident), waiting for the producers only for
// regions up to `need`.  Finished uploads free their staging slots for the producers.  A wait that
// sees no progress for 120 s is reported as a state error.
static gf_status stream_upload(Engine* e, Batch* b, int need) {
  const int K = b->plan.ring_slots > 0 ? b->plan.ring_slots : b->plan.nregions;
  auto poll = [&]() {
    if (b->plan.ring_slots <= 0) return;
    while (b->upload_done < b->uploaded) {
      if (cudaEventQuery(b->slot_upload[b->upload_done % K]) != cudaSuccess) break;
      b->upload_done += 1;
    }
    b->producible.store(std::min(b->plan.nregions, b->upload_done + K), std::memory_order_release);
  };
  const auto t0 = std::chrono::steady_clock::now();
  auto progress = t0;
  auto wait0 = t0;
  bool waiting = false;
  long long last = -1;
  auto account = [&]() {
    if (waiting)
      b->record_wait_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wait0).count();
    waiting = false;
  };
  for (;;) {
    poll();
    const int j = b->uploaded;
    if (j >= b->plan.nregions || j >= need + K) break;
    const long long done = b->region_done[j].load(std::memory_order_acquire);
    if (done == b->plan.region_jobs[j]) {
      const long long a = b->plan.slot_base(j), n = b->plan.region_base[j + 1] - b->plan.region_base[j];
      if (n > 0)
        GF_CUDA(e, cudaMemcpyAsync(b->d_all_recs + a, e->h_rec_stage + a, sizeof(WinGen) * n, cudaMemcpyHostToDevice,
                                   e->stream));
      if (b->plan.ring_slots > 0) GF_CUDA(e, cudaEventRecord(b->slot_upload[j % K], e->stream));
      b->uploaded += 1;
      continue;
    }
    if (j > need) break;   // not needed by this super-step
    const auto now = std::chrono::steady_clock::now();
    if (!waiting) {
      waiting = true;
      wait0 = now;
    }
    if (done != last) {
      last = done;
      progress = now;
    } else if (now - progress > std::chrono::seconds(120)) {
      account();
      return fail(e, GF_ERR_STATE, "record producers made no progress on region %d for 120 s", j);
    }
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  account();
  return GF_OK;
}

static gf_status batch_begin(Engine* e, const gf_replicate* in, int R) {
  if (!in || R <= 0) return fail(e, GF_ERR_INVALID_ARGUMENT, "no replicates");
  for (int r = 0; r < R; ++r) {
    const gf_replicate& p = in[r];
    if (p.N0 < 1 || p.N_min < 1 || p.N_max < p.N_min || p.compact_interval < 1 || p.num_generations < 0 ||
        !(p.num_sites > 0) || p.mu < 0 || p.F < 0 || p.F > 1)
      return fail(e, GF_ERR_INVALID_ARGUMENT, "replicate %d: invalid parameters", r);
    if (p.num_generations > GF_MAX_GENERATION)
      return fail(e, GF_ERR_CAPACITY, "replicate %d: %d generations above %d", r, p.num_generations, GF_MAX_GENERATION);
  }
  GF_CUDA(e, cudaSetDevice(e->device));
  GF_CUDA(e, cudaStreamSynchronize(e->stream));
  GF_TRACE_POINT(e, "begin");
  release_batch(e);
  GF_TRACE_POINT(e, "release previous batch");
  Batch* b = new Batch();
  e->batch = b;
  b->R = R;
  b->reps.resize(R);
  // ---- MSE classes ----
  std::vector<MseRep> mr(R);
  long long area_total = 0, class_total = 0;
  for (int r = 0; r < R; ++r) {
    BatchRep& br = b->reps[r];
    br.p = in[r];
    const gf_replicate& p = in[r];
    MseRep& m = mr[r];
    m.N0 = rep_population(p, 0);
    m.Nc0 = static_cast<int>(2 * m.N0 / (1 + p.F));
    m.selected = (p.sel_slope != 0.f || p.sel_intercept != 0.f) ? 1 : 0;
    m.mu = p.mu;
    m.L = p.num_sites;
    m.F = p.F;
    m.h = p.h;
    m.sa = p.sel_slope;
    m.sb = p.sel_intercept;
    m.seed1 = p.seed1;
    m.seed2 = p.seed2;
    m.area_off = area_total;
    m.class_off = class_total;
    area_total += std::max(m.Nc0, 1);
    class_total += std::max(m.Nc0 - 1, 0);
  }
  MseRep* d_mr = nullptr;
  float *d_area = nullptr, *d_integral = nullptr;
  unsigned *d_counts = nullptr, *d_starts = nullptr;
  int* d_M0 = nullptr;
  {
    gf_status ast = pool_alloc(e, reinterpret_cast<void**>(&d_mr), sizeof(MseRep) * R);
    if (ast == GF_OK) ast = pool_alloc(e, reinterpret_cast<void**>(&d_area), sizeof(float) * area_total);
    if (ast == GF_OK) ast = pool_alloc(e, reinterpret_cast<void**>(&d_integral), sizeof(float) * area_total);
    if (ast == GF_OK)
      ast = pool_alloc(e, reinterpret_cast<void**>(&d_counts), sizeof(unsigned) * std::max<long long>(class_total, 1));
    if (ast == GF_OK)
      ast = pool_alloc(e, reinterpret_cast<void**>(&d_starts), sizeof(unsigned) * std::max<long long>(class_total, 1));
    if (ast == GF_OK) ast = pool_alloc(e, reinterpret_cast<void**>(&d_M0), sizeof(int) * R);
    if (ast != GF_OK) return ast;
  }
  GF_CUDA(e, cudaMemcpyAsync(d_mr, mr.data(), sizeof(MseRep) * R, cudaMemcpyHostToDevice, e->stream));
  const int grid = e->num_sms * 8;
  batch_mse_area_kernel<<<grid, 256, 0, e->stream>>>(d_area, d_mr, R, area_total);
  batch_mse_integral_kernel<<<R, 1024, 0, e->stream>>>(d_area, d_integral, d_mr);
  if (class_total > 0) batch_mse_count_kernel<<<grid, 256, 0, e->stream>>>(d_counts, d_integral, d_mr, R, class_total);
  batch_class_scan_kernel<<<R, 1024, 0, e->stream>>>(d_counts, d_starts, d_mr, d_M0);
  GF_CUDA(e, cudaGetLastError());
  e->kernel_launches += 4;
  std::vector<int> M0(R);
  GF_CUDA(e, cudaMemcpyAsync(M0.data(), d_M0, sizeof(int) * R, cudaMemcpyDeviceToHost, e->stream));
  GF_CUDA(e, cudaStreamSynchronize(e->stream));
  GF_TRACE_POINT(e, "MSE classes and counts");
  // ---- arena ----
  long long arena = 0;
  for (int r = 0; r < R; ++r) {
    BatchRep& br = b->reps[r];
    br.base = arena;
    br.capacity = replicate_capacity(br.p, M0[r]);
    br.M = M0[r];
    br.generation = 0;
    br.next_compact = br.p.compact_interval;
    br.done = br.p.num_generations == 0;
    arena += br.capacity;
  }
  b->arena = arena;
  {
    // slices of one engine-owned allocation, 256-byte aligned, laid out in a fixed order
    size_t need = 0;
    auto sz = [](size_t bytes) { return (bytes + 255) / 256 * 256; };
    need += 2 * (sz(sizeof(float) * arena) + 2 * sz(sizeof(int) * arena) + sz(sizeof(int) * R));
    need += sz(sizeof(unsigned) * (arena / 32)) + 2 * sz(sizeof(unsigned) * (arena / kBatchTile));
    need += sz(sizeof(int) * R) + sz(sizeof(int));
    gf_status ast = grow_device(e, &e->batch_arena_mem, &e->batch_arena_bytes, need);
    if (ast != GF_OK) return ast;
    char* cur = static_cast<char*>(e->batch_arena_mem);
    auto pa = [&](void** p, size_t bytes) {
      *p = cur;
      cur += sz(bytes);
    };
    for (int k = 0; k < 2; ++k) {
      pa(reinterpret_cast<void**>(&b->freq[k]), sizeof(float) * arena);
      pa(reinterpret_cast<void**>(&b->id_gp[k]), sizeof(int) * arena);
      pa(reinterpret_cast<void**>(&b->id_tid[k]), sizeof(int) * arena);
      pa(reinterpret_cast<void**>(&b->d_M[k]), sizeof(int) * R);
    }
    pa(reinterpret_cast<void**>(&b->flags), sizeof(unsigned) * (arena / 32));
    pa(reinterpret_cast<void**>(&b->tile_count), sizeof(unsigned) * (arena / kBatchTile));
    pa(reinterpret_cast<void**>(&b->tile_offset), sizeof(unsigned) * (arena / kBatchTile));
    pa(reinterpret_cast<void**>(&b->d_Mend), sizeof(int) * R);
    pa(reinterpret_cast<void**>(&b->d_total_tiles), sizeof(int));
  }
  if (e->batch_h_M_cap < static_cast<size_t>(2 * R)) {
    if (e->batch_h_M) GF_CUDA(e, cudaFreeHost(e->batch_h_M));
    e->batch_h_M = nullptr;
    e->batch_h_M_cap = 0;
    GF_CUDA(e, cudaMallocHost(&e->batch_h_M, sizeof(int) * 2 * R));
    e->batch_h_M_cap = 2 * R;
  }
  b->h_M = e->batch_h_M;
  for (cudaEvent_t& ev : e->batch_ahead)
    if (!ev) GF_CUDA(e, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  b->step_ev = e->batch_ahead;
  b->slab_ev = e->batch_ahead + 64;
  GF_CUDA(e, cudaMemsetAsync(b->freq[0], 0, sizeof(float) * arena, e->stream));
  GF_CUDA(e, cudaMemsetAsync(b->freq[1], 0, sizeof(float) * arena, e->stream));
  GF_CUDA(e, cudaMemcpyAsync(b->d_M[0], M0.data(), sizeof(int) * R, cudaMemcpyHostToDevice, e->stream));
  // ---- fill ----
  std::vector<FillRep> fr(R);
  long long fill_total = 0;
  for (int r = 0; r < R; ++r) {
    fr[r].slot_prefix = fill_total;
    fr[r].class_off = mr[r].class_off;
    fr[r].base = b->reps[r].base;
    fr[r].Nc0 = mr[r].Nc0;
    fr[r].M0 = M0[r];
    fill_total += M0[r];
  }
  FillRep* d_fr = nullptr;
  {
    gf_status ast = pool_alloc(e, reinterpret_cast<void**>(&d_fr), sizeof(FillRep) * R);
    if (ast != GF_OK) return ast;
  }
  GF_CUDA(e, cudaMemcpyAsync(d_fr, fr.data(), sizeof(FillRep) * R, cudaMemcpyHostToDevice, e->stream));
  if (fill_total > 0)
    batch_mse_fill_kernel<<<grid, 256, 0, e->stream>>>(b->freq[0], b->id_gp[0], b->id_tid[0], d_starts, d_fr, R,
                                                        fill_total);
  GF_CUDA(e, cudaGetLastError());
  e->kernel_launches += 1;
  for (void* q : {static_cast<void*>(d_mr), static_cast<void*>(d_area), static_cast<void*>(d_integral),
                  static_cast<void*>(d_counts), static_cast<void*>(d_starts), static_cast<void*>(d_M0),
                  static_cast<void*>(d_fr)})
    cudaFreeAsync(q, e->stream);
  GF_CUDA(e, cudaMemsetAsync(e->d_stats, 0, sizeof(unsigned long long) * 2, e->stream));
  GF_CUDA(e, cudaMemsetAsync(e->d_count + 2, 0, sizeof(int), e->stream));
  GF_TRACE_POINT(e, "arena and MSE fill");
  const gf_status pst = precompute_records(e, b);
  GF_TRACE_POINT(e, "records");
  return pst;
}

// New-mutation draws of the window records, spread over host threads for large batches.
static void fill_records(std::vector<WinGen>& recs, const std::vector<std::pair<int, int>>& jobs,
                         const std::vector<BatchRep>& reps, const std::vector<int>& first) {
  auto work = [&](size_t a, size_t z) {
    for (size_t j = a; j < z; ++j) {
      const int r = jobs[j].first;
      const int ngen = jobs[j].second;
      const gf_replicate& p = reps[r].p;
      for (int k = 0; k < ngen; ++k) {
        const int g = reps[r].generation + 1 + k;
        const int N = rep_population(p, g);
        const int Nc = static_cast<int>(2 * N / (1 + p.F));
        WinGen& w = recs[first[j] + k];
        w.generation = g;
        w.Nc = Nc;
        w.new_count = (N > 0 && Nc > 0) ? host_new_mutation_count(p.seed1, p.seed2, p.mu, Nc, p.num_sites, g, 0) : 0;
        w.new_freq = Nc > 0 ? 1.f / Nc : 0.f;
        w.F = p.F;
        w.h = p.h;
        w.sel_a = p.sel_slope;
        w.sel_b = p.sel_intercept;
        w.alive = N > 0;
      }
    }
  };
  size_t total = 0;
  for (auto& j : jobs) total += j.second;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const unsigned nt = total > 20000 ? std::min<unsigned>(hw, 16) : 1;
  if (nt <= 1) {
    work(0, jobs.size());
    return;
  }
  std::vector<std::thread> th;
  const size_t per = (jobs.size() + nt - 1) / nt;
  for (unsigned t = 0; t < nt; ++t) {
    const size_t a = t * per, z = std::min(jobs.size(), a + per);
    if (a < z) th.emplace_back(work, a, z);
  }
  for (auto& x : th) x.join();
}

static gf_status batch_super_step_fallback(Engine* e, int* active_out);

// Survivor counts of every replicate back to the host (one transfer of both count arrays), and the
// device status word.
static gf_status sync_counts(Engine* e) {
  Batch* b = e->batch;
  if (!b->counts_stale) return GF_OK;
  GF_CUDA(e, cudaMemcpyAsync(b->h_M, b->d_M[0], sizeof(int) * b->R, cudaMemcpyDeviceToHost, e->stream));
  GF_CUDA(e, cudaMemcpyAsync(b->h_M + b->R, b->d_M[1], sizeof(int) * b->R, cudaMemcpyDeviceToHost, e->stream));
  int fault = 0;
  GF_CUDA(e, cudaMemcpyAsync(&fault, e->d_count + 2, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  GF_CUDA(e, cudaStreamSynchronize(e->stream));
  for (int r = 0; r < b->R; ++r) b->reps[r].M = b->h_M[b->reps[r].m_slot * b->R + r];
  b->counts_stale = false;
  if (fault)
    return fail(e, GF_ERR_DEVICE, "device status word reports fault %d (%s)", fault,
                fault == kFaultCapacity  ? "replicate capacity exceeded"
                : fault == kFaultRecords ? "a replicate's window has no generation records"
                                         : "bounded wait expired");
  return GF_OK;
}

// Fields of unfinished replicates after k lock-step super-steps (finished ones are final already).
static void sync_progress(Batch* b) {
  if (!b->precomputed) return;
  const long long k = b->super_steps;
  for (int r : b->active) {
    BatchRep& br = b->reps[r];
    if (br.done) continue;
    br.generation = static_cast<int>(k * br.p.compact_interval);
    br.next_compact = br.generation + br.p.compact_interval;
    br.id_buf = b->id_cur;
    br.m_slot = b->mslot;
  }
}

static void refresh_active(Batch* b) {
  if (!b->active_dirty) return;
  b->active.clear();
  b->active_cadence_sum = 0;
  for (int r = 0; r < b->R; ++r) {
    const BatchRep& br = b->reps[r];
    if (br.done) continue;
    b->active.push_back(r);
    b->active_cadence_sum += br.p.compact_interval;
  }
  b->active_dirty = false;
}

// The launches of one super-step at the batch's current buffer parity (precomputed records): a
// one-block kernel derives each replicate's window (records, generations) from the device's super-step
// counter and assigns its tiles from its device-side count (finished replicates get none; tiles past a
// replicate's end-of-window count return at once), then the window kernel and its compaction.  No
// host record work, no upload and no read-back.
static gf_status enqueue_step(Engine* e, Batch* b) {
  batch_step_tiles(e, b->d_table, b->R, b->d_M[b->mslot], b->d_all_recs, b->d_total_tiles, b->d_step, b->step_plan,
                   b->d_region_off, b->d_region_base, b->d_steprep, e->d_count + 2, b->d_list_rep, b->d_list_tile0,
                   b->d_list_count);
  GF_CUDA(e, cudaGetLastError());
  WindowLaunch w;
  w.A = b->freq[0];
  w.B = b->freq[1];
  w.id_gp_cur = b->id_gp[b->id_cur];
  w.id_tid_cur = b->id_tid[b->id_cur];
  w.id_gp_next = b->id_gp[b->id_cur ^ 1];
  w.id_tid_next = b->id_tid[b->id_cur ^ 1];
  w.flags = b->flags;
  w.tile_count = b->tile_count;
  w.tile_offset = b->tile_offset;
  w.M_in = b->d_M[b->mslot];
  w.M_end = b->d_Mend;
  w.M_next = nullptr;
  w.M_out = b->d_M[b->mslot ^ 1];
  w.reps = b->d_table;
  w.nreps = b->R;
  w.recs = b->d_all_recs;
  w.total_tiles = static_cast<int>(std::min<long long>(b->all_tiles, INT32_MAX));   // sizes the grids
  w.total_tiles_dev = b->d_total_tiles;
  w.any_compact = true;
  w.stats = e->d_stats;
  w.fault = e->d_count + 2;
  w.sched = e->d_count + kSchedWord;
  w.list.rep = b->d_list_rep;
  w.list.tile0 = b->d_list_tile0;
  w.list.count = b->d_list_count;
  return window_run(e, w, b->freq[0]);
}
constexpr int kLaunchesPerStep = 4;   // step kernel, window, segmented scan, scatter

// Host bookkeeping of the super-step just enqueued: buffer parity, generations, finished replicates.
// Returns how many replicates finished with it.
static int account_step(Batch* b) {
  refresh_active(b);
  const long long k = b->super_steps;
  b->mslot ^= 1;
  b->id_cur ^= 1;
  b->super_steps += 1;
  b->counts_stale = true;
  // generations of this step: every active replicate's cadence, less what the finishing ones lack
  long long gens = b->active_cadence_sum;
  int finishing = 0;
  if (k < static_cast<long long>(b->finish_at.size())) {
    for (int r : b->finish_at[k]) {
      BatchRep& br = b->reps[r];
      const long long gen = k * br.p.compact_interval;
      gens -= br.p.compact_interval - (br.p.num_generations - gen);
      br.generation = br.p.num_generations;
      br.next_compact = br.generation + br.p.compact_interval;
      br.id_buf = b->id_cur;
      br.m_slot = b->mslot;
      br.done = true;
      ++finishing;
    }
    if (finishing) b->active_dirty = true;
  }
  b->generations += gens;
  return finishing;
}

static gf_status batch_super_step(Engine* e, int* active_out) {
  Batch* b = e->batch;
  if (!b->precomputed) return batch_super_step_fallback(e, active_out);
  refresh_active(b);
  const int nj = static_cast<int>(b->active.size());
  if (nj == 0) {
    if (active_out) *active_out = 0;
    return GF_OK;
  }
  const long long k = b->super_steps;
  const int j = static_cast<int>(k / b->plan.slab_windows);   // the record region of every active replicate
  if (j >= b->plan.nregions) return fail(e, GF_ERR_STATE, "super-step %lld beyond the record regions", k);
  {
    gf_status ust = stream_upload(e, b, j);   // the records of this super-step, in stream order
    if (ust != GF_OK) return ust;
  }
  cudaEvent_t& ahead = b->step_ev[b->steps_enqueued % 64];
  GF_CUDA(e, cudaEventSynchronize(ahead));   // the step enqueued 64 steps ago has run
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (e->profiling) {
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    GF_CUDA(e, cudaEventRecord(ev0, e->stream));
  }
  gf_status st = enqueue_step(e, b);
  if (st != GF_OK) return st;
  if (e->profiling) {
    GF_CUDA(e, cudaEventRecord(ev1, e->stream));
    e->prof_drift.emplace_back(ev0, ev1);
  }
  GF_CUDA(e, cudaEventRecord(ahead, e->stream));
  b->steps_enqueued += 1;
  const int finishing = account_step(b);
  if (active_out) *active_out = nj - finishing;
  return GF_OK;
}

// The super-steps of one record slab (slab_windows of them, all in record region j) replayed as one
// CUDA graph: the steps read their window from the device's super-step counter, so the same launches
// serve every slab that starts at the same buffer parity (one graph per parity, captured on first use
// and again after the draw tuning changes).  Taken only at a slab's first step, after the first slab
// (which runs step by step, so launch set-up never happens inside a capture), when the whole slab
// lies before the batch's last super-step, and never while profiling; `*ran` says whether it ran.
static gf_status batch_slab(Engine* e, int* active_out, bool* ran) {
  *ran = false;
  Batch* b = e->batch;
  if (!b->precomputed || e->profiling || !e->stream || b->graphs_off) return GF_OK;
  refresh_active(b);
  const long long k = b->super_steps;
  const int W = b->plan.slab_windows;
  if (b->active.empty() || k == 0 || k % W != 0 || k + W > static_cast<long long>(b->finish_at.size())) return GF_OK;
  const int j = static_cast<int>(k / W);
  if (j >= b->plan.nregions) return GF_OK;
  {
    gf_status ust = stream_upload(e, b, j);
    if (ust != GF_OK) return ust;
  }
  const int parity = b->mslot;
  if (b->slab_graph[parity] &&
      (b->graph_draw[parity] != e->draw_strategy || b->graph_blocks[parity] != e->blocks_per_sm)) {
    cudaGraphExecDestroy(b->slab_graph[parity]);
    b->slab_graph[parity] = nullptr;
  }
  if (!b->slab_graph[parity]) {
    const long long launches0 = e->kernel_launches;
    const int m0 = b->mslot, i0 = b->id_cur;
    if (cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();   // a stream that cannot be captured: the batch runs step by step
      b->graphs_off = true;
      return GF_OK;
    }
    gf_status st = GF_OK;
    for (int i = 0; i < W && st == GF_OK; ++i) {
      st = enqueue_step(e, b);
      b->mslot ^= 1;
      b->id_cur ^= 1;
    }
    b->mslot = m0;
    b->id_cur = i0;
    e->kernel_launches = launches0;
    cudaGraph_t graph = nullptr;
    const cudaError_t cerr = cudaStreamEndCapture(e->stream, &graph);
    if (st != GF_OK) {
      if (graph) cudaGraphDestroy(graph);
      return st;
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ierr = cerr == cudaSuccess ? cudaGraphInstantiate(&exec, graph, 0) : cerr;
    if (graph) cudaGraphDestroy(graph);
    if (ierr != cudaSuccess) {   // nothing captured ran: the batch continues step by step
      cudaGetLastError();
      b->graphs_off = true;
      return GF_OK;
    }
    b->slab_graph[parity] = exec;
    b->graph_draw[parity] = e->draw_strategy;
    b->graph_blocks[parity] = e->blocks_per_sm;
  }
  cudaEvent_t& ahead = b->slab_ev[b->slabs_enqueued % 2];
  GF_CUDA(e, cudaEventSynchronize(ahead));   // the slab enqueued two slabs ago has run
  GF_CUDA(e, cudaGraphLaunch(b->slab_graph[parity], e->stream));
  GF_CUDA(e, cudaEventRecord(ahead, e->stream));
  b->slabs_enqueued += 1;
  e->kernel_launches += static_cast<long long>(kLaunchesPerStep) * W;
  for (int i = 0; i < W; ++i) account_step(b);
  refresh_active(b);
  if (active_out) *active_out = static_cast<int>(b->active.size());
  *ran = true;
  return GF_OK;
}

// Super-step for batches whose records do not fit the precomputation budget: records built per
// super-step and the counts read back every time.
static gf_status batch_super_step_fallback(Engine* e, int* active_out) {
  Batch* b = e->batch;
  std::vector<std::pair<int, int>> jobs;
  std::vector<int> first;
  int nrec = 0;
  for (int r = 0; r < b->R; ++r) {
    BatchRep& br = b->reps[r];
    if (br.done) continue;
    const int end = std::min(br.next_compact, br.p.num_generations);
    const int ngen = end - br.generation;
    jobs.emplace_back(r, ngen);
    first.push_back(nrec);
    nrec += ngen;
  }
  if (jobs.empty()) {
    if (active_out) *active_out = 0;
    return GF_OK;
  }
  std::vector<WinGen> recs(nrec);
  fill_records(recs, jobs, b->reps, first);
  gf_status st = grow_pinned(e, &b->d_recs, &b->h_recs, &b->recs_cap, nrec);
  if (st != GF_OK) return st;
  st = grow_pinned(e, &b->d_reps, &b->h_reps, &b->reps_cap, jobs.size());
  if (st != GF_OK) return st;
  std::memcpy(b->h_recs, recs.data(), sizeof(WinGen) * nrec);
  int tiles = 0;
  for (size_t j = 0; j < jobs.size(); ++j) {
    const int r = jobs[j].first;
    BatchRep& br = b->reps[r];
    long long news = 0;
    for (int k = 0; k < jobs[j].second; ++k) news += recs[first[j] + k].new_count;
    const long long need = br.M + news;
    if (need > br.capacity)
      return fail(e, GF_ERR_CAPACITY, "replicate %d needs %lld slots at generation %d, its segment holds %lld", r,
                  need, br.generation, br.capacity);
    WinRep& w = b->h_reps[j];
    w.base = br.base;
    w.capacity = br.capacity;
    w.rec = first[j];
    w.ngen = jobs[j].second;
    w.tile0 = tiles;
    w.ntiles = static_cast<int>(align_tiles(std::max<long long>(need, 1)) / kBatchTile);
    w.seed1 = br.p.seed1;
    w.seed2 = br.p.seed2;
    w.check_preserved = 0;
    w.compact = 1;
    w.preserve = 0;
    w.rep = r;
    w.births = news;
    tiles += w.ntiles;
  }
  GF_CUDA(e, cudaMemcpyAsync(b->d_recs, b->h_recs, sizeof(WinGen) * nrec, cudaMemcpyHostToDevice, e->stream));
  GF_CUDA(e, cudaMemcpyAsync(b->d_reps, b->h_reps, sizeof(WinRep) * jobs.size(), cudaMemcpyHostToDevice, e->stream));
  WindowLaunch w;
  w.A = b->freq[0];
  w.B = b->freq[1];
  w.id_gp_cur = b->id_gp[b->id_cur];
  w.id_tid_cur = b->id_tid[b->id_cur];
  w.id_gp_next = b->id_gp[b->id_cur ^ 1];
  w.id_tid_next = b->id_tid[b->id_cur ^ 1];
  w.flags = b->flags;
  w.tile_count = b->tile_count;
  w.tile_offset = b->tile_offset;
  w.M_in = b->d_M[b->mslot];
  w.M_end = b->d_Mend;
  w.M_next = nullptr;
  w.M_out = b->d_M[b->mslot ^ 1];
  w.reps = b->d_reps;
  w.nreps = static_cast<int>(jobs.size());
  w.recs = b->d_recs;
  w.total_tiles = tiles;
  w.any_compact = true;
  w.stats = e->d_stats;
  w.fault = e->d_count + 2;
  w.sched = e->d_count + kSchedWord;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (e->profiling) {
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    GF_CUDA(e, cudaEventRecord(ev0, e->stream));
  }
  st = window_run(e, w, b->freq[0]);
  if (st != GF_OK) return st;
  if (e->profiling) {
    GF_CUDA(e, cudaEventRecord(ev1, e->stream));
    e->prof_drift.emplace_back(ev0, ev1);
  }
  b->mslot ^= 1;
  b->id_cur ^= 1;
  b->super_steps += 1;
  // survivor counts of every replicate (one small read-back per super-step)
  GF_CUDA(e, cudaMemcpyAsync(b->h_M, b->d_M[b->mslot], sizeof(int) * b->R, cudaMemcpyDeviceToHost, e->stream));
  int fault = 0;
  GF_CUDA(e, cudaMemcpyAsync(&fault, e->d_count + 2, sizeof(int), cudaMemcpyDeviceToHost, e->stream));
  GF_CUDA(e, cudaStreamSynchronize(e->stream));
  if (fault) return fail(e, GF_ERR_DEVICE, "device status word reports fault %d", fault);
  int active = 0;
  for (size_t j = 0; j < jobs.size(); ++j) {
    BatchRep& br = b->reps[jobs[j].first];
    br.M = b->h_M[jobs[j].first];
    br.generation += jobs[j].second;
    b->generations += jobs[j].second;
    br.next_compact = br.generation + br.p.compact_interval;
    br.id_buf = b->id_cur;
    br.m_slot = b->mslot;
    if (br.generation >= br.p.num_generations) br.done = true;
    else ++active;
  }
  if (active_out) *active_out = active;
  return GF_OK;
}

}  // namespace gf

using namespace gf;

extern "C" {

int32_t gf_replicate_population(const gf_replicate* rep, int32_t generation) {
  return rep ? rep_population(*rep, generation) : 0;
}

void gf_replicate_population_table(const gf_replicate* rep, int32_t first, int32_t count, int32_t* out) {
  if (!rep || !out) return;
  for (int32_t k = 0; k < count; ++k) out[k] = rep_population(*rep, first + k);
}

gf_status gf_batch_begin(gf_engine* g, const gf_replicate* reps, int32_t R) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    return batch_begin(&g->impl, reps, R);
  });
}

gf_status gf_batch_set_record_budget(gf_engine* g, int64_t records) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    if (records < 0) return fail(&g->impl, GF_ERR_INVALID_ARGUMENT, "negative record budget");
    g->impl.batch_record_budget = records;
    return GF_OK;
  });
}

gf_status gf_batch_run(gf_engine* g, int32_t max_super_steps, int32_t* out_active) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (!e->batch) return fail(e, GF_ERR_STATE, "gf_batch_run before gf_batch_begin");
    GF_CUDA(e, cudaSetDevice(e->device));
    int active = 1;
    const int W = e->batch->precomputed ? e->batch->plan.slab_windows : 1;
    for (int s = 0; (max_super_steps <= 0 || s < max_super_steps) && active > 0;) {
      if (max_super_steps <= 0 || max_super_steps - s >= W) {
        bool ran = false;
        gf_status st = batch_slab(e, &active, &ran);   // a whole record slab as one graph, where it may
        if (st != GF_OK) {
          sync_progress(e->batch);
          return st;
        }
        if (ran) {
          s += W;
          continue;
        }
      }
      gf_status st = batch_super_step(e, &active);
      if (st != GF_OK) {
        sync_progress(e->batch);
        return st;
      }
      ++s;
    }
    sync_progress(e->batch);
    gf_status st = sync_counts(e);
    if (st != GF_OK) return st;
    if (out_active) {
      int a = 0;
      for (auto& br : e->batch->reps) a += br.done ? 0 : 1;
      *out_active = a;
    }
    return GF_OK;
  });
}

gf_status gf_batch_read_state(gf_engine* g, int32_t r, float* freq_out, int32_t* ids_out, int32_t max_mutations,
                              int32_t* out_num, int32_t* out_generation) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    Batch* b = e->batch;
    if (!b) return fail(e, GF_ERR_STATE, "no batch");
    if (r < 0 || r >= b->R) return fail(e, GF_ERR_INVALID_ARGUMENT, "replicate %d outside [0, %d)", r, b->R);
    GF_CUDA(e, cudaSetDevice(e->device));
    {
      gf_status st = sync_counts(e);
      if (st != GF_OK) return st;
    }
    GF_CUDA(e, cudaStreamSynchronize(e->stream));
    const BatchRep& br = b->reps[r];
    if (out_num) *out_num = br.M;
    if (out_generation) *out_generation = br.generation;
    if (br.M > max_mutations) return fail(e, GF_ERR_CAPACITY, "replicate %d holds %d mutations", r, br.M);
    if (br.M == 0) return GF_OK;
    if (freq_out)
      GF_CUDA(e, cudaMemcpy(freq_out, b->freq[0] + br.base, sizeof(float) * br.M, cudaMemcpyDeviceToHost));
    if (ids_out) {
      std::vector<int> gp(br.M), tid(br.M);
      GF_CUDA(e, cudaMemcpy(gp.data(), b->id_gp[br.id_buf] + br.base, sizeof(int) * br.M, cudaMemcpyDeviceToHost));
      GF_CUDA(e, cudaMemcpy(tid.data(), b->id_tid[br.id_buf] + br.base, sizeof(int) * br.M, cudaMemcpyDeviceToHost));
      for (int i = 0; i < br.M; ++i) {
        ids_out[4 * i + 0] = gp[i] & 0xFFFFFF;
        ids_out[4 * i + 1] = gp[i] >> 24;
        ids_out[4 * i + 2] = tid[i];
        ids_out[4 * i + 3] = 0;
      }
    }
    return GF_OK;
  });
}

gf_status gf_batch_sfs(gf_engine* g, int32_t n, float* out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g || !out) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    Batch* b = e->batch;
    if (!b) return fail(e, GF_ERR_STATE, "no batch");
    if (n < 1 || n + 1 > 8 * kBatchSfsThreads) return fail(e, GF_ERR_CAPACITY, "sample size %d outside [1, %d)", n, 8 * kBatchSfsThreads);
    for (int r = 0; r < b->R; ++r) {
      const int Nc = rep_nchrom(b->reps[r].p, b->reps[r].generation);   // Nchrom_e at its current generation
      if (n >= Nc) return fail(e, GF_ERR_INVALID_ARGUMENT, "replicate %d: sample size %d >= Nchrom_e %d", r, n, Nc);
    }
    GF_CUDA(e, cudaSetDevice(e->device));
    {
      gf_status st = sync_counts(e);
      if (st != GF_OK) return st;
    }
    std::vector<SfsRep> sr(b->R);
    for (int r = 0; r < b->R; ++r) sr[r] = {b->reps[r].base, b->reps[r].M, b->reps[r].p.num_sites};
    std::vector<double> lgc(n + 1);
    const double ln = std::lgamma(n + 1.0);
    for (int k = 0; k <= n; ++k) lgc[k] = ln - std::lgamma(k + 1.0) - std::lgamma(n - k + 1.0);
    SfsRep* d_sr = nullptr;
    double* d_lgc = nullptr;
    float* d_out = nullptr;
    {
      gf_status ast = pool_alloc(e, reinterpret_cast<void**>(&d_sr), sizeof(SfsRep) * b->R);
      if (ast == GF_OK) ast = pool_alloc(e, reinterpret_cast<void**>(&d_lgc), sizeof(double) * (n + 1));
      if (ast == GF_OK) ast = pool_alloc(e, reinterpret_cast<void**>(&d_out), sizeof(float) * b->R * n);
      if (ast != GF_OK) return ast;
    }
    GF_CUDA(e, cudaMemcpyAsync(d_sr, sr.data(), sizeof(SfsRep) * b->R, cudaMemcpyHostToDevice, e->stream));
    GF_CUDA(e, cudaMemcpyAsync(d_lgc, lgc.data(), sizeof(double) * (n + 1), cudaMemcpyHostToDevice, e->stream));
    batch_sfs_kernel<<<b->R, kBatchSfsThreads, 0, e->stream>>>(b->freq[0], d_sr, n, d_lgc, d_out);
    GF_CUDA(e, cudaGetLastError());
    e->kernel_launches += 1;
    GF_CUDA(e, cudaMemcpyAsync(out, d_out, sizeof(float) * b->R * n, cudaMemcpyDeviceToHost, e->stream));
    cudaFreeAsync(d_sr, e->stream);
    cudaFreeAsync(d_lgc, e->stream);
    cudaFreeAsync(d_out, e->stream);
    GF_CUDA(e, cudaStreamSynchronize(e->stream));
    return GF_OK;
  });
}

gf_status gf_batch_stats_read(gf_engine* g, gf_batch_stats* out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g || !out) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    Batch* b = e->batch;
    if (!b) return fail(e, GF_ERR_STATE, "no batch");
    GF_CUDA(e, cudaSetDevice(e->device));
    unsigned long long st[2] = {0, 0};
    GF_CUDA(e, cudaMemcpyAsync(st, e->d_stats, sizeof(st), cudaMemcpyDeviceToHost, e->stream));
    GF_CUDA(e, cudaStreamSynchronize(e->stream));
    out->mutation_generations = static_cast<double>(st[0]);
    out->generations = b->generations;
    out->super_steps = b->super_steps;
    out->replicates = b->R;
    int a = 0;
    for (auto& br : b->reps) a += br.done ? 0 : 1;
    out->active = a;
    out->record_wait_ms = b->record_wait_ms;
    out->record_producers = static_cast<int32_t>(b->producers.size());
    out->reserved = 0;
    out->arena_slots = b->arena;
    return GF_OK;
  });
}

}  // extern "C"
