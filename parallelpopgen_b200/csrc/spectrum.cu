// Spectrum: population frequency histogram and binomially projected site frequency spectrum
// (Spectrum::population_frequency_histogram / site_frequency_spectrum, spectrum.cu:74-294 of the
// reference).
//
// Both start from one integer histogram of allele counts j = round(Nc * p) over j in [0, Nc]
// (population_hist, spectrum.cu:74-83), built with a block-private shared-memory histogram for the
// low-count bins -- where a neutral SFS puts most of its mass -- and global atomics above them.
//
// The SFS then projects the histogram instead of every mutation: sum_i f(p_i) = sum_j c_j f(p_j),
// O(n * Nc) terms instead of the reference's O(n * M) (binom<1024>, spectrum.cu:111-139).  This is
// exact because engine frequencies are float(j) / Nc: the histogram kernel recomputes p_j with the
// same division and flags any mutation whose frequency differs from its class value, in which case
// the direct per-mutation projection runs instead.  Terms are evaluated in double precision from an
// exact log-binomial table and reduced in a fixed order, so the result is deterministic (the
// reference's float atomics are not, spectrum.cu:271-272).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "gf_internal.h"

namespace gf {

constexpr int kHistThreads = 512;
constexpr int kSmemBins = 40960;  // 160 KB of shared counters per block

// counts[j] for j in [0, Nc]; mismatch[0] != 0 if some frequency is not float(j) / Nc.
__global__ void __launch_bounds__(kHistThreads)
    hist_kernel(const float* __restrict__ freq, int M, int Nc, unsigned* __restrict__ counts,
                unsigned* __restrict__ mismatch, int smem_bins) {
  extern __shared__ unsigned s_bins[];
  for (int b = threadIdx.x; b < smem_bins; b += blockDim.x) s_bins[b] = 0;
  __syncthreads();
  unsigned bad = 0;
  const float Nf = static_cast<float>(Nc);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += blockDim.x * gridDim.x) {
    const float p = freq[i];
    int j = static_cast<int>(round(Nc * p));
    if (j < 0) j = 0;
    if (j > Nc) j = Nc;
    if (static_cast<float>(j) / Nf != p) bad = 1;
    if (j < smem_bins) {
      // warp-aggregated: one shared atomic per distinct bin in the warp
      const unsigned active = __activemask();
      const unsigned peers = __match_any_sync(active, j);
      const int leader = __ffs(peers) - 1;
      if ((threadIdx.x & 31) == leader) atomicAdd(&s_bins[j], __popc(peers));
    } else {
      atomicAdd(&counts[j], 1u);
    }
  }
  if (bad) atomicOr(mismatch, 1u);
  __syncthreads();
  for (int b = threadIdx.x; b < smem_bins; b += blockDim.x) {
    const unsigned v = s_bins[b];
    if (v) atomicAdd(&counts[b], v);
  }
}

// population_frequency_histogram output: out[k] = count of k (k in [1, Nc)), out[0] = count of 0,
// of Nc (fixed folds into 0) and of the (num_sites - M) monomorphic sites, in uint32 arithmetic as
// the reference accumulates it (spectrum.cu:78-82).
__global__ void hist_to_float_kernel(const unsigned* __restrict__ counts, int Nc, unsigned extra0, float* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < Nc; k += blockDim.x * gridDim.x) {
    unsigned v = counts[k];
    if (k == 0) v = v + counts[Nc] + extra0;
    out[k] = static_cast<float>(v);
  }
}

constexpr int kProjThreads = 256;
constexpr int kProjChunk = 256;

// Per-class binomial terms c * C(n, k) p^k q^(n-k): a thread owns kper consecutive levels
// [k0, k0 + kper); it evaluates the first in log space (one exp) and steps to the next with the pmf
// ratio (n - k) / (k + 1) * p / q, so a class costs one exp per thread instead of one per level.
// The recurrence adds ~1e-16 relative error per step (at most 7 steps); a first term that underflows
// only drops terms below 1e-300.
__device__ __forceinline__ void add_class_terms(double (&acc)[8], int k0, int kper, int levels, double c,
                                                double lp, double lq, double pq, int n, double lg0,
                                                const double (&ratio)[8]) {
  if (k0 >= levels) return;
  double t = c * exp(lg0 + k0 * lp + (n - k0) * lq);
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    if (u >= kper) break;
    if (k0 + u >= levels) break;
    if (u > 0) t *= ratio[u - 1] * pq;
    acc[u] += t;
  }
}

// The per-thread constants of add_class_terms: log C(n, k0) and (n - k) / (k + 1) for its levels.
__device__ __forceinline__ void thread_level_constants(const double* __restrict__ lgc, int n, int k0, int kper,
                                                       double& lg0, double (&ratio)[8]) {
  const int levels = n + 1;
  lg0 = k0 < levels ? lgc[k0] : 0.0;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int k = k0 + u;
    ratio[u] = (u < kper && k < n) ? static_cast<double>(n - k) / static_cast<double>(k + 1) : 0.0;
  }
}

// Partial projections: block b covers classes [j0, j1) and writes partial[b][k] for k in [0, n].
__global__ void __launch_bounds__(kProjThreads)
    project_hist_kernel(const unsigned* __restrict__ counts, int Nc, int n, const double* __restrict__ lgc,
                        double* __restrict__ partial, int classes_per_block) {
  __shared__ double s_lp[kProjChunk];
  __shared__ double s_lq[kProjChunk];
  __shared__ double s_pq[kProjChunk];
  __shared__ double s_c[kProjChunk];
  __shared__ int s_any;
  const int j0 = blockIdx.x * classes_per_block;
  const int j1 = min(Nc + 1, j0 + classes_per_block);
  const float Nf = static_cast<float>(Nc);
  const int levels = n + 1;
  const int kper = (levels + kProjThreads - 1) / kProjThreads;  // consecutive levels per thread
  const int k0 = threadIdx.x * kper;
  double lg0, ratio[8];
  thread_level_constants(lgc, n, k0, kper, lg0, ratio);
  double acc[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) acc[u] = 0.0;
  for (int c0 = j0; c0 < j1; c0 += kProjChunk) {
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    for (int t = threadIdx.x; t < kProjChunk; t += blockDim.x) {
      const int j = c0 + t;
      double c = 0.0, lp = 0.0, lq = 0.0, pq = 0.0;
      if (j < j1) {
        const float p = static_cast<float>(j) / Nf;
        const unsigned cnt = counts[j];
        if (cnt && p > 0.f && p < 1.f) {
          const double pd = static_cast<double>(p);
          c = static_cast<double>(cnt);
          lp = log(pd);
          lq = log1p(-pd);
          pq = pd / (1.0 - pd);
          s_any = 1;
        }
      }
      s_c[t] = c;
      s_lp[t] = lp;
      s_lq[t] = lq;
      s_pq[t] = pq;
    }
    __syncthreads();
    if (s_any) {
      const int cend = min(kProjChunk, j1 - c0);
      for (int t = 0; t < cend; ++t) {
        const double c = s_c[t];
        if (c == 0.0) continue;
        add_class_terms(acc, k0, kper, levels, c, s_lp[t], s_lq[t], s_pq[t], n, lg0, ratio);
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    if (u >= kper) break;
    const int k = k0 + u;
    if (k < levels) partial[static_cast<long long>(blockIdx.x) * levels + k] = acc[u];
  }
}

// Direct projection of every mutation (used when frequencies are not on the 1/Nc grid).
__global__ void __launch_bounds__(kProjThreads)
    project_direct_kernel(const float* __restrict__ freq, int M, int n, const double* __restrict__ lgc,
                          double* __restrict__ partial, int per_block, unsigned* __restrict__ nonseg) {
  __shared__ double s_lp[kProjChunk];
  __shared__ double s_lq[kProjChunk];
  __shared__ double s_pq[kProjChunk];
  __shared__ double s_c[kProjChunk];
  const int i0 = blockIdx.x * per_block;
  const int i1 = min(M, i0 + per_block);
  const int levels = n + 1;
  const int kper = (levels + kProjThreads - 1) / kProjThreads;
  const int k0 = threadIdx.x * kper;
  double lg0, ratio[8];
  thread_level_constants(lgc, n, k0, kper, lg0, ratio);
  double acc[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) acc[u] = 0.0;
  unsigned ns = 0;
  for (int c0 = i0; c0 < i1; c0 += kProjChunk) {
    for (int t = threadIdx.x; t < kProjChunk; t += blockDim.x) {
      const int i = c0 + t;
      double c = 0.0, lp = 0.0, lq = 0.0, pq = 0.0;
      if (i < i1) {
        const float p = freq[i];
        if (p > 0.f && p < 1.f) {
          const double pd = static_cast<double>(p);
          c = 1.0;
          lp = log(pd);
          lq = log1p(-pd);
          pq = pd / (1.0 - pd);
        } else {
          ++ns;
        }
      }
      s_c[t] = c;
      s_lp[t] = lp;
      s_lq[t] = lq;
      s_pq[t] = pq;
    }
    __syncthreads();
    const int cend = min(kProjChunk, i1 - c0);
    for (int t = 0; t < cend; ++t) {
      if (s_c[t] == 0.0) continue;
      add_class_terms(acc, k0, kper, levels, s_c[t], s_lp[t], s_lq[t], s_pq[t], n, lg0, ratio);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    if (u >= kper) break;
    const int k = k0 + u;
    if (k < levels) partial[static_cast<long long>(blockIdx.x) * levels + k] = acc[u];
  }
  if (ns) atomicAdd(nonseg, ns);
}

// Fixed-order reduction of the partials into float bins; k == n and every non-segregating mutation
// fold into bin 0, plus the (num_sites - M) monomorphic sites (spectrum.cu:130-138).  A block takes
// 32 levels (one per lane); its 8 warps sum fixed, contiguous eighths of the partial blocks and the
// eight sums are added in warp order, so the result does not depend on scheduling.
constexpr int kFinishWarps = 8;

__global__ void __launch_bounds__(32 * kFinishWarps)
    sfs_finish_kernel(const double* __restrict__ partial, int nblocks, int n, double extra0,
                      const unsigned* __restrict__ nonseg_count, float* __restrict__ out) {
  __shared__ double s_sum[kFinishWarps][33];   // column 32: the top level k == n (block 0 only)
  const int levels = n + 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int k = blockIdx.x * 32 + lane;
  const int per = (nblocks + kFinishWarps - 1) / kFinishWarps;
  const int b0 = warp * per, b1 = min(nblocks, b0 + per);
  double s = 0.0;
  if (k < n)
    for (int b = b0; b < b1; ++b) s += partial[static_cast<long long>(b) * levels + k];
  s_sum[warp][lane] = s;
  if (blockIdx.x == 0 && lane == 0) {
    double top = 0.0;
    for (int b = b0; b < b1; ++b) top += partial[static_cast<long long>(b) * levels + n];
    s_sum[warp][32] = top;
  }
  __syncthreads();
  if (warp == 0 && k < n) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kFinishWarps; ++w) t += s_sum[w][lane];
    if (k == 0) {
      double top = 0.0;
#pragma unroll
      for (int w = 0; w < kFinishWarps; ++w) top += s_sum[w][32];
      t += top + extra0 + static_cast<double>(*nonseg_count);
    }
    out[k] = static_cast<float>(t);
  }
}

// Non-segregating count from the histogram: classes whose p_j is not in (0, 1) -- only j == 0 and
// j == Nc can be (tested with the same division as the projection).
__global__ void nonseg_from_hist_kernel(const unsigned* __restrict__ counts, int Nc, unsigned* __restrict__ out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const float Nf = static_cast<float>(Nc);
  unsigned total = 0;
  for (int j : {0, Nc}) {
    if (j == Nc && Nc == 0) break;   // one class only
    const float p = static_cast<float>(j) / Nf;
    if (!(p > 0.f && p < 1.f)) total += counts[j];
  }
  *out = total;
}

// ------------------------------------------------------------------------------------------------
// host drivers
// ------------------------------------------------------------------------------------------------
struct SpecLayout {
  size_t counts_off, mismatch_off, nonseg_off, lgc_off, partial_off, total;
};

static size_t al256(size_t v) { return (v + 255) / 256 * 256; }

static int hist_blocks(int M) { return std::max(1, std::min(148 * 2, (M + kHistThreads - 1) / kHistThreads)); }

// Histogram into the scratch `counts` ([Nc + 1] uint32) and `mismatch` words.
static gf_status run_hist(Engine* e, const float* d_freq, int M, int Nc, unsigned* counts, unsigned* mismatch) {
  GF_CUDA(e, cudaMemsetAsync(counts, 0, sizeof(unsigned) * (Nc + 1), e->stream));
  GF_CUDA(e, cudaMemsetAsync(mismatch, 0, sizeof(unsigned), e->stream));
  if (M <= 0) return GF_OK;
  const int smem_bins = std::min(kSmemBins, Nc + 1);
  const size_t smem = sizeof(unsigned) * smem_bins;
  GF_CUDA(e, cudaFuncSetAttribute(hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(sizeof(unsigned) * kSmemBins)));
  hist_kernel<<<hist_blocks(M), kHistThreads, smem, e->stream>>>(d_freq, M, Nc, counts, mismatch, smem_bins);
  GF_CUDA(e, cudaGetLastError());
  e->kernel_launches += 1;
  return GF_OK;
}

static std::vector<double> log_binomial_row(int n) {
  std::vector<double> lgc(n + 1);
  const double ln = std::lgamma(n + 1.0);
  for (int k = 0; k <= n; ++k) lgc[k] = ln - std::lgamma(k + 1.0) - std::lgamma(n - k + 1.0);
  return lgc;
}

gf_status population_histogram_device(Engine* e, const float* d_freq, int M, int Nc, float num_sites, float* d_out) {
  if (Nc <= 0) return fail(e, GF_ERR_INVALID_ARGUMENT, "Nchrom_e must be > 0");
  if (M < 0) return fail(e, GF_ERR_INVALID_ARGUMENT, "num_mutations < 0");
  const size_t need = al256(sizeof(unsigned) * (Nc + 1)) + 256;
  gf_status st = ensure_scratch(e, &e->spec_scratch, &e->spec_scratch_bytes, need);
  if (st != GF_OK) return st;
  unsigned* counts = static_cast<unsigned*>(e->spec_scratch);
  unsigned* mismatch = reinterpret_cast<unsigned*>(static_cast<char*>(e->spec_scratch) + al256(sizeof(unsigned) * (Nc + 1)));
  st = run_hist(e, d_freq, M, Nc, counts, mismatch);
  if (st != GF_OK) return st;
  const unsigned extra0 = static_cast<unsigned>(static_cast<int>(num_sites) - M);
  hist_to_float_kernel<<<std::max(1, std::min(1024, (Nc + 255) / 256)), 256, 0, e->stream>>>(counts, Nc, extra0, d_out);
  GF_CUDA(e, cudaGetLastError());
  e->kernel_launches += 1;
  return GF_OK;
}

gf_status site_frequency_spectrum_device(Engine* e, const float* d_freq, int M, int Nc, int n, float num_sites,
                                         float* d_out) {
  if (n <= 0 || n >= Nc)
    return fail(e, GF_ERR_INVALID_ARGUMENT, "sample_size %d out of range [1, population_size %d)", n, Nc);
  if (M < 0) return fail(e, GF_ERR_INVALID_ARGUMENT, "num_mutations < 0");
  if (n + 1 > 8 * kProjThreads) return fail(e, GF_ERR_CAPACITY, "sample_size %d above the supported %d", n, 8 * kProjThreads - 1);
  const int levels = n + 1;
  // partial blocks: enough to fill the GPU, bounded so the partial buffer stays small
  const int hist_nblocks = std::max(1, std::min(592, (Nc + 1 + 255) / 256));
  const int classes_per_block = (Nc + 1 + hist_nblocks - 1) / hist_nblocks;
  const int direct_nblocks = std::max(1, std::min(592, (M + 1023) / 1024));
  const int nblocks = std::max(hist_nblocks, direct_nblocks);
  SpecLayout L;
  L.counts_off = 0;
  L.mismatch_off = al256(sizeof(unsigned) * (Nc + 1));
  L.nonseg_off = L.mismatch_off + 256;
  L.lgc_off = L.nonseg_off + 256;
  L.partial_off = L.lgc_off + al256(sizeof(double) * levels);
  L.total = L.partial_off + al256(sizeof(double) * levels * nblocks);
  gf_status st = ensure_scratch(e, &e->spec_scratch, &e->spec_scratch_bytes, L.total);
  if (st != GF_OK) return st;
  char* base = static_cast<char*>(e->spec_scratch);
  unsigned* counts = reinterpret_cast<unsigned*>(base + L.counts_off);
  unsigned* mismatch = reinterpret_cast<unsigned*>(base + L.mismatch_off);
  unsigned* nonseg = reinterpret_cast<unsigned*>(base + L.nonseg_off);
  double* lgc = reinterpret_cast<double*>(base + L.lgc_off);
  double* partial = reinterpret_cast<double*>(base + L.partial_off);
  const std::vector<double> h_lgc = log_binomial_row(n);
  GF_CUDA(e, cudaMemcpyAsync(lgc, h_lgc.data(), sizeof(double) * levels, cudaMemcpyHostToDevice, e->stream));
  st = run_hist(e, d_freq, M, Nc, counts, mismatch);
  if (st != GF_OK) return st;
  unsigned h_mismatch = 0;
  GF_CUDA(e, cudaMemcpyAsync(&h_mismatch, mismatch, sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
  GF_CUDA(e, cudaStreamSynchronize(e->stream));
  const double extra0 = static_cast<double>(num_sites - M);
  int used_blocks;
  if (!h_mismatch) {
    nonseg_from_hist_kernel<<<1, 32, 0, e->stream>>>(counts, Nc, nonseg);
    project_hist_kernel<<<hist_nblocks, kProjThreads, 0, e->stream>>>(counts, Nc, n, lgc, partial, classes_per_block);
    used_blocks = hist_nblocks;
  } else {
    GF_CUDA(e, cudaMemsetAsync(nonseg, 0, sizeof(unsigned), e->stream));
    const int per_block = (M + direct_nblocks - 1) / direct_nblocks;
    project_direct_kernel<<<direct_nblocks, kProjThreads, 0, e->stream>>>(d_freq, M, n, lgc, partial, std::max(per_block, 1),
                                                                           nonseg);
    used_blocks = direct_nblocks;
  }
  GF_CUDA(e, cudaGetLastError());
  sfs_finish_kernel<<<(n + 31) / 32, 32 * kFinishWarps, 0, e->stream>>>(partial, used_blocks, n, extra0, nonseg, d_out);
  GF_CUDA(e, cudaGetLastError());
  e->kernel_launches += h_mismatch ? 2 : 3;
  return GF_OK;
}

static gf_status stage_input(Engine* e, const float* h_freq, int M, const float** d_freq) {
  gf_status st = ensure_scratch(e, reinterpret_cast<void**>(&e->spec_in), &e->spec_in_bytes,
                                sizeof(float) * std::max(M, 1));
  if (st != GF_OK) return st;
  if (M > 0) GF_CUDA(e, cudaMemcpyAsync(e->spec_in, h_freq, sizeof(float) * M, cudaMemcpyHostToDevice, e->stream));
  *d_freq = e->spec_in;
  return GF_OK;
}

}  // namespace gf

using namespace gf;

extern "C" {

gf_status gf_population_histogram_device(gf_engine* g, const float* d_freq, int32_t M, int32_t Nc, float L, float* d_out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    GF_CUDA(e, cudaSetDevice(e->device));
    return population_histogram_device(e, d_freq, M, Nc, L, d_out);
  });
}

gf_status gf_site_frequency_spectrum_device(gf_engine* g, const float* d_freq, int32_t M, int32_t Nc, int32_t n, float L,
                                            float* d_out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    GF_CUDA(e, cudaSetDevice(e->device));
    return site_frequency_spectrum_device(e, d_freq, M, Nc, n, L, d_out);
  });
}

gf_status gf_population_histogram(gf_engine* g, const float* freq, int32_t M, int32_t Nc, float L, float* out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (!out || (M > 0 && !freq)) return fail(e, GF_ERR_INVALID_ARGUMENT, "NULL buffer");
    GF_CUDA(e, cudaSetDevice(e->device));
    const float* d_freq = nullptr;
    gf_status st = stage_input(e, freq, M, &d_freq);
    if (st != GF_OK) return st;
    st = ensure_scratch(e, reinterpret_cast<void**>(&e->spec_out), &e->spec_out_bytes, sizeof(float) * std::max(Nc, 1));
    if (st != GF_OK) return st;
    st = population_histogram_device(e, d_freq, M, Nc, L, e->spec_out);
    if (st != GF_OK) return st;
    GF_CUDA(e, cudaMemcpyAsync(out, e->spec_out, sizeof(float) * Nc, cudaMemcpyDeviceToHost, e->stream));
    GF_CUDA(e, cudaStreamSynchronize(e->stream));
    return GF_OK;
  });
}

gf_status gf_site_frequency_spectrum(gf_engine* g, const float* freq, int32_t M, int32_t Nc, int32_t n, float L, float* out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (!out || (M > 0 && !freq)) return fail(e, GF_ERR_INVALID_ARGUMENT, "NULL buffer");
    GF_CUDA(e, cudaSetDevice(e->device));
    const float* d_freq = nullptr;
    gf_status st = stage_input(e, freq, M, &d_freq);
    if (st != GF_OK) return st;
    st = ensure_scratch(e, reinterpret_cast<void**>(&e->spec_out), &e->spec_out_bytes, sizeof(float) * std::max(n, 1));
    if (st != GF_OK) return st;
    st = site_frequency_spectrum_device(e, d_freq, M, Nc, n, L, e->spec_out);
    if (st != GF_OK) return st;
    GF_CUDA(e, cudaMemcpyAsync(out, e->spec_out, sizeof(float) * n, cudaMemcpyDeviceToHost, e->stream));
    GF_CUDA(e, cudaStreamSynchronize(e->stream));
    return GF_OK;
  });
}

}  // extern "C"

// ==================================================================================================
// SFS without allocation.
//
// For callers that must not allocate device memory: code running inside a framework that owns the
// GPU's memory budget (a caching allocator or a pre-reserved pool, where a library's own cudaMalloc
// would bypass the budget and can fail mid-run), and code on a latency-critical path, where
// cudaMalloc / cudaFree would synchronize the device and stall work queued on other streams.  This
// entry point takes its scratch from one file-scope __device__ array instead of engine-owned
// allocations, and needs no gf_engine.
//
// The array is part of the library image: every GPU that loads libgofish_b200.so holds it
// (GF_NOALLOC_SCRATCH_BYTES, about 6.3 MB) until the process exits.  All calls on a device share it
// and it keeps the previous call's contents, so calls whose GPU work overlaps (concurrent streams, or
// several host threads) race and must be serialized by the caller.
// ==================================================================================================

#include <mutex>

namespace gf {

constexpr size_t kNoAllocCountsOff = 0;
constexpr size_t kNoAllocFlagsOff = (sizeof(unsigned) * (GF_NOALLOC_MAX_NCHROM + 1) + 255) / 256 * 256;
constexpr size_t kNoAllocLgcOff = kNoAllocFlagsOff + 256;
constexpr size_t kNoAllocPartialOff = kNoAllocLgcOff + sizeof(double) * (GF_NOALLOC_MAX_SAMPLE + 1);
constexpr int kNoAllocMaxBlocks = 256;
constexpr size_t kNoAllocBytes =
    kNoAllocPartialOff + sizeof(double) * static_cast<size_t>(kNoAllocMaxBlocks) * (GF_NOALLOC_MAX_SAMPLE + 1);
static_assert(kNoAllocBytes == GF_NOALLOC_SCRATCH_BYTES, "GF_NOALLOC_SCRATCH_BYTES out of date");

// Scratch of gf_site_frequency_spectrum_noalloc: [counts | mismatch, nonseg | log C(n,k) | partials]
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// log C(n, k) for k = 0 .. n, computed on the device so the call needs no host staging buffer
__global__ void log_binomial_kernel(double* __restrict__ lgc, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k <= n) lgc[k] = lgamma(n + 1.0) - lgamma(k + 1.0) - lgamma(n - k + 1.0);
}

// Per-device set-up, done once per device by the first call on it (with that device current): the
// scratch array's device address (in host code the array's name only stands for the symbol; kernels
// must be given this address) and the histogram kernel's dynamic shared-memory limit.  Under lazy
// module loading this first call may also load the module, which is when the array takes its device
// memory.  The cached set-up does not survive cudaDeviceReset.
static gf_status noalloc_scratch(int device, unsigned char** out) {
  static std::mutex mu;
  static unsigned char* addr[64] = {nullptr};
  if (device < 0 || device >= 64) return GF_ERR_NO_DEVICE;
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[device]) {
    void* p = nullptr;
    cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err == cudaSuccess && p)
      err = cudaFuncSetAttribute(hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(sizeof(unsigned) * kSmemBins));
    if (err != cudaSuccess || !p) {
      cudaGetLastError();
      return GF_ERR_CUDA;
    }
    addr[device] = static_cast<unsigned char*>(p);
  }
  *out = addr[device];
  return GF_OK;
}

#define GF_NA_CUDA(call)                     \
  do {                                       \
    if ((call) != cudaSuccess) {             \
      cudaGetLastError();                    \
      return GF_ERR_CUDA;                    \
    }                                        \
  } while (0)

}  // namespace gf

extern "C" {

gf_status gf_site_frequency_spectrum_noalloc(const float* d_freq, int32_t M, int32_t Nc, int32_t n, float num_sites,
                                             float* d_out, void* cuda_stream) {
  using namespace gf;
  if (!d_out || (M > 0 && !d_freq) || M < 0) return GF_ERR_INVALID_ARGUMENT;
  if (n <= 0 || n >= Nc) return GF_ERR_INVALID_ARGUMENT;
  if (Nc > GF_NOALLOC_MAX_NCHROM || n > GF_NOALLOC_MAX_SAMPLE) return GF_ERR_CAPACITY;
  int device = 0;
  GF_NA_CUDA(cudaGetDevice(&device));
  unsigned char* base = nullptr;
  const gf_status st = noalloc_scratch(device, &base);
  if (st != GF_OK) return st;
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  unsigned* counts = reinterpret_cast<unsigned*>(base + kNoAllocCountsOff);
  unsigned* mismatch = reinterpret_cast<unsigned*>(base + kNoAllocFlagsOff);
  unsigned* nonseg = mismatch + 1;
  double* lgc = reinterpret_cast<double*>(base + kNoAllocLgcOff);
  double* partial = reinterpret_cast<double*>(base + kNoAllocPartialOff);
  const int levels = n + 1;
  // the array keeps the previous call's contents: everything accumulated into starts from zero here
  GF_NA_CUDA(cudaMemsetAsync(counts, 0, sizeof(unsigned) * (Nc + 1), stream));
  GF_NA_CUDA(cudaMemsetAsync(mismatch, 0, sizeof(unsigned) * 2, stream));
  log_binomial_kernel<<<(levels + 255) / 256, 256, 0, stream>>>(lgc, n);
  GF_NA_CUDA(cudaGetLastError());
  if (M > 0) {
    const int smem_bins = std::min(kSmemBins, Nc + 1);
    hist_kernel<<<hist_blocks(M), kHistThreads, sizeof(unsigned) * smem_bins, stream>>>(d_freq, M, Nc, counts,
                                                                                       mismatch, smem_bins);
    GF_NA_CUDA(cudaGetLastError());
  }
  unsigned h_mismatch = 0;
  GF_NA_CUDA(cudaMemcpyAsync(&h_mismatch, mismatch, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
  GF_NA_CUDA(cudaStreamSynchronize(stream));
  int used_blocks;
  if (!h_mismatch) {
    const int nb = std::max(1, std::min(kNoAllocMaxBlocks, (Nc + 1 + 255) / 256));
    const int per_block = (Nc + 1 + nb - 1) / nb;
    nonseg_from_hist_kernel<<<1, 32, 0, stream>>>(counts, Nc, nonseg);
    project_hist_kernel<<<nb, kProjThreads, 0, stream>>>(counts, Nc, n, lgc, partial, per_block);
    used_blocks = nb;
  } else {
    const int nb = std::max(1, std::min(kNoAllocMaxBlocks, (M + 1023) / 1024));
    const int per_block = std::max(1, (M + nb - 1) / nb);
    project_direct_kernel<<<nb, kProjThreads, 0, stream>>>(d_freq, M, n, lgc, partial, per_block, nonseg);
    used_blocks = nb;
  }
  GF_NA_CUDA(cudaGetLastError());
  sfs_finish_kernel<<<(n + 31) / 32, 32 * kFinishWarps, 0, stream>>>(partial, used_blocks, n,
                                                                      static_cast<double>(num_sites - M), nonseg, d_out);
  GF_NA_CUDA(cudaGetLastError());
  return GF_OK;
}
}  // extern "C"
