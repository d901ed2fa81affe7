// Joint site frequency spectrum of two populations: the expected number of sites whose sample of n_a
// chromosomes from population a holds i derived copies and whose sample of n_b chromosomes from
// population b holds j, over the mutation sites (each site's two population frequencies projected
// binomially and independently), plus the num_sites - M monomorphic sites at (0, 0).  The same for
// three populations: bin (i, j, k), with population c's sample of n_c holding k copies.
//
// The reference computes single-population marginals only (Spectrum::site_frequency_spectrum,
// spectrum.cu:213-294, whose projection of one frequency is C(n,k) p^k (1-p)^(n-k), spectrum.cu:90-139);
// this is the two-population form of the same projection.  For 1 <= i <= n_a - 1 the row sums equal the
// single-population SFS of population a.
//
// Work: M x (n_a + 1) x (n_b + 1) FP64 multiply-adds, organised as a GEMM on the CUDA cores
// (JSFS = P_a^T P_b with the mutations as the reduction dimension): each block stages the binomial pmfs
// of a chunk of mutations for one 128 x 128 output tile in shared memory and every thread accumulates
// an 8 x 8 register tile in double; block partials are reduced in a fixed order (deterministic).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "gf_internal.h"

namespace gf {

constexpr int kJThreads = 256;   // 16 x 16
constexpr int kJTile = 128;      // output tile edge (8 rows / columns per thread)
constexpr int kJChunk = 16;      // mutations per shared-memory chunk
constexpr int kJMaxN = 1023;

// pmf of k derived copies in a sample of n from frequency p (exact point masses at p = 0 and p = 1)
__device__ __forceinline__ double sample_pmf(int k, int n, double lp, double lq, int edge, const double* lgc) {
  if (edge < 0) return k == 0 ? 1.0 : 0.0;
  if (edge > 0) return k == n ? 1.0 : 0.0;
  return exp(lgc[k] + k * lp + (n - k) * lq);
}

// THREE: a third population c; block row y covers output tile y / (n_c + 1) at k = y % (n_c + 1), and
// the b operand is weighted by the mutation's pmf of k copies in c.
template <bool THREE>
__global__ void __launch_bounds__(kJThreads)
    joint_sfs_kernel(const float* __restrict__ fa, const float* __restrict__ fb, const float* __restrict__ fc, int M,
                     int na, int nb, int nc, const double* __restrict__ lgca, const double* __restrict__ lgcb,
                     const double* __restrict__ lgcc, int per_block, int tiles_b, double* __restrict__ partial) {
  constexpr int NP = THREE ? 3 : 2;
  __shared__ double spa[kJChunk][kJTile];
  __shared__ double spb[kJChunk][kJTile];
  __shared__ double s_lp[NP][kJChunk], s_lq[NP][kJChunk];
  __shared__ int s_edge[NP][kJChunk];
  __shared__ double s_pc[kJChunk];
  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;
  const int tile = THREE ? static_cast<int>(blockIdx.y) / (nc + 1) : static_cast<int>(blockIdx.y);
  const int kc = THREE ? static_cast<int>(blockIdx.y) % (nc + 1) : 0;
  const int i0 = (tile / tiles_b) * kJTile;
  const int j0 = (tile % tiles_b) * kJTile;
  const int m0 = blockIdx.x * per_block;
  const int m1 = min(M, m0 + per_block);
  double acc[8][8];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[r][c] = 0.0;

  for (int c0 = m0; c0 < m1; c0 += kJChunk) {
    if (tid < NP * kJChunk) {
      const int w = tid / kJChunk, t = tid % kJChunk;
      const int m = c0 + t;
      double lp = 0.0, lq = 0.0;
      int edge = -1;   // beyond the block's range: contributes nothing (masked below)
      if (m < m1) {
        const float p = w == 0 ? fa[m] : w == 1 ? fb[m] : fc[m];
        if (p > 0.f && p < 1.f) {
          edge = 0;
          lp = log(static_cast<double>(p));
          lq = log1p(-static_cast<double>(p));
        } else {
          edge = p >= 1.f ? 1 : -1;
        }
      }
      s_lp[w][t] = lp;
      s_lq[w][t] = lq;
      s_edge[w][t] = edge;
    }
    __syncthreads();
    if (THREE && tid < kJChunk)
      s_pc[tid] = c0 + tid < m1 ? sample_pmf(kc, nc, s_lp[NP - 1][tid], s_lq[NP - 1][tid], s_edge[NP - 1][tid], lgcc)
                                : 0.0;
    if (THREE) __syncthreads();
    for (int e = tid; e < kJChunk * kJTile; e += kJThreads) {
      const int t = e / kJTile, k = e % kJTile;
      const bool live = c0 + t < m1;
      const int ia = i0 + k, jb = j0 + k;
      spa[t][k] = (live && ia <= na) ? sample_pmf(ia, na, s_lp[0][t], s_lq[0][t], s_edge[0][t], lgca) : 0.0;
      double pb = (live && jb <= nb) ? sample_pmf(jb, nb, s_lp[1][t], s_lq[1][t], s_edge[1][t], lgcb) : 0.0;
      if (THREE) pb *= s_pc[t];
      spb[t][k] = pb;
    }
    __syncthreads();
#pragma unroll 2
    for (int t = 0; t < kJChunk; ++t) {
      double a[8], b[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) a[r] = spa[t][ty + 16 * r];
#pragma unroll
      for (int c = 0; c < 8; ++c) b[c] = spb[t][tx + 16 * c];
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] = fma(a[r], b[c], acc[r][c]);
    }
    __syncthreads();
  }
  const long long bins = static_cast<long long>(na + 1) * (nb + 1) * (THREE ? nc + 1 : 1);
  double* out = partial + blockIdx.x * bins;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int i = i0 + ty + 16 * r;
    if (i > na) continue;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int j = j0 + tx + 16 * c;
      if (j <= nb) {
        const long long ij = static_cast<long long>(i) * (nb + 1) + j;
        out[THREE ? ij * (nc + 1) + kc : ij] = acc[r][c];
      }
    }
  }
}

// out[bin] = sum of the partials in block order, plus the monomorphic sites at (0, 0).
__global__ void joint_finish_kernel(const double* __restrict__ partial, int nblocks, long long bins, double extra0,
                                    float* __restrict__ out) {
  for (long long b = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; b < bins;
       b += static_cast<long long>(gridDim.x) * blockDim.x) {
    double s = b == 0 ? extra0 : 0.0;
    for (int k = 0; k < nblocks; ++k) s += partial[k * bins + b];
    out[b] = static_cast<float>(s);
  }
}

static std::vector<double> log_binomials(int n) {
  std::vector<double> v(n + 1);
  const double ln = std::lgamma(n + 1.0);
  for (int k = 0; k <= n; ++k) v[k] = ln - std::lgamma(k + 1.0) - std::lgamma(n - k + 1.0);
  return v;
}

// Largest number of bins of a three-population joint spectrum (the partial sums hold one copy per block).
constexpr long long kJMaxBins3 = 1ll << 24;

// d_fc == nullptr: two populations; else three (n_c >= 1).
gf_status joint_sfs_device(Engine* e, const float* d_fa, const float* d_fb, const float* d_fc, int M, int na, int nb,
                           int nc, float num_sites, float* d_out) {
  const bool three = d_fc != nullptr || nc > 0;
  if (na < 1 || nb < 1 || na > kJMaxN || nb > kJMaxN || (three && (nc < 1 || nc > kJMaxN)))
    return fail(e, GF_ERR_INVALID_ARGUMENT, "sample sizes %d, %d%s outside [1, %d]", na, nb, three ? " (or n_c)" : "",
                kJMaxN);
  if (M < 0) return fail(e, GF_ERR_INVALID_ARGUMENT, "negative mutation count");
  if (M > 0 && (!d_fa || !d_fb || (three && !d_fc))) return fail(e, GF_ERR_INVALID_ARGUMENT, "frequency rows are NULL");
  if (!d_out) return fail(e, GF_ERR_INVALID_ARGUMENT, "output is NULL");
  const long long bins = static_cast<long long>(na + 1) * (nb + 1) * (three ? nc + 1 : 1);
  if (three && bins > kJMaxBins3)
    return fail(e, GF_ERR_CAPACITY, "%lld bins exceed the three-population limit of %lld", bins, kJMaxBins3);
  const int tiles_a = (na + 1 + kJTile - 1) / kJTile, tiles_b = (nb + 1 + kJTile - 1) / kJTile;
  const int tiles = tiles_a * tiles_b * (three ? nc + 1 : 1);
  // about two blocks per SM over all tiles, each block a whole number of chunks; partials kept under
  // 256 MB
  int nblocks = std::max(1, (2 * e->num_sms + tiles - 1) / tiles);
  nblocks = std::min<long long>(nblocks, std::max<long long>(1, (256ll << 20) / (bins * 8)));
  nblocks = std::min(nblocks, std::max(1, (M + kJChunk - 1) / kJChunk));
  int per_block = (M + nblocks - 1) / std::max(nblocks, 1);
  per_block = std::max(kJChunk, (per_block + kJChunk - 1) / kJChunk * kJChunk);
  nblocks = std::max(1, (M + per_block - 1) / per_block);

  double* d_lgc = nullptr;
  double* d_partial = nullptr;
  gf_status st = pool_alloc(e, reinterpret_cast<void**>(&d_lgc), sizeof(double) * (na + 1 + nb + 1 + nc + 1));
  if (st != GF_OK) return st;
  st = pool_alloc(e, reinterpret_cast<void**>(&d_partial), sizeof(double) * bins * nblocks);
  if (st != GF_OK) {
    cudaFreeAsync(d_lgc, e->stream);
    return st;
  }
  std::vector<double> h = log_binomials(na);
  const std::vector<double> hb = log_binomials(nb);
  h.insert(h.end(), hb.begin(), hb.end());
  if (three) {
    const std::vector<double> hc = log_binomials(nc);
    h.insert(h.end(), hc.begin(), hc.end());
  }
  cudaError_t err = cudaMemcpyAsync(d_lgc, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, e->stream);
  if (err == cudaSuccess && M > 0) {
    if (tiles > 65535) {
      err = cudaErrorInvalidConfiguration;
    } else {
      dim3 grid(nblocks, tiles);
      if (three)
        joint_sfs_kernel<true><<<grid, kJThreads, 0, e->stream>>>(d_fa, d_fb, d_fc, M, na, nb, nc, d_lgc,
                                                                  d_lgc + (na + 1), d_lgc + (na + 1) + (nb + 1),
                                                                  per_block, tiles_b, d_partial);
      else
        joint_sfs_kernel<false><<<grid, kJThreads, 0, e->stream>>>(d_fa, d_fb, nullptr, M, na, nb, 0, d_lgc,
                                                                   d_lgc + (na + 1), nullptr, per_block, tiles_b,
                                                                   d_partial);
      err = cudaGetLastError();
      e->kernel_launches += 1;
    }
  }
  if (err == cudaSuccess) {
    const int fb = static_cast<int>(std::min<long long>(4 * e->num_sms, (bins + 255) / 256));
    joint_finish_kernel<<<std::max(fb, 1), 256, 0, e->stream>>>(d_partial, M > 0 ? nblocks : 0, bins,
                                                                static_cast<double>(num_sites) - M, d_out);
    err = cudaGetLastError();
    e->kernel_launches += 1;
  }
  cudaFreeAsync(d_partial, e->stream);
  cudaFreeAsync(d_lgc, e->stream);
  if (err != cudaSuccess) return cuda_fail(e, err, "joint SFS");
  return GF_OK;
}

}  // namespace gf

using namespace gf;

extern "C" {

gf_status gf_joint_site_frequency_spectrum_device(gf_engine* g, const float* d_freq_a, const float* d_freq_b,
                                                  int32_t M, int32_t n_a, int32_t n_b, float num_sites,
                                                  float* d_out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    GF_CUDA(e, cudaSetDevice(e->device));
    return joint_sfs_device(e, d_freq_a, d_freq_b, nullptr, M, n_a, n_b, 0, num_sites, d_out);
  });
}

gf_status gf_joint3_site_frequency_spectrum_device(gf_engine* g, const float* d_freq_a, const float* d_freq_b,
                                                   const float* d_freq_c, int32_t M, int32_t n_a, int32_t n_b,
                                                   int32_t n_c, float num_sites, float* d_out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (n_c < 1) return fail(e, GF_ERR_INVALID_ARGUMENT, "sample size n_c %d below 1", n_c);
    GF_CUDA(e, cudaSetDevice(e->device));
    return joint_sfs_device(e, d_freq_a, d_freq_b, d_freq_c, M, n_a, n_b, n_c, num_sites, d_out);
  });
}

}  // extern "C"

namespace gf {

// Host rows in, host spectrum out (freq_c == nullptr: two populations).
static gf_status joint_sfs_host(Engine* e, const float* freq_a, const float* freq_b, const float* freq_c, int M,
                                int n_a, int n_b, int n_c, float num_sites, float* out) {
  const bool three = freq_c != nullptr || n_c > 0;
  if (M < 0 || (M > 0 && (!freq_a || !freq_b || (three && !freq_c))) || !out)
    return fail(e, GF_ERR_INVALID_ARGUMENT, "bad buffers");
  if (n_a < 1 || n_b < 1 || n_a > kJMaxN || n_b > kJMaxN || (three && (n_c < 1 || n_c > kJMaxN)))
    return fail(e, GF_ERR_INVALID_ARGUMENT, "sample sizes %d, %d%s outside [1, %d]", n_a, n_b, three ? " (or n_c)" : "",
                kJMaxN);
  const long long bins = static_cast<long long>(n_a + 1) * (n_b + 1) * (three ? n_c + 1 : 1);
  if (three && bins > kJMaxBins3)
    return fail(e, GF_ERR_CAPACITY, "%lld bins exceed the three-population limit of %lld", bins, kJMaxBins3);
  GF_CUDA(e, cudaSetDevice(e->device));
  const long long rows = three ? 3 : 2;
  float* d = nullptr;
  gf_status st = pool_alloc(e, reinterpret_cast<void**>(&d), sizeof(float) * (rows * std::max(M, 1) + bins));
  if (st != GF_OK) return st;
  float* d_fa = d;
  float* d_fb = d + std::max(M, 1);
  float* d_fc = three ? d + 2ll * std::max(M, 1) : nullptr;
  float* d_out = d + rows * std::max(M, 1);
  cudaError_t err = cudaSuccess;
  if (M > 0) {
    err = cudaMemcpyAsync(d_fa, freq_a, sizeof(float) * M, cudaMemcpyHostToDevice, e->stream);
    if (err == cudaSuccess) err = cudaMemcpyAsync(d_fb, freq_b, sizeof(float) * M, cudaMemcpyHostToDevice, e->stream);
    if (err == cudaSuccess && three)
      err = cudaMemcpyAsync(d_fc, freq_c, sizeof(float) * M, cudaMemcpyHostToDevice, e->stream);
  }
  if (err == cudaSuccess) {
    st = joint_sfs_device(e, d_fa, d_fb, d_fc, M, n_a, n_b, three ? n_c : 0, num_sites, d_out);
    if (st == GF_OK) err = cudaMemcpyAsync(out, d_out, sizeof(float) * bins, cudaMemcpyDeviceToHost, e->stream);
  }
  cudaFreeAsync(d, e->stream);
  if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
  if (st != GF_OK) return st;
  if (err != cudaSuccess) return cuda_fail(e, err, "joint SFS transfer");
  return GF_OK;
}

}  // namespace gf

extern "C" {

gf_status gf_joint_site_frequency_spectrum(gf_engine* g, const float* freq_a, const float* freq_b, int32_t M,
                                           int32_t n_a, int32_t n_b, float num_sites, float* out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    return joint_sfs_host(&g->impl, freq_a, freq_b, nullptr, M, n_a, n_b, 0, num_sites, out);
  });
}

gf_status gf_joint3_site_frequency_spectrum(gf_engine* g, const float* freq_a, const float* freq_b, const float* freq_c,
                                            int32_t M, int32_t n_a, int32_t n_b, int32_t n_c, float num_sites,
                                            float* out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    if (n_c < 1) return fail(&g->impl, GF_ERR_INVALID_ARGUMENT, "sample size n_c %d below 1", n_c);
    return joint_sfs_host(&g->impl, freq_a, freq_b, freq_c, M, n_a, n_b, n_c, num_sites, out);
  });
}

}  // extern "C"
