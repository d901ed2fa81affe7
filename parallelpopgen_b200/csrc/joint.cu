// Joint site frequency spectrum of two populations: the expected number of sites whose sample of n_a
// chromosomes from population a holds i derived copies and whose sample of n_b chromosomes from
// population b holds j, over the mutation sites (each site's two population frequencies projected
// binomially and independently), plus the num_sites - M monomorphic sites at (0, 0).
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

__global__ void __launch_bounds__(kJThreads)
    joint_sfs_kernel(const float* __restrict__ fa, const float* __restrict__ fb, int M, int na, int nb,
                     const double* __restrict__ lgca, const double* __restrict__ lgcb, int per_block,
                     int tiles_b, double* __restrict__ partial) {
  __shared__ double spa[kJChunk][kJTile];
  __shared__ double spb[kJChunk][kJTile];
  __shared__ double s_lp[2][kJChunk], s_lq[2][kJChunk];
  __shared__ int s_edge[2][kJChunk];
  const int tid = threadIdx.x;
  const int ty = tid >> 4, tx = tid & 15;
  const int i0 = (blockIdx.y / tiles_b) * kJTile;
  const int j0 = (blockIdx.y % tiles_b) * kJTile;
  const int m0 = blockIdx.x * per_block;
  const int m1 = min(M, m0 + per_block);
  double acc[8][8];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[r][c] = 0.0;

  for (int c0 = m0; c0 < m1; c0 += kJChunk) {
    if (tid < 2 * kJChunk) {
      const int w = tid / kJChunk, t = tid % kJChunk;
      const int m = c0 + t;
      double lp = 0.0, lq = 0.0;
      int edge = -1;   // beyond the block's range: contributes nothing (masked below)
      if (m < m1) {
        const float p = w == 0 ? fa[m] : fb[m];
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
    for (int e = tid; e < kJChunk * kJTile; e += kJThreads) {
      const int t = e / kJTile, k = e % kJTile;
      const bool live = c0 + t < m1;
      const int ia = i0 + k, jb = j0 + k;
      spa[t][k] = (live && ia <= na) ? sample_pmf(ia, na, s_lp[0][t], s_lq[0][t], s_edge[0][t], lgca) : 0.0;
      spb[t][k] = (live && jb <= nb) ? sample_pmf(jb, nb, s_lp[1][t], s_lq[1][t], s_edge[1][t], lgcb) : 0.0;
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
  const long long bins = static_cast<long long>(na + 1) * (nb + 1);
  double* out = partial + blockIdx.x * bins;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int i = i0 + ty + 16 * r;
    if (i > na) continue;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int j = j0 + tx + 16 * c;
      if (j <= nb) out[static_cast<long long>(i) * (nb + 1) + j] = acc[r][c];
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

gf_status joint_sfs_device(Engine* e, const float* d_fa, const float* d_fb, int M, int na, int nb, float num_sites,
                           float* d_out) {
  if (na < 1 || nb < 1 || na > kJMaxN || nb > kJMaxN)
    return fail(e, GF_ERR_INVALID_ARGUMENT, "sample sizes %d, %d outside [1, %d]", na, nb, kJMaxN);
  if (M < 0) return fail(e, GF_ERR_INVALID_ARGUMENT, "negative mutation count");
  if (M > 0 && (!d_fa || !d_fb)) return fail(e, GF_ERR_INVALID_ARGUMENT, "frequency rows are NULL");
  if (!d_out) return fail(e, GF_ERR_INVALID_ARGUMENT, "output is NULL");
  const long long bins = static_cast<long long>(na + 1) * (nb + 1);
  const int tiles_a = (na + 1 + kJTile - 1) / kJTile, tiles_b = (nb + 1 + kJTile - 1) / kJTile;
  const int tiles = tiles_a * tiles_b;
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
  gf_status st = pool_alloc(e, reinterpret_cast<void**>(&d_lgc), sizeof(double) * (na + 1 + nb + 1));
  if (st != GF_OK) return st;
  st = pool_alloc(e, reinterpret_cast<void**>(&d_partial), sizeof(double) * bins * nblocks);
  if (st != GF_OK) {
    cudaFreeAsync(d_lgc, e->stream);
    return st;
  }
  std::vector<double> h = log_binomials(na);
  const std::vector<double> hb = log_binomials(nb);
  h.insert(h.end(), hb.begin(), hb.end());
  cudaError_t err = cudaMemcpyAsync(d_lgc, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, e->stream);
  if (err == cudaSuccess && M > 0) {
    dim3 grid(nblocks, tiles);
    joint_sfs_kernel<<<grid, kJThreads, 0, e->stream>>>(d_fa, d_fb, M, na, nb, d_lgc, d_lgc + (na + 1), per_block,
                                                        tiles_b, d_partial);
    err = cudaGetLastError();
    e->kernel_launches += 1;
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
    return joint_sfs_device(e, d_freq_a, d_freq_b, M, n_a, n_b, num_sites, d_out);
  });
}

gf_status gf_joint_site_frequency_spectrum(gf_engine* g, const float* freq_a, const float* freq_b, int32_t M,
                                           int32_t n_a, int32_t n_b, float num_sites, float* out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g) return GF_ERR_INVALID_ARGUMENT;
    Engine* e = &g->impl;
    if (M < 0 || (M > 0 && (!freq_a || !freq_b)) || !out) return fail(e, GF_ERR_INVALID_ARGUMENT, "bad buffers");
    if (n_a < 1 || n_b < 1 || n_a > kJMaxN || n_b > kJMaxN)
      return fail(e, GF_ERR_INVALID_ARGUMENT, "sample sizes %d, %d outside [1, %d]", n_a, n_b, kJMaxN);
    GF_CUDA(e, cudaSetDevice(e->device));
    const long long bins = static_cast<long long>(n_a + 1) * (n_b + 1);
    float* d = nullptr;
    gf_status st = pool_alloc(e, reinterpret_cast<void**>(&d), sizeof(float) * (2ll * std::max(M, 1) + bins));
    if (st != GF_OK) return st;
    float* d_fa = d;
    float* d_fb = d + std::max(M, 1);
    float* d_out = d + 2ll * std::max(M, 1);
    cudaError_t err = cudaSuccess;
    if (M > 0) {
      err = cudaMemcpyAsync(d_fa, freq_a, sizeof(float) * M, cudaMemcpyHostToDevice, e->stream);
      if (err == cudaSuccess) err = cudaMemcpyAsync(d_fb, freq_b, sizeof(float) * M, cudaMemcpyHostToDevice, e->stream);
    }
    if (err == cudaSuccess) {
      st = joint_sfs_device(e, d_fa, d_fb, M, n_a, n_b, num_sites, d_out);
      if (st == GF_OK)
        err = cudaMemcpyAsync(out, d_out, sizeof(float) * bins, cudaMemcpyDeviceToHost, e->stream);
    }
    cudaFreeAsync(d, e->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    if (st != GF_OK) return st;
    if (err != cudaSuccess) return cuda_fail(e, err, "joint SFS transfer");
    return GF_OK;
  });
}

}  // extern "C"
