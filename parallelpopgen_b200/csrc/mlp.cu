// SFS surrogate network on sm_100a tensor cores: a bf16 GEMM built on TMA + tcgen05 with the
// accumulator in tensor memory, fused epilogues (bias + GELU forward, GELU' backward with bias
// gradients, split-K weight-gradient partials), the loss, the gradient reduction and Adam.
//
// Every GEMM is C[M][N] = A[M][K] * B[N][K]^T with both operands K-contiguous:
//   forward   Z_l  = Y_{l-1} W_l^T          A = Y_{l-1} [batch][in]      B = W_l   [out][in]
//   input     dY_{l-1} = dZ_l W_l           A = dZ_l    [batch][out]     B = W_l^T [in][out]
//   weights   dW_l = dZ_l^T Y_{l-1}         A = dZ_l^T  [out][batch]     B = Y_{l-1}^T [in][batch]
// so the forward epilogue writes each activation twice (row-major and transposed), the backward
// epilogue does the same for dZ, and Adam keeps bf16 copies of W and W^T.  Layer 1's six inputs are
// zero-padded to 64 columns and layer 5's 99 outputs to 128 rows; padding stays exactly zero.
//
// The reference has no network (3P answers every SFS query by simulation, go_fish.cuh:280 and
// spectrum.h:90); this file serves the surrogate that stands in for those calls.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "gf_surrogate.h"
#include "gf_umma.cuh"

namespace gfm {

constexpr int BM = 128;       // tile rows = tensor-memory lanes
constexpr int BK = 64;        // K per pipeline stage: one 128-byte swizzle row of bf16
constexpr long long WAIT_LIMIT = 1ll << 31;   // SM cycles (about a second) before a wait gives up
constexpr long long INJECT_WAIT_LIMIT = 1ll << 22;   // the same under fault injection (about 2 ms)
constexpr int HID = GF_MLP_HIDDEN;
constexpr int IN_PAD = 64;
constexpr int OUT_PAD = 128;
constexpr int MAX_SPLITS = 16;

enum Epi : int {
  EPI_STORE_F32 = 0,     // C (fp32)
  EPI_FWD_GELU = 1,      // Z = acc + bias (fp32), Y = GELU(Z) (bf16) and Y^T (bf16)
  EPI_FWD_LINEAR = 2,    // out = acc + bias (fp32)
  EPI_BWD_GELU = 3,      // dZ = acc * GELU'(Z) (bf16) and dZ^T (bf16), bias partials
  EPI_PARTIAL = 4,       // split-K partial slice of C (fp32)
  EPI_FWD_GELU_INFER = 5,// Y = GELU(acc + bias) (bf16) only
  EPI_FWD_OUT = 6        // out = acc + bias written straight to the caller's [rows][99] array
};

struct EpiArgs {
  const float* bias;         // [N]
  const float* z;            // forward pre-activation read by the backward epilogue
  long long ldz;
  float* bias_part;          // [M / 128][ld_bias_part] column sums of the backward output
  long long ld_bias_part;
  int rows_per_split;        // row offset of split s in the partial-slice map (EPI_PARTIAL)
  float* out;                // caller's output [rows][out_cols] (EPI_FWD_OUT)
  int out_cols;
  int* fault;                // set when a bounded wait ran out
};

constexpr int EPI_WARPS = 8;                        // two per tensor-memory lane quarter
constexpr int GEMM_THREADS = 64 + 32 * EPI_WARPS;   // TMA warp, MMA warp, 8 epilogue warps
constexpr int SMEM_LIMIT = 232448;                  // dynamic shared memory per CTA on sm_100

// Per-epilogue-warp staging of one 32 x 32 output chunk, double-buffered: fp32 rows with the 128-byte
// swizzle, bf16 rows with the 64-byte swizzle, bf16 transposed rows unswizzled -- the layouts the
// output tensor maps expect, and conflict-free for the row-per-lane writes.  Only the outputs the
// epilogue writes get space.
template <int EPI>
struct Stage {
  static constexpr bool F32 = EPI == EPI_STORE_F32 || EPI == EPI_PARTIAL || EPI == EPI_FWD_LINEAR || EPI == EPI_FWD_GELU;
  static constexpr bool BF16 = EPI == EPI_FWD_GELU || EPI == EPI_FWD_GELU_INFER || EPI == EPI_BWD_GELU;
  static constexpr bool T = EPI == EPI_FWD_GELU || EPI == EPI_BWD_GELU;
  static constexpr int F32_OFF = 0;
  static constexpr int BF16_OFF = F32 ? 4096 : 0;
  static constexpr int T_OFF = BF16_OFF + (BF16 ? 2048 : 0);
  static constexpr int BUF = ((T_OFF + (T ? 2048 : 0)) + 1023) / 1024 * 1024;
  static constexpr int WARP = 2 * BUF;
};

template <int BN, int EPI>
struct Smem {
  static constexpr int A_BYTES = BM * BK * 2;
  static constexpr int B_BYTES = BN * BK * 2;
  static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
  static constexpr int BIAS_FLOATS = 512;   // the bias vector of the whole output width
  // EPI_FWD_OUT stages a whole 128-row tile of the caller's [rows][99] output (one contiguous span)
  static constexpr int OUT_TILE = EPI == EPI_FWD_OUT ? (BM * GF_MLP_OUTPUTS * 4 + 1023) / 1024 * 1024 : 0;
  static constexpr int EXTRA = EPI_WARPS * Stage<EPI>::WARP + OUT_TILE + 256 + 2 * 4 * 32 * 4 + 4 * BIAS_FLOATS + 1024;
  static constexpr int STAGES = (4 * STAGE_BYTES + EXTRA <= SMEM_LIMIT)   ? 4
                                : (3 * STAGE_BYTES + EXTRA <= SMEM_LIMIT) ? 3
                                                                          : 2;
  static constexpr int STG_OFFSET = STAGES * STAGE_BYTES;
  static constexpr int BAR_OFFSET = STG_OFFSET + EPI_WARPS * Stage<EPI>::WARP + OUT_TILE;
  static constexpr int OUT_OFFSET = BAR_OFFSET - OUT_TILE;
  static constexpr int BIAS_OFFSET = BAR_OFFSET + 256 + 2 * 4 * 32 * 4;
  static constexpr int BYTES = BIAS_OFFSET + 4 * BIAS_FLOATS + 1024;   // + barriers, reductions, bias, alignment
  static_assert(BYTES <= SMEM_LIMIT, "shared memory");
};

// GELU in its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), on the hardware tanh.
constexpr float GELU_C = 0.7978845608028654f;
constexpr float GELU_A = 0.044715f;

__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Written as tanh(z (c + c a z^2)) and (z/2) t + z/2: six instructions, one of them on the MUFU pipe.
// The fused forward's epilogue is bound by instruction issue, and this form issues two fewer than
// c (z + a z^3) and (z/2)(1 + t).
__device__ __forceinline__ float gelu(float z) {
  const float t = tanh_hw(z * fmaf(GELU_C * GELU_A, z * z, GELU_C));
  const float hz = 0.5f * z;
  return fmaf(hz, t, hz);
}

__device__ __forceinline__ float gelu_grad(float z) {
  const float z2 = z * z;
  const float t = tanh_hw(GELU_C * fmaf(GELU_A * z, z2, z));
  return 0.5f * (1.f + t) + 0.5f * z * (1.f - t * t) * GELU_C * fmaf(3.f * GELU_A, z2, 1.f);
}

// row `r` of a 32 x 32 fp32 chunk, 128-byte swizzle (16-byte unit q of row r sits at q ^ (r % 8))
__device__ __forceinline__ void stage_f32_row(uint8_t* buf, int r, const float* v) {
#pragma unroll
  for (int q = 0; q < 8; ++q)
    *reinterpret_cast<float4*>(buf + r * 128 + ((q ^ (r & 7)) << 4)) =
        make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
}

// row `r` of a 32 x 32 bf16 chunk, 64-byte swizzle (16-byte unit q of row r sits at q ^ ((r / 2) % 4))
__device__ __forceinline__ void stage_bf16_row(uint8_t* buf, int r, const float* v) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint32_t w[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      __nv_bfloat162 p = __floats2bfloat162_rn(v[q * 8 + 2 * t], v[q * 8 + 2 * t + 1]);
      w[t] = *reinterpret_cast<uint32_t*>(&p);
    }
    *reinterpret_cast<uint4*>(buf + r * 64 + ((q ^ ((r >> 1) & 3)) << 4)) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// column `r` of the transposed chunk: element (j, r) at j * 64 + 2 r
__device__ __forceinline__ void stage_bf16_col(uint8_t* buf, int r, const float* v) {
#pragma unroll
  for (int j = 0; j < 32; ++j) *reinterpret_cast<__nv_bfloat16*>(buf + j * 64 + 2 * r) = __float2bfloat16_rn(v[j]);
}

// Persistent tensor-core GEMM: CTAs stride over 128 x BN output tiles (N fastest, then M, then the
// K split).  Warp 0 streams A/B K-blocks with TMA into a 4-stage ring, warp 1 issues tcgen05 MMAs
// into one of two tensor-memory accumulators, warps 2-5 drain the other accumulator through the
// epilogue (tcgen05.ld -> registers -> swizzled shared staging -> TMA store), so a tile's epilogue
// overlaps the next tile's MMAs.
template <int BN, int EPI>
__global__ void __launch_bounds__(GEMM_THREADS, 1)
umma_gemm_kernel(const __grid_constant__ CUtensorMap tma_a, const __grid_constant__ CUtensorMap tma_b,
                 const __grid_constant__ CUtensorMap tma_c, const __grid_constant__ CUtensorMap tma_y,
                 const __grid_constant__ CUtensorMap tma_yt, int m_tiles, int n_tiles, int splits, int k_blocks,
                 EpiArgs ep, long long wait_limit, int inject) {
  using L = Smem<BN, EPI>;
  using SG = Stage<EPI>;
  constexpr int STAGES = L::STAGES;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L::BAR_OFFSET);
  uint64_t* empty = full + STAGES;
  uint64_t* tfull = empty + STAGES;      // accumulator ready (MMA -> epilogue)
  uint64_t* tempty = tfull + 2;          // accumulator drained (epilogue -> MMA)
  uint64_t* drain = tempty + 2;           // MMA completion before tensor memory is released (abort path)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  int* timed_out = reinterpret_cast<int*>(tmem_slot + 1);
  int* epi_fail = timed_out + 1;         // the epilogue warps' joint verdict (sticky)
  int* consumed_s = timed_out + 2;       // K-blocks the MMA thread received (for the drain)
  float* red = reinterpret_cast<float*>(smem + L::BAR_OFFSET + 256);   // [2 halves][4 quarters][32]
  float* s_bias = reinterpret_cast<float*>(smem + L::BIAS_OFFSET);
  volatile int* abort_flag = timed_out;
  constexpr bool HAS_BIAS = EPI == EPI_FWD_GELU || EPI == EPI_FWD_GELU_INFER || EPI == EPI_FWD_LINEAR ||
                            EPI == EPI_FWD_OUT;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tiles = m_tiles * n_tiles * splits;
  // Bounded waits.  The producer and MMA threads stop issuing work as soon as any wait of the CTA has
  // run out (`wait`); the epilogue warps wait on the barrier alone and then agree on the outcome, so
  // all of them leave the tile loop together.  An aborted CTA never touches unsynchronised data: it
  // drains what it issued and releases tensor memory.
  auto wait = [&](uint64_t* bar, uint32_t parity) -> bool {
    if (*abort_flag) return false;
    const uint32_t addr = smem_u32(bar);
    const long long t0 = clock64();
    while (!mbar_try_wait(addr, parity)) {
      if (*abort_flag) return false;
      if (clock64() - t0 > wait_limit) {
        *abort_flag = 1;
        return false;
      }
    }
    return true;
  };

  if (threadIdx.x == 0) {
    tma_prefetch_desc(&tma_a);
    tma_prefetch_desc(&tma_b);
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&tfull[a], 1);
      mbar_init(&tempty[a], EPI_WARPS);
    }
    mbar_init(drain, 1);
    *timed_out = 0;
    *epi_fail = 0;
    *consumed_s = 0;
    mbar_fence_init();
  }
  if constexpr (HAS_BIAS) {
    for (int i = threadIdx.x; i < n_tiles * BN && i < L::BIAS_FLOATS; i += blockDim.x) s_bias[i] = ep.bias[i];
  }
  __syncwarp();
  if (warp == 1) tmem_alloc(tmem_slot, 2 * BN);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool late = false;
  int issued = 0;   // K-blocks the producer issued (for the drain after a timeout)

  if (warp == 0) {
    if (lane == 0) {
      int it = 0;
      for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int nt = tile % n_tiles;
        const int rest = tile / n_tiles;
        const int mt = rest % m_tiles;
        const int sp = rest / m_tiles;
        for (int kb = 0; kb < k_blocks; ++kb, ++it) {
          const int s = it % STAGES;
          const uint32_t ph = (it / STAGES) & 1;
          if (!wait(&empty[s], ph ^ 1)) {
            late = true;
            goto producer_done;
          }
          uint8_t* a = smem + s * L::STAGE_BYTES;
          mbar_arrive_expect_tx(&full[s], L::STAGE_BYTES);
          const int kx = (sp * k_blocks + kb) * BK;
          tma_load_2d(a, &tma_a, kx, mt * BM, &full[s]);
          tma_load_2d(a + L::A_BYTES, &tma_b, kx, nt * BN, &full[s]);
        }
      }
    producer_done:
      issued = it;
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t idesc = bf16_idesc(BM, BN);
      int it = 0, local = 0;
      for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++local) {
        const int acc = local & 1;
        const uint32_t use = static_cast<uint32_t>(local >> 1);
        if (!wait(&tempty[acc], (use & 1) ^ 1)) {
          late = true;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + static_cast<uint32_t>(acc * BN);
        bool stop = false;
        for (int kb = 0; kb < k_blocks; ++kb, ++it) {
          const int s = it % STAGES;
          const uint32_t ph = (it / STAGES) & 1;
          if (!wait(&full[s], ph)) {
            late = true;
            stop = true;
            break;
          }
          tc_fence_after();
          const uint32_t a_addr = smem_u32(smem + s * L::STAGE_BYTES);
          const uint32_t b_addr = a_addr + L::A_BYTES;
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk)
            umma_bf16(d, sw128_kmajor_desc(a_addr + kk * 32), sw128_kmajor_desc(b_addr + kk * 32), idesc,
                      (kb | kk) != 0);
          umma_commit(&empty[s]);
        }
        if (stop) break;
        // fault injection for tests: withhold the first accumulator hand-off
        if (!((inject & 1) && local == 0)) umma_commit(&tfull[acc]);
      }
      *consumed_s = it;
    }
    __syncwarp();
  } else {
    // epilogue warps: TMEM lane quarter = warp % 4; the two warps of a quarter take alternate
    // 32-column chunks
    const int qd = warp & 3;
    const int ew = warp - 2;
    const int half = ew >> 2;
    uint8_t* stg = smem + L::STG_OFFSET + ew * SG::WARP;
    int chunk = 0, local = 0;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x, ++local) {
      const int nt = tile % n_tiles;
      const int rest = tile / n_tiles;
      const int mt = rest % m_tiles;
      const int sp = rest / m_tiles;
      const int acc = local & 1;
      const uint32_t use = static_cast<uint32_t>(local >> 1);
      if (lane == 0 && !mbar_wait(&tfull[acc], use & 1, wait_limit)) atomicOr(epi_fail, 1);
      named_barrier_sync(4, 32 * EPI_WARPS);     // every epilogue warp has its verdict in epi_fail
      if (*reinterpret_cast<volatile int*>(epi_fail)) {
        late = true;
        break;
      }
      __syncwarp();
      tc_fence_after();
      const int row0 = mt * BM + qd * 32;        // first output row of this warp
      const int row = row0 + lane;
      float* s_out = reinterpret_cast<float*>(smem + L::OUT_OFFSET);
      if constexpr (EPI == EPI_FWD_OUT) {
        // the previous tile's bulk store has read the staging tile
        if (ew == 0 && lane == 0) bulk_wait_read<0>();
        named_barrier_sync(3, 32 * EPI_WARPS);
      }
      const uint32_t tbase = tmem + (static_cast<uint32_t>(qd * 32) << 16) + static_cast<uint32_t>(acc * BN);
#pragma unroll 1
      for (int c0 = 32 * half; c0 < BN; c0 += 64, ++chunk) {
        const int n = nt * BN + c0;
        uint8_t* buf = stg + (chunk & 1) * SG::BUF;
        if (lane == 0) bulk_wait_read<1>();     // the store that last used this buffer has read it
        __syncwarp();
        float v[32];
        tmem_ld_32cols(tbase + c0, v);
        if constexpr (EPI == EPI_STORE_F32 || EPI == EPI_PARTIAL) {
          stage_f32_row(buf + SG::F32_OFF, lane, v);
        } else if constexpr (EPI == EPI_FWD_LINEAR) {
#pragma unroll
          for (int j = 0; j < 32; ++j) v[j] += s_bias[n + j];
          stage_f32_row(buf + SG::F32_OFF, lane, v);
        } else if constexpr (EPI == EPI_FWD_OUT) {
          // row stride 99 words: lanes (rows) hit distinct banks
          float* o = s_out + (qd * 32 + lane) * GF_MLP_OUTPUTS;
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (n + j < GF_MLP_OUTPUTS) o[n + j] = v[j] + s_bias[n + j];
        } else if constexpr (EPI == EPI_FWD_GELU || EPI == EPI_FWD_GELU_INFER) {
#pragma unroll
          for (int j = 0; j < 32; ++j) v[j] += s_bias[n + j];
          if constexpr (EPI == EPI_FWD_GELU) stage_f32_row(buf + SG::F32_OFF, lane, v);
#pragma unroll
          for (int j = 0; j < 32; ++j) v[j] = gelu(v[j]);
          stage_bf16_row(buf + SG::BF16_OFF, lane, v);
          if constexpr (EPI == EPI_FWD_GELU) stage_bf16_col(buf + SG::T_OFF, lane, v);
        } else if constexpr (EPI == EPI_BWD_GELU) {
          const float4* zp = reinterpret_cast<const float4*>(ep.z + static_cast<long long>(row) * ep.ldz + n);
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const float4 z = __ldg(zp + q);
            v[4 * q] *= gelu_grad(z.x);
            v[4 * q + 1] *= gelu_grad(z.y);
            v[4 * q + 2] *= gelu_grad(z.z);
            v[4 * q + 3] *= gelu_grad(z.w);
          }
          stage_bf16_row(buf + SG::BF16_OFF, lane, v);
          stage_bf16_col(buf + SG::T_OFF, lane, v);
          // column sums over the tile's 128 rows (fixed order: lanes, then quarters 0..3); the four
          // warps of a half work on the same chunk and meet at their own named barrier
          float mine = 0.f;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            float t = v[j];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == j) mine = t;
          }
          float* rh = red + half * 128;
          rh[qd * 32 + lane] = mine;
          named_barrier_sync(1 + half, 128);
          if (qd == 0) {
            const float t = ((rh[lane] + rh[32 + lane]) + rh[64 + lane]) + rh[96 + lane];
            ep.bias_part[mt * ep.ld_bias_part + n + lane] = t;
          }
          named_barrier_sync(1 + half, 128);
        }
        if constexpr (EPI == EPI_FWD_OUT) continue;   // written directly
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) {
          if constexpr (EPI == EPI_STORE_F32 || EPI == EPI_FWD_LINEAR || EPI == EPI_FWD_GELU) {
            tma_store_2d(&tma_c, n, row0, buf + SG::F32_OFF);
          } else if constexpr (EPI == EPI_PARTIAL) {
            tma_store_2d(&tma_c, n, sp * ep.rows_per_split + row0, buf + SG::F32_OFF);
          }
          if constexpr (SG::BF16) tma_store_2d(&tma_y, n, row0, buf + SG::BF16_OFF);
          if constexpr (SG::T) tma_store_2d(&tma_yt, row0, n, buf + SG::T_OFF);
          bulk_commit();
        }
      }
      if constexpr (EPI == EPI_FWD_OUT) {
        // rows [mt*128, mt*128 + 128) of a [rows][99] array are one contiguous span
        fence_proxy_async_smem();
        named_barrier_sync(3, 32 * EPI_WARPS);
        if (ew == 0 && lane == 0) {
          bulk_store_1d(ep.out + static_cast<long long>(mt) * BM * GF_MLP_OUTPUTS, s_out, BM * GF_MLP_OUTPUTS * 4);
          bulk_commit();
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[acc]);
    }
    if (lane == 0) bulk_wait_all();
    __syncwarp();
  }

  tc_fence_before();
  if (late) *abort_flag = 1;
  __syncthreads();
  if (*abort_flag) {
    // a wait ran out: let every load and MMA this CTA issued finish before its shared and tensor
    // memory are released (each wait again bounded)
    if (threadIdx.x == 0) {
      // loads issued but never received by the MMA thread are still landing
      for (int it = *consumed_s; it < issued; ++it) mbar_wait(&full[it % STAGES], (it / STAGES) & 1, wait_limit);
      if (ep.fault) atomicOr(ep.fault, 1);
    } else if (threadIdx.x == 32) {
      umma_commit(drain);   // arrives once every MMA this thread issued has completed
      mbar_wait(drain, 0, wait_limit);
    }
    __syncthreads();
  }
  if (warp == 1) tmem_dealloc(tmem, 2 * BN);
}

// ---------------------------------------------------------------------------------------------
// Fused inference forward: all five layers of a 128-row tile in one CTA, the activations on chip.
//
// The layered path writes each hidden activation (batch x 512 bf16) to memory and reads it back in
// the next layer's GEMM.  Here a CTA keeps its tile's activation H (128 x 512 bf16 = 128 KB) in
// shared memory, in the 128-byte-swizzled K-major layout the MMA reads (eight 64-column K blocks of
// 16 KB), and the layer's fp32 accumulator (128 x 512) in all 512 tensor-memory columns: N half 0
// in region A (columns 0-255), N half 1 in region B (256-511).  Warp 1 issues the MMAs (A = H from
// shared memory, B = weight K-blocks streamed by warp 0's TMA through a 3-stage ring from L2, where
// every CTA finds the 1.3 MB of weights); 16 epilogue warps drain the accumulators (bias, GELU, bf16)
// back into H for the next layer, overlapped with the MMAs: region A while N half 1 accumulates
// (staged in tensor memory, since H is still being read), region B while the next layer's first
// K blocks accumulate.  The last layer's epilogue writes acc + bias to the caller's [batch][99]
// array.  Each layer's MMAs run in the order of the layered GEMMs (N halves of 256, K blocks 0..7,
// four 16-wide slices each; layer 5 one 128-wide N tile), so the outputs are bit-identical to the
// layered path.
// ---------------------------------------------------------------------------------------------
constexpr int FF_EPI_WARPS = 16;                          // four per tensor-memory lane quarter
constexpr int FF_THREADS = 64 + 32 * FF_EPI_WARPS;        // TMA warp, MMA warp, 16 epilogue warps
constexpr int FF_WSTAGES = 3;
constexpr int FF_KB_BYTES = BM * BK * 2;                  // one 128 x 64 bf16 K block of H: 16 KB
constexpr int FF_H_BYTES = BM * HID * 2;                  // H: 128 KB
constexpr int FF_WSTAGE_BYTES = 256 * BK * 2;             // a 256-row x 64 weight block: 32 KB
constexpr int FF_BIAS_OFFSET = FF_H_BYTES + FF_WSTAGES * FF_WSTAGE_BYTES;   // the layer's bias (512 fp32)
constexpr int FF_BAR_OFFSET = FF_BIAS_OFFSET + HID * 4;
constexpr int FF_ALIGN_SLACK = 256;   // dynamic shared memory starts 1024-aligned when a kernel has no static
                                      // shared memory; up to this much misalignment is absorbed, more is a fault
constexpr int FF_SMEM = FF_BAR_OFFSET + 256 + FF_ALIGN_SLACK;   // + barriers and flags
static_assert(FF_SMEM <= SMEM_LIMIT, "fused forward shared memory");
constexpr int FF_STAGES_PER_TILE = 2 + 3 * 16 + 8;        // weight blocks streamed per tile (58)
constexpr int kFfStoreThread = 64;                         // the epilogue thread that issues the output stores
constexpr int kFfPollThread = 64;                          // the epilogue thread that waits for the MMA hand-offs
static_assert(BM * GF_MLP_OUTPUTS * 4 <= 4 * FF_KB_BYTES, "staged outputs fit in H's K blocks 1-4");

// Weight block `i` of a tile's stream: layer, the N offset of its rows, the K block, its rows.
struct FfBlock {
  int layer, n0, kb, rows;
};
__device__ __forceinline__ FfBlock ff_block(int i) {
  if (i < 2) return {0, 256 * i, 0, 256};                           // layer 1: K = 64, two N halves
  if (i < 50) {                                                      // layers 2-4: N halves x 8 K blocks
    const int j = i - 2;
    return {1 + j / 16, 256 * ((j % 16) / 8), j % 8, 256};
  }
  return {4, 0, i - 50, OUT_PAD};                                    // layer 5: 128 rows x 8 K blocks
}

__global__ void __launch_bounds__(FF_THREADS, 1)
fused_forward_kernel(const __grid_constant__ CUtensorMap tma_x, const __grid_constant__ CUtensorMap tma_w1,
                     const __grid_constant__ CUtensorMap tma_w2, const __grid_constant__ CUtensorMap tma_w3,
                     const __grid_constant__ CUtensorMap tma_w4, const __grid_constant__ CUtensorMap tma_w5,
                     const float* __restrict__ b1, const float* __restrict__ b2, const float* __restrict__ b3,
                     const float* __restrict__ b4, const float* __restrict__ b5, float* __restrict__ out,
                     int batch, int m_tiles, long long wait_limit, int inject, int* fault) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  if (smem - smem_raw > FF_ALIGN_SLACK) {   // the layout would not fit (uniform over the CTA)
    if (threadIdx.x == 0 && fault) atomicOr(fault, 1);
    return;
  }
  uint8_t* H = smem;
  uint8_t* W = smem + FF_H_BYTES;
  float* s_bias = reinterpret_cast<float*>(smem + FF_BIAS_OFFSET);
  uint64_t* wfull = reinterpret_cast<uint64_t*>(smem + FF_BAR_OFFSET);
  uint64_t* wempty = wfull + FF_WSTAGES;
  uint64_t* xfull = wempty + FF_WSTAGES;   // the tile's inputs have landed in H's first K block
  uint64_t* accA = xfull + 1;              // N half 0 (region A) accumulated (MMA -> epilogue)
  uint64_t* accB = accA + 1;               // N half 1 (region B) accumulated: the layer's MMAs are done
  uint64_t* hlo = accB + 1;                // H's K blocks 0-3 written, region A drained (epilogue -> MMA)
  uint64_t* hhi = hlo + 1;                 // H's K blocks 4-7 written, region B drained (epilogue -> MMA)
  uint64_t* hfree = hhi + 1;               // the tile's last MMAs have read H (MMA -> producer)
  uint64_t* drain = hfree + 1;             // MMA completion before tensor memory is released (abort)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  int* flags = reinterpret_cast<int*>(tmem_slot + 1);
  volatile int* abort_flag = flags;        // [0] a wait ran out; [1] epilogue verdict; [2] consumed
  int* epi_fail = flags + 1;
  int* consumed_s = flags + 2;             // weight blocks the MMA thread received (for the drain)
  int* x_consumed_s = flags + 3;           // input tiles the MMA thread received

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto wait = [&](uint64_t* bar, uint32_t parity) -> bool {
    if (*abort_flag) return false;
    const uint32_t addr = smem_u32(bar);
    const long long t0 = clock64();
    while (!mbar_try_wait(addr, parity)) {
      if (*abort_flag) return false;
      if (clock64() - t0 > wait_limit) {
        *abort_flag = 1;
        return false;
      }
    }
    return true;
  };

  // the same, sleeping between polls: for the producer, whose polls otherwise take issue slots and
  // barrier accesses from the MMA thread (~2%)
  auto wait_sleep = [&](uint64_t* bar, uint32_t parity) -> bool {
    if (*abort_flag) return false;
    const uint32_t addr = smem_u32(bar);
    const long long t0 = clock64();
    while (!mbar_try_wait(addr, parity)) {
      if (*abort_flag) return false;
      if (clock64() - t0 > wait_limit) {
        *abort_flag = 1;
        return false;
      }
      __nanosleep(32);
    }
    return true;
  };

  if (threadIdx.x == 0) {
    tma_prefetch_desc(&tma_x);
    for (int s = 0; s < FF_WSTAGES; ++s) {
      mbar_init(&wfull[s], 1);
      mbar_init(&wempty[s], 1);
    }
    mbar_init(xfull, 1);
    mbar_init(accA, 1);
    mbar_init(accB, 1);
    mbar_init(hlo, FF_EPI_WARPS);
    mbar_init(hhi, FF_EPI_WARPS);
    mbar_init(hfree, 1);
    mbar_init(drain, 1);
    flags[0] = flags[1] = flags[2] = flags[3] = 0;
    mbar_fence_init();
  }
  __syncwarp();
  if (warp == 1) tmem_alloc(tmem_slot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool late = false;
  int issued = 0, x_issued = 0;

  if (warp == 0) {
    // ---- producer: the tile's inputs, then its 58 weight blocks in the order the MMAs use them ----
    if (lane == 0) {
      int it = 0, local = 0;
      for (int tile = blockIdx.x; tile < m_tiles; tile += gridDim.x, ++local) {
        if (local > 0 && !wait(hfree, (local - 1) & 1)) {   // the previous tile's MMAs are done with H
          late = true;
          break;
        }
        mbar_arrive_expect_tx(xfull, FF_KB_BYTES);
        tma_load_2d(H, &tma_x, 0, tile * BM, xfull);
        ++x_issued;
        bool stop = false;
        for (int i = 0; i < FF_STAGES_PER_TILE; ++i, ++it) {
          const int s = it % FF_WSTAGES;
          if (!wait_sleep(&wempty[s], ((it / FF_WSTAGES) & 1) ^ 1)) {
            stop = true;
            break;
          }
          const FfBlock blk = ff_block(i);
          const CUtensorMap* map = blk.layer == 0 ? &tma_w1 : blk.layer == 1 ? &tma_w2 : blk.layer == 2 ? &tma_w3
                                   : blk.layer == 3 ? &tma_w4 : &tma_w5;
          mbar_arrive_expect_tx(&wfull[s], blk.rows * BK * 2);
          tma_load_2d(W + s * FF_WSTAGE_BYTES, map, blk.kb * BK, blk.n0, &wfull[s]);
        }
        if (stop) {
          late = true;
          break;
        }
      }
      issued = it;
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---- MMA issue (one thread) ----
    if (lane == 0) {
      constexpr uint32_t idesc256 = bf16_idesc(BM, 256);
      constexpr uint32_t idesc128 = bf16_idesc(BM, OUT_PAD);
      int it = 0, local = 0, lo_waits = 0, hi_waits = 0, xs = 0;
      const uint32_t h_addr = smem_u32(H);
      // the four MMAs of weight block i of the tile's stream (ring slot it % 3): A = H's K block
      auto stage = [&](int i, uint32_t d, uint32_t idesc) -> bool {
        const int s = it % FF_WSTAGES;
        if (!wait(&wfull[s], (it / FF_WSTAGES) & 1)) return false;
        tc_fence_after();
        const FfBlock blk = ff_block(i);
        const uint32_t w_addr = smem_u32(W + s * FF_WSTAGE_BYTES);
        const uint32_t a_addr = h_addr + blk.kb * FF_KB_BYTES;
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk)
          umma_bf16(d, sw128_kmajor_desc(a_addr + kk * 32), sw128_kmajor_desc(w_addr + kk * 32), idesc,
                    (blk.kb | kk) != 0);
        umma_commit(&wempty[s]);
        ++it;
        return true;
      };
      for (int tile = blockIdx.x; tile < m_tiles && !late; tile += gridDim.x, ++local) {
        if (!wait(xfull, local & 1)) {
          late = true;
          break;
        }
        ++xs;
        int i = 0;
        for (int layer = 0; layer < GF_MLP_LAYERS; ++layer) {
          // region A drained (by the previous layer's staging copy, or the previous tile's output) and,
          // from the second layer on, H's K blocks 0-3 written
          if (local > 0 || layer > 0) {
            if (!wait(hlo, lo_waits & 1)) {
              late = true;
              break;
            }
            ++lo_waits;
          }
          tc_fence_after();
          const int kblocks = layer == 0 ? 1 : 8;
          // N half 0 (the output layer's only N tile) into region A; K blocks 4-7 once H's K blocks 4-7
          // are written (which also means region B is drained)
          for (int kb = 0; kb < kblocks && !late; ++kb, ++i) {
            if (kb == 4) {
              if (!wait(hhi, hi_waits & 1)) {
                late = true;
                break;
              }
              ++hi_waits;
              tc_fence_after();
            }
            if (!stage(i, tmem, layer == 4 ? idesc128 : idesc256)) late = true;
          }
          if (late) break;
          // fault injection for tests: withhold the first accumulator hand-off
          if (!((inject & 1) && local == 0 && layer == 0)) umma_commit(accA);
          if (layer < 4) {
            // N half 1 into region B, while the epilogue drains region A
            for (int kb = 0; kb < kblocks && !late; ++kb, ++i)
              if (!stage(i, tmem + 256, idesc256)) late = true;
            if (late) break;
            umma_commit(accB);   // also: every MMA of the layer has read H
          }
        }
        if (late) break;
        umma_commit(hfree);
      }
      *consumed_s = it;
      *x_consumed_s = xs;
    }
    __syncwarp();
  } else {
    // ---- epilogue: lane quarter qd of tensor memory, column group cg of each N half ----
    // A hidden layer's N half 0 (region A, tensor-memory columns 0-255) is drained while the MMAs of
    // N half 1 run: bias + GELU, rounded to bf16 pairs and stored back into the first half of the
    // warp's own region-A columns (H is still being read).  Once every MMA of the layer is done, the
    // staged half is copied into H's K blocks 0-3, which releases region A and lets the next layer's
    // MMAs start on K blocks 0-3 while N half 1 (region B) is drained straight into K blocks 4-7.
    const int qd = warp & 3;
    const int cg = (warp - 2) >> 2;
    const int r = qd * 32 + lane;                 // row within the tile
    float* s_out = reinterpret_cast<float*>(H + FF_KB_BYTES);   // the last layer's staged outputs
    const uint32_t tlane = tmem + (static_cast<uint32_t>(qd * 32) << 16);
    int a_waits = 0, b_waits = 0;
    // one thread waits for the MMA hand-off (sixteen pollers of the same barrier slow the MMAs down by
    // ~5%); every epilogue warp then learns the verdict at the named barrier
    auto handoff = [&](uint64_t* bar, int& n, bool store_read) -> bool {
      if (threadIdx.x == kFfPollThread && !mbar_wait_sleep(bar, n & 1, wait_limit)) atomicOr(epi_fail, 1);
      ++n;
      // the previous tile's output store has read its staging rows before this tile writes H
      if (store_read && threadIdx.x == kFfStoreThread) bulk_wait_read<0>();
      named_barrier_sync(4, 32 * FF_EPI_WARPS);
      if (*reinterpret_cast<volatile int*>(epi_fail)) return false;
      __syncwarp();
      tc_fence_after();
      return true;
    };
    // bias + GELU of the 32 accumulator columns at tensor-memory column tcol (output columns c0 ..
    // c0 + 31), rounded to 16 bf16 pairs
    auto gelu_pack = [&](uint32_t tcol, int c0, uint32_t (&w)[16]) {
      float v[32];
      tmem_ld_32cols(tlane + tcol, v);
      const float4* b4v = reinterpret_cast<const float4*>(s_bias + c0);
#pragma unroll
      for (int q4 = 0; q4 < 8; ++q4) {
        const float4 bb = b4v[q4];
        v[4 * q4] = gelu(v[4 * q4] + bb.x);
        v[4 * q4 + 1] = gelu(v[4 * q4 + 1] + bb.y);
        v[4 * q4 + 2] = gelu(v[4 * q4 + 2] + bb.z);
        v[4 * q4 + 3] = gelu(v[4 * q4 + 3] + bb.w);
      }
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        __nv_bfloat162 pr = __floats2bfloat162_rn(v[2 * t], v[2 * t + 1]);
        w[t] = *reinterpret_cast<uint32_t*>(&pr);
      }
    };
    // row r, output columns c0 .. c0+31 of H: K block c0 / 64, 16-byte units (c0 % 64) / 8 + q, placed
    // at unit ^ (r % 8) of the row (128-byte swizzle)
    auto store_h = [&](int c0, const uint32_t (&w)[16]) {
      uint8_t* rowp = H + (c0 >> 6) * FF_KB_BYTES + r * 128;
      const int u0 = (c0 & 63) >> 3;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        *reinterpret_cast<uint4*>(rowp + (((u0 + q) ^ (r & 7)) << 4)) =
            make_uint4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]);
    };
    for (int tile = blockIdx.x; tile < m_tiles; tile += gridDim.x) {
      bool stop = false;
      for (int layer = 0; layer < GF_MLP_LAYERS; ++layer) {
        // the layer's bias into shared memory while its MMAs run (every epilogue warp passed the
        // barrier at the end of the previous layer, so the buffer is free)
        {
          const float* bias = layer == 0 ? b1 : layer == 1 ? b2 : layer == 2 ? b3 : layer == 3 ? b4 : b5;
          const int nb = layer < 4 ? HID : OUT_PAD;
          const int et = threadIdx.x - 64;
          if (et < nb) s_bias[et] = __ldg(bias + et);
        }
        if (!handoff(accA, a_waits, false)) {
          stop = true;
          break;
        }
        if (layer < 4) {
          // N half 0: output columns cg*64 .. cg*64+63, staged as bf16 pairs in tensor-memory columns
          // cg*64 .. cg*64+31 (each chunk's pairs land on columns this warp has already read)
#pragma unroll 1
          for (int h = 0; h < 2; ++h) {
            uint32_t w[16];
            gelu_pack(cg * 64 + 32 * h, cg * 64 + 32 * h, w);
            tmem_st_16cols(tlane + cg * 64 + 16 * h, w);
          }
          tmem_st_wait();
          if (!handoff(accB, b_waits, layer == 0)) {   // every MMA of the layer is done with H
            stop = true;
            break;
          }
          {
            float v[32];
            tmem_ld_32cols(tlane + cg * 64, v);
            uint32_t w0[16], w1[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              w0[j] = __float_as_uint(v[j]);
              w1[j] = __float_as_uint(v[16 + j]);
            }
            store_h(cg * 64, w0);
            store_h(cg * 64 + 32, w1);
          }
          fence_proxy_async_smem();   // H is read by the tensor cores (async proxy)
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(hlo);   // H's K blocks 0-3 written, region A drained
          // N half 1: output columns 256 + cg*64 .. +63 straight into H's K block 4 + cg
#pragma unroll 1
          for (int h = 0; h < 2; ++h) {
            uint32_t w[16];
            const int c0 = 256 + cg * 64 + 32 * h;
            gelu_pack(c0, c0, w);
            store_h(c0, w);
          }
          fence_proxy_async_smem();
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(hhi);   // H's K blocks 4-7 written, region B drained
        } else {
          // layer 5: 128 padded outputs, one 32-column chunk per warp.  The first 99 of each row are
          // staged in H's K blocks 1-4 (row stride 99 words: the lanes' rows fall in distinct banks), and
          // the tile's rows, one contiguous span of the caller's [batch][99] array, leave in one bulk
          // store.  K block 0 may already be receiving the next tile's inputs; blocks 1-7 are next
          // written by the next tile's first epilogue, which waits until this store has read them.
          const int c0 = cg * 32;
          float v[32];
          tmem_ld_32cols(tlane + c0, v);
          float* o = s_out + r * GF_MLP_OUTPUTS;
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (c0 + j < GF_MLP_OUTPUTS) o[c0 + j] = v[j] + s_bias[c0 + j];
          fence_proxy_async_smem();   // the staged rows are read by the bulk copy (async proxy)
          tc_fence_before();
          named_barrier_sync(4, 32 * FF_EPI_WARPS);   // every row is staged
          if (threadIdx.x == kFfStoreThread) {
            // batch is a multiple of 128 (checked by the caller): the tile's rows are all in range
            bulk_store_1d(out + static_cast<long long>(tile) * BM * GF_MLP_OUTPUTS, s_out,
                          BM * GF_MLP_OUTPUTS * 4);
            bulk_commit();
          }
          if (lane == 0) mbar_arrive(hlo);   // region A drained: the next tile's first MMAs may write it
        }
        named_barrier_sync(4, 32 * FF_EPI_WARPS);   // every warp is done with s_bias before it is refilled
      }
      if (stop) {
        late = true;
        break;
      }
    }
    if (threadIdx.x == kFfStoreThread) bulk_wait_all();   // the outputs are written before the CTA exits
  }

  tc_fence_before();
  if (late) *abort_flag = 1;
  __syncthreads();
  if (*abort_flag) {
    // a wait ran out: every load and MMA this CTA issued completes before its shared and tensor memory
    // are released (each wait again bounded)
    if (threadIdx.x == 0) {
      for (int it = *consumed_s; it < issued; ++it)
        mbar_wait(&wfull[it % FF_WSTAGES], (it / FF_WSTAGES) & 1, wait_limit);
      for (int x = *x_consumed_s; x < x_issued; ++x) mbar_wait(xfull, x & 1, wait_limit);
      if (fault) atomicOr(fault, 1);
    } else if (threadIdx.x == 32) {
      umma_commit(drain);
      mbar_wait(drain, 0, wait_limit);
    }
    __syncthreads();
  }
  if (warp == 1) tmem_dealloc(tmem, 512);
}

// ---------------------------------------------------------------------------------------------
// small kernels
// ---------------------------------------------------------------------------------------------

// Inputs [batch][6] fp32 -> X0 [cap][64] bf16 (one 16-byte store of columns 0..7 per row; columns
// 8..63 stay zero) and, for training, X0^T [64][cap].
__global__ void encode_inputs_kernel(const float* __restrict__ x, int batch, __nv_bfloat16* __restrict__ x0,
                                     __nv_bfloat16* __restrict__ x0t, long long cap, int transposed) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  float v[8];
#pragma unroll
  for (int j = 0; j < GF_MLP_INPUTS; ++j) v[j] = x[b * GF_MLP_INPUTS + j];
  v[6] = 0.f;
  v[7] = 0.f;
  uint32_t w[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    __nv_bfloat162 p = __floats2bfloat162_rn(v[2 * t], v[2 * t + 1]);
    w[t] = *reinterpret_cast<uint32_t*>(&p);
  }
  *reinterpret_cast<uint4*>(x0 + static_cast<long long>(b) * IN_PAD) = make_uint4(w[0], w[1], w[2], w[3]);
  if (transposed) {
#pragma unroll
    for (int j = 0; j < GF_MLP_INPUTS; ++j) x0t[j * cap + b] = __float2bfloat16_rn(v[j]);
  }
}

// Squared-error loss of one 128-row tile and its gradient: dOut = 2 (out - target) / (batch * 99),
// written row-major and transposed in bf16, with the tile's column sums (bias gradient of layer 5)
// and loss sum.  One block of 128 threads per tile; thread = row for the gradient, thread = column
// for the column sums (recomputed, same expression, fixed row order).
__global__ void __launch_bounds__(128)
loss_kernel(const float* __restrict__ out, const float* __restrict__ target, int batch,
            __nv_bfloat16* __restrict__ dout, __nv_bfloat16* __restrict__ doutt, long long cap,
            float* __restrict__ bias_part, float* __restrict__ loss_part) {
  __shared__ float rl[BM];
  const int r = threadIdx.x;
  const int row0 = blockIdx.x * BM;
  const int row = row0 + r;
  const float scale = 2.f / (static_cast<float>(batch) * GF_MLP_OUTPUTS);
  float l = 0.f;
  for (int j = 0; j < GF_MLP_OUTPUTS; ++j) {
    const float d = out[row * OUT_PAD + j] - target[row * GF_MLP_OUTPUTS + j];
    l += d * d;
    const __nv_bfloat16 b = __float2bfloat16_rn(scale * d);
    dout[row * OUT_PAD + j] = b;
    doutt[j * cap + row] = b;
  }
  rl[r] = l;
  if (r < GF_MLP_OUTPUTS) {
    float s = 0.f;
    for (int i = 0; i < BM; ++i) s += scale * (out[(row0 + i) * OUT_PAD + r] - target[(row0 + i) * GF_MLP_OUTPUTS + r]);
    bias_part[blockIdx.x * OUT_PAD + r] = s;
  }
  __syncthreads();
  if (r == 0) {
    float s = 0.f;
    for (int i = 0; i < BM; ++i) s += rl[i];
    loss_part[blockIdx.x] = s / (static_cast<float>(batch) * GF_MLP_OUTPUTS);
  }
}

__global__ void loss_finish_kernel(const float* __restrict__ loss_part, int tiles, float* __restrict__ loss) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    float s = 0.f;
    for (int i = 0; i < tiles; ++i) s += loss_part[i];
    *loss = s;
  }
}

// One parameter tensor (padded shape rows x cols) and where its gradient partials are.
struct ParamSlot {
  float* w;
  float* m;
  float* v;
  float* g;
  __nv_bfloat16* wb;     // bf16 copy [rows][cols] (weights only)
  __nv_bfloat16* wt;     // bf16 transposed copy [cols][rows] (weights only)
  const float* part;     // gradient partials
  long long part_stride;
  int nparts;
  int rows, cols, rows_true, cols_true;
  long long offset;      // first element in the concatenated index space
};

struct ParamTable {
  ParamSlot s[2 * GF_MLP_LAYERS];
  long long total;
};

__device__ __forceinline__ int find_slot(const ParamTable& t, long long i) {
  int k = 0;
#pragma unroll 1
  while (k + 1 < 2 * GF_MLP_LAYERS && t.s[k + 1].offset <= i) ++k;
  return k;
}

// g = sum of the partials in a fixed order.
__global__ void reduce_grads_kernel(const __grid_constant__ ParamTable t) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < t.total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const ParamSlot& p = t.s[find_slot(t, i)];
    const long long e = i - p.offset;
    float acc = 0.f;
    for (int k = 0; k < p.nparts; ++k) acc += p.part[k * p.part_stride + e];
    p.g[e] = acc;
  }
}

// Adam (with optional decoupled weight decay) on the master weights, then the bf16 copies.
__global__ void adam_kernel(const __grid_constant__ ParamTable t, float lr, float beta1, float beta2, float eps,
                            float bc1, float bc2, float decay) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < t.total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const ParamSlot& p = t.s[find_slot(t, i)];
    const long long e = i - p.offset;
    const int r = static_cast<int>(e / p.cols), c = static_cast<int>(e % p.cols);
    if (r >= p.rows_true || c >= p.cols_true) continue;
    const float g = p.g[e];
    const float m = beta1 * p.m[e] + (1.f - beta1) * g;
    const float v = beta2 * p.v[e] + (1.f - beta2) * g * g;
    p.m[e] = m;
    p.v[e] = v;
    float w = p.w[e];
    w -= lr * decay * w;
    w -= lr * (m / bc1) / (sqrtf(v / bc2) + eps);
    p.w[e] = w;
    if (p.wb) {
      const __nv_bfloat16 b = __float2bfloat16_rn(w);
      p.wb[e] = b;
      p.wt[static_cast<long long>(c) * p.rows + r] = b;
    }
  }
}

// bf16 copies of the master weights (after set_params).
__global__ void refresh_bf16_kernel(const __grid_constant__ ParamTable t) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < t.total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const ParamSlot& p = t.s[find_slot(t, i)];
    if (!p.wb) continue;
    const long long e = i - p.offset;
    const int r = static_cast<int>(e / p.cols), c = static_cast<int>(e % p.cols);
    const __nv_bfloat16 b = __float2bfloat16_rn(p.w[e]);
    p.wb[e] = b;
    p.wt[static_cast<long long>(c) * p.rows + r] = b;
  }
}


// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// Operand map: row-major bf16 [rows][cols] (cols contiguous), box box_rows x 64, 128-byte swizzle
// (the layout the UMMA matrix descriptors name).
bool make_map(CUtensorMap* m, const void* base, long long rows, long long cols, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(cols) * 2};
  cuuint32_t box[2] = {static_cast<cuuint32_t>(BK), static_cast<cuuint32_t>(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Output map of a row-major [rows][cols] matrix with 32 x 32 boxes, in the staging layout of the
// epilogue: fp32 with the 128-byte swizzle, bf16 with the 64-byte swizzle, or (transposed outputs) bf16
// unswizzled.
enum OutKind { OUT_F32 = 0, OUT_BF16 = 1, OUT_BF16_T = 2 };
bool make_out_map(CUtensorMap* m, const void* base, long long rows, long long cols, OutKind kind) {
  auto fn = encode_fn();
  if (!fn) return false;
  const int esize = kind == OUT_F32 ? 4 : 2;
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(cols), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(cols) * esize};
  cuuint32_t box[2] = {32, 32};
  cuuint32_t estr[2] = {1, 1};
  const CUtensorMapSwizzle sw = kind == OUT_F32    ? CU_TENSOR_MAP_SWIZZLE_128B
                                : kind == OUT_BF16 ? CU_TENSOR_MAP_SWIZZLE_64B
                                                   : CU_TENSOR_MAP_SWIZZLE_NONE;
  return fn(m, kind == OUT_F32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
            const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// SM count of the current device (cached per device)
int sm_count() {
  static std::atomic<int> counts[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 148;
  if (counts[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) {
      cudaGetLastError();
      n = 148;
    }
    counts[dev] = n;
  }
  return counts[dev];
}

// Outputs the epilogue does not write get the A map in their slot (never used).
template <int BN, int EPI>
cudaError_t launch_gemm(const CUtensorMap& a, const CUtensorMap& b, const CUtensorMap* c, const CUtensorMap* y,
                        const CUtensorMap* yt, int M, int N, int K, int splits, const EpiArgs& ep,
                        cudaStream_t stream, int inject = 0) {
  static std::atomic<bool> attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_set[dev]) {
    cudaError_t err = cudaFuncSetAttribute(umma_gemm_kernel<BN, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           Smem<BN, EPI>::BYTES);
    if (err != cudaSuccess) return err;
    attr_set[dev] = true;
  }
  const int m_tiles = M / BM, n_tiles = N / BN;
  const int tiles = m_tiles * n_tiles * splits;
  const int grid = tiles < sm_count() ? tiles : sm_count();
  umma_gemm_kernel<BN, EPI><<<grid, GEMM_THREADS, Smem<BN, EPI>::BYTES, stream>>>(
      a, b, c ? *c : a, y ? *y : a, yt ? *yt : a, m_tiles, n_tiles, splits, K / BK / splits, ep,
      inject ? INJECT_WAIT_LIMIT : WAIT_LIMIT, inject);
  return cudaGetLastError();
}

cudaError_t launch_fused_forward(const CUtensorMap& x, const CUtensorMap* w256, const CUtensorMap& w5,
                                 float* const* bias, float* out, int batch, cudaStream_t stream, int inject,
                                 int* fault) {
  static std::atomic<bool> attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_set[dev]) {
    cudaError_t err = cudaFuncSetAttribute(fused_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, FF_SMEM);
    if (err != cudaSuccess) return err;
    attr_set[dev] = true;
  }
  const int m_tiles = batch / BM;
  const int grid = m_tiles < sm_count() ? m_tiles : sm_count();
  fused_forward_kernel<<<grid, FF_THREADS, FF_SMEM, stream>>>(
      x, w256[0], w256[1], w256[2], w256[3], w5, bias[0], bias[1], bias[2], bias[3], bias[4], out, batch, m_tiles,
      inject ? INJECT_WAIT_LIMIT : WAIT_LIMIT, inject, fault);
  return cudaGetLastError();
}

// Split count for a weight-gradient GEMM: enough CTAs to cover the SMs, each split a whole number
// of 64-wide K blocks.
int choose_splits(int tiles, int K) {
  const int kblocks = K / BK;
  int s = 1;
  while (s < MAX_SPLITS && tiles * s < 148 && kblocks % (2 * s) == 0 && kblocks / (2 * s) >= 2) s *= 2;
  return s;
}

}  // namespace gfm

using namespace gfm;

struct gf_mlp {
  int device = 0;
  cudaStream_t stream = nullptr;
  gf_mlp_config cfg{};
  long long cap = 0;
  long long step = 0;
  std::string error;

  // layer geometry (padded): out x in
  int rows[GF_MLP_LAYERS] = {HID, HID, HID, HID, OUT_PAD};
  int cols[GF_MLP_LAYERS] = {IN_PAD, HID, HID, HID, HID};
  int rows_true[GF_MLP_LAYERS] = {HID, HID, HID, HID, GF_MLP_OUTPUTS};
  int cols_true[GF_MLP_LAYERS] = {GF_MLP_INPUTS, HID, HID, HID, HID};

  // parameters (fp32 master, Adam moments, gradient) -- one allocation each, weights then biases
  float* w[GF_MLP_LAYERS] = {};
  float* b[GF_MLP_LAYERS] = {};
  float* m_all = nullptr;
  float* v_all = nullptr;
  float* g_all = nullptr;
  float* w_all = nullptr;
  __nv_bfloat16* wb[GF_MLP_LAYERS] = {};
  __nv_bfloat16* wt[GF_MLP_LAYERS] = {};
  long long off_w[GF_MLP_LAYERS] = {}, off_b[GF_MLP_LAYERS] = {};
  long long n_params_padded = 0;

  // activations
  __nv_bfloat16 *x0 = nullptr, *x0t = nullptr;
  float* z[4] = {};
  __nv_bfloat16 *y[4] = {}, *yt[4] = {};
  float* out = nullptr;
  __nv_bfloat16 *dout = nullptr, *doutt = nullptr;
  __nv_bfloat16 *dz[4] = {}, *dzt[4] = {};
  float* wpart[GF_MLP_LAYERS] = {};
  float* bpart[GF_MLP_LAYERS] = {};
  int wsplits[GF_MLP_LAYERS] = {};
  float* loss_part = nullptr;
  float* loss = nullptr;
  int* fault = nullptr;

  // tensor maps
  CUtensorMap fwd_a[GF_MLP_LAYERS], fwd_b[GF_MLP_LAYERS];     // A = input activations, B = W
  CUtensorMap fwd_b256[4];                                    // B = W in 256-row boxes (inference tiles)
  CUtensorMap bwd_a[GF_MLP_LAYERS], bwd_b[GF_MLP_LAYERS];     // A = dZ_l (dOut), B = W_l^T  (l >= 2)
  CUtensorMap dw_a[GF_MLP_LAYERS], dw_b[GF_MLP_LAYERS];       // A = dZ_l^T, B = Y_{l-1}^T
  CUtensorMap out_z[4], out_y[4], out_yt[4];                  // forward outputs of the hidden layers
  CUtensorMap out_final;                                      // layer-5 output (fp32)
  CUtensorMap out_dz[4], out_dzt[4];                          // backward outputs dZ, dZ^T
  CUtensorMap out_wpart[GF_MLP_LAYERS];                       // split-K weight-gradient slices

  std::vector<void*> allocations;
  int inject = 0;   // fault injection armed for the next forward pass (tests)
  int fused = 1;    // inference runs the fused five-layer kernel (0: one GEMM per layer)
};

namespace {

gf_status mlp_fail(gf_mlp* m, gf_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (m) m->error = buf;
  return st;
}

#define MLP_CUDA(m, call)                                                                         \
  do {                                                                                            \
    cudaError_t _e = (call);                                                                      \
    if (_e != cudaSuccess) return mlp_fail((m), GF_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e)); \
  } while (0)

template <class T>
gf_status alloc(gf_mlp* m, T** p, long long count) {
  void* q = nullptr;
  if (cudaMalloc(&q, static_cast<size_t>(count) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    return mlp_fail(m, GF_ERR_OUT_OF_MEMORY, "device allocation of %lld bytes failed",
                    static_cast<long long>(count * sizeof(T)));
  }
  m->allocations.push_back(q);
  *p = static_cast<T*>(q);
  if (cudaMemsetAsync(q, 0, static_cast<size_t>(count) * sizeof(T), m->stream) != cudaSuccess)
    return mlp_fail(m, GF_ERR_CUDA, "memset failed");
  return GF_OK;
}

ParamTable param_table(gf_mlp* m, int batch) {
  ParamTable t{};
  long long off = 0;
  for (int l = 0; l < GF_MLP_LAYERS; ++l) {
    ParamSlot& s = t.s[l];
    s.w = m->w[l];
    s.m = m->m_all + m->off_w[l];
    s.v = m->v_all + m->off_w[l];
    s.g = m->g_all + m->off_w[l];
    s.wb = m->wb[l];
    s.wt = m->wt[l];
    s.part = m->wpart[l];
    s.part_stride = static_cast<long long>(m->rows[l]) * m->cols[l];
    s.nparts = m->wsplits[l];
    s.rows = m->rows[l];
    s.cols = m->cols[l];
    s.rows_true = m->rows_true[l];
    s.cols_true = m->cols_true[l];
    s.offset = off;
    off += s.part_stride;
  }
  for (int l = 0; l < GF_MLP_LAYERS; ++l) {
    ParamSlot& s = t.s[GF_MLP_LAYERS + l];
    s.w = m->b[l];
    s.m = m->m_all + m->off_b[l];
    s.v = m->v_all + m->off_b[l];
    s.g = m->g_all + m->off_b[l];
    s.wb = nullptr;
    s.wt = nullptr;
    s.part = m->bpart[l];
    s.part_stride = m->rows[l];
    s.nparts = batch / BM;
    s.rows = 1;
    s.cols = m->rows[l];
    s.rows_true = 1;
    s.cols_true = m->rows_true[l];
    s.offset = off;
    off += m->rows[l];
  }
  t.total = off;
  return t;
}

gf_status check_batch(gf_mlp* m, int batch) {
  if (batch <= 0 || batch % BM != 0 || batch > m->cap)
    return mlp_fail(m, GF_ERR_INVALID_ARGUMENT, "batch %d must be a positive multiple of %d and at most %lld",
                    batch, BM, m->cap);
  return GF_OK;
}

// Forward pass.  Training writes Z, Y, Y^T and the padded fp32 output; inference (d_out != nullptr)
// writes Y only, on 128 x 256 tiles, and the last layer writes the caller's [batch][99] array.
gf_status run_forward(gf_mlp* m, const float* d_inputs, int batch, bool train, float* d_out = nullptr) {
  encode_inputs_kernel<<<(batch + 255) / 256, 256, 0, m->stream>>>(d_inputs, batch, m->x0, m->x0t, m->cap,
                                                                  train ? 1 : 0);
  MLP_CUDA(m, cudaGetLastError());
  if (!train && m->fused) {
    cudaError_t err = launch_fused_forward(m->fwd_a[0], m->fwd_b256, m->fwd_b[4], m->b, d_out, batch, m->stream,
                                           m->inject, m->fault);
    m->inject = 0;
    if (err != cudaSuccess) return mlp_fail(m, GF_ERR_CUDA, "fused forward: %s", cudaGetErrorString(err));
    return GF_OK;
  }
  for (int l = 0; l < GF_MLP_LAYERS; ++l) {
    EpiArgs ep{};
    ep.bias = m->b[l];
    ep.fault = m->fault;
    cudaError_t err;
    if (l < 4) {
      err = train ? launch_gemm<128, EPI_FWD_GELU>(m->fwd_a[l], m->fwd_b[l], &m->out_z[l], &m->out_y[l],
                                                   &m->out_yt[l], batch, HID, m->cols[l], 1, ep, m->stream)
                  : launch_gemm<256, EPI_FWD_GELU_INFER>(m->fwd_a[l], m->fwd_b256[l], nullptr, &m->out_y[l],
                                                         nullptr, batch, HID, m->cols[l], 1, ep, m->stream,
                                                         l == 0 ? m->inject : 0);
      if (l == 0) m->inject = 0;
    } else if (train) {
      err = launch_gemm<128, EPI_FWD_LINEAR>(m->fwd_a[l], m->fwd_b[l], &m->out_final, nullptr, nullptr, batch,
                                             OUT_PAD, HID, 1, ep, m->stream);
    } else {
      ep.out = d_out;
      ep.out_cols = GF_MLP_OUTPUTS;
      err = launch_gemm<128, EPI_FWD_OUT>(m->fwd_a[l], m->fwd_b[l], nullptr, nullptr, nullptr, batch, OUT_PAD, HID,
                                          1, ep, m->stream);
    }
    if (err != cudaSuccess) return mlp_fail(m, GF_ERR_CUDA, "forward GEMM %d: %s", l + 1, cudaGetErrorString(err));
  }
  return GF_OK;
}

gf_status run_backward(gf_mlp* m, const float* d_targets, int batch) {
  const int tiles = batch / BM;
  loss_kernel<<<tiles, BM, 0, m->stream>>>(m->out, d_targets, batch, m->dout, m->doutt, m->cap, m->bpart[4],
                                          m->loss_part);
  MLP_CUDA(m, cudaGetLastError());
  loss_finish_kernel<<<1, 32, 0, m->stream>>>(m->loss_part, tiles, m->loss);
  MLP_CUDA(m, cudaGetLastError());
  for (int l = GF_MLP_LAYERS - 1; l >= 0; --l) {
    // weight gradient partials of layer l+1
    {
      EpiArgs ep{};
      ep.rows_per_split = m->rows[l];
      ep.fault = m->fault;
      const int M = m->rows[l], N = m->cols[l];
      const int bn = (N % 128 == 0) ? 128 : 64;
      const int splits = choose_splits((M / BM) * (N / bn), batch);
      m->wsplits[l] = splits;
      cudaError_t err = bn == 128
          ? launch_gemm<128, EPI_PARTIAL>(m->dw_a[l], m->dw_b[l], &m->out_wpart[l], nullptr, nullptr, M, N, batch,
                                          splits, ep, m->stream)
          : launch_gemm<64, EPI_PARTIAL>(m->dw_a[l], m->dw_b[l], &m->out_wpart[l], nullptr, nullptr, M, N, batch,
                                         splits, ep, m->stream);
      if (err != cudaSuccess)
        return mlp_fail(m, GF_ERR_CUDA, "weight-gradient GEMM %d: %s", l + 1, cudaGetErrorString(err));
    }
    if (l == 0) break;
    // input gradient of layer l+1 = output gradient of layer l, times GELU'(Z_l)
    EpiArgs ep{};
    ep.z = m->z[l - 1];
    ep.ldz = HID;
    ep.bias_part = m->bpart[l - 1];
    ep.ld_bias_part = HID;
    ep.fault = m->fault;
    cudaError_t err = launch_gemm<128, EPI_BWD_GELU>(m->bwd_a[l], m->bwd_b[l], nullptr, &m->out_dz[l - 1],
                                                    &m->out_dzt[l - 1], batch, HID, m->rows[l], 1, ep, m->stream);
    if (err != cudaSuccess)
      return mlp_fail(m, GF_ERR_CUDA, "input-gradient GEMM %d: %s", l + 1, cudaGetErrorString(err));
  }
  ParamTable t = param_table(m, batch);
  reduce_grads_kernel<<<2 * 148, 256, 0, m->stream>>>(t);
  MLP_CUDA(m, cudaGetLastError());
  return GF_OK;
}

}  // namespace

extern "C" {

int64_t gf_mlp_param_count(void) {
  int64_t n = 0;
  const int r[GF_MLP_LAYERS] = {HID, HID, HID, HID, GF_MLP_OUTPUTS};
  const int c[GF_MLP_LAYERS] = {GF_MLP_INPUTS, HID, HID, HID, HID};
  for (int l = 0; l < GF_MLP_LAYERS; ++l) n += static_cast<int64_t>(r[l]) * c[l] + r[l];
  return n;
}

const char* gf_mlp_last_error(const gf_mlp* mlp) { return mlp ? mlp->error.c_str() : "null network"; }

gf_status gf_mlp_create(int32_t device, void* stream, const gf_mlp_config* config, gf_mlp** out) {
  if (!out || !config) return GF_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return GF_ERR_NO_DEVICE;
  }
  if (config->batch_capacity <= 0 || config->batch_capacity % BM != 0) return GF_ERR_INVALID_ARGUMENT;
  if (!encode_fn()) return GF_ERR_CUDA;
  auto* m = new (std::nothrow) gf_mlp();
  if (!m) return GF_ERR_OUT_OF_MEMORY;
  m->device = device;
  m->cfg = *config;
  m->cap = config->batch_capacity;
  if (cudaSetDevice(device) != cudaSuccess) {
    delete m;
    return GF_ERR_CUDA;
  }
  m->stream = static_cast<cudaStream_t>(stream);
  gf_status st = GF_OK;
#define MLP_TRY(x)            \
  do {                        \
    st = (x);                 \
    if (st != GF_OK) goto bad; \
  } while (0)
  {
    long long off = 0;
    for (int l = 0; l < GF_MLP_LAYERS; ++l) {
      m->off_w[l] = off;
      off += static_cast<long long>(m->rows[l]) * m->cols[l];
    }
    for (int l = 0; l < GF_MLP_LAYERS; ++l) {
      m->off_b[l] = off;
      off += m->rows[l];
    }
    m->n_params_padded = off;
    MLP_TRY(alloc(m, &m->w_all, off));
    MLP_TRY(alloc(m, &m->m_all, off));
    MLP_TRY(alloc(m, &m->v_all, off));
    MLP_TRY(alloc(m, &m->g_all, off));
    for (int l = 0; l < GF_MLP_LAYERS; ++l) {
      m->w[l] = m->w_all + m->off_w[l];
      m->b[l] = m->w_all + m->off_b[l];
      const long long n = static_cast<long long>(m->rows[l]) * m->cols[l];
      MLP_TRY(alloc(m, &m->wb[l], n));
      MLP_TRY(alloc(m, &m->wt[l], n));
      MLP_TRY(alloc(m, &m->wpart[l], n * MAX_SPLITS));
      MLP_TRY(alloc(m, &m->bpart[l], (m->cap / BM) * m->rows[l]));
    }
    const long long cap = m->cap;
    MLP_TRY(alloc(m, &m->x0, cap * IN_PAD));
    MLP_TRY(alloc(m, &m->x0t, cap * IN_PAD));
    for (int l = 0; l < 4; ++l) {
      MLP_TRY(alloc(m, &m->z[l], cap * HID));
      MLP_TRY(alloc(m, &m->y[l], cap * HID));
      MLP_TRY(alloc(m, &m->yt[l], cap * HID));
      MLP_TRY(alloc(m, &m->dz[l], cap * HID));
      MLP_TRY(alloc(m, &m->dzt[l], cap * HID));
    }
    MLP_TRY(alloc(m, &m->out, cap * OUT_PAD));
    MLP_TRY(alloc(m, &m->dout, cap * OUT_PAD));
    MLP_TRY(alloc(m, &m->doutt, cap * OUT_PAD));
    MLP_TRY(alloc(m, &m->loss_part, cap / BM));
    MLP_TRY(alloc(m, &m->loss, 1));
    MLP_TRY(alloc(m, &m->fault, 1));

    bool ok = true;
    for (int l = 0; l < GF_MLP_LAYERS; ++l) {
      const void* in = l == 0 ? static_cast<const void*>(m->x0) : m->y[l - 1];
      const void* in_t = l == 0 ? static_cast<const void*>(m->x0t) : m->yt[l - 1];
      const void* g = l == 4 ? static_cast<const void*>(m->dout) : m->dz[l];
      const void* g_t = l == 4 ? static_cast<const void*>(m->doutt) : m->dzt[l];
      ok = ok && make_map(&m->fwd_a[l], in, cap, m->cols[l], BM);
      ok = ok && make_map(&m->fwd_b[l], m->wb[l], m->rows[l], m->cols[l], 128);
      if (l < 4) ok = ok && make_map(&m->fwd_b256[l], m->wb[l], m->rows[l], m->cols[l], 256);
      if (l > 0) {   // layer 1's input gradient is never formed
        ok = ok && make_map(&m->bwd_a[l], g, cap, m->rows[l], BM);
        ok = ok && make_map(&m->bwd_b[l], m->wt[l], m->cols[l], m->rows[l], 128);
      }
      ok = ok && make_map(&m->dw_a[l], g_t, m->rows[l], cap, BM);
      ok = ok && make_map(&m->dw_b[l], in_t, m->cols[l], cap, m->cols[l] % 128 == 0 ? 128 : 64);
      ok = ok && make_out_map(&m->out_wpart[l], m->wpart[l], static_cast<long long>(MAX_SPLITS) * m->rows[l],
                              m->cols[l], OUT_F32);
    }
    for (int l = 0; l < 4; ++l) {
      ok = ok && make_out_map(&m->out_z[l], m->z[l], cap, HID, OUT_F32);
      ok = ok && make_out_map(&m->out_y[l], m->y[l], cap, HID, OUT_BF16);
      ok = ok && make_out_map(&m->out_yt[l], m->yt[l], HID, cap, OUT_BF16_T);
      ok = ok && make_out_map(&m->out_dz[l], m->dz[l], cap, HID, OUT_BF16);
      ok = ok && make_out_map(&m->out_dzt[l], m->dzt[l], HID, cap, OUT_BF16_T);
    }
    ok = ok && make_out_map(&m->out_final, m->out, cap, OUT_PAD, OUT_F32);
    if (!ok) {
      st = mlp_fail(m, GF_ERR_CUDA, "tensor map encoding failed");
      goto bad;
    }
    if (cudaStreamSynchronize(m->stream) != cudaSuccess) {
      st = GF_ERR_CUDA;
      goto bad;
    }
  }
#undef MLP_TRY
  *out = m;
  return GF_OK;
bad:
  for (void* p : m->allocations) cudaFree(p);
  delete m;
  return st == GF_OK ? GF_ERR_CUDA : st;
}

gf_status gf_mlp_destroy(gf_mlp* mlp) {
  if (!mlp) return GF_OK;
  cudaSetDevice(mlp->device);
  cudaStreamSynchronize(mlp->stream);
  for (void* p : mlp->allocations) cudaFree(p);
  delete mlp;
  return GF_OK;
}

gf_status gf_mlp_set_params(gf_mlp* m, const float* params, int64_t count) {
  if (!m || !params) return GF_ERR_INVALID_ARGUMENT;
  if (count != gf_mlp_param_count())
    return mlp_fail(m, GF_ERR_INVALID_ARGUMENT, "expected %lld parameters, got %lld",
                    static_cast<long long>(gf_mlp_param_count()), static_cast<long long>(count));
  MLP_CUDA(m, cudaSetDevice(m->device));
  std::vector<float> h;
  try {
    h.assign(m->n_params_padded, 0.f);
  } catch (const std::bad_alloc&) {
    return mlp_fail(m, GF_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
  const float* p = params;
  for (int l = 0; l < GF_MLP_LAYERS; ++l) {
    for (int r = 0; r < m->rows_true[l]; ++r)
      for (int c = 0; c < m->cols_true[l]; ++c) h[m->off_w[l] + static_cast<long long>(r) * m->cols[l] + c] = *p++;
    for (int r = 0; r < m->rows_true[l]; ++r) h[m->off_b[l] + r] = *p++;
  }
  MLP_CUDA(m, cudaMemcpyAsync(m->w_all, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, m->stream));
  MLP_CUDA(m, cudaMemsetAsync(m->m_all, 0, h.size() * sizeof(float), m->stream));
  MLP_CUDA(m, cudaMemsetAsync(m->v_all, 0, h.size() * sizeof(float), m->stream));
  ParamTable t = param_table(m, BM);
  refresh_bf16_kernel<<<2 * 148, 256, 0, m->stream>>>(t);
  MLP_CUDA(m, cudaGetLastError());
  MLP_CUDA(m, cudaStreamSynchronize(m->stream));
  m->step = 0;
  return GF_OK;
}

static gf_status unpad_to_host(gf_mlp* m, const float* d_all, float* out) {
  std::vector<float> h;
  try {
    h.resize(m->n_params_padded);
  } catch (const std::bad_alloc&) {
    return mlp_fail(m, GF_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
  MLP_CUDA(m, cudaMemcpyAsync(h.data(), d_all, h.size() * sizeof(float), cudaMemcpyDeviceToHost, m->stream));
  MLP_CUDA(m, cudaStreamSynchronize(m->stream));
  float* p = out;
  for (int l = 0; l < GF_MLP_LAYERS; ++l) {
    for (int r = 0; r < m->rows_true[l]; ++r)
      for (int c = 0; c < m->cols_true[l]; ++c) *p++ = h[m->off_w[l] + static_cast<long long>(r) * m->cols[l] + c];
    for (int r = 0; r < m->rows_true[l]; ++r) *p++ = h[m->off_b[l] + r];
  }
  return GF_OK;
}

gf_status gf_mlp_get_params(gf_mlp* m, float* params, int64_t count) {
  if (!m || !params) return GF_ERR_INVALID_ARGUMENT;
  if (count != gf_mlp_param_count()) return mlp_fail(m, GF_ERR_INVALID_ARGUMENT, "parameter count mismatch");
  MLP_CUDA(m, cudaSetDevice(m->device));
  return unpad_to_host(m, m->w_all, params);
}

gf_status gf_mlp_set_learning_rate(gf_mlp* m, float lr) {
  if (!m || !(lr >= 0.f)) return GF_ERR_INVALID_ARGUMENT;
  m->cfg.lr = lr;
  return GF_OK;
}

gf_status gf_mlp_forward(gf_mlp* m, const float* d_inputs, int32_t batch, float* d_outputs) {
  if (!m || !d_inputs || !d_outputs) return GF_ERR_INVALID_ARGUMENT;
  gf_status st = check_batch(m, batch);
  if (st != GF_OK) return st;
  MLP_CUDA(m, cudaSetDevice(m->device));
  if (reinterpret_cast<uintptr_t>(d_outputs) & 15)
    return mlp_fail(m, GF_ERR_INVALID_ARGUMENT, "d_outputs must be 16-byte aligned");
  return run_forward(m, d_inputs, batch, false, d_outputs);
}

gf_status gf_mlp_gradients(gf_mlp* m, const float* d_inputs, const float* d_targets, int32_t batch, float* grads,
                           float* loss) {
  if (!m || !d_inputs || !d_targets) return GF_ERR_INVALID_ARGUMENT;
  gf_status st = check_batch(m, batch);
  if (st != GF_OK) return st;
  MLP_CUDA(m, cudaSetDevice(m->device));
  if ((st = run_forward(m, d_inputs, batch, true)) != GF_OK) return st;
  if ((st = run_backward(m, d_targets, batch)) != GF_OK) return st;
  if (loss) {
    MLP_CUDA(m, cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->stream));
  }
  if (grads) {
    if ((st = unpad_to_host(m, m->g_all, grads)) != GF_OK) return st;
  }
  MLP_CUDA(m, cudaStreamSynchronize(m->stream));
  return gf_mlp_check(m);
}

gf_status gf_mlp_train_step(gf_mlp* m, const float* d_inputs, const float* d_targets, int32_t batch,
                            float* d_loss) {
  if (!m || !d_inputs || !d_targets) return GF_ERR_INVALID_ARGUMENT;
  gf_status st = check_batch(m, batch);
  if (st != GF_OK) return st;
  MLP_CUDA(m, cudaSetDevice(m->device));
  if ((st = run_forward(m, d_inputs, batch, true)) != GF_OK) return st;
  if ((st = run_backward(m, d_targets, batch)) != GF_OK) return st;
  m->step += 1;
  const double bc1 = 1.0 - std::pow(static_cast<double>(m->cfg.beta1), static_cast<double>(m->step));
  const double bc2 = 1.0 - std::pow(static_cast<double>(m->cfg.beta2), static_cast<double>(m->step));
  ParamTable t = param_table(m, batch);
  adam_kernel<<<2 * 148, 256, 0, m->stream>>>(t, m->cfg.lr, m->cfg.beta1, m->cfg.beta2, m->cfg.eps,
                                             static_cast<float>(bc1), static_cast<float>(bc2), m->cfg.weight_decay);
  MLP_CUDA(m, cudaGetLastError());
  if (d_loss) MLP_CUDA(m, cudaMemcpyAsync(d_loss, m->loss, sizeof(float), cudaMemcpyDeviceToDevice, m->stream));
  return GF_OK;
}

gf_status gf_mlp_check(gf_mlp* m) {
  if (!m) return GF_ERR_INVALID_ARGUMENT;
  MLP_CUDA(m, cudaSetDevice(m->device));
  int f = 0;
  MLP_CUDA(m, cudaMemcpyAsync(&f, m->fault, sizeof(int), cudaMemcpyDeviceToHost, m->stream));
  MLP_CUDA(m, cudaStreamSynchronize(m->stream));
  if (f) {
    MLP_CUDA(m, cudaMemsetAsync(m->fault, 0, sizeof(int), m->stream));
    MLP_CUDA(m, cudaStreamSynchronize(m->stream));
    return mlp_fail(m, GF_ERR_DEVICE, "a tensor-core GEMM wait ran out of time");
  }
  return GF_OK;
}

gf_status gf_mlp_set_fused_inference(gf_mlp* m, int32_t enable) {
  if (!m || enable < 0 || enable > 1) return GF_ERR_INVALID_ARGUMENT;
  m->fused = enable;
  return GF_OK;
}

gf_status gf_mlp_inject_fault(gf_mlp* m, int32_t kind) {
  if (!m || kind < 0 || kind > 1) return GF_ERR_INVALID_ARGUMENT;
  m->inject = kind;
  return GF_OK;
}

gf_status gf_bf16_gemm(const void* d_a, const void* d_b, int32_t M, int32_t N, int32_t K, float* d_c,
                       void* stream) {
  if (!d_a || !d_b || !d_c || M <= 0 || N <= 0 || K <= 0 || M % BM || N % 64 || K % BK)
    return GF_ERR_INVALID_ARGUMENT;
  if ((reinterpret_cast<uintptr_t>(d_a) | reinterpret_cast<uintptr_t>(d_b) | reinterpret_cast<uintptr_t>(d_c)) & 15)
    return GF_ERR_INVALID_ARGUMENT;
  const int bn = N % 128 == 0 ? 128 : 64;
  CUtensorMap a, b, c;
  if (!make_map(&a, d_a, M, K, BM) || !make_map(&b, d_b, N, K, bn) || !make_out_map(&c, d_c, M, N, OUT_F32))
    return GF_ERR_CUDA;
  EpiArgs ep{};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t err = bn == 128 ? launch_gemm<128, EPI_STORE_F32>(a, b, &c, nullptr, nullptr, M, N, K, 1, ep, s)
                              : launch_gemm<64, EPI_STORE_F32>(a, b, &c, nullptr, nullptr, M, N, K, 1, ep, s);
  return err == cudaSuccess ? GF_OK : GF_ERR_CUDA;
}

}  // extern "C"
