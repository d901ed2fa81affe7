// Values of model functions that the reference evaluates inside its device kernels, computed here on
// the device with the same expression and the same fast-math flags, so that the host front-end (which
// evaluates the Sim_Model functors once per population and generation) hands the engine the same
// float the reference's kernel computes.
#include <cuda_runtime.h>

#include "gf_internal.h"

namespace gf {

// Sim_Model::selection_sine_wave::operator() (template_inline_simulation_functors.cuh:92):
// s = A sin(pi (generation - generation_shift) + rho) + D, with t = generation - generation_shift.
// Under --use_fast_math the sine is the hardware approximation, whose value the host's sinf does not
// reproduce; this kernel is compiled with the flags the reference compiles its kernels with.
__global__ void sine_selection_kernel(float A, float pi, float rho, float D, int t0, int count, float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) {
    const int t = t0 + i;
    out[i] = A * sin(pi * t + rho) + D;
  }
}

}  // namespace gf

using namespace gf;

extern "C" gf_status gf_selection_sine_values(gf_engine* g, float A, float pi, float rho, float D, int32_t t0,
                                              int32_t count, float* out) {
  return guard_host(g, [&]() -> gf_status {
    if (!g || !out || count < 0) return GF_ERR_INVALID_ARGUMENT;
    if (count == 0) return GF_OK;
    if (static_cast<long long>(t0) + count - 1 > 0x7FFFFFFFll)
      return fail(&g->impl, GF_ERR_INVALID_ARGUMENT, "gf_selection_sine_values: t0 + count overflows int");
    Engine* e = &g->impl;
    GF_CUDA(e, cudaSetDevice(e->device));
    float* d_out = nullptr;
    GF_CUDA(e, cudaMallocAsync(reinterpret_cast<void**>(&d_out), sizeof(float) * count, e->stream));
    sine_selection_kernel<<<(count + 255) / 256, 256, 0, e->stream>>>(A, pi, rho, D, t0, count, d_out);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess) err = cudaMemcpyAsync(out, d_out, sizeof(float) * count, cudaMemcpyDeviceToHost, e->stream);
    cudaFreeAsync(d_out, e->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    if (err != cudaSuccess) return cuda_fail(e, err, "gf_selection_sine_values");
    return GF_OK;
  });
}
