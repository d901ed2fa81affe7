/* C ABI of the SFS surrogate network: a 6 -> 512 -> 512 -> 512 -> 512 -> 99 multilayer perceptron
 * with GELU activations (tanh form), bf16 weights and activations, fp32 accumulation (tcgen05 tensor cores, sm_100a),
 * fp32 master weights and Adam.
 *
 * The reference has no counterpart: 3P answers every SFS query with a forward simulation
 * (GO_Fish::run_sim, go_fish.cuh:280, then Spectrum::site_frequency_spectrum, spectrum.h:90).  The
 * network maps six model parameters (log N, gamma, h, F, growth rate, duration / 2N, each scaled to
 * [-1, 1] by the caller) to the log of the normalised expected SFS of a sample of 100 (bins 1..99),
 * and is trained on spectra the batched simulator produces.
 *
 * Parameter vector (fp32, gf_mlp_param_count() values), layer by layer: W1[512][6], b1[512],
 * W2[512][512], b2[512], W3[512][512], b3[512], W4[512][512], b4[512], W5[99][512], b5[99]
 * (row-major, out x in).
 *
 * Batches are a multiple of 128 rows and at most the capacity given at creation.  Device pointers
 * are used on the network's stream; calls are asynchronous unless they return host data.
 */
#ifndef GF_SURROGATE_H_
#define GF_SURROGATE_H_

#include <stdint.h>

#include "gofish_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define GF_MLP_INPUTS 6
#define GF_MLP_HIDDEN 512
#define GF_MLP_LAYERS 5
#define GF_MLP_OUTPUTS 99
#define GF_MLP_BATCH_ALIGN 128

typedef struct gf_mlp gf_mlp;

typedef struct gf_mlp_config {
  int32_t batch_capacity; /* largest batch (rows), a multiple of 128 */
  float lr;               /* Adam step size */
  float beta1;            /* Adam first-moment decay (0.9) */
  float beta2;            /* Adam second-moment decay (0.999) */
  float eps;              /* Adam epsilon (1e-8) */
  float weight_decay;     /* decoupled weight decay per step, as a fraction of lr (0: none) */
} gf_mlp_config;

gf_status gf_mlp_create(int32_t device, void* stream, const gf_mlp_config* config, gf_mlp** out);
gf_status gf_mlp_destroy(gf_mlp* mlp);
const char* gf_mlp_last_error(const gf_mlp* mlp);
int64_t gf_mlp_param_count(void);

/* Master weights in and out (host fp32, the layout above).  set_params also resets Adam's moments
 * and step count. */
gf_status gf_mlp_set_params(gf_mlp* mlp, const float* params, int64_t count);
gf_status gf_mlp_get_params(gf_mlp* mlp, float* params, int64_t count);
gf_status gf_mlp_set_learning_rate(gf_mlp* mlp, float lr);

/* Inference: d_inputs [batch][6] fp32 -> d_outputs [batch][99] fp32 (device pointers; d_outputs
 * 16-byte aligned).  By default one fused kernel runs all five layers of each 128-row tile with the
 * activations kept on chip; gf_mlp_set_fused_inference(mlp, 0) runs one tensor-core GEMM per layer
 * instead (the same outputs, bit for bit). */
gf_status gf_mlp_forward(gf_mlp* mlp, const float* d_inputs, int32_t batch, float* d_outputs);
gf_status gf_mlp_set_fused_inference(gf_mlp* mlp, int32_t enable);

/* Mean-squared-error gradients of the loss (1 / (batch * 99)) sum (out - target)^2 with respect to
 * the master parameters, without an update: host fp32 gradients in the parameter layout, and the
 * loss.  Synchronous. */
gf_status gf_mlp_gradients(gf_mlp* mlp, const float* d_inputs, const float* d_targets, int32_t batch,
                           float* grads, float* loss);

/* One training step (forward, backward, Adam update); the batch loss is written to d_loss (a device
 * float, may be NULL).  Asynchronous. */
gf_status gf_mlp_train_step(gf_mlp* mlp, const float* d_inputs, const float* d_targets, int32_t batch,
                            float* d_loss);

/* Kernel-fault word of the network's kernels (bounded waits that ran out); synchronous.  Returns
 * GF_ERR_DEVICE once per fault and clears the word; the network stays usable. */
gf_status gf_mlp_check(gf_mlp* mlp);

/* Failure-path testing: kind 1 arms the next inference pass so that its first GEMM (or the fused
 * kernel's first layer) withholds the hand-off of one accumulator; the epilogue's bounded wait (about 2 ms under injection) runs out, the
 * kernel stops, drains what it issued, releases tensor memory and sets the fault word.  Outputs of
 * that pass are undefined.  kind 0 disarms. */
gf_status gf_mlp_inject_fault(gf_mlp* mlp, int32_t kind);

/* Plain tensor-core GEMM C[M][N] = A[M][K] * B[N][K]^T (bf16 operands, both K-contiguous, fp32 out),
 * the kernel the network is built on.  M a multiple of 128, N of 64, K of 64; 16-byte aligned device
 * pointers.  Asynchronous on `stream`. */
gf_status gf_bf16_gemm(const void* d_a, const void* d_b, int32_t M, int32_t N, int32_t K, float* d_c,
                       void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GF_SURROGATE_H_ */
