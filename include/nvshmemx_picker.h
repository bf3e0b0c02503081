/*
 * nvshmemx_picker.h -- learned transfer-variant picker (plain C ABI).
 *
 * No counterpart in the reference, which has a single transfer method (one
 * thread's scalar loop, nvshmem_device.cu:498-500).  Here a request group can
 * be carried out by NVSHMEMX_PICKER_VARIANTS variants (per-call thread / warp
 * / CTA / CTA-TMA, and batch-engine shapes with register or TMA copies); a
 * small FP32 MLP -- 6 inputs, three hidden layers of 64 with ReLU, 12 outputs
 * -- predicts each variant's log2 time from
 *   (log2 bytes, element width, log2 alignment, log2 PEs, pattern id,
 *    log2 requests in flight)
 * and the picker takes the fastest prediction, falling back to the measured
 * table (nvshmemx_tune.h) when the inputs leave the range the network was
 * trained on.  The network is trained on the GPU by this library's own
 * forward, backward and Adam kernels.
 */
#ifndef NVSHMEM_B200_NVSHMEMX_PICKER_H_
#define NVSHMEM_B200_NVSHMEMX_PICKER_H_

#include "nvshmemx_batch.h"

#define NVSHMEMX_PICKER_NIN 6
#define NVSHMEMX_PICKER_HIDDEN 64
#define NVSHMEMX_PICKER_VARIANTS 12

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nvshmemx_mlp nvshmemx_mlp;

/* Parameter count and layout: W1[64][6] b1[64] W2[64][64] b2[64]
 * W3[64][64] b3[64] W4[12][64] b4[12], row-major, concatenated. */
int nvshmemx_mlp_num_params(void);

/* He-initialised weights from `seed` (splitmix64 + Box-Muller), zero biases
 * and Adam state; inputs are standardised with (mean, std) set below
 * (initially 0 / 1). */
int nvshmemx_mlp_create(unsigned long long seed, nvshmemx_mlp **out);
int nvshmemx_mlp_destroy(nvshmemx_mlp *m);
int nvshmemx_mlp_get_params(const nvshmemx_mlp *m, float *host_params);
int nvshmemx_mlp_set_params(nvshmemx_mlp *m, const float *host_params);
int nvshmemx_mlp_set_normalization(nvshmemx_mlp *m, const float *mean, const float *std_dev);

/* Y[n][12] = network(X[n][6]) (host arrays). */
int nvshmemx_mlp_forward(nvshmemx_mlp *m, const float *X, int n, float *Y);

/* Masked mean squared error over the n x 12 outputs (M = 1 where Y is
 * measured) and its gradient with respect to every parameter (host array of
 * nvshmemx_mlp_num_params() floats). */
int nvshmemx_mlp_loss_grad(nvshmemx_mlp *m, const float *X, const float *Y, const float *M, int n, float *loss,
                           float *grad);

/* Adam (beta1 0.9, beta2 0.999, eps 1e-8) on mini-batches of `batch`
 * samples, reshuffled every epoch from `seed`; loss_curve[epochs] receives the
 * mean training loss of each epoch (may be NULL). */
int nvshmemx_mlp_train(nvshmemx_mlp *m, const float *X, const float *Y, const float *M, int n, int epochs,
                       int batch, float lr, unsigned long long seed, float *loss_curve);

/* For each of n feature rows: the variant with the smallest predicted time
 * and the predicted gap to the runner-up (log2 units). */
int nvshmemx_mlp_pick(nvshmemx_mlp *m, const float *X, int n, int *variant, float *margin);

/* Execution of variant v (0..11) on b's uploaded requests, with L2 flushed
 * before each of `reps` runs; *out_ms = median device time. */
int nvshmemx_variant_time(nvshmemx_batch *b, int variant, int reps, size_t flush_bytes, float *out_ms);
/* The batch configuration (variants 4..11) or per-call mode (0..3) of v. */
int nvshmemx_variant_describe(int variant, int *percall_mode, nvshmemx_batch_config *cfg);

#ifdef __cplusplus
}
#endif

#endif /* NVSHMEM_B200_NVSHMEMX_PICKER_H_ */
