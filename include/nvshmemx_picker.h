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
 * table of variant timings it was trained on when the inputs leave the range
 * of that table (nvshmemx_picker_pick); nvshmemx_batch_execute_picked groups
 * a request array and runs every group with its picked variant.  The
 * network is trained on the GPU by this library's own forward, backward and
 * Adam kernels.
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

/* ---- picking at run time --------------------------------------------------
 * A picker couples a trained network with the measured table it learned
 * from: nt classes with features table_x[nt][6] and measured times
 * table_t[nt][12] (ms; NaN or <= 0 where a variant did not run).  It sets
 * the network's input normalisation to the table's per-feature mean and
 * standard deviation (so create the picker before training the network) and
 * keeps the per-feature range of the table as the range the network is
 * trusted in.  The network must outlive the picker. */
typedef struct nvshmemx_picker nvshmemx_picker;

int nvshmemx_picker_create(nvshmemx_mlp *net, const float *table_x, const float *table_t, int nt,
                           nvshmemx_picker **out);
int nvshmemx_picker_destroy(nvshmemx_picker *p);

/* For each of n feature rows: the network's fastest variant when every
 * feature lies inside the table's range (source 0), else the best measured
 * variant of the nearest table class -- Euclidean distance of the
 * standardised features -- (source 1).  source may be NULL. */
int nvshmemx_picker_pick(nvshmemx_picker *p, const float *X, int n, int *variant, int *source);

/* The table's choice alone (nearest class's best measured variant). */
int nvshmemx_picker_table_pick(nvshmemx_picker *p, const float *X, int n, int *variant);

/* Pattern ids of the feature vector. */
#define NVSHMEMX_PATTERN_PAIRS 0      /* PE pairs (put sweeps, ping-pong)     */
#define NVSHMEMX_PATTERN_ALLTOALL 1   /* every PE to every other              */
#define NVSHMEMX_PATTERN_NEIGHBOR 2   /* nearest neighbours on a PE grid      */
#define NVSHMEMX_PATTERN_RANDOM 3     /* uniform random PE pairs              */

/* One group of a picked execution. */
typedef struct nvshmemx_picked_group {
  int first;        /* index of its first request in the grouped order     */
  int count;        /* requests in the group                               */
  int variant;      /* variant that ran it (0..11)                          */
  int source;       /* 0 network, 1 table fallback, 2 fixed (SIGNAL/P/G)    */
  float features[NVSHMEMX_PICKER_NIN];
} nvshmemx_picked_group;

/* Executes n requests (a host array, any host memory) through the picker.
 * Requests are validated on the host first (PEs, op, type, every range
 * inside its slice, SIGNAL/P alignment); an invalid one fails the call with
 * nothing executed.  PUT/GET requests are grouped by element width,
 * relative source/destination alignment (4, 8 or 16 bytes) and size class
 * (floor(log2 bytes)); each group's features are (log2 of its mean size,
 * width, log2 alignment, log2 PE count, `pattern`, log2 of its request
 * count), and the picker chooses its variant (network, or table outside the
 * trained range).  SIGNAL, P and G requests form one group run by the batch
 * engine's default configuration.  Groups that chose the same variant run
 * together: one batch run per batch-engine shape, one after the other on the
 * batch's stream, and one launch per per-call mode, each on a stream of the
 * picker's own, beside the batch runs (the requests of one call touch
 * disjoint bytes); the call returns when all are done.  The requests occupy
 * the batch's device
 * request array (so n <= its max_requests) in grouped order.  groups
 * (room for max_groups entries, may be NULL) receives the groups, *ngroups
 * their count; *out_status the first execution error (0: every request
 * done); *out_ms the device time from the start of the request copy to the
 * end of the last run, *out_run_ms the part after the copy (both may be
 * NULL).  The requests reach the device through the batch's pinned host
 * buffer (nvshmemx_batch_host_buffer), which the call overwrites; passing
 * that buffer itself as reqs is allowed. */
int nvshmemx_batch_execute_picked(nvshmemx_batch *b, nvshmemx_picker *p, const nvshmemx_request *reqs, int n,
                                  int pattern, nvshmemx_picked_group *groups, int max_groups, int *ngroups,
                                  int *out_status, float *out_ms, float *out_run_ms);

/* Execution of variant v (0..11) on b's uploaded requests, with L2 flushed
 * before each of `reps` runs; *out_ms = median device time. */
int nvshmemx_variant_time(nvshmemx_batch *b, int variant, int reps, size_t flush_bytes, float *out_ms);
/* The batch configuration (variants 4..11) or per-call mode (0..3) of v. */
int nvshmemx_variant_describe(int variant, int *percall_mode, nvshmemx_batch_config *cfg);

#ifdef __cplusplus
}
#endif

#endif /* NVSHMEM_B200_NVSHMEMX_PICKER_H_ */
