/*
 * nvshmemx_tune.h -- autotuner for the batched engine (plain C ABI).
 *
 * No counterpart in the reference: the prototype copies with one calling
 * thread and a fixed scalar loop (nvshmem_device.cu:498-500), so it has
 * nothing to tune.  Here a batch's copy shape (nvshmemx_batch_config) is
 * chosen by measuring candidates on the device: each candidate runs the
 * uploaded batch `reps` times with L2 flushed before every run, timed with
 * CUDA events; the median decides.  The measured table is also what the
 * learned picker falls back to and the yardstick for its regret.
 */
#ifndef NVSHMEM_B200_NVSHMEMX_TUNE_H_
#define NVSHMEM_B200_NVSHMEMX_TUNE_H_

#include "nvshmemx_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nvshmemx_tune_result {
  nvshmemx_batch_config cfg;
  float ms_median;  /* median over reps of one graph execution            */
  float ms_min;
  float exec_ms_median;  /* the exec kernel alone (direct path, events)   */
  int status;       /* 0, or the error the candidate hit                    */
} nvshmemx_tune_result;

/* Writes up to max candidates of the standard search grid (vector width x
 * accesses in flight x chunk size x threads x chunks per claim, every chunk
 * >= min_chunk_bytes) to out; returns how many. */
int nvshmemx_tune_candidates(nvshmemx_batch_config *out, int max, int min_chunk_bytes);

/* Measures each candidate on b's uploaded requests; results[i] for
 * candidates[i]; *best receives the index of the smallest median.  The
 * batch is left configured with the best candidate.  Each run is preceded by
 * a write of flush_bytes (>= 2x L2 recommended) so no run starts with the
 * batch's data in L2. */
int nvshmemx_tune_batch(nvshmemx_batch *b, const nvshmemx_batch_config *candidates, int ncand, int reps,
                        size_t flush_bytes, nvshmemx_tune_result *results, int *best);

#ifdef __cplusplus
}
#endif

#endif /* NVSHMEM_B200_NVSHMEMX_TUNE_H_ */
