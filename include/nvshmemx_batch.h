/*
 * nvshmemx_batch.h -- batched one-sided traffic for the B200 virtual-PE
 * library (plain C ABI).
 *
 * The prototype has no batching: every put/get is one call of the per-thread
 * device API (nvshmem_device.cu:488-540) and the caller decides how many
 * threads issue how many calls.  A batch here is an array of
 * nvshmemx_request descriptors (nvshmemx_ops.h) that one CUDA graph executes
 * with two kernels:
 *   plan  -- validates and translates each request and cuts it into chunks of
 *            at most chunk_bytes (a 0-byte SIGNAL/P is one chunk);
 *   exec  -- a persistent grid whose warps claim chunks from a device-wide
 *            cursor and copy them with coalesced vector accesses,
 * so uneven request sizes and random PE pairs spread over every SM.  Results
 * are bit-identical to issuing the same requests one by one (requests of one
 * batch must not write bytes that another request of the batch reads or
 * writes).
 *
 * How the copy is shaped (vector width, chunk size, accesses in flight,
 * threads and CTAs per SM) is a nvshmemx_batch_config; the autotuner
 * (nvshmemx_tune_batch) measures candidate configurations and keeps the best
 * in a table, and the learned picker (nvshmemx_mlp_*) can predict it.
 */
#ifndef NVSHMEM_B200_NVSHMEMX_BATCH_H_
#define NVSHMEM_B200_NVSHMEMX_BATCH_H_

#include <stddef.h>
#include <stdint.h>

#include "nvshmemx_ops.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nvshmemx_batch_config {
  int vec_bytes;    /* widest access: 4, 8 or 16                              */
  int chunk_bytes;  /* work unit: multiple of 256 in [256, 1 MiB]             */
  int unroll;       /* accesses in flight per lane: 1, 2, 4 or 8              */
  int threads;      /* threads per CTA: 128, 256, 512 or 1024 (TMA: <= 256)   */
  int ctas_per_sm;  /* resident CTAs per SM (0: as many as fit)               */
  int grab;         /* chunks claimed per cursor atomic: 1..16                */
  int tma_stages;   /* 0: copy through registers; 2, 3 or 4: every warp
                       streams 16-byte-aligned bodies through a ring of this
                       many shared-memory stages with cp.async.bulk          */
  int tma_stage_bytes; /* bytes per stage: multiple of 1024, 1 KiB..32 KiB    */
  int tma_min_bytes;   /* chunks shorter than this use the register copy    */
  int stream;          /* 1: plan and execute in one persistent cooperative
                          launch, planning warps feeding executing warps
                          (needs tma_stages > 0); the end-to-end call then
                          reads the requests straight from the pinned host
                          buffer.  An invalid request is skipped on its own
                          and reported, the others still run.  0: a graph of
                          plan then exec; an invalid request stops the batch */
  int stream_planners; /* planning warps per CTA in stream mode: 1..4        */
} nvshmemx_batch_config;

/* Defaults for B200: one of the leading configurations the autotuner
 * measured on the 64-PE, 100,000-request workload (tuned/batch_c4.json holds
 * the measured table and its best). */
void nvshmemx_batch_default_config(nvshmemx_batch_config *cfg);

typedef struct nvshmemx_batch nvshmemx_batch;

/* Device buffers for up to max_requests requests moving up to
 * max_payload_bytes in total (sizes the chunk table for the smallest chunk
 * size a configuration may use, 256 bytes, unless min_chunk_bytes is larger;
 * 32 bytes per chunk). */
int nvshmemx_batch_create(int max_requests, unsigned long long max_payload_bytes, int min_chunk_bytes,
                          nvshmemx_batch **out);
int nvshmemx_batch_destroy(nvshmemx_batch *b);
int nvshmemx_batch_set_config(nvshmemx_batch *b, const nvshmemx_batch_config *cfg);
int nvshmemx_batch_get_config(const nvshmemx_batch *b, nvshmemx_batch_config *cfg);

/* Pinned host staging buffer of max_requests descriptors owned by the batch;
 * callers fill it and pass it to nvshmemx_batch_submit. */
nvshmemx_request *nvshmemx_batch_host_buffer(nvshmemx_batch *b);

/* Copies n requests to the device (synchronously) for later executions. */
int nvshmemx_batch_upload(nvshmemx_batch *b, const nvshmemx_request *reqs, int n);

/* Executes the uploaded requests `reps` times back to back (one graph launch
 * each; the CUDA graph is rebuilt when n or the configuration changes).
 * *out_ms receives the device time of all reps (CUDA events). */
int nvshmemx_batch_execute(nvshmemx_batch *b, int reps, float *out_ms);

/* End-to-end call: copies n requests from host memory (pinned if it is the
 * batch's host buffer), executes them and reads back the batch status word;
 * *out_status receives the status (0 = every request done), *out_ms the
 * device time of the whole sequence.  With a graph configuration (stream 0)
 * the copy precedes the plan and exec kernels on the batch's stream; from
 * 8192 requests on, the batch runs as two pieces: a second stream copies
 * and plans the first quarter (in whole 256-request blocks), then the rest,
 * while the batch's stream executes each piece once it is planned, and a
 * one-thread kernel writes the status word into pinned host memory.  An
 * invalid request in the second piece is reported after the first piece has
 * run (with one piece, nothing runs).  In stream mode the copy precedes the
 * streaming kernel.  The requests stay resident: nvshmemx_batch_execute
 * afterwards runs the same batch. */
int nvshmemx_batch_submit(nvshmemx_batch *b, const nvshmemx_request *reqs, int n, int *out_status,
                          float *out_ms);

/* nvshmemx_batch_submit for requests in the 16-byte compact form
 * (nvshmemx_ops.h), which halves the host-to-device copy; the batch's host
 * buffer, viewed as nvshmemx_request_compact, is the pinned place for them.
 * Same pieces, order and error rules as nvshmemx_batch_submit; the plan
 * kernels expand each request as they read it and leave the full 32-byte
 * form resident, so nvshmemx_batch_execute afterwards runs the same batch.
 * A compact request with bits set outside its fields is reported as
 * NVSHMEMX_ERR_INVALID.  Needs a graph configuration (stream 0). */
int nvshmemx_batch_submit_compact(nvshmemx_batch *b, const nvshmemx_request_compact *reqs, int n,
                                  int *out_status, float *out_ms);

/* The same work as nvshmemx_batch_execute, enqueued without a graph and with
 * CUDA events around the plan and exec kernels on the batch's stream:
 * *out_ms is the time of all reps, *out_exec_ms the exec kernel's share. */
int nvshmemx_batch_execute_direct(nvshmemx_batch *b, int reps, float *out_ms, float *out_exec_ms);

/* Statistics of the last execution: chunk count, and the plan and exec kernel
 * times of the last nvshmemx_batch_execute_direct (0 before one ran). */
int nvshmemx_batch_last_stats(const nvshmemx_batch *b, unsigned long long *chunks, float *plan_ms,
                              float *exec_ms);

/* Algorithmic bytes of n requests: 2*bytes for PUT/GET (read + write),
 * 2*width for G, 4 for SIGNAL, width for P. */
unsigned long long nvshmemx_requests_bytes(const nvshmemx_request *reqs, int n);

/* The per-call path on the same device-resident requests: one caller unit
 * per request (mode NVSHMEMX_MODE_*) through the public device API, `reps`
 * launches back to back; *out_ms the device time of all reps. */
int nvshmemx_batch_execute_percall(nvshmemx_batch *b, int mode, int reps, float *out_ms);

/* Work items (chunks) the allocation-free entry point below can hold:
 * 32768 x 32 bytes = 1 MiB of scratch, plus a 256-byte control block. */
#define NVSHMEMX_NOALLOC_MAX_CHUNKS 32768

/* Allocation-free batch execution.  No counterpart in the reference (the
 * prototype has no batching at all).
 *
 * Executes n requests that are already in device memory (d_reqs, owned by
 * the caller) on `stream` (a cudaStream_t; NULL for the legacy default
 * stream) and waits for them, without allocating: it calls no cudaMalloc,
 * cudaFree or allocating library routine.  It is for callers that cannot
 * allocate device memory while they run -- a serving loop that must not take
 * cudaMalloc's device-wide synchronisation and unbounded latency, a process
 * whose device memory is owned by another allocator or a budget fixed at
 * start-up, a foreign-language caller that cannot release device memory it
 * would have to own.
 *
 * Its scratch is a fixed array inside this library that every GPU loading
 * the library holds until the process exits.  Limits: at most
 * NVSHMEMX_NOALLOC_MAX_CHUNKS requests and at most that many chunks of
 * cfg->chunk_bytes in total; larger batches are rejected with
 * NVSHMEMX_ERR_NOMEM and nothing is executed.  cfg NULL uses
 * nvshmemx_batch_default_config.  Every field of cfg is honoured as in
 * nvshmemx_batch_execute (tma_stages > 0 runs the TMA-ring exec kernel,
 * whose stages are shared memory, not scratch), except stream: stream mode
 * keeps state across calls that the shared scratch cannot hold, so a cfg
 * with stream != 0 is rejected with NVSHMEMX_ERR_INVALID.  As in the graph
 * path, one invalid request stops the whole batch (nothing is executed).
 *
 * The first call on a device looks up the scratch array's device address
 * (cudaGetSymbolAddress, with that device current); make that first call
 * before any stream capture.  All calls share the one array: the control
 * block is cleared at the start of every call, so sequential calls are
 * independent, but calls whose executions overlap on the GPU (from several
 * host threads or streams at once) race on it and must be serialised by the
 * caller.  Results are bit-identical to nvshmemx_batch_execute on the same
 * requests. */
int nvshmemx_batch_execute_noalloc(const nvshmemx_request *d_reqs, int n, const nvshmemx_batch_config *cfg,
                                   void *stream);

#ifdef __cplusplus
}
#endif

#endif /* NVSHMEM_B200_NVSHMEMX_BATCH_H_ */
