// batch.h -- internals shared by the batch engine, the autotuner and the
// learned picker.
#pragma once

#include <cuda_runtime.h>

#include "nvshmemx_batch.h"
#include "runtime.h"

namespace nvshm {

// Launches the one-caller-unit-per-request kernel of nvshmemx_exec_requests
// on device-resident requests (ops.cu).
int launch_exec_requests(int mode, const nvshmemx_request *d_reqs, int n, cudaStream_t stream);

// Validates a batch configuration; returns 0 or NVSHMEMX_ERR_INVALID.
int check_batch_config(const nvshmemx_batch_config &c);

// Writes `bytes` of a library-owned buffer and waits, so the next run does
// not start with its data in L2 (tuner.cu).
int l2_flush(size_t bytes);

// For the picker's grouped execution (picker.cu): b's stream, its
// device-resident request array (room for batch_capacity requests), and an
// enqueue (no graph, no wait) of zeroing + plan + exec of requests
// [first, first + n) with configuration cfg.  A plan or exec error of the
// run is kept in a status word that later runs do not clear; read it with
// batch_sticky_status after the stream has finished, clear it with
// batch_clear_sticky before the first run.
cudaStream_t batch_stream(const nvshmemx_batch *b);
nvshmemx_request *batch_device_requests(nvshmemx_batch *b);
int batch_capacity(const nvshmemx_batch *b);
int batch_min_chunk(const nvshmemx_batch *b);
int batch_enqueue_range(nvshmemx_batch *b, int first, int n, const nvshmemx_batch_config &cfg);
int batch_clear_sticky(nvshmemx_batch *b);
int batch_sticky_status(nvshmemx_batch *b, int *status, int *bad_request);

}  // namespace nvshm
