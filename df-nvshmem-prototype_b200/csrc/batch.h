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

}  // namespace nvshm
