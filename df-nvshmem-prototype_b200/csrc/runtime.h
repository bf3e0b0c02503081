// runtime.h -- host-side state of the virtual-PE library shared by the
// runtime, the operation launchers and the batch engine.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "nvshm_core.cuh"

namespace nvshm {

// Host copy of everything nvstart_pes sets up (the prototype keeps the same
// facts in globals, nvshmem.cu:119-135).
struct Runtime {
  std::recursive_mutex mu;
  bool started = false;
  int device = 0;
  int sm_count = 0;
  int npes = 0;
  size_t heap_bytes = 0;     // usable bytes per PE (NVSHMEM_HEAP_SIZE)
  size_t slice_mapped = 0;   // bytes mapped at the start of each slice
  size_t stride = 0;         // power of two >= slice_mapped
  int log2_stride = 0;
  char *arena = nullptr;
  std::vector<CUmemGenericAllocationHandle> handles;
  std::vector<size_t> tail;  // per-PE bump pointer (offset in the slice)
  // control block in device memory: status word, barrier counters
  char *ctrl = nullptr;
  int *d_status = nullptr;
  unsigned long long *d_coll_bar = nullptr;
  unsigned long long *d_pe_bar = nullptr;
  size_t bar_reset_bytes = 0;  // bytes from d_coll_bar to reset before a collective launch
  long long wait_timeout_ns = 5000000000LL;
  int error_mode = NVSHMEMX_ERRORS_EXIT;
  int host_err = 0;
  long long host_detail = -1;
  long long last_detail = -1;
  // trace ring
  nvshmemx_trace_record *d_trace = nullptr;
  unsigned long long *d_trace_head = nullptr;
  unsigned trace_cap = 0;
  bool trace_from_env = false;  // NVSHMEM_ENABLE_TRACING: write the CSV files at stop
  Cfg cfg{};
  // SPMD host threads
  bool spmd_active = false;
};

Runtime &rt();
const Cfg &cfg();
bool is_started();

// Records `code` (first error wins) and prints; exits in NVSHMEMX_ERRORS_EXIT
// mode as the prototype's CUDA_CHECK/ERROR_PRINT paths do.
int fail(int code, const char *fmt, ...);
int check_cuda(cudaError_t e, const char *what);

// Uploads rt().cfg to the __constant__ copy.
int publish_cfg();

extern thread_local int t_pe;
extern thread_local bool t_spmd;

// Cooperative launch of `func` over (grid.x, grid.y, npes) after zeroing the
// barrier counters on `stream`.
int launch_collective(const void *func, dim3 grid_per_pe, dim3 block, void **args, size_t smem,
                      cudaStream_t stream);
// Largest grid.x (CTAs per PE, grid.y == 1) that is co-resident.
int max_ctas_per_pe(const void *func, int block_threads, size_t smem);

cudaError_t upload_cfg(const Cfg &c);

}  // namespace nvshm
