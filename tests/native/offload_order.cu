// nvshmem_barrier_all_offload orders the work of blocking streams, as a
// kernel on the legacy default stream does: a kernel on one blocking stream
// writes a flag after about 100 us, then the barrier, then a kernel on another
// blocking stream reads the flag.  Without the barrier the reader runs beside
// the writer and reads the old value (the control); with it, it must read the
// new one.  Prints both counts and exits 0 when no read after a barrier missed
// the write.
#include <cuda_runtime.h>
#include <stdio.h>

#include "nvshmem.h"
#include "nvshmemx.h"

__global__ void late_write(volatile int *flag, int value, long long cycles) {
  const long long t0 = clock64();
  while (clock64() - t0 < cycles) {
  }
  *flag = value;
}

__global__ void read_flag(const volatile int *flag, int *out) { *out = *flag; }

int main() {
  nvshmemx_set_error_mode(NVSHMEMX_ERRORS_RETURN);
  if (nvshmemx_init_attr(2, 1 << 20) != 0) return 2;
  cudaStream_t a, b;  // default flags: blocking streams
  if (cudaStreamCreate(&a) != cudaSuccess || cudaStreamCreate(&b) != cudaSuccess) return 3;
  int *flag = nullptr, *out = nullptr;
  if (cudaMalloc(&flag, sizeof(int)) != cudaSuccess || cudaMallocHost(&out, sizeof(int)) != cudaSuccess) return 3;
  if (cudaMemset(flag, 0, sizeof(int)) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return 3;
  const int reps = 32;
  int misses = 0, races = 0;
  for (int with_barrier = 0; with_barrier < 2; ++with_barrier) {
    for (int i = 0; i < reps; ++i) {
      const int value = 1 + i + 1000 * with_barrier;
      *out = -1;
      late_write<<<1, 1, 0, a>>>(flag, value, 200000);
      if (with_barrier) nvshmem_barrier_all_offload();
      read_flag<<<1, 1, 0, b>>>(flag, out);
      if (cudaDeviceSynchronize() != cudaSuccess) return 4;
      if (*out != value) ++(with_barrier ? misses : races);
    }
  }
  if (nvshmemx_status() != 0) return 5;
  printf("misses_with_barrier=%d races_without=%d of %d\n", misses, races, reps);
  cudaStreamDestroy(a);
  cudaStreamDestroy(b);
  cudaFree(flag);
  cudaFreeHost(out);
  nvstop_pes();
  return misses ? 1 : 0;
}
