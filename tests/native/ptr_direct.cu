// Direct loads and stores through the addresses nvshmem_ptr and nvshmemx_ptr
// return, the way applications of the prototype use nvshmem_ptr
// (nvshmem.cu:880-883: "the actual address of the symmetric object at the
// remote PE for direct loads/stores from inside CUDA kernel").
//   1. one collective launch: PE p stores its send block straight into PE
//      p+1's receive block (plain 16-byte stores through nvshmemx_ptr), then
//      quiet + device barrier, then loads PE p-1's send block into its own
//      `got` block (plain loads);
//   2. ordinary launches with pointers from the host-side nvshmem_ptr: PE q's
//      copy2 block <- PE q+1's receive block.
// Every slice starts from a fixed byte pattern; the heap images are written
// to argv[1] and the symmetric offsets printed, for the test to compare with
// the CPU oracle.  NVSHMEM_NPES and NVSHMEM_HEAP_SIZE come from the
// environment.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "nvshmem.h"
#include "nvshmem_device.h"
#include "nvshmemx.h"

__global__ void ring_direct(char *send, char *recv, char *got, size_t n) {
  const int pe = nvshmemx_my_pe(), np = nvshmemx_n_pes();
  const int next = (pe + 1) % np, prev = (pe + np - 1) % np;
  const size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x, step = (size_t)gridDim.x * blockDim.x;
  const uint4 *src = (const uint4 *)nvshmemx_ptr(send, pe);
  uint4 *dst = (uint4 *)nvshmemx_ptr(recv, next);
  for (size_t i = i0; i < n / 16; i += step) dst[i] = src[i];
  nvshmem_quiet();
  nvshmemx_barrier_all();
  const uint4 *rsrc = (const uint4 *)nvshmemx_ptr(send, prev);
  uint4 *mine = (uint4 *)nvshmemx_ptr(got, pe);
  for (size_t i = i0; i < n / 16; i += step) mine[i] = rsrc[i];
}

__global__ void copy_plain(uint4 *dst, const uint4 *src, size_t n16) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

static unsigned char pattern(int pe, size_t i) { return (unsigned char)((pe * 131 + i * 7 + (i >> 8)) & 0xff); }

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  nvshmemx_set_error_mode(NVSHMEMX_ERRORS_RETURN);
  nvstart_pes();
  if (!nvshmemx_is_started()) return 3;
  const int np = nvshmem_n_pes();
  const size_t heap = nvshmemx_heap_size();
  const size_t n = 65536 - 48;  // a multiple of 16
  char *send = (char *)nvshmalloc(65536), *recv = (char *)nvshmalloc(65536);
  char *got = (char *)nvshmalloc(65536), *copy2 = (char *)nvshmalloc(65536);
  if (!send || !recv || !got || !copy2) return 4;
  char *arena = (char *)nvshmemx_arena_base();
  std::vector<unsigned char> h(heap);
  for (int pe = 0; pe < np; ++pe) {
    for (size_t i = 0; i < heap; ++i) h[i] = pattern(pe, i);
    if (cudaMemcpy(nvshmem_ptr(arena, pe), h.data(), heap, cudaMemcpyHostToDevice) != cudaSuccess) return 5;
  }
  void *args[] = {&send, &recv, &got, (void *)&n};
  if (nvshmemx_collective_launch((const void *)ring_direct, dim3(4), dim3(256), args, 0, 0)) return 6;
  if (cudaDeviceSynchronize() != cudaSuccess) return 7;
  for (int q = 0; q < np; ++q)
    copy_plain<<<64, 256>>>((uint4 *)nvshmem_ptr(copy2, q), (const uint4 *)nvshmem_ptr(recv, (q + 1) % np), n / 16);
  if (cudaDeviceSynchronize() != cudaSuccess || nvshmemx_status() != 0) return 8;
  FILE *f = fopen(argv[1], "wb");
  if (!f) return 9;
  for (int pe = 0; pe < np; ++pe) {
    if (cudaMemcpy(h.data(), nvshmem_ptr(arena, pe), heap, cudaMemcpyDeviceToHost) != cudaSuccess) return 10;
    fwrite(h.data(), 1, heap, f);
  }
  fclose(f);
  printf("%zu %zu %zu %zu %zu %d %zu\n", (size_t)(send - arena), (size_t)(recv - arena), (size_t)(got - arena),
         (size_t)(copy2 - arena), n, np, heap);
  nvstop_pes();
  return 0;
}
