// A prototype-style application, one process per PE (started by
// python -m nvshmem_b200.launch): every process calls nvstart_pes, allocates
// the same symmetric objects, launches its own kernels with ordinary <<<>>>
// launches and meets the others in nvshmem_barrier_all, as the prototype's
// MPI ranks do.
//   exchange <dir>: PE p puts its block into PE p+1's slot p (nvshmem_int_put
//     from many threads, then nvshmem_quiet), barrier, gets PE p-1's block
//     into its `got` area (nvshmem_int_get), barrier, then writes its own
//     slice to <dir>/pe<p>.bin and its symmetric offsets to <dir>/pe<p>.txt.
//   depart <dir>: PE 1 leaves without stopping; the others' barrier must
//     report an error instead of waiting for it (exit status 3 = error seen).
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <string>
#include <vector>

#include "nvshmem.h"
#include "nvshmem_device.h"
#include "nvshmemx.h"

__global__ void put_block(int *dst, const int *src, int n, int pe) {
  const int per = 256;  // elements per thread
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) * per;
  if (i < n) nvshmem_int_put(dst + i, (int *)src + i, n - i < per ? n - i : per, pe);
  nvshmem_quiet();
}

__global__ void get_block(int *dst, const int *src, int n, int pe) {
  const int per = 256;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) * per;
  if (i < n) nvshmem_int_get(dst + i, (int *)src + i, n - i < per ? n - i : per, pe);
}

static unsigned pattern(int pe, size_t i) { return (unsigned)(pe * 2654435761u + i * 40503u + 7u); }

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  const std::string mode = argv[1], dir = argv[2];
  nvshmemx_set_error_mode(NVSHMEMX_ERRORS_RETURN);
  nvstart_pes();
  if (!nvshmemx_is_started()) return 4;
  const int me = nvshmem_my_pe(), np = nvshmem_n_pes();
  const int n = 100000;  // ints per block
  int *send = (int *)nvshmalloc(n * sizeof(int));
  int *recv = (int *)nvshmalloc((size_t)np * n * sizeof(int));
  int *got = (int *)nvshmalloc(n * sizeof(int));
  if (!send || !recv || !got) return 5;
  std::vector<unsigned> h(n);
  for (int i = 0; i < n; ++i) h[i] = pattern(me, i);
  if (cudaMemcpy(send, h.data(), n * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) return 6;
  nvshmem_barrier_all();  // every PE's block is in place
  if (mode == "depart") {
    if (me == 1) _exit(0);  // leaves between steps, nothing of it in flight
    nvshmem_barrier_all();
    return nvshmemx_status() != 0 ? 3 : 0;
  }
  const int next = (me + 1) % np, prev = (me + np - 1) % np;
  const int threads = 128, blocks = (n / 256 + threads) / threads;
  put_block<<<blocks, threads>>>(recv + (size_t)me * n, send, n, next);
  nvshmem_barrier_all();
  get_block<<<blocks, threads>>>(got, send, n, prev);
  nvshmem_barrier_all();
  if (nvshmemx_status() != 0) return 7;
  const size_t heap = nvshmemx_heap_size();
  std::vector<unsigned char> img(heap);
  char *base = (char *)nvshmemx_arena_base() + (size_t)me * nvshmemx_slice_stride();
  if (cudaMemcpy(img.data(), base, heap, cudaMemcpyDeviceToHost) != cudaSuccess) return 8;
  FILE *f = fopen((dir + "/pe" + std::to_string(me) + ".bin").c_str(), "wb");
  if (!f) return 9;
  fwrite(img.data(), 1, heap, f);
  fclose(f);
  char *arena0 = (char *)nvshmemx_arena_base() + (size_t)me * nvshmemx_slice_stride();
  FILE *o = fopen((dir + "/pe" + std::to_string(me) + ".txt").c_str(), "w");
  if (!o) return 11;
  fprintf(o, "%d %zu %zu %zu %d\n", me, (size_t)((char *)send - arena0), (size_t)((char *)recv - arena0),
          (size_t)((char *)got - arena0), n);
  fclose(o);
  nvstop_pes();
  return nvshmemx_status() != 0 ? 10 : 0;
}
