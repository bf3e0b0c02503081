// ref_driver.cu -- runs scenarios through the REFERENCE's own build (its
// nvshmem.cu / nvshmem_device.cu / nvshmem_kernels.cu /
// nvshmem_cuda_constants.cu compiled for sm_100a, see Makefile) with every
// MPI rank on the same GPU, and prints per-rank FNV-1a hashes of the heap so
// the CPU oracle can be pinned to the reference's behaviour.
// TEST INFRASTRUCTURE ONLY.
//
// Ranks never wait on each other inside a kernel: kernels launched by
// different processes are not guaranteed to run at the same time on one
// GPU, so every ordering step goes through the host barrier
// (nvshmem_barrier_all = cuCtxSynchronize + MPI_Barrier, nvshmem.cu:858-867).
//
//   MPI_SHIM_NP=N ref_driver alloc
//   MPI_SHIM_NP=N ref_driver requests <file> <heap_bytes> <seed>
//   MPI_SHIM_NP=N ref_driver alltoall <bytes> <rounds> <seed>
//   MPI_SHIM_NP=8 ref_driver halo <n> <iters>           (2x2x2, blocks from <file prefix>)
//   MPI_SHIM_NP=2 ref_driver pingpong <len> <iters> <seed>
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mpi.h"
#include "nvshmem.h"
#include "nvshmem_device.h"
#include "../shmem_model.h"

extern long long _nvshmem_heap_size;  // nvshmem.cu:184 (a plain global)

#define CK(x)                                                                            \
  do {                                                                                   \
    cudaError_t e_ = (x);                                                                \
    if (e_ != cudaSuccess) {                                                             \
      fprintf(stderr, "ref_driver %s:%d %s\n", __FILE__, __LINE__, cudaGetErrorString(e_)); \
      exit(2);                                                                           \
    }                                                                                    \
  } while (0)

typedef struct {
  uint64_t src_off, dst_off;
  uint32_t bytes;
  uint16_t src_pe, dst_pe;
  uint8_t op, dtype;
  uint16_t flags;
  int32_t value;
} req_t;

static int g_rank, g_npes;

// Fill this rank's heap with the library's deterministic pattern (the
// oracle's om_fill_random), through a host image.
static void fill_heap(char *heap, size_t bytes, uint64_t seed) {
  om_model *m = om_create(g_npes, bytes, bytes);
  om_fill_random(m, g_rank, 0, bytes, seed);
  CK(cudaMemcpy(heap, om_slice(m, g_rank), bytes, cudaMemcpyHostToDevice));
  om_destroy(m);
}

static void print_hash(const char *scen, char *heap, size_t bytes) {
  unsigned char *h = (unsigned char *)malloc(bytes);
  CK(cudaMemcpy(h, heap, bytes, cudaMemcpyDeviceToHost));
  printf("{\"scenario\": \"%s\", \"rank\": %d, \"npes\": %d, \"bytes\": %zu, \"fnv\": \"%016llx\"}\n", scen, g_rank,
         g_npes, bytes, (unsigned long long)om_fnv1a(h, bytes));
  fflush(stdout);
  free(h);
}

// ------------------------------------------------------------ request lists
// One thread per request this rank initiates, through the reference's
// per-thread device calls.
__global__ void run_requests(const req_t *reqs, int n, int mype, char *heap) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  req_t r = reqs[i];
  const bool by_dst = r.op == 1 || r.op == 4;
  if ((by_dst ? r.dst_pe : r.src_pe) != mype) return;
  const int w = r.dtype == 2 ? 8 : 4;
  const int len = (int)(r.bytes / w);
  char *dst = heap + r.dst_off, *src = heap + r.src_off;
  switch (r.op) {
    case 0:
      if (r.dtype == 0) nvshmem_int_put((int *)dst, (int *)src, len, r.dst_pe);
      else if (r.dtype == 1) nvshmem_float_put((float *)dst, (float *)src, len, r.dst_pe);
      else nvshmem_double_put((double *)dst, (double *)src, len, r.dst_pe);
      break;
    case 1:
      if (r.dtype == 0) nvshmem_int_get((int *)dst, (int *)src, len, r.src_pe);
      else if (r.dtype == 1) nvshmem_float_get((float *)dst, (float *)src, len, r.src_pe);
      else nvshmem_double_get((double *)dst, (double *)src, len, r.src_pe);
      break;
    case 2: nvshmem_int_p((int *)dst, r.value, r.dst_pe); break;
    case 3:
      if (r.dtype == 0) nvshmem_int_p((int *)dst, (int)(uint32_t)r.src_off, r.dst_pe);
      else if (r.dtype == 1) nvshmem_float_p((float *)dst, __uint_as_float((uint32_t)r.src_off), r.dst_pe);
      else nvshmem_double_p((double *)dst, __longlong_as_double((long long)r.src_off), r.dst_pe);
      break;
    case 4:
      if (r.dtype == 0) *(int *)dst = nvshmem_int_g((int *)src, r.src_pe);
      else if (r.dtype == 1) *(float *)dst = nvshmem_float_g((float *)src, r.src_pe);
      else *(double *)dst = nvshmem_double_g((double *)src, r.src_pe);
      break;
  }
  nvshmem_quiet();
}

static int scen_requests(const char *file, size_t heap_bytes, uint64_t seed) {
  FILE *f = fopen(file, "rb");
  if (!f) return 1;
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  int n = (int)(sz / (long)sizeof(req_t));
  req_t *h = (req_t *)malloc(sz);
  if (fread(h, sizeof(req_t), n, f) != (size_t)n) return 1;
  fclose(f);
  char *heap = (char *)nvshmalloc(heap_bytes);
  fill_heap(heap, heap_bytes, seed);
  req_t *d;
  CK(cudaMalloc(&d, sz));
  CK(cudaMemcpy(d, h, sz, cudaMemcpyHostToDevice));
  nvshmem_barrier_all();
  if (n) run_requests<<<(n + 127) / 128, 128>>>(d, n, g_rank, heap);
  CK(cudaGetLastError());
  nvshmem_barrier_all();
  print_hash("requests", heap, heap_bytes);
  cudaFree(d);
  free(h);
  return 0;
}

// ---------------------------------------------------------------- all-to-all
// Message to peer q = (me+1+k) % npes: block q of the send region into slot
// `me` of q's receive region (one thread per message, nvshmem_float_put).
__global__ void alltoall_put(char *send, char *recv, size_t bytes, int mype, int npes) {
  int k = threadIdx.x;
  if (k >= npes - 1) return;
  int q = (mype + 1 + k) % npes;
  nvshmem_float_put((float *)(recv + (size_t)mype * bytes), (float *)(send + (size_t)q * bytes), (int)(bytes / 4), q);
  nvshmem_quiet();
}

static int scen_alltoall(size_t bytes, int rounds, uint64_t seed) {
  size_t heap_bytes = 2 * (size_t)g_npes * bytes;
  char *heap = (char *)nvshmalloc(heap_bytes);
  fill_heap(heap, heap_bytes, seed);
  nvshmem_barrier_all();
  for (int r = 0; r < rounds; ++r) {
    alltoall_put<<<1, 32 * ((g_npes - 1 + 31) / 32)>>>(heap, heap + (size_t)g_npes * bytes, bytes, g_rank, g_npes);
    CK(cudaGetLastError());
    nvshmem_barrier_all();
  }
  print_hash("alltoall", heap, heap_bytes);
  return 0;
}

// --------------------------------------------------------------------- halo
__device__ int halo_nbr(int pe, int d) {
  int x = pe % 2, y = (pe / 2) % 2, z = pe / 4;
  if (d < 2) x ^= 1;
  else if (d < 4) y ^= 1;
  else z ^= 1;
  return x + 2 * (y + 2 * z);
}

// One thread per face row: x faces element by element with nvshmem_double_p
// (stride-n gather), y and z rows with nvshmem_double_put.
__global__ void halo_faces(double *blk, double *ghost, int n, int mype) {
  int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= 6 * n) return;
  int d = u / n, j = u % n;
  int nb = halo_nbr(mype, d);
  double *dst = ghost + (size_t)(d ^ 1) * n * n + (size_t)j * n;
  int e = (d & 1) ? n - 1 : 0;
  if (d < 2) {
    for (int k = 0; k < n; ++k) nvshmem_double_p(dst + k, blk[((size_t)j * n + k) * n + e], nb);
  } else if (d < 4) {
    nvshmem_double_put(dst, blk + ((size_t)j * n + e) * n, n, nb);
  } else {
    nvshmem_double_put(dst, blk + ((size_t)e * n + j) * n, n, nb);
  }
  nvshmem_quiet();
}

__global__ void halo_signal(int *sig, int it, int mype) {
  int d = threadIdx.x;
  if (d < 6) nvshmem_int_p(sig + (d ^ 1), it + 1, halo_nbr(mype, d));
  nvshmem_quiet();
}

static int scen_halo(int n, int iters, const char *prefix) {
  const size_t nn = (size_t)n, block = nn * nn * nn * 8, ghosts = 6 * nn * nn * 8;
  size_t heap_bytes = block + ghosts + 64;
  heap_bytes = (heap_bytes + 4095) / 4096 * 4096;
  char *heap = (char *)nvshmalloc(heap_bytes);
  CK(cudaMemset(heap, 0, heap_bytes));
  char path[512];
  snprintf(path, sizeof path, "%s%d", prefix, g_rank);
  FILE *f = fopen(path, "rb");
  if (!f) return 1;
  double *h = (double *)malloc(block);
  if (fread(h, 1, block, f) != block) return 1;
  fclose(f);
  CK(cudaMemcpy(heap, h, block, cudaMemcpyHostToDevice));
  free(h);
  nvshmem_barrier_all();
  for (int it = 0; it < iters; ++it) {
    halo_faces<<<(6 * n + 127) / 128, 128>>>((double *)heap, (double *)(heap + block), n, g_rank);
    CK(cudaGetLastError());
    nvshmem_barrier_all();
    halo_signal<<<1, 32>>>((int *)(heap + block + ghosts), it, g_rank);
    CK(cudaGetLastError());
    nvshmem_barrier_all();
  }
  print_hash("halo", heap, heap_bytes);
  return 0;
}

// ----------------------------------------------------------------- ping-pong
// The put + flag exchange of microbench/shmem_latency.cu with each half-step
// separated by the host barrier instead of a device wait.
__global__ void pp_step(int *data, int *flag, int len, int i, int peer) {
  if (len) nvshmem_int_put(data, data, len, peer);
  nvshmem_quiet();
  nvshmem_int_p(flag, i + 1, peer);
  nvshmem_quiet();
}

static int scen_pingpong(int len, int iters, uint64_t seed) {
  if (g_npes != 2) return 1;
  size_t heap_bytes = 4096 + (size_t)len * 4;
  heap_bytes = (heap_bytes + 4095) / 4096 * 4096;
  char *heap = (char *)nvshmalloc(heap_bytes);
  fill_heap(heap, heap_bytes, seed);
  CK(cudaMemset(heap, 0, 4));  // the flag starts at 0
  nvshmem_barrier_all();
  for (int i = 0; i < iters; ++i) {
    if (g_rank == 0) pp_step<<<1, 1>>>((int *)(heap + 64), (int *)heap, len, i, 1);
    nvshmem_barrier_all();
    if (g_rank == 1) pp_step<<<1, 1>>>((int *)(heap + 64), (int *)heap, len, i, 0);
    nvshmem_barrier_all();
  }
  print_hash("pingpong", heap, heap_bytes);
  return 0;
}

// ------------------------------------------------------------------- alloc
static int scen_alloc(void) {
  const size_t sizes[] = {3, 1, 8, 0, 17, 70, 4096, 5};
  char *base = (char *)nvshmalloc(0);
  printf("{\"scenario\": \"alloc\", \"rank\": %d, \"offsets\": [", g_rank);
  for (int i = 0; i < 8; ++i) {
    char *p = (char *)nvshmalloc(sizes[i]);
    printf("%s%ld", i ? ", " : "", (long)(p - base));
  }
  nvshmcleanup();
  char *again = (char *)nvshmalloc(16);
  char *peer = (char *)nvshmem_ptr(again, (g_rank + 1) % g_npes);
  printf("], \"after_cleanup\": %ld, \"ptr_is_peer_heap\": %d}\n", (long)(again - base), peer != again || g_npes == 1);
  fflush(stdout);
  return 0;
}

int main(int argc, char **argv) {
  MPI_Init(&argc, &argv);  // forks the ranks before any CUDA call
  MPI_Comm_rank(MPI_COMM_WORLD, &g_rank);
  MPI_Comm_size(MPI_COMM_WORLD, &g_npes);
  CK(cudaSetDevice(0));
  _nvshmem_heap_size = 64ll << 20;
  if (argc >= 2 && !strcmp(argv[1], "requests") && argc >= 5) _nvshmem_heap_size = atoll(argv[3]) + 4096;
  if (argc >= 2 && !strcmp(argv[1], "alltoall") && argc >= 3) _nvshmem_heap_size = 2ll * g_npes * atoll(argv[2]) + 4096;
  nvstart_pes();
  int rc = 2;
  if (argc >= 2 && !strcmp(argv[1], "alloc")) rc = scen_alloc();
  else if (argc >= 5 && !strcmp(argv[1], "requests")) rc = scen_requests(argv[2], (size_t)atoll(argv[3]), strtoull(argv[4], 0, 10));
  else if (argc >= 5 && !strcmp(argv[1], "alltoall")) rc = scen_alltoall((size_t)atoll(argv[2]), atoi(argv[3]), strtoull(argv[4], 0, 10));
  else if (argc >= 5 && !strcmp(argv[1], "halo")) rc = scen_halo(atoi(argv[2]), atoi(argv[3]), argv[4]);
  else if (argc >= 5 && !strcmp(argv[1], "pingpong")) rc = scen_pingpong(atoi(argv[2]), atoi(argv[3]), strtoull(argv[4], 0, 10));
  nvshmem_barrier_all();
  // The reference's nvshmcleanup frees its region list but leaves the list
  // head and tail pointing at the freed entries (nvshmem.cu:805-819), so a
  // second call double-frees; the alloc scenario has already called it.
  if (!(argc >= 2 && !strcmp(argv[1], "alloc"))) nvshmcleanup();
  nvstop_pes();
  MPI_Finalize();
  return rc;
}
