// An application that starts its PE processes itself and bootstraps the
// library through its own collective, as an MPI program would with
// MPI_Allgather (nvshmemx_init_bootstrap).  There is no MPI on this machine,
// so the stand-in is in this file: the first process forks the others before
// any CUDA call, and the allgather goes through a shared anonymous mapping
// between two waits on a process-shared barrier.
//   boot_pes <npes> <dir>: every PE puts its block into PE p+1's slot p and
//   gets PE p-1's block (the exchange of proc_pes.cu), then writes its slice
//   to <dir>/pe<p>.bin and its symmetric offsets to <dir>/pe<p>.txt.  The
//   first process exits 0 when every PE process did.
#include <cuda_runtime.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <unistd.h>

#include <string>
#include <vector>

#include "nvshmem.h"
#include "nvshmem_device.h"
#include "nvshmemx.h"

namespace {

struct Shared {  // the launcher's collective state, shared by every process
  pthread_barrier_t bar;
  unsigned char scratch[1 << 16];
};

struct Comm {
  Shared *sh;
  int rank, size;
};

// MPI_Allgather of `len` bytes, in rank order.
int allgather(const void *in, void *out, size_t len, void *ctx) {
  Comm *c = static_cast<Comm *>(ctx);
  if ((size_t)c->size * len > sizeof c->sh->scratch) return -1;
  memcpy(c->sh->scratch + (size_t)c->rank * len, in, len);
  pthread_barrier_wait(&c->sh->bar);
  memcpy(out, c->sh->scratch, (size_t)c->size * len);
  pthread_barrier_wait(&c->sh->bar);  // nobody writes the scratch again before all have read it
  return 0;
}

__global__ void put_block(int *dst, const int *src, int n, int pe) {
  const int per = 256;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) * per;
  if (i < n) nvshmem_int_put(dst + i, (int *)src + i, n - i < per ? n - i : per, pe);
  nvshmem_quiet();
}

__global__ void get_block(int *dst, const int *src, int n, int pe) {
  const int per = 256;
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) * per;
  if (i < n) nvshmem_int_get(dst + i, (int *)src + i, n - i < per ? n - i : per, pe);
}

unsigned pattern(int pe, size_t i) { return (unsigned)(pe * 2654435761u + i * 40503u + 7u); }

int run_pe(Comm *comm, const std::string &dir) {
  nvshmemx_set_error_mode(NVSHMEMX_ERRORS_RETURN);
  nvshmemx_bootstrap bs;
  bs.rank = comm->rank;
  bs.size = comm->size;
  bs.allgather = allgather;
  bs.ctx = comm;
  if (nvshmemx_init_bootstrap(&bs, 4 << 20) != 0) return 4;
  const int me = nvshmem_my_pe(), np = nvshmem_n_pes();
  if (me != comm->rank || np != comm->size) return 5;
  const int n = 100000;
  int *send = (int *)nvshmalloc(n * sizeof(int));
  int *recv = (int *)nvshmalloc((size_t)np * n * sizeof(int));
  int *got = (int *)nvshmalloc(n * sizeof(int));
  if (!send || !recv || !got) return 6;
  std::vector<unsigned> h(n);
  for (int i = 0; i < n; ++i) h[i] = pattern(me, i);
  if (cudaMemcpy(send, h.data(), n * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) return 7;
  nvshmem_barrier_all();
  const int next = (me + 1) % np, prev = (me + np - 1) % np;
  const int threads = 128, blocks = (n / 256 + threads) / threads;
  put_block<<<blocks, threads>>>(recv + (size_t)me * n, send, n, next);
  nvshmem_barrier_all();
  get_block<<<blocks, threads>>>(got, send, n, prev);
  nvshmem_barrier_all();
  if (nvshmemx_status() != 0) return 8;
  const size_t heap = nvshmemx_heap_size();
  std::vector<unsigned char> img(heap);
  char *base = (char *)nvshmemx_arena_base() + (size_t)me * nvshmemx_slice_stride();
  if (cudaMemcpy(img.data(), base, heap, cudaMemcpyDeviceToHost) != cudaSuccess) return 9;
  FILE *f = fopen((dir + "/pe" + std::to_string(me) + ".bin").c_str(), "wb");
  if (!f) return 10;
  fwrite(img.data(), 1, heap, f);
  fclose(f);
  FILE *o = fopen((dir + "/pe" + std::to_string(me) + ".txt").c_str(), "w");
  if (!o) return 11;
  fprintf(o, "%d %zu %zu %zu %d\n", me, (size_t)((char *)send - base), (size_t)((char *)recv - base),
          (size_t)((char *)got - base), n);
  fclose(o);
  nvshmem_barrier_all();
  nvstop_pes();
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  const int np = atoi(argv[1]);
  const std::string dir = argv[2];
  if (np < 1 || np > 64) return 2;
  Shared *sh = (Shared *)mmap(nullptr, sizeof(Shared), PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
  if (sh == MAP_FAILED) return 3;
  pthread_barrierattr_t ba;
  pthread_barrierattr_init(&ba);
  pthread_barrierattr_setpshared(&ba, PTHREAD_PROCESS_SHARED);
  pthread_barrier_init(&sh->bar, &ba, np);
  std::vector<pid_t> kids;
  int rank = 0;
  for (int r = 1; r < np; ++r) {  // before any CUDA call
    const pid_t pid = fork();
    if (pid < 0) return 3;
    if (pid == 0) {
      rank = r;
      kids.clear();
      break;
    }
    kids.push_back(pid);
  }
  Comm comm{sh, rank, np};
  const int rc = run_pe(&comm, dir);
  if (rank != 0) _exit(rc);
  int worst = rc;
  for (pid_t k : kids) {
    int st = 0;
    waitpid(k, &st, 0);
    const int code = WIFEXITED(st) ? WEXITSTATUS(st) : 100;
    if (code && !worst) worst = code;
  }
  return worst;
}
