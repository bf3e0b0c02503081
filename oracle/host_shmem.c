/*
 * host_shmem.c -- CPU baseline for the benchmark.  TEST / BENCHMARK
 * INFRASTRUCTURE ONLY: the library never links or calls it.
 *
 * It times the reference's host path as stated for this project: one OS
 * process per PE (the prototype's MPI ranks, nvshmem.cu:480-481), a shared
 * symmetric heap (a MAP_SHARED anonymous mapping created before fork, in
 * place of the prototype's CUDA-IPC mapped peer heaps, nvshmem.cu:548-589),
 * every put/get a memcpy between slices and every signal a 4-byte store, and
 * the host barrier a process-shared pthread barrier in place of MPI_Barrier
 * (nvshmem.cu:858-867).  No MPI is installed here, so the barrier and the
 * process launch are the stand-ins.
 *
 *   host_shmem_bench batch <reqfile> <npes> <slice_bytes> <max_reps> <max_seconds> [seed]
 *   host_shmem_bench alltoall <npes> <bytes> <max_reps> <max_seconds>
 *   host_shmem_bench pingpong <iters>
 *   host_shmem_bench barrier <npes> <iters>
 * Each prints one JSON line.
 */
#define _GNU_SOURCE
#include <errno.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#include "shmem_model.h"

typedef struct {
  uint64_t src_off, dst_off;
  uint32_t bytes;
  uint16_t src_pe, dst_pe;
  uint8_t op, dtype;
  uint16_t flags;
  int32_t value;
} req_t;

typedef struct {
  pthread_barrier_t bar;
  volatile int stop;
  volatile int32_t flag[2][16];
  double t[4096];
} ctl_t;

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static int ncores(void) {
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (int)n : 1;
}

static void *shared_map(size_t bytes) {
  void *p = mmap(NULL, bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
  return p == MAP_FAILED ? NULL : p;
}

static ctl_t *make_ctl(int nranks) {
  ctl_t *c = (ctl_t *)shared_map(sizeof(ctl_t));
  if (!c) return NULL;
  memset(c, 0, sizeof *c);
  pthread_barrierattr_t a;
  pthread_barrierattr_init(&a);
  pthread_barrierattr_setpshared(&a, PTHREAD_PROCESS_SHARED);
  pthread_barrier_init(&c->bar, &a, (unsigned)nranks);
  return c;
}

/* Forks nranks-1 children; returns this process's rank (0 for the parent). */
static int spawn_ranks(int nranks) {
  for (int r = 1; r < nranks; ++r) {
    pid_t pid = fork();
    if (pid < 0) {
      perror("fork");
      exit(1);
    }
    if (pid == 0) return r;
  }
  return 0;
}

static void reap(int nranks) {
  for (int r = 1; r < nranks; ++r) wait(NULL);
}

static int initiator(const req_t *q) { return (q->op == 1 || q->op == 4) ? q->dst_pe : q->src_pe; }

static void run_req(unsigned char *heap, size_t slice, const req_t *q) {
  unsigned char *s = heap + (size_t)q->src_pe * slice + q->src_off;
  unsigned char *d = heap + (size_t)q->dst_pe * slice + q->dst_off;
  const int w = q->dtype == 2 ? 8 : 4;
  switch (q->op) {
    case 0:
    case 1: memcpy(d, s, q->bytes); break;
    case 2: __atomic_store_n((int32_t *)d, q->value, __ATOMIC_RELEASE); break;
    case 3: memcpy(d, &q->src_off, (size_t)w); break;
    case 4: memcpy(d, s, (size_t)w); break;
  }
}

/* Runs reps until max_reps or max_seconds; rank 0 reports seconds per rep
 * (between the barrier before and the barrier after the work, so the time
 * of the slowest rank). */
static int cmd_batch(const char *file, int npes, size_t slice, int max_reps, double max_s, long long seed,
                     int warmup) {
  FILE *f = fopen(file, "rb");
  if (!f) {
    perror(file);
    return 1;
  }
  fseek(f, 0, SEEK_END);
  long sz = ftell(f);
  fseek(f, 0, SEEK_SET);
  int n = (int)(sz / (long)sizeof(req_t));
  req_t *reqs = (req_t *)malloc((size_t)n * sizeof(req_t));
  if (fread(reqs, sizeof(req_t), (size_t)n, f) != (size_t)n) {
    fclose(f);
    return 1;
  }
  fclose(f);
  unsigned long long alg = 0;
  for (int i = 0; i < n; ++i) {
    const req_t *q = &reqs[i];
    const unsigned w = q->dtype == 2 ? 8u : 4u;
    alg += q->op <= 1 ? 2ull * q->bytes : (q->op == 2 ? 4ull : (q->op == 3 ? w : 2ull * w));
  }
  unsigned char *heap = (unsigned char *)shared_map((size_t)npes * slice);
  ctl_t *c = make_ctl(npes);
  if (!heap || !c) {
    fprintf(stderr, "mmap failed\n");
    return 1;
  }
  const int rank = spawn_ranks(npes);
  /* first touch of this rank's own slice: the library's deterministic fill
   * when a seed is given (so the final heap can be checked against the GPU
   * run), zeros otherwise */
  if (seed >= 0) {
    om_model m = {npes, slice, slice, heap, NULL};
    om_fill_random(&m, rank, 0, slice, (uint64_t)seed);
  } else {
    memset(heap + (size_t)rank * slice, 0, slice);
  }
  int *mine = (int *)malloc((size_t)n * sizeof(int));
  int nm = 0;
  for (int i = 0; i < n; ++i)
    if (initiator(&reqs[i]) == rank) mine[nm++] = i;
  int reps = 0;
  double total = 0;
  const double start = now_s();
  if (warmup < 0) warmup = 0;
  for (int rep = -warmup; rep < max_reps; ++rep) { /* negative reps: untimed warm-up */
    pthread_barrier_wait(&c->bar);
    const double t0 = now_s();
    for (int k = 0; k < nm; ++k) run_req(heap, slice, &reqs[mine[k]]);
    pthread_barrier_wait(&c->bar);
    const double t1 = now_s();
    if (rank == 0 && rep >= 0) {
      total += t1 - t0;
      ++reps;
      if (now_s() - start > max_s) c->stop = 1;
    }
    pthread_barrier_wait(&c->bar);
    if (c->stop) break;
  }
  if (rank != 0) _exit(0);
  reap(npes);
  unsigned long long sum = 0;
  for (int p = 0; p < npes; ++p) sum += om_checksum(heap + (size_t)p * slice, slice);
  const int cores = npes < ncores() ? npes : ncores();
  printf("{\"mode\": \"batch\", \"requests\": %d, \"npes\": %d, \"reps\": %d, \"seconds_per_rep\": %.9f, "
         "\"alg_bytes\": %llu, \"gbs\": %.4f, \"cores\": %d, \"host_cores\": %d, \"heap_checksum\": %llu}\n",
         n, npes, reps, total / reps, alg, alg / (total / reps) / 1e9, cores, ncores(), sum);
  return 0;
}

static int cmd_alltoall(int npes, size_t bytes, int max_reps, double max_s) {
  const size_t slice = 2 * (size_t)npes * bytes;
  unsigned char *heap = (unsigned char *)shared_map((size_t)npes * slice);
  ctl_t *c = make_ctl(npes);
  if (!heap || !c) return 1;
  const int rank = spawn_ranks(npes);
  memset(heap + (size_t)rank * slice, rank + 1, slice);
  int reps = 0;
  double total = 0;
  const double start = now_s();
  for (int rep = -1; rep < max_reps; ++rep) {
    pthread_barrier_wait(&c->bar);
    const double t0 = now_s();
    for (int k = 0; k < npes - 1; ++k) {
      const int q = (rank + 1 + k) % npes;
      memcpy(heap + (size_t)q * slice + (size_t)npes * bytes + (size_t)rank * bytes,
             heap + (size_t)rank * slice + (size_t)q * bytes, bytes);
    }
    pthread_barrier_wait(&c->bar);
    const double t1 = now_s();
    if (rank == 0 && rep >= 0) {
      total += t1 - t0;
      ++reps;
      if (now_s() - start > max_s) c->stop = 1;
    }
    pthread_barrier_wait(&c->bar);
    if (c->stop) break;
  }
  if (rank != 0) _exit(0);
  reap(npes);
  const double alg = 2.0 * npes * (npes - 1) * (double)bytes;
  const int cores = npes < ncores() ? npes : ncores();
  printf("{\"mode\": \"alltoall\", \"npes\": %d, \"bytes\": %zu, \"reps\": %d, \"seconds_per_rep\": %.9f, "
         "\"gbs\": %.4f, \"cores\": %d, \"host_cores\": %d}\n",
         npes, bytes, reps, total / reps, alg / (total / reps) / 1e9, cores, ncores());
  return 0;
}

static int cmp_d(const void *a, const void *b) {
  double x = *(const double *)a, y = *(const double *)b;
  return x < y ? -1 : x > y;
}

/* Rank 0 stores i+1 into rank 1's flag and spins for the echo. */
static int cmd_pingpong(int iters) {
  ctl_t *c = make_ctl(2);
  if (!c) return 1;
  double *lat = (double *)shared_map((size_t)iters * sizeof(double));
  const int rank = spawn_ranks(2);
  pthread_barrier_wait(&c->bar);
  for (int i = 0; i < iters; ++i) {
    if (rank == 0) {
      const double t0 = now_s();
      __atomic_store_n(&c->flag[1][0], i + 1, __ATOMIC_RELEASE);
      while (__atomic_load_n(&c->flag[0][0], __ATOMIC_ACQUIRE) == i) {
      }
      lat[i] = (now_s() - t0) * 1e9;
    } else {
      while (__atomic_load_n(&c->flag[1][0], __ATOMIC_ACQUIRE) == i) {
      }
      __atomic_store_n(&c->flag[0][0], i + 1, __ATOMIC_RELEASE);
    }
  }
  if (rank != 0) _exit(0);
  reap(2);
  qsort(lat, (size_t)iters, sizeof(double), cmp_d);
  printf("{\"mode\": \"pingpong\", \"iters\": %d, \"p50_ns\": %.1f, \"p99_ns\": %.1f, \"cores\": 2, "
         "\"host_cores\": %d}\n",
         iters, lat[iters / 2], lat[(int)(iters * 0.99)], ncores());
  return 0;
}

static int cmd_barrier(int npes, int iters) {
  ctl_t *c = make_ctl(npes);
  if (!c) return 1;
  double *lat = (double *)shared_map((size_t)iters * sizeof(double));
  const int rank = spawn_ranks(npes);
  pthread_barrier_wait(&c->bar);
  double t = now_s();
  for (int i = 0; i < iters; ++i) {
    pthread_barrier_wait(&c->bar);
    if (rank == 0) {
      const double t1 = now_s();
      lat[i] = (t1 - t) * 1e9;
      t = t1;
    }
  }
  if (rank != 0) _exit(0);
  reap(npes);
  qsort(lat, (size_t)iters, sizeof(double), cmp_d);
  const int cores = npes < ncores() ? npes : ncores();
  printf("{\"mode\": \"barrier\", \"npes\": %d, \"iters\": %d, \"p50_ns\": %.1f, \"p99_ns\": %.1f, \"cores\": %d, "
         "\"host_cores\": %d}\n",
         npes, iters, lat[iters / 2], lat[(int)(iters * 0.99)], cores, ncores());
  return 0;
}

int main(int argc, char **argv) {
  if (argc >= 7 && strcmp(argv[1], "batch") == 0)
    return cmd_batch(argv[2], atoi(argv[3]), (size_t)atoll(argv[4]), atoi(argv[5]), atof(argv[6]),
                     argc >= 8 ? atoll(argv[7]) : -1, argc >= 9 ? atoi(argv[8]) : 1);
  if (argc >= 6 && strcmp(argv[1], "alltoall") == 0)
    return cmd_alltoall(atoi(argv[2]), (size_t)atoll(argv[3]), atoi(argv[4]), atof(argv[5]));
  if (argc >= 3 && strcmp(argv[1], "pingpong") == 0) return cmd_pingpong(atoi(argv[2]));
  if (argc >= 4 && strcmp(argv[1], "barrier") == 0) return cmd_barrier(atoi(argv[2]), atoi(argv[3]));
  fprintf(stderr, "usage: see host_shmem.c\n");
  return 2;
}
