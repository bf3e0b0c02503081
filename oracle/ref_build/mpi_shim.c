/*
 * mpi_shim.c -- fork-based implementation of the MPI subset in mpi.h.
 * TEST INFRASTRUCTURE ONLY.  Every rank is a process forked by MPI_Init before
 * any CUDA call, so all ranks may then open the same GPU; collectives copy
 * through a shared scratch area between process-shared barrier waits.  A
 * barrier that waits longer than MPI_SHIM_TIMEOUT_S (default 120 s) aborts the
 * rank instead of waiting forever.
 */
#define _GNU_SOURCE
#include "mpi.h"

#include <errno.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#define SHIM_SCRATCH (1 << 20)

typedef struct {
  pthread_mutex_t mu;
  pthread_cond_t cv;
  int count;
  unsigned long long gen;
  int failed;
  unsigned char scratch[SHIM_SCRATCH];
} shim_ctl;

static shim_ctl *g_ctl;
static int g_rank, g_size = 1;
static pid_t g_children[1024];

static int shim_barrier(void) {
  double to = getenv("MPI_SHIM_TIMEOUT_S") ? atof(getenv("MPI_SHIM_TIMEOUT_S")) : 120.0;
  struct timespec dl;
  clock_gettime(CLOCK_REALTIME, &dl);
  dl.tv_sec += (time_t)to;
  pthread_mutex_lock(&g_ctl->mu);
  unsigned long long g = g_ctl->gen;
  if (++g_ctl->count == g_size) {
    g_ctl->count = 0;
    g_ctl->gen++;
    pthread_cond_broadcast(&g_ctl->cv);
  } else {
    while (g_ctl->gen == g && !g_ctl->failed) {
      if (pthread_cond_timedwait(&g_ctl->cv, &g_ctl->mu, &dl) == ETIMEDOUT) {
        g_ctl->failed = 1;
        pthread_cond_broadcast(&g_ctl->cv);
        break;
      }
    }
  }
  int failed = g_ctl->failed;
  pthread_mutex_unlock(&g_ctl->mu);
  if (failed) {
    fprintf(stderr, "[mpi shim %d] barrier timed out\n", g_rank);
    _exit(3);
  }
  return MPI_SUCCESS;
}

int MPI_Init(int *argc, char ***argv) {
  (void)argc;
  (void)argv;
  const char *np = getenv("MPI_SHIM_NP");
  g_size = np ? atoi(np) : 1;
  if (g_size < 1 || g_size > 1024) g_size = 1;
  g_ctl = (shim_ctl *)mmap(NULL, sizeof(shim_ctl), PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
  if (g_ctl == MAP_FAILED) {
    perror("mmap");
    exit(1);
  }
  pthread_mutexattr_t ma;
  pthread_mutexattr_init(&ma);
  pthread_mutexattr_setpshared(&ma, PTHREAD_PROCESS_SHARED);
  pthread_mutex_init(&g_ctl->mu, &ma);
  pthread_condattr_t ca;
  pthread_condattr_init(&ca);
  pthread_condattr_setpshared(&ca, PTHREAD_PROCESS_SHARED);
  pthread_cond_init(&g_ctl->cv, &ca);
  g_rank = 0;
  for (int r = 1; r < g_size; ++r) {
    pid_t pid = fork();
    if (pid < 0) {
      perror("fork");
      exit(1);
    }
    if (pid == 0) {
      g_rank = r;
      break;
    }
    g_children[r] = pid;
  }
  return MPI_SUCCESS;
}

int MPI_Finalize(void) {
  shim_barrier();
  if (g_rank == 0) {
    int bad = 0;
    for (int r = 1; r < g_size; ++r) {
      int st = 0;
      waitpid(g_children[r], &st, 0);
      if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) bad = 1;
    }
    if (bad) fprintf(stderr, "[mpi shim] a rank exited with an error\n");
  }
  return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm c, int *rank) {
  (void)c;
  *rank = g_rank;
  return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm c, int *size) {
  (void)c;
  *size = g_size;
  return MPI_SUCCESS;
}

int MPI_Allgather(void *sendbuf, int sendcount, MPI_Datatype st, void *recvbuf, int recvcount, MPI_Datatype rt,
                  MPI_Comm comm) {
  (void)st;
  (void)rt;
  (void)comm;
  (void)recvcount;
  if ((size_t)sendcount * (size_t)g_size > SHIM_SCRATCH) return 1;
  shim_barrier();
  memcpy(g_ctl->scratch + (size_t)g_rank * sendcount, sendbuf, (size_t)sendcount);
  shim_barrier();
  memcpy(recvbuf, g_ctl->scratch, (size_t)sendcount * (size_t)g_size);
  shim_barrier();
  return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm) {
  (void)t;
  (void)comm;
  if ((size_t)count > SHIM_SCRATCH) return 1;
  shim_barrier();
  if (g_rank == root) memcpy(g_ctl->scratch, buf, (size_t)count);
  shim_barrier();
  if (g_rank != root) memcpy(buf, g_ctl->scratch, (size_t)count);
  shim_barrier();
  return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) {
  (void)comm;
  return shim_barrier();
}
