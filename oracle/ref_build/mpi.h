/*
 * mpi.h -- the subset of MPI the reference's host code calls
 * (nvshmem.cu:480-481, :509, :551, :372, :863; microbench/*.cu MPI_Init /
 * MPI_Finalize), written for this project so the reference can be built and
 * run without an MPI installation.  TEST INFRASTRUCTURE ONLY.
 *
 * MPI_Init forks MPI_SHIM_NP - 1 children (default 1 rank); collectives go
 * through a MAP_SHARED anonymous mapping created before the fork and a
 * process-shared pthread barrier.
 */
#ifndef ORACLE_MPI_SHIM_H_
#define ORACLE_MPI_SHIM_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;

#define MPI_COMM_WORLD 0
#define MPI_BYTE 1
#define MPI_SUCCESS 0

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Allgather(void *sendbuf, int sendcount, MPI_Datatype st, void *recvbuf, int recvcount,
                  MPI_Datatype rt, MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Barrier(MPI_Comm comm);

#ifdef __cplusplus
}
#endif

#endif
