/*
 * nvshmemx.h -- extensions of the B200 virtual-PE library that the prototype
 * does not have.  Nothing here changes the meaning of nvshmem.h /
 * nvshmem_device.h; it adds
 *   - error codes and a status query (the prototype has none: it calls
 *     exit(-1) on host errors, nvshmem.cu:57-91, and its device waits never
 *     fail, nvshmem_device.cu:542-584);
 *   - the virtual-PE launcher: one cooperative launch whose grid carries every
 *     PE along blockIdx.z (stands in for mpirun + one process per PE);
 *   - cooperative (warp / block / TMA-bulk) forms of put and get;
 *   - bounded waits and a device-side barrier across all CTAs of a launch;
 *   - the %globaltimer trace ring that replaces the prototype's trace buffers
 *     (nvshmem_device.cu:49-429, nvshmem.cu:206-467).
 */
#ifndef NVSHMEM_B200_NVSHMEMX_H_
#define NVSHMEM_B200_NVSHMEMX_H_

#include <stddef.h>
#include "nvshmem.h"

/* ---- status codes ------------------------------------------------------- */
#define NVSHMEMX_SUCCESS 0
#define NVSHMEMX_ERR_INVALID 1  /* bad argument (npes, size, pe, dtype ...)     */
#define NVSHMEMX_ERR_NOMEM 2    /* arena or heap exhausted                      */
#define NVSHMEMX_ERR_CUDA 3     /* a CUDA runtime call failed                   */
#define NVSHMEMX_ERR_STATE 4    /* library not started / already started        */
#define NVSHMEMX_ERR_TIMEOUT 5  /* a device wait or barrier passed its deadline */
#define NVSHMEMX_ERR_BOUNDS 6   /* device access outside the arena (skipped)    */
#define NVSHMEMX_ERR_COOP 7     /* grid too large to be co-resident             */
#define NVSHMEMX_ERR_UNSUPPORTED 8

#define NVSHMEMX_ERRORS_EXIT 0   /* prototype behaviour: print, exit(-1) */
#define NVSHMEMX_ERRORS_RETURN 1 /* return NULL / error code, keep going */

#define NVSHMEMX_MAX_NPES 1024

/* Comparison operators for nvshmemx_int_wait_until_cmp (OpenSHMEM names). */
#define NVSHMEMX_CMP_EQ 0
#define NVSHMEMX_CMP_NE 1
#define NVSHMEMX_CMP_GT 2
#define NVSHMEMX_CMP_GE 3
#define NVSHMEMX_CMP_LT 4
#define NVSHMEMX_CMP_LE 5

/* Trace op codes; the first eight keep the prototype's op_type order
 * (nvshmem.cu:117). */
#define NVSHMEMX_TRACE_PUT_INT 0
#define NVSHMEMX_TRACE_PUT_FLOAT 1
#define NVSHMEMX_TRACE_PUT_DOUBLE 2
#define NVSHMEMX_TRACE_GET_INT 3
#define NVSHMEMX_TRACE_GET_FLOAT 4
#define NVSHMEMX_TRACE_GET_DOUBLE 5
#define NVSHMEMX_TRACE_WAIT_INT 6
#define NVSHMEMX_TRACE_WAIT_UNTIL_INT 7
#define NVSHMEMX_TRACE_BARRIER 8
#define NVSHMEMX_TRACE_QUIET 9
#define NVSHMEMX_TRACE_P 10
#define NVSHMEMX_TRACE_G 11
#define NVSHMEMX_TRACE_BEGIN 12
#define NVSHMEMX_TRACE_END 13

/* One trace-ring record (48 bytes). */
typedef struct nvshmemx_trace_record {
  long long t_ns;                  /* %globaltimer when the op started        */
  long long spin_ns;               /* time spent in the op (waits: spinning)  */
  unsigned long long local_addr;   /* local operand                           */
  unsigned long long remote_addr;  /* translated remote operand               */
  unsigned int bytes;              /* payload bytes                           */
  unsigned short op;               /* NVSHMEMX_TRACE_*                        */
  unsigned short pe;               /* calling PE                              */
  unsigned short peer;             /* target PE                               */
  unsigned short tid;              /* thread index in the block               */
  unsigned int block;              /* linear block index within the PE        */
} nvshmemx_trace_record;

#ifdef __cplusplus
extern "C" {
#endif

/* ---- host: lifetime and status ------------------------------------------ */
/* nvstart_pes with explicit values instead of NVSHMEM_NPES/NVSHMEM_HEAP_SIZE;
 * returns a status code instead of exiting. */
int nvshmemx_init_attr(int npes, size_t heap_bytes_per_pe);
/* Process-per-PE mode, the prototype's own model (one process per PE, as its
 * MPI ranks were; nvshmem.cu:472-561): this process becomes PE `pe` of `npes`
 * processes that meet in the directory `rendezvous_dir`, where they exchange
 * their slices' VMM handles over Unix sockets and share the host barrier.
 * Every slice is mapped in every process at the same arena layout, so device
 * calls work unchanged; nvshmem_barrier_all synchronises the device and meets
 * the other processes on the host, and nvshmem_barrier_all_offload does the
 * same (kernels of different processes cannot wait for each other on one GPU,
 * so device-side waits on another process's data are not supported).
 * nvstart_pes enters this mode when NVSHMEM_PROCESS_PE and
 * NVSHMEM_RENDEZVOUS are set (python -m nvshmem_b200.launch sets them);
 * NVSHMEM_DEVICE, when set, selects this process's device first. */
int nvshmemx_init_process(int pe, int npes, size_t heap_bytes_per_pe, const char *rendezvous_dir);

/* Process-per-PE mode started by the application's own launcher: the
 * prototype bootstraps through MPI inside nvstart_pes (MPI_Comm_rank/size,
 * MPI_Allgather of its IPC handles, MPI_Barrier; nvshmem.cu:480-561).  Here
 * the caller hands over its rank, size and an allgather callback (for an MPI
 * program, a wrapper of MPI_Allgather with MPI_BYTE on its communicator), and
 * this process becomes PE `rank` of `size` as with nvshmemx_init_process.
 * The callback is called with identical `len` by every rank and must fill
 * out[size * len] with every rank's `len` bytes in rank order, returning 0 on
 * success.  Rank 0 makes a private rendezvous directory under $TMPDIR (or
 * /tmp) and shares its name through the callback; once every process has
 * mapped every slice (a second allgather of each rank's start status), rank 0
 * removes the directory's entries, which nothing uses after start-up.  All
 * processes must be on one node (slices are exchanged as POSIX file
 * descriptors).  Returns 0 when every rank started; otherwise no rank is
 * left started. */
typedef struct nvshmemx_bootstrap {
  int rank;
  int size;
  int (*allgather)(const void *in, void *out, size_t len, void *ctx);
  void *ctx;
} nvshmemx_bootstrap;
int nvshmemx_init_bootstrap(const nvshmemx_bootstrap *bs, size_t heap_bytes_per_pe);
/* nvstop_pes with a status code. */
int nvshmemx_finalize(void);
int nvshmemx_is_started(void);
/* First error recorded since the last call (host side or the device status
 * word, which this call reads after synchronising), then clears it. */
int nvshmemx_status(void);
/* Extra detail of the last device error: the PE and the address or counter
 * value involved (-1 if none). */
long long nvshmemx_status_detail(void);
void nvshmemx_set_error_mode(int mode);
int nvshmemx_get_error_mode(void);
const char *nvshmemx_strerror(int code);
/* Message of the most recent host-side failure ("" if none yet). */
const char *nvshmemx_last_error_string(void);

/* ---- host: arena queries and direct access ------------------------------ */
void *nvshmemx_arena_base(void);
size_t nvshmemx_slice_stride(void);  /* distance between slices (power of 2) */
size_t nvshmemx_heap_size(void);     /* usable bytes per slice               */
size_t nvshmemx_heap_used(int pe);   /* bump-allocator tail of PE `pe`       */
int nvshmemx_heap_write(int pe, size_t offset, const void *src, size_t bytes);
int nvshmemx_heap_read(int pe, size_t offset, void *dst, size_t bytes);
int nvshmemx_heap_memset(int pe, size_t offset, int value, size_t bytes);
int nvshmemx_sm_count(void);
int nvshmemx_device_sync(void);

/* ---- host: waits, SPMD threads ------------------------------------------ */
void nvshmemx_set_wait_timeout_ns(long long ns);
long long nvshmemx_get_wait_timeout_ns(void);
/* Run fn(arg) on one host thread per PE; nvshmem_my_pe() answers each
 * thread's PE, nvshmalloc advances that PE's tail only, and
 * nvshmem_barrier_all also meets the other PE threads. */
int nvshmemx_spmd_run(void (*fn)(void *), void *arg);

/* ---- host: trace ring --------------------------------------------------- */
int nvshmemx_trace_enable(unsigned int records_per_pe);
int nvshmemx_trace_disable(void);
/* Copies up to max_records of PE `pe`'s ring (oldest first); returns the
 * number copied, or -1.  *dropped receives how many were overwritten. */
long long nvshmemx_trace_read(int pe, nvshmemx_trace_record *out,
                              size_t max_records, long long *dropped);
int nvshmemx_trace_reset(void);
/* Writes <prefix>_<pe> per PE in the prototype's processed-trace CSV format
 * (nvshmem.cu:390,411-433). */
int nvshmemx_trace_write_csv(const char *prefix);

#ifdef __cplusplus
}
#endif

/* ---- CUDA-typed host API ------------------------------------------------ */
#if defined(__CUDACC__) || defined(__CUDA_RUNTIME_API_H__)
#include <cuda_runtime_api.h>
#ifdef __cplusplus
extern "C" {
#endif
/* Launch `func` once for all PEs: the grid becomes (grid.x, grid.y, n_pes),
 * PE p runs blocks with blockIdx.z == p.  The launch is cooperative, so every
 * CTA of every PE is co-resident and device waits between PEs make progress;
 * a grid that cannot be co-resident fails with NVSHMEMX_ERR_COOP.  The
 * device barrier counter is reset on `stream` before the launch, so
 * collective launches must not overlap each other. */
int nvshmemx_collective_launch(const void *func, dim3 grid_per_pe, dim3 block,
                               void **args, size_t smem_bytes,
                               cudaStream_t stream);
/* Largest CTA count per PE for which `func` with this block and dynamic
 * shared memory still fits a collective launch. */
int nvshmemx_collective_max_ctas_per_pe(const void *func, int block_threads,
                                        size_t smem_bytes);
#ifdef __cplusplus
}
#endif
#endif

/* ---- device extensions -------------------------------------------------- */
#ifdef __CUDACC__
#ifdef __cplusplus
extern "C" {
#endif
/* PE of the calling CTA: blockIdx.z in a collective launch, 0 otherwise. */
__device__ int nvshmemx_my_pe(void);
__device__ int nvshmemx_n_pes(void);
/* Device-side nvshmem_ptr: the object `sym` in PE `pe`'s slice (NULL if out
 * of the arena). */
__device__ void *nvshmemx_ptr(const void *sym, int pe);
/* The object `sym` in the calling PE's slice. */
__device__ void *nvshmemx_local_ptr(const void *sym);

/* Cooperative put/get: every thread of the warp (block) calls with the same
 * arguments; copies use coalesced 16-byte accesses. */
__device__ void nvshmemx_putmem_warp(void *target, const void *source, size_t bytes, int pe);
__device__ void nvshmemx_getmem_warp(void *target, const void *source, size_t bytes, int pe);
__device__ void nvshmemx_putmem_block(void *target, const void *source, size_t bytes, int pe);
__device__ void nvshmemx_getmem_block(void *target, const void *source, size_t bytes, int pe);
__device__ void nvshmemx_int_put_warp(int *target, int *source, int len, int pe);
__device__ void nvshmemx_float_put_warp(float *target, float *source, int len, int pe);
__device__ void nvshmemx_double_put_warp(double *target, double *source, int len, int pe);
__device__ void nvshmemx_int_get_warp(int *target, int *source, int len, int pe);
__device__ void nvshmemx_float_get_warp(float *target, float *source, int len, int pe);
__device__ void nvshmemx_double_get_warp(double *target, double *source, int len, int pe);
__device__ void nvshmemx_int_put_block(int *target, int *source, int len, int pe);
__device__ void nvshmemx_float_put_block(float *target, float *source, int len, int pe);
__device__ void nvshmemx_double_put_block(double *target, double *source, int len, int pe);
__device__ void nvshmemx_int_get_block(int *target, int *source, int len, int pe);
__device__ void nvshmemx_float_get_block(float *target, float *source, int len, int pe);
__device__ void nvshmemx_double_get_block(double *target, double *source, int len, int pe);

/* Block-cooperative copy staged through shared memory with cp.async.bulk
 * (global -> shared -> global, mbarrier-tracked ring of six stages).  `smem`
 * must be 128-byte aligned shared memory; with `smem_bytes` below 6272 (six
 * stages of 1 KiB plus 128 bytes of mbarriers) the copy takes the generic
 * path, and 64 KiB is what the library's own launches give it.  Unaligned
 * heads and tails are copied by the generic path.  All threads of the block
 * call. */
__device__ void nvshmemx_putmem_bulk_block(void *target, const void *source, size_t bytes,
                                           int pe, void *smem, unsigned int smem_bytes);
__device__ void nvshmemx_getmem_bulk_block(void *target, const void *source, size_t bytes,
                                           int pe, void *smem, unsigned int smem_bytes);

/* Release store of a 4-byte signal: orders the caller's earlier stores
 * before it (nvshmem_quiet + nvshmem_int_p in one). */
__device__ void nvshmemx_int_signal(int *target, int value, int pe);
/* Bounded wait with an OpenSHMEM comparison; returns NVSHMEMX_SUCCESS or
 * NVSHMEMX_ERR_TIMEOUT (and then also records it in the status word).
 * timeout_ns <= 0 uses the library deadline. */
__device__ int nvshmemx_int_wait_until_cmp(int *ivar, int cmp, int value, long long timeout_ns);
/* Barrier over every CTA of the current collective launch (all PEs): orders
 * all earlier stores of all participants before everything after it.
 * Returns NVSHMEMX_ERR_TIMEOUT if the deadline passed. */
__device__ int nvshmemx_barrier_all(void);
/* Barrier over the CTAs of the calling PE only. */
__device__ int nvshmemx_barrier_pe(void);
/* nvshmemx_barrier_all for callers that count their barriers: `episode` is
 * the number of earlier device barriers of this collective launch (0 for the
 * first).  Every CTA must pass the same sequence.  Saves one atomic round
 * trip per barrier. */
__device__ int nvshmemx_barrier_all_ep(unsigned long long episode);
#ifdef __cplusplus
}
#endif
#endif /* __CUDACC__ */

#endif /* NVSHMEM_B200_NVSHMEMX_H_ */
