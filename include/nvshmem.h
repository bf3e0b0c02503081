/*
 * nvshmem.h -- host API of the B200 virtual-PE symmetric-memory library.
 *
 * Every declaration keeps the name, signature and argument meaning of the
 * prototype's host API (nvshmem.h:34-55 of NVIDIA/df-nvshmem-prototype), so
 * applications written against it recompile unchanged.
 *
 * What differs underneath: all PEs ("processing elements") live on ONE GPU.
 * The symmetric heap is a single HBM arena cut into equal per-PE slices whose
 * stride is a power of two; a PE is a group of CTAs inside one launch
 * (see nvshmemx.h: nvshmemx_collective_launch) and, on the host, optionally a
 * thread started by nvshmemx_spmd_run.  No MPI is needed: nvstart_pes() reads
 * the PE count from NVSHMEM_NPES (default 2) and the per-PE heap size from
 * NVSHMEM_HEAP_SIZE (default 1 GiB, the prototype's HEAP_SIZE).
 *
 * Error behaviour matches the prototype by default: a failing CUDA call, a bad
 * argument or an exhausted heap prints a message and calls exit(-1)
 * (nvshmem.cu:57-91, :780-783).  nvshmemx_set_error_mode(NVSHMEMX_ERRORS_RETURN)
 * or NVSHMEM_ERROR_MODE=return switches to returning NULL / recording a code
 * that nvshmemx_status() reports.
 */
#ifndef NVSHMEM_B200_NVSHMEM_H_
#define NVSHMEM_B200_NVSHMEM_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same macro as nvshmem.h:38-42: a volatile view of a pointer unless the
 * application opts out with NONVOLATILE_UPDATES. */
#ifndef NONVOLATILE_UPDATES
#define VOLATILE_POINTER(x) ((volatile __typeof__(*(x)) *)(x))
#else
#define VOLATILE_POINTER(x) (x)
#endif

/* Start the PEs: allocate the arena (npes x slice), zero the signal and
 * barrier words and publish the device-side configuration.
 * Replaces nvstart_pes, nvshmem.h:44 / nvshmem.cu:472-773. */
void nvstart_pes(void);

/* Release the arena and all library state.  nvshmem.h:45 / nvshmem.cu:821-856. */
void nvstop_pes(void);

/* PE of the calling host thread: its PE inside nvshmemx_spmd_run, 0 on any
 * other thread (the launching thread speaks for PE 0).
 * nvshmem.h:46 / nvshmem.cu:193-196. */
int nvshmem_my_pe(void);

/* Number of virtual PEs.  nvshmem.h:47 / nvshmem.cu:198-201. */
int nvshmem_n_pes(void);

/* Symmetric bump allocation of `size` bytes, with no alignment padding, as in
 * nvshmem.cu:775-802: the k-th allocation lands at the same offset in every
 * slice.  Returns the address inside the calling thread's PE slice. */
void *nvshmalloc(size_t size);

/* Drop every allocation and reset the heap tail.  nvshmem.h:49 /
 * nvshmem.cu:805-819. */
void nvshmcleanup(void);

/* Host barrier: waits for all device work of every PE, then (inside
 * nvshmemx_spmd_run) for every PE thread.  Replaces cuCtxSynchronize +
 * MPI_Barrier, nvshmem.h:50 / nvshmem.cu:858-867. */
void nvshmem_barrier_all(void);

/* Device-side barrier enqueued on the legacy default stream without blocking
 * the host: a one-CTA-per-PE cooperative kernel whose CTAs meet on a ticket
 * counter.  nvshmem.h:51 / nvshmem.cu:869-878, nvshmem_kernels.cu:56-102. */
void nvshmem_barrier_all_offload(void);

/* Address of the symmetric object `local` in PE `pe`'s slice; NULL when
 * `local` is not inside the arena or `pe` is out of range.
 * nvshmem.h:52 / nvshmem.cu:880-883. */
void *nvshmem_ptr(void *local, int pe);

#ifdef __cplusplus
}
#endif

#endif /* NVSHMEM_B200_NVSHMEM_H_ */
