/*
 * nvshmem_device.h -- device API of the B200 virtual-PE symmetric-memory
 * library.  Same names and signatures as the prototype's nvshmem_device.h:34-75
 * (extern "C" __device__ functions), so kernels written against it recompile
 * unchanged with -rdc=true and link against libnvshmem.a.
 *
 * Semantics (identical to nvshmem_device.cu:431-584 unless noted):
 *  - `target` of p/put and `source` of g/get are symmetric addresses: any
 *    address of the object in any PE's slice names it.  They are translated to
 *    PE `pe`'s slice as  arena + pe*stride + ((addr - arena) & (stride-1)).
 *  - the other pointer of put/get is used as given (a local device pointer).
 *  - put/get copy `len` ELEMENTS; the calling thread copies all of them (the
 *    warp/block/bulk cooperative forms are in nvshmemx.h).  From 32 KiB on,
 *    the thread also has the TMA unit prefetch its source into L2 16 KiB
 *    ahead of its loads (a hint: the bytes copied are the same).
 *  - nvshmem_quiet orders all earlier stores of the calling thread before its
 *    later ones at GPU scope (all PEs share one GPU, so L2 is the coherence
 *    point; the prototype needed the system-scope fence of PCIe P2P).
 *  - nvshmem_int_wait returns once *ivar != cmp_value; nvshmem_int_wait_until
 *    returns once *ivar == cmp_value and, like the prototype, ignores `cmp`.
 *    Unlike the prototype, both give up after the wait deadline
 *    (NVSHMEM_WAIT_TIMEOUT_NS, default 5 s) and record NVSHMEMX_ERR_TIMEOUT
 *    in the device status word instead of spinning forever.
 *  - an address outside the arena or a PE out of range is not accessed; the
 *    call records NVSHMEMX_ERR_BOUNDS instead of faulting.
 */
#ifndef NVSHMEM_B200_NVSHMEM_DEVICE_H_
#define NVSHMEM_B200_NVSHMEM_DEVICE_H_

#ifdef __cplusplus
extern "C" {
#endif

/* Open/close a tracing scope; records go to the %globaltimer trace ring when
 * tracing is enabled (nvshmem_device.h:38-39). */
__device__ void nvshmem_trace_begin(void);
__device__ void nvshmem_trace_end(void);

/* nvshmem_device.h:40 / nvshmem_device.cu:431-436. */
__device__ void nvshmem_quiet(void);

/* Single-element remote store, nvshmem_device.h:42-48 / nvshmem_device.cu:439-460. */
__device__ void nvshmem_int_p(int *target, const int value, int pe);
__device__ void nvshmem_float_p(float *target, const float value, int pe);
__device__ void nvshmem_double_p(double *target, const double value, int pe);

/* Single-element remote load, nvshmem_device.h:50-55 / nvshmem_device.cu:463-485. */
__device__ int nvshmem_int_g(int *source, int pe);
__device__ float nvshmem_float_g(float *source, int pe);
__device__ double nvshmem_double_g(double *source, int pe);

/* Bulk put of `len` elements from local `source` to symmetric `target` on `pe`,
 * nvshmem_device.h:57-62 / nvshmem_device.cu:488-512. */
__device__ void nvshmem_int_put(int *target, int *source, int len, int pe);
__device__ void nvshmem_float_put(float *target, float *source, int len, int pe);
__device__ void nvshmem_double_put(double *target, double *source, int len, int pe);

/* Bulk get of `len` elements from symmetric `source` on `pe` to local `target`,
 * nvshmem_device.h:64-69 / nvshmem_device.cu:515-540. */
__device__ void nvshmem_int_get(int *target, int *source, int len, int pe);
__device__ void nvshmem_float_get(float *target, float *source, int len, int pe);
__device__ void nvshmem_double_get(double *target, double *source, int len, int pe);

/* nvshmem_device.h:71-72 / nvshmem_device.cu:542-584. */
__device__ void nvshmem_int_wait(int *ivar, int cmp_value);
__device__ void nvshmem_int_wait_until(int *ivar, int cmp, int cmp_value);

#ifdef __cplusplus
}
#endif

#endif /* NVSHMEM_B200_NVSHMEM_DEVICE_H_ */
