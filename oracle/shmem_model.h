/*
 * shmem_model.h -- CPU oracle for the one-sided path.  TEST INFRASTRUCTURE
 * ONLY: tests, the smoke check and the CPU-baseline leg of the benchmark use
 * it as the checker; the library never links or calls it.
 *
 * It restates, sequentially and byte-for-byte, what the prototype's device
 * API and allocator do to the PEs' heaps (NVIDIA/df-nvshmem-prototype):
 *   nvshmalloc / nvshmcleanup     nvshmem.cu:775-819 (bump, no padding)
 *   nvshmem_ptr                   nvshmem.cu:880-883
 *   nvshmem_T_p / _g              nvshmem_device.cu:439-485
 *   nvshmem_T_put / _get          nvshmem_device.cu:488-540
 *   nvshmem_quiet                 nvshmem_device.cu:431-436 (no-op here)
 *   nvshmem_int_wait(_until)      nvshmem_device.cu:542-584 (predicates)
 *   barriers                      phase boundaries of the sequential model
 * plus scenario drivers composed only of those calls: the ping-pong of
 * microbench/shmem_latency.cu:48-81, all-to-all rounds, the halo exchange
 * and request lists.
 *
 * Parity anchoring: the prototype ships no tests or golden vectors; this
 * model is pinned against the prototype's own build run multi-process on one
 * GPU (oracle/ref_build) through heap hashes committed in tests/golden.
 */
#ifndef ORACLE_SHMEM_MODEL_H_
#define ORACLE_SHMEM_MODEL_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct om_model {
  int npes;
  size_t slice;        /* bytes per PE image                 */
  size_t heap_limit;   /* allocator limit (NVSHMEM_HEAP_SIZE) */
  unsigned char *heap; /* npes * slice bytes                 */
  size_t *tail;        /* per-PE bump pointer                */
} om_model;

om_model *om_create(int npes, size_t slice, size_t heap_limit);
void om_destroy(om_model *m);
unsigned char *om_slice(om_model *m, int pe);

/* nvshmalloc for PE pe (pe < 0: every PE, the collective call).  Returns
 * the offset, or -1 when the reference would exit for lack of heap. */
long long om_alloc(om_model *m, int pe, size_t size);
void om_cleanup(om_model *m, int pe);
/* nvshmem_ptr on offsets: offset of `off` on PE pe, or -1 if out of range. */
long long om_ptr(const om_model *m, size_t off, int pe);

void om_p(om_model *m, int width, size_t target_off, uint64_t bits, int pe);
uint64_t om_g(const om_model *m, int width, size_t source_off, int pe);
/* The calling PE `me` copies len elements of `width` bytes. */
void om_put(om_model *m, int width, size_t target_off, int me, size_t source_off, int len, int pe);
void om_get(om_model *m, int width, int me, size_t target_off, size_t source_off, int len, int pe);

/* nvshmemx_request list applied in order (32-byte records). */
int om_apply_requests(om_model *m, const void *reqs, int n);

/* All-to-all rounds (see nvshmemx_op_alltoall). op 0 = put, 1 = get. */
void om_alltoall(om_model *m, int op, size_t send_off, size_t recv_off, size_t bytes, int rounds, int nsets,
                 size_t set_stride);

/* Halo exchange (see nvshmemx_op_halo). */
void om_halo(om_model *m, int px, int py, int pz, int n, size_t block_off, size_t ghost_off, size_t sig_off,
             int iters);

/* Ping-pong between PE 0 and 1 (microbench/shmem_latency.cu:54-72):
 * iterations i = 0..total-1; returns the sequence of flag values each PE
 * observes when its wait is satisfied into seen0/seen1 (may be NULL). */
void om_pingpong(om_model *m, size_t flag_off, size_t data_off, int len, int total, int32_t *seen0,
                 int32_t *seen1);

/* The library's deterministic fill (splitmix64 keyed on seed and PE). */
void om_fill_random(om_model *m, int pe, size_t off, size_t bytes, uint64_t seed);
uint64_t om_splitmix64(uint64_t x);
/* The library's checksum of 8-byte words. */
uint64_t om_checksum(const unsigned char *p, size_t bytes);
/* FNV-1a 64 of a byte range (heap-image hashes for golden files). */
uint64_t om_fnv1a(const unsigned char *p, size_t bytes);

#ifdef __cplusplus
}
#endif

#endif
