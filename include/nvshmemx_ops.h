/*
 * nvshmemx_ops.h -- host-callable operations of the B200 virtual-PE library,
 * plain C ABI (pointers, sizes, integers; no CUDA or framework types) for
 * foreign-function callers such as Python ctypes, cgo or JNI.
 *
 * The prototype exposes its one-sided path only as __device__ functions
 * (nvshmem_device.h:34-75) called from the application's own kernels, which
 * a foreign caller cannot reach.  Each entry point here launches a library
 * kernel that drives those same device functions for one of the patterns the
 * prototype's users run: request lists (one put/get/p/g/signal per call, the
 * plain path), the put + flag ping-pong of microbench/shmem_latency.cu:48-81
 * and microbench/shmem_sync_latency.cu:48-78, the device barrier of
 * nvshmem_kernels.cu:56-102, all-to-all rounds and halo exchanges.
 *
 * Every function returns NVSHMEMX_SUCCESS (0) or an NVSHMEMX_ERR_* code and,
 * unlike the void API of nvshmem.h, never exits the process.  Offsets are
 * byte offsets inside a PE's slice of the symmetric heap.  Times are measured
 * with CUDA events on the launching stream.
 */
#ifndef NVSHMEM_B200_NVSHMEMX_OPS_H_
#define NVSHMEM_B200_NVSHMEMX_OPS_H_

#include <stddef.h>
#include <stdint.h>

#include "nvshmemx.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- request descriptors (32 bytes, 16-byte aligned in arrays) ----------- */
#define NVSHMEMX_REQ_PUT 0    /* src_pe copies bytes to dst_pe (nvshmem_T_put)       */
#define NVSHMEMX_REQ_GET 1    /* dst_pe fetches bytes from src_pe (nvshmem_T_get)    */
#define NVSHMEMX_REQ_SIGNAL 2 /* src_pe release-stores int `value` at dst_pe/dst_off */
#define NVSHMEMX_REQ_P 3      /* src_pe stores one element (bits in src_off) at dst  */
#define NVSHMEMX_REQ_G 4      /* dst_pe loads one element of src_pe into dst_off     */

#define NVSHMEMX_DT_INT 0    /* 4-byte elements */
#define NVSHMEMX_DT_FLOAT 1  /* 4-byte elements */
#define NVSHMEMX_DT_DOUBLE 2 /* 8-byte elements */

typedef struct nvshmemx_request {
  uint64_t src_off;  /* byte offset in src_pe's slice (P: the element's bits) */
  uint64_t dst_off;  /* byte offset in dst_pe's slice                        */
  uint32_t bytes;    /* payload bytes, a multiple of the element width       */
  uint16_t src_pe;
  uint16_t dst_pe;
  uint8_t op;        /* NVSHMEMX_REQ_*                                       */
  uint8_t dtype;     /* NVSHMEMX_DT_*                                        */
  uint16_t flags;    /* reserved, 0                                          */
  int32_t value;     /* SIGNAL value                                         */
} nvshmemx_request;

/* Compact form of a request (16 bytes) for nvshmemx_batch_submit_compact,
 * which halves what crosses the host link.  It holds every request whose
 * offsets and sizes are multiples of 4 below 16 GiB and whose PEs are below
 * 1024, except P of a double (64-bit value):
 *   src_off4  src_off / 4 (P: the int or float element's bits)
 *   dst_off4  dst_off / 4
 *   arg       PUT / GET: bytes / 4; SIGNAL: value; P, G: 0
 *   meta      src_pe | dst_pe << 10 | op << 20 | dtype << 23 (bits 25-31 0) */
typedef struct nvshmemx_request_compact {
  uint32_t src_off4;
  uint32_t dst_off4;
  uint32_t arg;
  uint32_t meta;
} nvshmemx_request_compact;

/* How a request is carried out (the per-call variants). */
#define NVSHMEMX_MODE_THREAD 0 /* one thread per request, nvshmem_{T}_put/get/p/g */
#define NVSHMEMX_MODE_WARP 1   /* one warp per request, nvshmemx_{T}_put/get_warp  */
#define NVSHMEMX_MODE_BLOCK 2  /* one CTA per request, nvshmemx_{T}_put/get_block  */
#define NVSHMEMX_MODE_BULK 3   /* one CTA per request, TMA bulk ring               */

/* Runs n requests (host array) as one launch, one caller unit per request,
 * through the public device API; requests must not overlap in their
 * destinations.  *out_ms receives the kernel time (may be NULL). */
int nvshmemx_exec_requests(const nvshmemx_request *reqs, int n, int mode, float *out_ms);

/* ---- deterministic fill and on-device comparison ------------------------- */
/* Fills [off, off+bytes) of PE pe with the splitmix64 stream of `seed`:
 * 8-byte word w (counted from slice offset 0) = splitmix64(seed, pe, w). */
int nvshmemx_fill_random(int pe, size_t off, size_t bytes, uint64_t seed);
/* Number of bytes that differ between [a_off, +bytes) of PE a and
 * [b_off, +bytes) of PE b (0 means bit-identical). */
int nvshmemx_compare(int a_pe, size_t a_off, int b_pe, size_t b_off, size_t bytes,
                     unsigned long long *out_mismatches);
/* 64-bit checksum of [off, off+bytes) of PE pe: sum over 8-byte words w of
 * splitmix64(word ^ (w_index * golden)); bytes must be a multiple of 8. */
int nvshmemx_checksum(int pe, size_t off, size_t bytes, unsigned long long *out_sum);

/* ---- C1: put + flag ping-pong between PE 0 and PE 1 ----------------------
 * Iteration i: PE 0 puts len_elems ints (nvshmem_int_put), quiets and sets
 * PE 1's flag to i+1 (nvshmem_int_p), then waits for its own flag to leave i
 * (nvshmem_int_wait); PE 1 waits for its flag to leave i, puts its data back
 * and echoes i+1 -- the put + flag exchange of
 * microbench/shmem_latency.cu:54-72; len_elems == 0 gives the flag-only
 * exchange of microbench/shmem_sync_latency.cu:54-70.  flag_off / data_off
 * are symmetric offsets; both PEs' flag words are set to 0 first, so calls
 * may reuse one flag.  out_ns[iters]
 * receives PE 0's per-iteration round trip in ns (may be NULL);
 * *out_total_ns the timed total. */
int nvshmemx_op_pingpong(size_t flag_off, size_t data_off, int len_elems, int iters, int skip,
                         double *out_ns, double *out_total_ns);

/* ---- device barrier latency --------------------------------------------- */
/* iters back-to-back device barriers over ctas_per_pe CTAs per PE:
 * nvshmemx_barrier_all() (counted == 0) or nvshmemx_barrier_all_ep(i)
 * (counted != 0); out_ns[iters] = per-barrier interval seen by PE 0's first
 * CTA (may be NULL), *out_total_ns the total. */
int nvshmemx_op_barrier_latency(int ctas_per_pe, int iters, int counted, double *out_ns, double *out_total_ns);
/* iters host calls of nvshmem_barrier_all_offload(); *out_us_per_call. */
int nvshmemx_op_offload_barrier(int iters, double *out_us_per_call);

/* ---- C2: all-to-all rounds ----------------------------------------------
 * Each PE p holds npes blocks of `bytes` at send_off (block q is for PE q)
 * and receives block p of every peer into slot p of recv_off.  PUT: p writes
 * its block q into q's slot p; GET: p reads q's block p into its slot q.  The
 * PE itself is skipped (npes-1 messages per PE).  Each round is followed by
 * nvshmem_quiet and the device barrier.  Round r uses buffer set r % nsets,
 * set s at send_off + s*set_stride / recv_off + s*set_stride, so the working
 * set can exceed L2.  mode: NVSHMEMX_MODE_* (THREAD = one thread per message
 * through nvshmem_{T}_put/get).  dtype selects the typed call for THREAD.
 * ctas_per_pe 0: NVSHMEM_CTAS_PER_PE if set, else SMs / npes. */
int nvshmemx_op_alltoall(int op, int dtype, size_t send_off, size_t recv_off, size_t bytes,
                         int rounds, int nsets, size_t set_stride, int mode, int ctas_per_pe,
                         float *out_ms);
/* The same rounds in the prototype's own structure: one collective launch
 * per round (puts or gets, then nvshmem_quiet) followed by the host's
 * nvshmem_barrier_all(); the heaps end identical. */
int nvshmemx_op_alltoall_host(int op, int dtype, size_t send_off, size_t recv_off, size_t bytes,
                              int rounds, int nsets, size_t set_stride, int mode, int ctas_per_pe,
                              float *out_ms);

/* ---- C3: halo exchange on a periodic px x py x pz PE grid ----------------
 * Each PE owns an n^3 float64 block at block_off (x fastest).  Per iteration
 * it puts its 6 faces (n x n doubles; x faces gathered with stride n, y faces
 * row by row) into the neighbours' ghost buffers at ghost_off (6 consecutive
 * n*n*8-byte buffers ordered -x,+x,-y,+y,-z,+z of the RECEIVER: the face a
 * receiver gets from its -x neighbour goes to its -x ghost), then quiets,
 * sets the neighbour's signal (int at sig_off + 4*face) to it+1 with
 * nvshmem_int_p, waits for its own 6 signals with nvshmem_int_wait_until,
 * and meets the others at the device barrier.  ctas_per_pe 0 launches
 * NVSHMEM_CTAS_PER_PE CTAs per PE if that is set, else as many as stay
 * co-resident. */
int nvshmemx_op_halo(int px, int py, int pz, int n, size_t block_off, size_t ghost_off,
                     size_t sig_off, int iters, int ctas_per_pe, float *out_ms);
/* The same exchange in the prototype's own structure: one collective launch
 * per iteration (faces, quiet, signals, waits) followed by the host's
 * nvshmem_barrier_all_offload(), iters times; the heaps end identical. */
int nvshmemx_op_halo_offload(int px, int py, int pz, int n, size_t block_off, size_t ghost_off,
                             size_t sig_off, int iters, int ctas_per_pe, float *out_ms);

/* ---- measurement: the halo's gather ceiling ------------------------------
 * No counterpart in the reference.  Every PE reads nsets x rows 8-byte
 * elements of its own slice, element i of set t at off + t * set_off +
 * i * stride, with ctas_per_pe CTAs of 256 threads per PE and 8 loads in
 * flight per thread, `iters` launches back to back; *out_ms their device
 * time.  With the halo's x faces (rows = n*n, stride = 8n, sets at x = 0 and
 * x = n-1) it is the time those faces need at best: the same scattered
 * reads with nothing else to do. */
int nvshmemx_op_strided_read(size_t off, size_t set_off, int nsets, size_t rows, size_t stride, int ctas_per_pe,
                             int iters, float *out_ms);

/* ---- failure detection ---------------------------------------------------
 * One thread of PE 0 waits (nvshmemx_int_wait_until_cmp EQ) on the int at
 * flag_off for `value` with the given deadline; returns the wait's status
 * (NVSHMEMX_ERR_TIMEOUT if nothing set it) in *out_status. */
int nvshmemx_op_wait_test(size_t flag_off, int value, long long timeout_ns, int *out_status);
/* A collective barrier in which PE `skip_pe` never arrives: every other CTA
 * must leave with NVSHMEMX_ERR_TIMEOUT after timeout_ns. */
int nvshmemx_op_barrier_fault_test(int skip_pe, long long timeout_ns, int *out_status);

#ifdef __cplusplus
}
#endif

#endif /* NVSHMEM_B200_NVSHMEMX_OPS_H_ */
