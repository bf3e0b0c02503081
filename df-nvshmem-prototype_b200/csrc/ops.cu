// ops.cu -- host-callable operations (nvshmemx_ops.h) built on the public
// device API of nvshmem_device.h / nvshmemx.h.  The kernels here are what an
// application of the prototype writes by hand: they call nvshmem_int_put,
// nvshmem_int_p, nvshmem_int_wait_until, nvshmem_quiet ... from inside one
// collective launch in which blockIdx.z is the PE.
#include <cuda_runtime.h>
#include <stdio.h>

#include <algorithm>
#include <vector>

#include "nvshmem_device.h"
#include "nvshmemx.h"
#include "nvshmemx_ops.h"
#include "procs.h"
#include "runtime.h"

namespace nvshm {

// Grow-only device scratch owned by the library (request uploads, results).
struct DevScratch {
  void *p = nullptr;
  size_t n = 0;
  void *get(size_t bytes) {
    if (bytes > n) {
      if (p) cudaFree(p);
      p = nullptr;
      n = 0;
      if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
      n = bytes;
    }
    return p;
  }
};
static DevScratch g_req_buf, g_out_buf;

struct EventTimer {
  cudaEvent_t a = nullptr, b = nullptr;
  EventTimer() {
    cudaEventCreate(&a);
    cudaEventCreate(&b);
  }
  ~EventTimer() {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
  }
  void start(cudaStream_t s = 0) { cudaEventRecord(a, s); }
  void stop(cudaStream_t s = 0) { cudaEventRecord(b, s); }
  float ms() {
    float m = 0;
    cudaEventSynchronize(b);
    cudaEventElapsedTime(&m, a, b);
    return m;
  }
};

__device__ __forceinline__ char *slice_ptr(const Cfg &c, int pe, unsigned long long off) {
  return c.arena + ((unsigned long long)(unsigned)pe << c.log2_stride) + off;
}

// ------------------------------------------------------------ request lists
// One caller unit per request: a thread (MODE_THREAD), a warp (MODE_WARP) or
// a CTA (MODE_BLOCK / MODE_BULK).  The symmetric operand is passed as PE 0's
// copy of the object (any slice names the same object).
template <int MODE>
__global__ void exec_requests_kernel(Cfg c, const nvshmemx_request *__restrict__ reqs, int n,
                                     unsigned bulk_smem) {
  extern __shared__ __align__(128) char smem[];
  long long u;
  if (MODE == NVSHMEMX_MODE_THREAD)
    u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  else if (MODE == NVSHMEMX_MODE_WARP)
    u = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  else
    u = blockIdx.x;
  if (u >= n) return;
  const nvshmemx_request r = reqs[u];
  const bool leader = MODE == NVSHMEMX_MODE_THREAD || (MODE == NVSHMEMX_MODE_WARP ? (threadIdx.x & 31) == 0
                                                                                 : threadIdx.x == 0);
  const int w = r.dtype == NVSHMEMX_DT_DOUBLE ? 8 : 4;
  const int len = (int)(r.bytes / (unsigned)w);
  switch (r.op) {
    case NVSHMEMX_REQ_PUT: {
      char *sym = c.arena + r.dst_off;
      char *src = slice_ptr(c, r.src_pe, r.src_off);
      if (MODE == NVSHMEMX_MODE_THREAD) {
        if (r.dtype == NVSHMEMX_DT_INT) nvshmem_int_put((int *)sym, (int *)src, len, r.dst_pe);
        else if (r.dtype == NVSHMEMX_DT_FLOAT) nvshmem_float_put((float *)sym, (float *)src, len, r.dst_pe);
        else nvshmem_double_put((double *)sym, (double *)src, len, r.dst_pe);
      } else if (MODE == NVSHMEMX_MODE_WARP) {
        if (r.dtype == NVSHMEMX_DT_INT) nvshmemx_int_put_warp((int *)sym, (int *)src, len, r.dst_pe);
        else if (r.dtype == NVSHMEMX_DT_FLOAT) nvshmemx_float_put_warp((float *)sym, (float *)src, len, r.dst_pe);
        else nvshmemx_double_put_warp((double *)sym, (double *)src, len, r.dst_pe);
      } else if (MODE == NVSHMEMX_MODE_BLOCK) {
        if (r.dtype == NVSHMEMX_DT_INT) nvshmemx_int_put_block((int *)sym, (int *)src, len, r.dst_pe);
        else if (r.dtype == NVSHMEMX_DT_FLOAT) nvshmemx_float_put_block((float *)sym, (float *)src, len, r.dst_pe);
        else nvshmemx_double_put_block((double *)sym, (double *)src, len, r.dst_pe);
      } else {
        nvshmemx_putmem_bulk_block(sym, src, (size_t)len * w, r.dst_pe, smem, bulk_smem);
      }
      break;
    }
    case NVSHMEMX_REQ_GET: {
      char *sym = c.arena + r.src_off;
      char *dst = slice_ptr(c, r.dst_pe, r.dst_off);
      if (MODE == NVSHMEMX_MODE_THREAD) {
        if (r.dtype == NVSHMEMX_DT_INT) nvshmem_int_get((int *)dst, (int *)sym, len, r.src_pe);
        else if (r.dtype == NVSHMEMX_DT_FLOAT) nvshmem_float_get((float *)dst, (float *)sym, len, r.src_pe);
        else nvshmem_double_get((double *)dst, (double *)sym, len, r.src_pe);
      } else if (MODE == NVSHMEMX_MODE_WARP) {
        if (r.dtype == NVSHMEMX_DT_INT) nvshmemx_int_get_warp((int *)dst, (int *)sym, len, r.src_pe);
        else if (r.dtype == NVSHMEMX_DT_FLOAT) nvshmemx_float_get_warp((float *)dst, (float *)sym, len, r.src_pe);
        else nvshmemx_double_get_warp((double *)dst, (double *)sym, len, r.src_pe);
      } else if (MODE == NVSHMEMX_MODE_BLOCK) {
        if (r.dtype == NVSHMEMX_DT_INT) nvshmemx_int_get_block((int *)dst, (int *)sym, len, r.src_pe);
        else if (r.dtype == NVSHMEMX_DT_FLOAT) nvshmemx_float_get_block((float *)dst, (float *)sym, len, r.src_pe);
        else nvshmemx_double_get_block((double *)dst, (double *)sym, len, r.src_pe);
      } else {
        nvshmemx_getmem_bulk_block(dst, sym, (size_t)len * w, r.src_pe, smem, bulk_smem);
      }
      break;
    }
    case NVSHMEMX_REQ_SIGNAL:
      if (leader) nvshmemx_int_signal((int *)(c.arena + r.dst_off), r.value, r.dst_pe);
      break;
    case NVSHMEMX_REQ_P:
      if (leader) {
        char *sym = c.arena + r.dst_off;
        if (r.dtype == NVSHMEMX_DT_INT) nvshmem_int_p((int *)sym, (int)(unsigned)r.src_off, r.dst_pe);
        else if (r.dtype == NVSHMEMX_DT_FLOAT)
          nvshmem_float_p((float *)sym, __uint_as_float((unsigned)r.src_off), r.dst_pe);
        else nvshmem_double_p((double *)sym, __longlong_as_double((long long)r.src_off), r.dst_pe);
      }
      break;
    case NVSHMEMX_REQ_G:
      if (leader) {
        char *sym = c.arena + r.src_off;
        char *dst = slice_ptr(c, r.dst_pe, r.dst_off);
        if (check_local(c, dst, w) && check_align(c, dst, w)) {
          if (r.dtype == NVSHMEMX_DT_INT) *(int *)dst = nvshmem_int_g((int *)sym, r.src_pe);
          else if (r.dtype == NVSHMEMX_DT_FLOAT) *(float *)dst = nvshmem_float_g((float *)sym, r.src_pe);
          else *(double *)dst = nvshmem_double_g((double *)sym, r.src_pe);
        }
      }
      break;
    default:
      if (leader) record_error(c, NVSHMEMX_ERR_INVALID, (long long)u);
  }
}

// ---------------------------------------------------------------- fill etc.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// Word w of PE p's slice for `seed`: the stream is keyed on (seed, pe) so
// every PE and every seed gets independent contents.
__device__ __forceinline__ unsigned long long fill_word(unsigned long long seed, int pe, unsigned long long w) {
  return splitmix64(splitmix64(seed ^ ((unsigned long long)pe << 48)) + w);
}

__global__ void fill_random_kernel(char *slice, unsigned long long off, unsigned long long bytes,
                                   unsigned long long seed, int pe) {
  // byte b (slice offset off+b) takes byte (off+b)%8 of word (off+b)/8
  const unsigned long long first_w = off >> 3, last_w = (off + bytes + 7) >> 3;
  const unsigned long long nthr = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long w = first_w + blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; w < last_w;
       w += nthr) {
    unsigned long long v = fill_word(seed, pe, w);
    unsigned long long lo = w << 3, hi = lo + 8;
    if (lo >= off && hi <= off + bytes) {
      *(unsigned long long *)(slice + lo) = v;
    } else {
      for (unsigned long long b = lo; b < hi; ++b)
        if (b >= off && b < off + bytes) slice[b] = (char)((v >> (8 * (b - lo))) & 0xff);
    }
  }
}

__global__ void compare_kernel(const unsigned char *a, const unsigned char *b, unsigned long long bytes,
                               unsigned long long *mismatches) {
  unsigned long long local = 0;
  const unsigned long long nthr = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long tid = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  if ((((uintptr_t)a | (uintptr_t)b) & 15) == 0) {
    const unsigned long long nv = bytes >> 4;
    const uint4 *a4 = (const uint4 *)a, *b4 = (const uint4 *)b;
    for (unsigned long long i = tid; i < nv; i += nthr) {
      uint4 x = a4[i], y = b4[i];
      if (x.x != y.x || x.y != y.y || x.z != y.z || x.w != y.w) {
        for (int k = 0; k < 16; ++k) local += a[i * 16 + k] != b[i * 16 + k];
      }
    }
    for (unsigned long long i = (nv << 4) + tid; i < bytes; i += nthr) local += a[i] != b[i];
  } else {
    for (unsigned long long i = tid; i < bytes; i += nthr) local += a[i] != b[i];
  }
  for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(mismatches, local);
}

__global__ void checksum_kernel(const unsigned long long *p, unsigned long long nwords, unsigned long long *out) {
  unsigned long long local = 0;
  const unsigned long long nthr = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < nwords; i += nthr)
    local += splitmix64(p[i] ^ (i * 0x9E3779B97F4A7C15ull));
  for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, local);
}

// ------------------------------------------------------------- C1 ping-pong
// The put + flag exchange of microbench/shmem_latency.cu:48-81 (and, with
// len == 0, the flag-only one of shmem_sync_latency.cu:48-78), with the PE
// taken from the launch instead of a kernel argument and the local copies of
// the symmetric objects named through nvshmemx_local_ptr.  PE 0 puts its data
// and sets PE 1's flag to i+1; PE 1 waits for its flag to leave i
// (nvshmem_int_wait), puts its data back and echoes i+1 into PE 0's flag.
// Each side has one value in flight, so no flag value can be overwritten
// before it is seen (the microbench's alternating equality waits can miss an
// i+1 that the peer already replaced with i+2).
__global__ void pingpong_kernel(int *data, int *flag, int len, int iters, int skip, long long *cycles,
                                unsigned long long *gt) {
  const int pe = nvshmemx_my_pe();
  if (pe > 1 || threadIdx.x != 0 || blockIdx.x != 0) return;
  int *my_flag = (int *)nvshmemx_local_ptr(flag);
  int *my_data = (int *)nvshmemx_local_ptr(data);
  unsigned long long g0 = 0;
  for (int i = 0; i < iters + skip; ++i) {
    if (i == skip) g0 = nvshm::gtimer();
    long long t = clock64();
    if (pe == 0) {
      if (len > 0) {
        nvshmem_int_put(data, my_data, len, 1);
        nvshmem_quiet();
      }
      nvshmem_int_p(flag, i + 1, 1);
      nvshmem_int_wait(my_flag, i);
    } else {
      nvshmem_int_wait(my_flag, i);
      if (len > 0) {
        nvshmem_int_put(data, my_data, len, 0);
        nvshmem_quiet();
      }
      nvshmem_int_p(flag, i + 1, 0);
    }
    if (pe == 0 && i >= skip) cycles[i - skip] = clock64() - t;
  }
  if (pe == 0) gt[0] = nvshm::gtimer() - g0;
}

// ------------------------------------------------------------ barrier latency
__global__ void barrier_latency_kernel(int iters, int counted, long long *cycles, unsigned long long *gt) {
  const bool rec = blockIdx.x == 0 && blockIdx.z == 0 && threadIdx.x == 0;
  unsigned long long g0 = nvshm::gtimer();
  long long t = clock64();
  for (int i = 0; i < iters; ++i) {
    if (counted)
      nvshmemx_barrier_all_ep((unsigned long long)i);
    else
      nvshmemx_barrier_all();
    if (rec) {
      long long t1 = clock64();
      cycles[i] = t1 - t;
      t = t1;
    }
  }
  if (rec) gt[0] = nvshm::gtimer() - g0;
}

// -------------------------------------------------------------- C2 all-to-all
// A CTA's share of one all-to-all round, [b, e) of the PE's (npes-1) *
// `bytes` outgoing (put) or incoming (get) bytes, streamed by one thread
// through one TMA ring of kA2aStages stages: the ring runs across message
// boundaries, so a share that spans two messages is loaded and stored
// without draining the ring between them (a cooperative bulk copy per
// message fills and drains its ring once per message).  Every chunk stays
// inside one message; all addresses are 16-byte aligned (the caller checks).
// Shared memory: 8 mbarriers, the destination and length of each stage's
// chunk (256 bytes), then the stages.  Stage reuse lags one store behind,
// as in bulk_copy_1t.  Returns false if an mbarrier wait passed `deadline`.
constexpr unsigned kA2aStages = 6;

// Where message k of the share starts: its destination and source.
__device__ __forceinline__ void a2a_message(const Cfg &c, int op, int pe, unsigned long long so, unsigned long long ro,
                                            unsigned long long bytes, unsigned long long k, char **dst,
                                            const char **src) {
  const int q = (pe + 1 + (int)k) % c.npes;
  if (op == NVSHMEMX_REQ_PUT) {
    *dst = xlate(c, c.arena + ro + (unsigned long long)pe * bytes, q);
    *src = slice_ptr(c, pe, so + (unsigned long long)q * bytes);
  } else {
    *dst = slice_ptr(c, pe, ro + (unsigned long long)q * bytes);
    *src = xlate(c, c.arena + so + (unsigned long long)pe * bytes, q);
  }
}

// The issuing thread walks the share message by message (one division at
// the start, none per chunk): a chunk costs it a few instructions, since at
// tens of GB/s per CTA a 10 KiB chunk leaves it a few hundred cycles.
__device__ __forceinline__ bool a2a_stream_1t(const Cfg &c, char *smem, unsigned smem_bytes, int op, int pe,
                                              unsigned long long so, unsigned long long ro, unsigned long long bytes,
                                              unsigned long long b, unsigned long long e,
                                              unsigned long long deadline) {
  if (b >= e) return true;
  const unsigned S = kA2aStages;
  unsigned long long *mbar = reinterpret_cast<unsigned long long *>(smem);
  unsigned long long *sdst = reinterpret_cast<unsigned long long *>(smem + 64);
  unsigned *slen = reinterpret_cast<unsigned *>(smem + 128);
  char *buf = smem + 256;
  const unsigned SB = ((smem_bytes - 256) / S) & ~127u;
  for (unsigned s = 0; s < S; ++s) mbar_init(mbar + s, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  unsigned long long k = b / bytes, off = b - k * bytes, left = e - b;
  char *dbase;
  const char *sbase;
  a2a_message(c, op, pe, so, ro, bytes, k, &dbase, &sbase);
  unsigned issued = 0, stored = 0;
  while (issued < S && left) {
    unsigned long long len = bytes - off;
    if (len > left) len = left;
    if (len > SB) len = SB;
    sdst[issued] = (unsigned long long)(dbase + off);
    slen[issued] = (unsigned)len;
    mbar_expect_tx(mbar + issued, (unsigned)len);
    bulk_g2s(buf + (size_t)issued * SB, sbase + off, (unsigned)len, mbar + issued);
    ++issued;
    off += len;
    left -= len;
    if (off == bytes && left) {
      off = 0;
      a2a_message(c, op, pe, so, ro, bytes, ++k, &dbase, &sbase);
    }
  }
  bool ok = true;
  while (stored < issued) {
    const unsigned s = stored % S;
    if (!mbar_wait(mbar + s, (stored / S) & 1u, deadline)) {
      ok = false;
      break;
    }
    bulk_s2g(reinterpret_cast<void *>(sdst[s]), buf + (size_t)s * SB, slen[s]);
    bulk_commit();
    // refill the stage the previous store read, not this one (see bulk_copy_1t)
    if (stored >= 1 && left) {
      bulk_wait_read1();
      const unsigned ps = (stored - 1) % S;
      unsigned long long len = bytes - off;
      if (len > left) len = left;
      if (len > SB) len = SB;
      sdst[ps] = (unsigned long long)(dbase + off);
      slen[ps] = (unsigned)len;
      mbar_expect_tx(mbar + ps, (unsigned)len);
      bulk_g2s(buf + (size_t)ps * SB, sbase + off, (unsigned)len, mbar + ps);
      ++issued;
      off += len;
      left -= len;
      if (off == bytes && left) {
        off = 0;
        a2a_message(c, op, pe, so, ro, bytes, ++k, &dbase, &sbase);
      }
    }
    ++stored;
  }
  bulk_wait_all();
  if (ok)
    for (unsigned s = 0; s < S; ++s) mbar_inval(mbar + s);
  return ok;
}

// Message k (0..npes-2) of PE p goes to / comes from peer q = (p+1+k) % npes.
// For the cooperative modes the PE's (npes-1)*bytes are cut into one
// contiguous, 16-byte-rounded segment per caller unit (warp or CTA), so every
// unit streams one range; MODE_THREAD keeps the prototype's shape, one thread
// per message through the typed per-thread call.
template <int MODE>
__global__ void alltoall_kernel(Cfg c, int op, int dtype, unsigned long long send_off,
                                unsigned long long recv_off, unsigned long long bytes, int rounds, int nsets,
                                unsigned long long set_stride, unsigned bulk_smem, int device_barrier) {
  extern __shared__ __align__(128) char smem[];
  const int pe = blockIdx.z, np = c.npes;
  const unsigned long long total = (unsigned long long)(np - 1) * bytes;
  unsigned long long unit, nunits;
  if (MODE == NVSHMEMX_MODE_THREAD) {
    unit = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    nunits = (unsigned long long)(np - 1);
  } else if (MODE == NVSHMEMX_MODE_WARP) {
    unit = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    nunits = (unsigned long long)gridDim.x * (blockDim.x >> 5);
  } else {
    unit = blockIdx.x;
    nunits = gridDim.x;
  }
  const int w = dtype == NVSHMEMX_DT_DOUBLE ? 8 : 4;
  for (int r = 0; r < rounds; ++r) {
    const unsigned long long so = send_off + (unsigned long long)(r % nsets) * set_stride;
    const unsigned long long ro = recv_off + (unsigned long long)(r % nsets) * set_stride;
    if (MODE == NVSHMEMX_MODE_THREAD) {
      if (unit < nunits) {
        const int q = (pe + 1 + (int)unit) % np;
        const int len = (int)(bytes / w);
        if (op == NVSHMEMX_REQ_PUT) {
          char *sym = c.arena + ro + (unsigned long long)pe * bytes;
          char *src = slice_ptr(c, pe, so + (unsigned long long)q * bytes);
          if (dtype == NVSHMEMX_DT_INT) nvshmem_int_put((int *)sym, (int *)src, len, q);
          else if (dtype == NVSHMEMX_DT_FLOAT) nvshmem_float_put((float *)sym, (float *)src, len, q);
          else nvshmem_double_put((double *)sym, (double *)src, len, q);
        } else {
          char *sym = c.arena + so + (unsigned long long)pe * bytes;
          char *dst = slice_ptr(c, pe, ro + (unsigned long long)q * bytes);
          if (dtype == NVSHMEMX_DT_INT) nvshmem_int_get((int *)dst, (int *)sym, len, q);
          else if (dtype == NVSHMEMX_DT_FLOAT) nvshmem_float_get((float *)dst, (float *)sym, len, q);
          else nvshmem_double_get((double *)dst, (double *)sym, len, q);
        }
      }
    } else if (MODE == NVSHMEMX_MODE_BULK && ((bytes | so | ro) & 15) == 0) {
      // one ring per CTA across its whole share of the round
      const unsigned long long seg = (((total + nunits - 1) / nunits) + 15) & ~15ull;
      const unsigned long long b = unit * seg;
      const unsigned long long e = b + seg < total ? b + seg : total;
      if (threadIdx.x == 0 && b < e &&
          !a2a_stream_1t(c, smem, bulk_smem, op, pe, so, ro, bytes, b, e, gtimer() + (unsigned long long)c.wait_timeout_ns))
        record_error(c, NVSHMEMX_ERR_TIMEOUT, -2);
    } else {
      const unsigned long long seg = (((total + nunits - 1) / nunits) + 15) & ~15ull;
      unsigned long long b = unit * seg;
      const unsigned long long e = b + seg < total ? b + seg : total;
      while (b < e) {
        const unsigned long long k = b / bytes, off = b - k * bytes;
        const unsigned long long len = (e - b) < (bytes - off) ? (e - b) : (bytes - off);
        const int q = (pe + 1 + (int)k) % np;
        if (op == NVSHMEMX_REQ_PUT) {
          char *sym = c.arena + ro + (unsigned long long)pe * bytes + off;
          char *src = slice_ptr(c, pe, so + (unsigned long long)q * bytes + off);
          if (MODE == NVSHMEMX_MODE_WARP) nvshmemx_putmem_warp(sym, src, len, q);
          else if (MODE == NVSHMEMX_MODE_BLOCK) nvshmemx_putmem_block(sym, src, len, q);
          else nvshmemx_putmem_bulk_block(sym, src, len, q, smem, bulk_smem);
        } else {
          char *sym = c.arena + so + (unsigned long long)pe * bytes + off;
          char *dst = slice_ptr(c, pe, ro + (unsigned long long)q * bytes + off);
          if (MODE == NVSHMEMX_MODE_WARP) nvshmemx_getmem_warp(dst, sym, len, q);
          else if (MODE == NVSHMEMX_MODE_BLOCK) nvshmemx_getmem_block(dst, sym, len, q);
          else nvshmemx_getmem_bulk_block(dst, sym, len, q, smem, bulk_smem);
        }
        b += len;
      }
    }
    // quiet + barrier: the barrier's __syncthreads orders every thread's
    // stores before the leader, whose quiet and release cover them all
    __syncthreads();
    if (threadIdx.x == 0) nvshmem_quiet();
    if (device_barrier) nvshmemx_barrier_all_ep((unsigned long long)r);
  }
}

// ------------------------------------------------------------------ C3 halo
// Face d (0..5 = -x,+x,-y,+y,-z,+z) of the sender goes to the neighbour in
// direction d, into that neighbour's ghost buffer for direction d^1.  A face
// is n rows of n doubles; one warp moves one row per step.
__device__ __forceinline__ int halo_nbr(int pe, int d, int px, int py, int pz) {
  int x = pe % px, y = (pe / px) % py, z = pe / (px * py);
  const int s = (d & 1) ? 1 : -1;
  if (d < 2) x = (x + s + px) % px;
  else if (d < 4) y = (y + s + py) % py;
  else z = (z + s + pz) % pz;
  return x + px * (y + py * z);
}

// `iters` iterations numbered from it0 (signal values it0 + it + 1); with
// device_barrier each iteration ends at the device barrier, without it the
// caller follows the launch with nvshmem_barrier_all_offload (one iteration
// per launch, the prototype's own structure).
// The face rows are 2 KiB warp copies; they use the same checks and
// translation as nvshmemx_putmem_warp, inlined with a 4-deep copy loop (the
// public call is a shared out-of-line helper with a deeper loop tuned for
// long copies, which costs this short-row kernel registers and a call).
__device__ __forceinline__ void halo_row_put(const Cfg &c, double *dst_sym, const double *src, size_t bytes, int pe,
                                             unsigned lane) {
  if (!check_remote(c, dst_sym, bytes, pe) || !check_local(c, src, bytes)) return;
  char *dst = xlate(c, dst_sym, pe);
  const unsigned long long t0 = (c.trace && lane == 0) ? gtimer() : 0;
  copy_coop<16, 4>(dst, reinterpret_cast<const char *>(src), bytes, lane, 32);
  if (c.trace && lane == 0) trace_rec(c, NVSHMEMX_TRACE_PUT_INT, src, dst, bytes, pe, t0, gtimer());
}

// One x-face row: n doubles at stride n (src[k * n]) to n contiguous doubles
// at dst_sym on PE pe, with the checks of nvshmem_double_p made once for the
// row.  The gather is bound by DRAM access latency (every element is in its
// own row of the block), so each lane keeps 8 loads in flight, read through
// the non-coherent path without L1 allocation (the block is not written
// during the exchange), before storing them; stores are relaxed, ordered by
// the quiet that follows the faces.
__device__ __forceinline__ void halo_xrow_put(const Cfg &c, double *dst_sym, const double *src, int n, int pe,
                                              unsigned lane) {
  const unsigned long long bytes = (unsigned long long)n * 8ull;
  if (!check_remote(c, dst_sym, bytes, pe) || !check_local(c, src, (unsigned long long)(n - 1) * bytes + 8)) return;
  unsigned long long *dst = reinterpret_cast<unsigned long long *>(xlate(c, dst_sym, pe));
  const unsigned long long *s = reinterpret_cast<const unsigned long long *>(src);
  const long long stride = n;
  if (c.trace && lane == 0) {
    const unsigned long long t = gtimer();
    trace_rec(c, NVSHMEMX_TRACE_PUT_DOUBLE, src, dst, bytes, pe, t, t);
  }
  for (int k0 = 0; k0 < n; k0 += 256) {
    unsigned long long v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = k0 + u * 32 + (int)lane;
      if (k < n)
        asm volatile("ld.global.nc.L1::no_allocate.L2::64B.b64 %0, [%1];" : "=l"(v[u]) : "l"(s + k * stride));
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = k0 + u * 32 + (int)lane;
      if (k < n) st_relaxed_b64(dst + k, v[u]);
    }
  }
}

__global__ void __launch_bounds__(256, 4) halo_kernel(Cfg c, int px, int py, int pz, int n, unsigned long long block_off,
                            unsigned long long ghost_off, unsigned long long sig_off, int iters, int it0,
                            int device_barrier) {
  const int pe = blockIdx.z;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned long long face_bytes = (unsigned long long)n * n * 8ull;
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  const double *blk = (const double *)slice_ptr(c, pe, block_off);
  int *my_sig = (int *)slice_ptr(c, pe, sig_off);
  for (int it = 0; it < iters; ++it) {
    for (long long u = gw; u < 6ll * n; u += nw) {
      // units 0 .. 2n-1 pair the two x faces row by row (unit 2j reads
      // element x = 0 and unit 2j+1 element x = n-1 of the same 2 KiB rows,
      // on neighbouring warps at about the same time), then the y and z faces
      const int d = u < 2ll * n ? (int)(u & 1) : (int)(u / n), j = u < 2ll * n ? (int)(u >> 1) : (int)(u % n);
      const int nb = halo_nbr(pe, d, px, py, pz);
      double *dst = (double *)(c.arena + ghost_off + (unsigned long long)(d ^ 1) * face_bytes +
                               (unsigned long long)j * n * 8ull);
      if (d < 2) {
        // x face: element (z=j, y=k) sits at blk[(j*n + k)*n + x0]; gather
        // with stride n (one 8-byte element per n*8-byte row) and store the
        // row contiguously on the neighbour
        const int x0 = (d & 1) ? n - 1 : 0;
        halo_xrow_put(c, dst, blk + (long long)j * n * n + x0, n, nb, lane);
      } else if (d < 4) {
        // y face: row j is z=j, contiguous in x
        const int y0 = (d & 1) ? n - 1 : 0;
        halo_row_put(c, dst, blk + ((long long)j * n + y0) * n, (size_t)n * 8, nb, lane);
      } else {
        // z face: row j is y=j of plane z0
        const int z0 = (d & 1) ? n - 1 : 0;
        halo_row_put(c, dst, blk + ((long long)z0 * n + j) * n, (size_t)n * 8, nb, lane);
      }
    }
    nvshmem_quiet();
    nvshmemx_barrier_pe();
    if (blockIdx.x == 0 && threadIdx.x < 6) {
      const int d = threadIdx.x;
      nvshmem_quiet();
      nvshmem_int_p((int *)(c.arena + sig_off) + (d ^ 1), it0 + it + 1, halo_nbr(pe, d, px, py, pz));
      nvshmem_int_wait_until(my_sig + d, 0, it0 + it + 1);
    }
    if (device_barrier) nvshmemx_barrier_all_ep((unsigned long long)it);
  }
}

// ------------------------------------------------ strided-read ceiling
// What the halo's x faces cost at best: every PE reads nsets x rows 8-byte
// elements, element i of set t at slice offset off + t * set_off +
// i * stride, with ctas_per_pe CTAs per PE and 8 loads in flight per lane
// (the access pattern of halo_xrow_put without its stores; consecutive
// threads take the sets of one row in turn, as the halo pairs its two x
// faces), and adds them into one word per warp so that nothing is optimised
// away.
__global__ void __launch_bounds__(256) strided_read_kernel(Cfg c, unsigned long long off, unsigned long long set_off,
                                                           int nsets, unsigned long long rows,
                                                           unsigned long long stride, unsigned long long *sink) {
  const int pe = blockIdx.y;
  const char *base = slice_ptr(c, pe, off);
  const unsigned long long total = (unsigned long long)nsets * rows;
  const unsigned long long nthr = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long t0 = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long acc = 0;
  for (unsigned long long i0 = t0; i0 < total; i0 += 8 * nthr) {
    unsigned long long v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const unsigned long long i = i0 + (unsigned long long)u * nthr;
      v[u] = 0;
      if (i < total) {
        const unsigned long long set = i % (unsigned long long)nsets, row = i / (unsigned long long)nsets;
        const char *p = base + set * set_off + row * stride;
        asm volatile("ld.global.nc.L1::no_allocate.L2::64B.b64 %0, [%1];" : "=l"(v[u]) : "l"(p));
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) acc += v[u];
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(sink, acc);
}

// ------------------------------------------------------- failure detection
__global__ void wait_test_kernel(Cfg c, int *flag, int value, long long timeout_ns, int *out) {
  if (threadIdx.x == 0) out[0] = wait_cmp(c, flag, NVSHMEMX_CMP_EQ, value, timeout_ns);
}

__global__ void barrier_fault_kernel(Cfg c, int skip_pe, int *out) {
  if ((int)blockIdx.z == skip_pe) return;  // this PE never arrives
  int rc = barrier_all(c);
  if (threadIdx.x == 0 && rc) atomicMax(out, rc);
}

}  // namespace nvshm

using namespace nvshm;

static int need_started() {
  if (!is_started()) return fail(NVSHMEMX_ERR_STATE, "operation before nvstart_pes");
  // Drop a non-sticky error left by an earlier, unrelated runtime call so the
  // launch checks below report only this operation's own failures (sticky
  // device errors persist and are still reported).
  (void)cudaGetLastError();
  return 0;
}

// The C1-C3 operations run every PE in one collective launch and meet at
// device barriers; with one process per PE those barriers would see only
// this process's CTAs, so the operations refuse instead.
static int need_collective() {
  int rc;
  if ((rc = need_started())) return rc;
  if (proc_mode())
    return fail(NVSHMEMX_ERR_STATE, "operation needs every PE in one process (one process per PE is active)");
  return 0;
}

static int last_launch(const char *what) {
  return check_cuda(cudaGetLastError(), what);
}

// [off, off + bytes) lies inside [0, limit).  Arguments come from the caller
// as size_t, so the test never forms a sum that could wrap.
static bool range_ok(size_t off, size_t bytes, size_t limit) { return off <= limit && bytes <= limit - off; }

// *out = a * b, false when the product does not fit a size_t.
static bool mul_ok(size_t a, size_t b, size_t *out) {
  if (a != 0 && b > (size_t)-1 / a) return false;
  *out = a * b;
  return true;
}

// Shared memory for the CTA-wide TMA copies: a 64 KiB ring (six stages)
// plus 128 bytes of mbarriers (three CTAs fit an SM).
static const unsigned kBulkSmem = 4 * 16384 + 128;

namespace nvshm {
int launch_exec_requests(int mode, const nvshmemx_request *dr, int n, cudaStream_t s) {
  const Cfg c = rt().cfg;
  if (n <= 0) return 0;
  switch (mode) {
    case NVSHMEMX_MODE_THREAD:
      exec_requests_kernel<NVSHMEMX_MODE_THREAD><<<(n + 255) / 256, 256, 0, s>>>(c, dr, n, 0);
      break;
    case NVSHMEMX_MODE_WARP:
      exec_requests_kernel<NVSHMEMX_MODE_WARP><<<(n + 7) / 8, 256, 0, s>>>(c, dr, n, 0);
      break;
    case NVSHMEMX_MODE_BLOCK:
      exec_requests_kernel<NVSHMEMX_MODE_BLOCK><<<n, 256, 0, s>>>(c, dr, n, 0);
      break;
    default:
      cudaFuncSetAttribute(exec_requests_kernel<NVSHMEMX_MODE_BULK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kBulkSmem);
      exec_requests_kernel<NVSHMEMX_MODE_BULK><<<n, 256, kBulkSmem, s>>>(c, dr, n, kBulkSmem);
  }
  return check_cuda(cudaGetLastError(), "exec_requests launch");
}
}  // namespace nvshm

extern "C" {

int nvshmemx_exec_requests(const nvshmemx_request *reqs, int n, int mode, float *out_ms) {
  int rc;
  if ((rc = need_started())) return rc;
  if (n < 0 || mode < 0 || mode > NVSHMEMX_MODE_BULK) return fail(NVSHMEMX_ERR_INVALID, "exec_requests: bad n/mode");
  if (out_ms) *out_ms = 0.f;
  if (n == 0) return 0;
  const Runtime &r = rt();
  for (int i = 0; i < n; ++i) {
    const nvshmemx_request &q = reqs[i];
    if (q.src_pe >= r.npes || q.dst_pe >= r.npes || q.op > NVSHMEMX_REQ_G || q.dtype > NVSHMEMX_DT_DOUBLE)
      return fail(NVSHMEMX_ERR_INVALID, "exec_requests: request %d has a bad pe/op/dtype", i);
  }
  void *d = g_req_buf.get((size_t)n * sizeof(nvshmemx_request));
  if (!d) return fail(NVSHMEMX_ERR_NOMEM, "exec_requests: cannot allocate request buffer");
  if ((rc = check_cuda(cudaMemcpy(d, reqs, (size_t)n * sizeof(nvshmemx_request), cudaMemcpyHostToDevice),
                       "cudaMemcpy(requests)")))
    return rc;
  const nvshmemx_request *dr = (const nvshmemx_request *)d;
  EventTimer t;
  t.start();
  rc = launch_exec_requests(mode, dr, n, 0);
  t.stop();
  if (rc) return rc;
  float ms = t.ms();
  if (out_ms) *out_ms = ms;
  return check_cuda(cudaDeviceSynchronize(), "exec_requests");
}

int nvshmemx_fill_random(int pe, size_t off, size_t bytes, uint64_t seed) {
  int rc;
  if ((rc = need_started())) return rc;
  const Runtime &r = rt();
  if (pe < 0 || pe >= r.npes || off > r.heap_bytes || bytes > r.heap_bytes - off)
    return fail(NVSHMEMX_ERR_INVALID, "fill_random: range outside the slice");
  if (bytes == 0) return 0;
  fill_random_kernel<<<r.sm_count * 8, 256>>>(r.arena + (size_t)pe * r.stride, off, bytes, seed, pe);
  if ((rc = last_launch("fill_random"))) return rc;
  return check_cuda(cudaDeviceSynchronize(), "fill_random");
}

int nvshmemx_compare(int a_pe, size_t a_off, int b_pe, size_t b_off, size_t bytes, unsigned long long *out) {
  int rc;
  if ((rc = need_started())) return rc;
  const Runtime &r = rt();
  if (a_pe < 0 || a_pe >= r.npes || b_pe < 0 || b_pe >= r.npes || a_off > r.heap_bytes ||
      bytes > r.heap_bytes - a_off || b_off > r.heap_bytes || bytes > r.heap_bytes - b_off)
    return fail(NVSHMEMX_ERR_INVALID, "compare: range outside the slice");
  unsigned long long *d = (unsigned long long *)g_out_buf.get(64);
  if (!d) return fail(NVSHMEMX_ERR_NOMEM, "compare: scratch");
  cudaMemset(d, 0, 8);
  if (bytes)
    compare_kernel<<<r.sm_count * 8, 256>>>((const unsigned char *)(r.arena + (size_t)a_pe * r.stride + a_off),
                                            (const unsigned char *)(r.arena + (size_t)b_pe * r.stride + b_off),
                                            bytes, d);
  if ((rc = last_launch("compare"))) return rc;
  return check_cuda(cudaMemcpy(out, d, 8, cudaMemcpyDeviceToHost), "compare result");
}

int nvshmemx_checksum(int pe, size_t off, size_t bytes, unsigned long long *out) {
  int rc;
  if ((rc = need_started())) return rc;
  const Runtime &r = rt();
  if (pe < 0 || pe >= r.npes || off > r.heap_bytes || bytes > r.heap_bytes - off || (bytes & 7) || (off & 7))
    return fail(NVSHMEMX_ERR_INVALID, "checksum: range outside the slice or not 8-byte aligned");
  unsigned long long *d = (unsigned long long *)g_out_buf.get(64);
  if (!d) return fail(NVSHMEMX_ERR_NOMEM, "checksum: scratch");
  cudaMemset(d, 0, 8);
  if (bytes)
    checksum_kernel<<<r.sm_count * 8, 256>>>((const unsigned long long *)(r.arena + (size_t)pe * r.stride + off),
                                             bytes / 8, d);
  if ((rc = last_launch("checksum"))) return rc;
  return check_cuda(cudaMemcpy(out, d, 8, cudaMemcpyDeviceToHost), "checksum result");
}

int nvshmemx_op_pingpong(size_t flag_off, size_t data_off, int len_elems, int iters, int skip, double *out_ns,
                         double *out_total_ns) {
  int rc;
  if ((rc = need_collective())) return rc;
  const Runtime &r = rt();
  if (r.npes < 2) return fail(NVSHMEMX_ERR_INVALID, "pingpong needs at least 2 PEs");
  if (iters < 1 || skip < 0 || len_elems < 0 || !range_ok(flag_off, 4, r.heap_bytes) ||
      !range_ok(data_off, (size_t)len_elems * 4, r.heap_bytes))
    return fail(NVSHMEMX_ERR_INVALID, "pingpong: bad arguments");
  long long *cyc = (long long *)g_out_buf.get((size_t)iters * 8 + 64);
  if (!cyc) return fail(NVSHMEMX_ERR_NOMEM, "pingpong scratch");
  unsigned long long *gt = (unsigned long long *)(cyc + iters);
  int *data = (int *)(r.arena + data_off);
  int *flag = (int *)(r.arena + flag_off);
  // both flag words start at 0, whatever an earlier exchange left there
  for (int pe = 0; pe < 2; ++pe)
    if ((rc = check_cuda(cudaMemsetAsync(r.arena + (size_t)pe * r.stride + flag_off, 0, 4, 0), "pingpong flags")))
      return rc;
  void *args[] = {&data, &flag, &len_elems, &iters, &skip, &cyc, &gt};
  if ((rc = launch_collective((const void *)pingpong_kernel, dim3(1), dim3(32), args, 0, 0))) return rc;
  if ((rc = check_cuda(cudaDeviceSynchronize(), "pingpong"))) return rc;
  std::vector<long long> h(iters);
  unsigned long long total = 0;
  cudaMemcpy(h.data(), cyc, (size_t)iters * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(&total, gt, 8, cudaMemcpyDeviceToHost);
  double sum = 0;
  for (long long v : h) sum += (double)v;
  const double ns_per_cycle = sum > 0 ? (double)total / sum : 0.0;
  if (out_ns)
    for (int i = 0; i < iters; ++i) out_ns[i] = (double)h[i] * ns_per_cycle;
  if (out_total_ns) *out_total_ns = (double)total;
  return 0;
}

int nvshmemx_op_barrier_latency(int ctas_per_pe, int iters, int counted, double *out_ns, double *out_total_ns) {
  int rc;
  if ((rc = need_collective())) return rc;
  if (ctas_per_pe < 1 || iters < 1) return fail(NVSHMEMX_ERR_INVALID, "barrier_latency: bad arguments");
  long long *cyc = (long long *)g_out_buf.get((size_t)iters * 8 + 64);
  if (!cyc) return fail(NVSHMEMX_ERR_NOMEM, "barrier scratch");
  unsigned long long *gt = (unsigned long long *)(cyc + iters);
  void *args[] = {&iters, &counted, &cyc, &gt};
  if ((rc = launch_collective((const void *)barrier_latency_kernel, dim3(ctas_per_pe), dim3(128), args, 0, 0)))
    return rc;
  if ((rc = check_cuda(cudaDeviceSynchronize(), "barrier_latency"))) return rc;
  std::vector<long long> h(iters);
  unsigned long long total = 0;
  cudaMemcpy(h.data(), cyc, (size_t)iters * 8, cudaMemcpyDeviceToHost);
  cudaMemcpy(&total, gt, 8, cudaMemcpyDeviceToHost);
  double sum = 0;
  for (long long v : h) sum += (double)v;
  const double ns_per_cycle = sum > 0 ? (double)total / sum : 0.0;
  if (out_ns)
    for (int i = 0; i < iters; ++i) out_ns[i] = (double)h[i] * ns_per_cycle;
  if (out_total_ns) *out_total_ns = (double)total;
  return 0;
}

int nvshmemx_op_offload_barrier(int iters, double *out_us_per_call) {
  int rc;
  if ((rc = need_collective())) return rc;
  if (iters < 1) return fail(NVSHMEMX_ERR_INVALID, "offload_barrier: iters < 1");
  nvshmem_barrier_all_offload();  // warm-up
  if ((rc = check_cuda(cudaDeviceSynchronize(), "offload barrier"))) return rc;
  EventTimer t;
  t.start();
  for (int i = 0; i < iters; ++i) nvshmem_barrier_all_offload();
  t.stop();
  float ms = t.ms();
  if (out_us_per_call) *out_us_per_call = 1000.0 * ms / iters;
  return check_cuda(cudaDeviceSynchronize(), "offload barrier");
}

// Validates the arguments and picks the kernel, grid and block of an
// all-to-all in `mode`.
// CTAs per PE for an operation called with 0: NVSHMEM_CTAS_PER_PE when it is
// set to a positive count, else the operation's own choice `fallback`.
static int default_ctas_per_pe(int fallback) {
  const char *v = getenv("NVSHMEM_CTAS_PER_PE");
  const int k = v ? atoi(v) : 0;
  return k > 0 ? k : fallback;
}

static int alltoall_setup(int op, int dtype, size_t send_off, size_t recv_off, size_t bytes, int rounds, int nsets,
                          size_t set_stride, int mode, int ctas_per_pe, const void **fn, dim3 *grid, dim3 *block,
                          unsigned *smem) {
  int rc;
  if ((rc = need_collective())) return rc;
  const Runtime &r = rt();
  // 0: one CTA per PE per 1/npes of the SMs (18 for 8 PEs on 148 SMs: one
  // ring-driving CTA per SM measured fastest from 4 MiB messages on)
  if (ctas_per_pe == 0) ctas_per_pe = default_ctas_per_pe(r.sm_count / r.npes > 0 ? r.sm_count / r.npes : 1);
  if ((op != NVSHMEMX_REQ_PUT && op != NVSHMEMX_REQ_GET) || dtype < 0 || dtype > NVSHMEMX_DT_DOUBLE ||
      mode < 0 || mode > NVSHMEMX_MODE_BULK || rounds < 1 || nsets < 1 || ctas_per_pe < 1 || r.npes < 2)
    return fail(NVSHMEMX_ERR_INVALID, "alltoall: bad arguments");
  const int w = dtype == NVSHMEMX_DT_DOUBLE ? 8 : 4;
  if (bytes % w) return fail(NVSHMEMX_ERR_INVALID, "alltoall: bytes not a multiple of the element width");
  if (mode == NVSHMEMX_MODE_THREAD && bytes / w > 0x7fffffffull)
    return fail(NVSHMEMX_ERR_INVALID, "alltoall: message too long for an int element count");
  // every set of send and receive buffers, [off + s * set_stride, + npes * bytes)
  // for s < nsets, must lie inside the heap; no product or sum may wrap
  size_t span = 0, last = 0;
  if (!mul_ok((size_t)r.npes, bytes, &span) || !mul_ok((size_t)(nsets - 1), set_stride, &last) ||
      !range_ok(last, span, r.heap_bytes) || !range_ok(send_off, last + span, r.heap_bytes) ||
      !range_ok(recv_off, last + span, r.heap_bytes))
    return fail(NVSHMEMX_ERR_INVALID, "alltoall: buffers exceed the heap");
  *smem = mode == NVSHMEMX_MODE_BULK ? kBulkSmem : 0;
  *grid = dim3(ctas_per_pe);
  *block = dim3(256);
  switch (mode) {
    case NVSHMEMX_MODE_THREAD:
      *fn = (const void *)alltoall_kernel<NVSHMEMX_MODE_THREAD>;
      *grid = dim3(1);
      *block = dim3(32 * ((r.npes - 1 + 31) / 32));
      break;
    case NVSHMEMX_MODE_WARP: *fn = (const void *)alltoall_kernel<NVSHMEMX_MODE_WARP>; break;
    case NVSHMEMX_MODE_BLOCK: *fn = (const void *)alltoall_kernel<NVSHMEMX_MODE_BLOCK>; break;
    default: *fn = (const void *)alltoall_kernel<NVSHMEMX_MODE_BULK>;
  }
  return 0;
}

int nvshmemx_op_alltoall(int op, int dtype, size_t send_off, size_t recv_off, size_t bytes, int rounds, int nsets,
                         size_t set_stride, int mode, int ctas_per_pe, float *out_ms) {
  int rc;
  const void *fn;
  dim3 grid, block;
  unsigned smem;
  if ((rc = alltoall_setup(op, dtype, send_off, recv_off, bytes, rounds, nsets, set_stride, mode, ctas_per_pe, &fn,
                           &grid, &block, &smem)))
    return rc;
  Cfg c = rt().cfg;
  unsigned long long so = send_off, ro = recv_off, by = bytes, ss = set_stride;
  int device_barrier = 1;
  void *args[] = {&c, &op, &dtype, &so, &ro, &by, &rounds, &nsets, &ss, &smem, &device_barrier};
  EventTimer t;
  t.start();
  if ((rc = launch_collective(fn, grid, block, args, smem, 0))) return rc;
  t.stop();
  float ms = t.ms();
  if (out_ms) *out_ms = ms;
  return check_cuda(cudaDeviceSynchronize(), "alltoall");
}

int nvshmemx_op_alltoall_host(int op, int dtype, size_t send_off, size_t recv_off, size_t bytes, int rounds,
                              int nsets, size_t set_stride, int mode, int ctas_per_pe, float *out_ms) {
  int rc;
  const void *fn;
  dim3 grid, block;
  unsigned smem;
  if ((rc = alltoall_setup(op, dtype, send_off, recv_off, bytes, rounds, nsets, set_stride, mode, ctas_per_pe, &fn,
                           &grid, &block, &smem)))
    return rc;
  Cfg c = rt().cfg;
  unsigned long long by = bytes, ss = 0;
  int one = 1, device_barrier = 0;
  EventTimer t;
  t.start();
  for (int rd = 0; rd < rounds; ++rd) {
    unsigned long long so = send_off + (size_t)(rd % nsets) * set_stride;
    unsigned long long ro = recv_off + (size_t)(rd % nsets) * set_stride;
    void *args[] = {&c, &op, &dtype, &so, &ro, &by, &one, &one, &ss, &smem, &device_barrier};
    if ((rc = launch_collective(fn, grid, block, args, smem, 0))) return rc;
    nvshmem_barrier_all();
    if ((rc = last_launch("alltoall_host round"))) return rc;
  }
  t.stop();
  float ms = t.ms();
  if (out_ms) *out_ms = ms;
  return check_cuda(cudaDeviceSynchronize(), "alltoall_host");
}

// ctas_per_pe 0: NVSHMEM_CTAS_PER_PE if set, else as many CTAs per PE as stay
// co-resident (the exchange is latency-bound, so more warps in flight help).
static int halo_check(int px, int py, int pz, int n, size_t block_off, size_t ghost_off, size_t sig_off, int iters,
                      int *ctas_per_pe) {
  int rc;
  if ((rc = need_collective())) return rc;
  const Runtime &r = rt();
  if (*ctas_per_pe == 0) *ctas_per_pe = default_ctas_per_pe(max_ctas_per_pe((const void *)halo_kernel, 256, 0));
  if (px < 1 || py < 1 || pz < 1 || px * py * pz != r.npes || n < 1 || iters < 1 || *ctas_per_pe < 1)
    return fail(NVSHMEMX_ERR_INVALID, "halo: grid %dx%dx%d does not match %d PEs", px, py, pz, r.npes);
  const size_t nn = (size_t)n;
  size_t face = 0, block = 0, ghosts = 0;
  if (!mul_ok(nn * 8, nn, &face) || !mul_ok(face, nn, &block) || !mul_ok(face, 6, &ghosts) ||
      !range_ok(block_off, block, r.heap_bytes) || !range_ok(ghost_off, ghosts, r.heap_bytes) ||
      !range_ok(sig_off, 24, r.heap_bytes) || (block_off | ghost_off) % 16 || sig_off % 4)
    return fail(NVSHMEMX_ERR_INVALID, "halo: buffers exceed the heap or are misaligned");
  return 0;
}

int nvshmemx_op_halo(int px, int py, int pz, int n, size_t block_off, size_t ghost_off, size_t sig_off, int iters,
                     int ctas_per_pe, float *out_ms) {
  int rc;
  if ((rc = halo_check(px, py, pz, n, block_off, ghost_off, sig_off, iters, &ctas_per_pe))) return rc;
  Cfg c = rt().cfg;
  unsigned long long bo = block_off, go = ghost_off, so = sig_off;
  int it0 = 0, device_barrier = 1;
  void *args[] = {&c, &px, &py, &pz, &n, &bo, &go, &so, &iters, &it0, &device_barrier};
  EventTimer t;
  t.start();
  if ((rc = launch_collective((const void *)halo_kernel, dim3(ctas_per_pe), dim3(256), args, 0, 0))) return rc;
  t.stop();
  float ms = t.ms();
  if (out_ms) *out_ms = ms;
  return check_cuda(cudaDeviceSynchronize(), "halo");
}

int nvshmemx_op_halo_offload(int px, int py, int pz, int n, size_t block_off, size_t ghost_off, size_t sig_off,
                             int iters, int ctas_per_pe, float *out_ms) {
  int rc;
  if ((rc = halo_check(px, py, pz, n, block_off, ghost_off, sig_off, iters, &ctas_per_pe))) return rc;
  Cfg c = rt().cfg;
  unsigned long long bo = block_off, go = ghost_off, so = sig_off;
  int one = 1, device_barrier = 0;
  EventTimer t;
  t.start();
  for (int it = 0; it < iters; ++it) {
    void *args[] = {&c, &px, &py, &pz, &n, &bo, &go, &so, &one, &it, &device_barrier};
    if ((rc = launch_collective((const void *)halo_kernel, dim3(ctas_per_pe), dim3(256), args, 0, 0))) return rc;
    nvshmem_barrier_all_offload();
    if ((rc = last_launch("halo_offload barrier"))) return rc;
  }
  t.stop();
  float ms = t.ms();
  if (out_ms) *out_ms = ms;
  return check_cuda(cudaDeviceSynchronize(), "halo_offload");
}

int nvshmemx_op_strided_read(size_t off, size_t set_off, int nsets, size_t rows, size_t stride, int ctas_per_pe,
                             int iters, float *out_ms) {
  int rc;
  if ((rc = need_started())) return rc;
  const Runtime &r = rt();
  size_t span = 0, last = 0;
  if (nsets < 1 || ctas_per_pe < 1 || iters < 1 || rows < 1 || stride < 8 || (off | set_off | stride) % 8 ||
      !mul_ok(rows - 1, stride, &span) || !mul_ok((size_t)(nsets - 1), set_off, &last) ||
      span > r.heap_bytes ||  // so that span + 8 cannot wrap
      !range_ok(last, span + 8, r.heap_bytes) || !range_ok(off, last + span + 8, r.heap_bytes))
    return fail(NVSHMEMX_ERR_INVALID, "strided_read: bad arguments or elements outside the heap");
  unsigned long long *sink = (unsigned long long *)g_out_buf.get(64);
  if (!sink) return fail(NVSHMEMX_ERR_NOMEM, "strided_read scratch");
  EventTimer t;
  t.start();
  for (int i = 0; i < iters; ++i)
    strided_read_kernel<<<dim3(ctas_per_pe, r.npes), 256>>>(r.cfg, off, set_off, nsets, rows, stride, sink);
  t.stop();
  if ((rc = last_launch("strided_read"))) return rc;
  float ms = t.ms();
  if (out_ms) *out_ms = ms;
  return check_cuda(cudaDeviceSynchronize(), "strided_read");
}

int nvshmemx_op_wait_test(size_t flag_off, int value, long long timeout_ns, int *out_status) {
  int rc;
  if ((rc = need_collective())) return rc;
  const Runtime &r = rt();
  if (!range_ok(flag_off, 4, r.heap_bytes) || flag_off % 4)
    return fail(NVSHMEMX_ERR_INVALID, "wait_test: bad flag offset");
  int *d = (int *)g_out_buf.get(64);
  if (!d) return fail(NVSHMEMX_ERR_NOMEM, "wait_test scratch");
  cudaMemset(d, 0, 4);
  wait_test_kernel<<<1, 32>>>(r.cfg, (int *)(r.arena + flag_off), value, timeout_ns, d);
  if ((rc = last_launch("wait_test"))) return rc;
  return check_cuda(cudaMemcpy(out_status, d, 4, cudaMemcpyDeviceToHost), "wait_test result");
}

int nvshmemx_op_barrier_fault_test(int skip_pe, long long timeout_ns, int *out_status) {
  int rc;
  if ((rc = need_collective())) return rc;
  const Runtime &r = rt();
  if (skip_pe < 0 || skip_pe >= r.npes || timeout_ns <= 0) return fail(NVSHMEMX_ERR_INVALID, "barrier_fault_test");
  int *d = (int *)g_out_buf.get(64);
  if (!d) return fail(NVSHMEMX_ERR_NOMEM, "barrier_fault_test scratch");
  cudaMemset(d, 0, 4);
  Cfg c = r.cfg;
  c.wait_timeout_ns = timeout_ns;
  void *args[] = {&c, &skip_pe, &d};
  if ((rc = launch_collective((const void *)barrier_fault_kernel, dim3(1), dim3(32), args, 0, 0))) return rc;
  if ((rc = check_cuda(cudaDeviceSynchronize(), "barrier_fault_test"))) return rc;
  return check_cuda(cudaMemcpy(out_status, d, 4, cudaMemcpyDeviceToHost), "barrier_fault_test result");
}

}  // extern "C"

