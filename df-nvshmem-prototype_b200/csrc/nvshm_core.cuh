// nvshm_core.cuh -- device-side building blocks of the virtual-PE library.
//
// Everything on the hot path is here as inline functions taking the arena
// configuration explicitly, so the library's own kernels get it through the
// kernel parameter bank and inline every call, while the public extern "C"
// device API (device_api.cu) forwards to the same code with the __constant__
// copy.
//
// Memory layout (one B200):
//   arena = npes slices of `stride` bytes (stride a power of two), slice p at
//   arena + p*stride.  A symmetric address names an object by its offset in
//   its slice, so translating it to PE `pe` needs no table:
//       arena + pe*stride + ((addr - arena) & (stride - 1)).
//   (The prototype looked the peer base up in a __constant__ table of IPC
//   mappings, nvshmem_device.cu:446-447, which serialises lanes that name
//   different PEs; the shift/mask form is uniform-cost.)
#pragma once

#include <stdint.h>
#include <cuda_runtime.h>
#include "nvshmemx.h"

namespace nvshm {

// Arena configuration visible to device code.  One copy lives in __constant__
// memory for the public API; library kernels receive it by value.
struct Cfg {
  char *arena;
  unsigned long long arena_bytes;  // npes << log2_stride
  unsigned long long mask;         // stride - 1
  unsigned long long slice_bytes;  // mapped (usable) bytes at the start of each slice
  int log2_stride;
  int npes;
  int *status;                     // [0] code, [1] pe, [2..3] 64-bit detail
  unsigned long long *coll_bar;    // collective-launch ticket counter
  unsigned long long *pe_bar;      // per-PE ticket counters [npes]
  long long wait_timeout_ns;
  nvshmemx_trace_record *trace;    // npes * trace_cap records, or nullptr
  unsigned long long *trace_head;  // per-PE record counters
  unsigned int trace_cap;          // power of two
  int proc_pe;                     // process-per-PE mode: this process's PE; -1
                                   // when all PEs share one collective launch
};

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned int ld_relaxed_b32(const void *p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_b64(const void *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_b32(void *p, unsigned int v) {
  asm volatile("st.relaxed.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_b64(void *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void st_release_b32(void *p, unsigned int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long atom_add_acq_rel_u64(unsigned long long *p,
                                                                   unsigned long long v) {
  unsigned long long old;
  asm volatile("atom.add.acq_rel.gpu.global.u64 %0, [%1], %2;"
               : "=l"(old) : "l"(p), "l"(v) : "memory");
  return old;
}
__device__ __forceinline__ void fence_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

// ------------------------------------------------------------- PE / addresses
// The calling PE: blockIdx.z of a collective launch, or the process's PE when
// every PE is a process of its own.
__device__ __forceinline__ int my_pe(const Cfg &c) { return c.proc_pe >= 0 ? c.proc_pe : (int)blockIdx.z; }

__device__ __forceinline__ bool in_arena(const Cfg &c, const void *p) {
  return (unsigned long long)((const char *)p - c.arena) < c.arena_bytes;
}

__device__ __forceinline__ unsigned long long slice_off(const Cfg &c, const void *sym) {
  return (unsigned long long)((const char *)sym - c.arena) & c.mask;
}

__device__ __forceinline__ char *xlate(const Cfg &c, const void *sym, int pe) {
  return c.arena + ((unsigned long long)(unsigned)pe << c.log2_stride) + slice_off(c, sym);
}

// Records the first device-side error; later ones are dropped.
__device__ __forceinline__ void record_error(const Cfg &c, int code, long long detail) {
  if (atomicCAS(c.status, 0, code) == 0) {
    c.status[1] = my_pe(c);
    *(volatile long long *)(c.status + 2) = detail;
  }
}

// A symmetric range [sym, sym+bytes) on `pe` is valid when sym lies in the
// arena, pe is a PE and the range stays inside the mapped part of one slice.
__device__ __forceinline__ bool check_remote(const Cfg &c, const void *sym, unsigned long long bytes,
                                             int pe) {
  bool ok = in_arena(c, sym) && (unsigned)pe < (unsigned)c.npes &&
            slice_off(c, sym) + bytes <= c.slice_bytes;
  if (!ok) record_error(c, NVSHMEMX_ERR_BOUNDS, (long long)((const char *)sym - c.arena));
  return ok;
}

// A local operand may point anywhere in device memory; if it points into the
// arena's address range it must stay inside the mapped part of its slice
// (the rest of each slice's stride is reserved address space, not memory).
__device__ __forceinline__ bool check_local(const Cfg &c, const void *p, unsigned long long bytes) {
  if (!in_arena(c, p)) return true;
  bool ok = slice_off(c, p) + bytes <= c.slice_bytes;
  if (!ok) record_error(c, NVSHMEMX_ERR_BOUNDS, (long long)((const char *)p - c.arena));
  return ok;
}

// ------------------------------------------------------------------- tracing
__device__ __forceinline__ void trace_rec(const Cfg &c, int op, const void *local,
                                          const void *remote, unsigned long long bytes, int peer,
                                          unsigned long long t0, unsigned long long t1) {
  int pe = my_pe(c);
  if ((unsigned)pe >= (unsigned)c.npes) pe = 0;
  unsigned long long idx = atomicAdd(&c.trace_head[pe], 1ull);
  nvshmemx_trace_record *r =
      c.trace + (size_t)pe * c.trace_cap + (size_t)(idx & (unsigned long long)(c.trace_cap - 1));
  r->t_ns = (long long)t0;
  r->spin_ns = (long long)(t1 - t0);
  r->local_addr = (unsigned long long)local;
  r->remote_addr = (unsigned long long)remote;
  r->bytes = (unsigned)bytes;
  r->op = (unsigned short)op;
  r->pe = (unsigned short)pe;
  r->peer = (unsigned short)peer;
  r->tid = (unsigned short)(threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z));
  r->block = blockIdx.x + gridDim.x * blockIdx.y;
}

// --------------------------------------------------------------- copy engines
template <int VB> struct VecT;
template <> struct VecT<16> { typedef uint4 T; };
template <> struct VecT<8> { typedef uint2 T; };
template <> struct VecT<4> { typedef unsigned int T; };
template <> struct VecT<1> { typedef unsigned char T; };

// Asks the TMA unit to stage [p, p + bytes) in L2 (16-byte aligned address,
// size a multiple of 16; nothing to wait for -- later loads just hit L2).
__device__ __forceinline__ void l2_prefetch_bulk(uintptr_t p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes));
}

// Copies `bytes` with `nthr` cooperating threads (this one is `r`), VB-byte
// accesses for the aligned body and U accesses in flight per thread.  dst and
// src must have the same alignment modulo VB.
//
// PFI > 0: a copy by one thread or one warp is bound by the latency of its
// loads (U accesses per thread per round).  Its thread 0 keeps an L2
// prefetch of the source PFI rounds in front of the loads (never past the
// source range), so the loads hit L2 instead of DRAM.  Copies shorter than
// twice that distance skip it.
template <int VB, int U, unsigned PFI = 0>
__device__ __forceinline__ void copy_body(char *__restrict__ dst, const char *__restrict__ src,
                                          unsigned long long bytes, unsigned r, unsigned nthr) {
  typedef typename VecT<VB>::T V;
  unsigned long long head = (VB - ((uintptr_t)dst & (VB - 1))) & (VB - 1);
  if (head > bytes) head = bytes;
  for (unsigned long long i = r; i < head; i += nthr) dst[i] = src[i];
  const unsigned long long nv = (bytes - head) / VB;
  const V *s = reinterpret_cast<const V *>(src + head);
  V *d = reinterpret_cast<V *>(dst + head);
  unsigned long long i = r;
  const unsigned long long step = (unsigned long long)nthr * U;
  const unsigned long long dist = (unsigned long long)PFI * step * VB;  // bytes ahead
  const bool pf_on = PFI > 0 && r == 0 && nthr <= 32 && bytes >= 2 * dist;
  const uintptr_t pf_end = ((uintptr_t)src + bytes) & ~(uintptr_t)15;
  uintptr_t pf = ((uintptr_t)src + 15) & ~(uintptr_t)15;  // next source byte to stage
  if (nv >= (unsigned long long)(U - 1) * nthr) {
    for (; i + (unsigned long long)(U - 1) * nthr < nv; i += step) {
      V v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) v[u] = s[i + (unsigned long long)u * nthr];
      // between this iteration's loads and its stores: the stores of one
      // iteration and the loads of the next stay free to interleave
      // (measured: placed before the loads, the prefetch cost 15-23% on
      // copies already in L2)
      if (pf_on) {
        uintptr_t want = ((uintptr_t)(s + i) + dist) & ~(uintptr_t)15;
        if (want > pf_end) want = pf_end;
        if (want >= pf + 4096 || (want == pf_end && want > pf)) {
          const unsigned n = (unsigned)(want - pf < 65536 ? want - pf : 65536);
          l2_prefetch_bulk(pf, n);
          pf += n;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) d[i + (unsigned long long)u * nthr] = v[u];
    }
  }
  // copies too short for U accesses per thread still get 4 in flight
  if (U > 4) {
    for (; i + 3ull * nthr < nv; i += 4ull * nthr) {
      V v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = s[i + (unsigned long long)u * nthr];
#pragma unroll
      for (int u = 0; u < 4; ++u) d[i + (unsigned long long)u * nthr] = v[u];
    }
  }
  for (; i < nv; i += nthr) d[i] = s[i];
  for (unsigned long long j = head + nv * VB + r; j < bytes; j += nthr) dst[j] = src[j];
}

// Widest access the relative alignment of dst and src allows, capped at MAXV.
template <int MAXV = 16, int U = 4, unsigned PFI = 0>
__device__ __forceinline__ void copy_coop(char *dst, const char *src, unsigned long long bytes,
                                          unsigned r, unsigned nthr) {
  const unsigned mis = (unsigned)((uintptr_t)dst ^ (uintptr_t)src);
  if (MAXV >= 16 && (mis & 15) == 0)
    copy_body<16, U, PFI>(dst, src, bytes, r, nthr);
  else if (MAXV >= 8 && (mis & 7) == 0)
    copy_body<8, U, PFI>(dst, src, bytes, r, nthr);
  else if ((mis & 3) == 0)
    copy_body<4, U, PFI>(dst, src, bytes, r, nthr);
  else
    copy_body<1, U, PFI>(dst, src, bytes, r, nthr);
}

__device__ __forceinline__ unsigned block_rank() {
  return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
}
__device__ __forceinline__ unsigned block_size() { return blockDim.x * blockDim.y * blockDim.z; }

// ------------------------------------------------- TMA bulk (cp.async.bulk) ring
__device__ __forceinline__ void mbar_init(unsigned long long *m, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_inval(unsigned long long *m) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(m)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long *m, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)),
               "r"(bytes)
               : "memory");
}
// Bounded wait on an mbarrier phase; returns false when `deadline` passed.
__device__ __forceinline__ bool mbar_wait(unsigned long long *m, unsigned parity,
                                          unsigned long long deadline) {
  unsigned addr = smem_u32(m);
  for (unsigned it = 0;; ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    if (ok) return true;
    if ((it & 63) == 63 && gtimer() > deadline) return false;
  }
}
__device__ __forceinline__ void bulk_g2s(void *smem_dst, const void *gsrc, unsigned bytes,
                                         unsigned long long *m) {
  asm volatile(
      "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(smem_dst)),
      "l"(gsrc), "r"(bytes), "r"(smem_u32(m))
      : "memory");
}
__device__ __forceinline__ void bulk_s2g(void *gdst, const void *smem_src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst),
               "r"(smem_u32(smem_src)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// at most one bulk group (the newest store) may still be reading shared memory
__device__ __forceinline__ void bulk_wait_read1() {
  asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

// Shared-memory layout of a bulk ring: up to 8 mbarriers in the first 128
// bytes, then `stages` buffers of `stage_bytes` (a multiple of 16).
struct BulkRing {
  unsigned long long *mbar;
  char *buf;
  unsigned stages;
  unsigned stage_bytes;
};

__device__ __forceinline__ BulkRing make_ring(void *smem, unsigned smem_bytes, unsigned want_stages) {
  BulkRing r;
  r.mbar = reinterpret_cast<unsigned long long *>(smem);
  r.buf = reinterpret_cast<char *>(smem) + 128;
  unsigned avail = smem_bytes > 128 ? smem_bytes - 128 : 0;
  unsigned st = want_stages < 2 ? 2 : (want_stages > 8 ? 8 : want_stages);
  unsigned sb = (avail / st) & ~127u;
  r.stages = st;
  r.stage_bytes = sb;
  return r;
}

// Single-thread bulk pipeline for a 16-byte aligned body (dst, src 16-aligned,
// bytes a multiple of 16): loads run up to `stages` - 1 ahead of the stores,
// and a stage is reloaded one store later than it could be, so the issuing
// thread never waits on the store it has just started (measured against
// reloading the stage of the newest store: one CTA's 1 MiB put 51 -> 60 GB/s,
// the 16 MiB all-to-all 6350 -> 6565 GB/s with 6 stages).
// Returns false if an mbarrier wait passed `deadline` (the copy is then
// incomplete; every issued store is still drained before returning).
__device__ __forceinline__ bool bulk_copy_1t(const BulkRing &ring, char *dst, const char *src,
                                             unsigned long long bytes, unsigned long long deadline) {
  if (bytes == 0) return true;
  const unsigned S = ring.stages, SB = ring.stage_bytes;
  const unsigned long long nch = (bytes + SB - 1) / SB;
  for (unsigned s = 0; s < S; ++s) mbar_init(ring.mbar + s, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  const unsigned long long pre = nch < S ? nch : S;
  for (unsigned long long c = 0; c < pre; ++c) {
    unsigned len = (unsigned)((bytes - c * SB) < SB ? (bytes - c * SB) : SB);
    mbar_expect_tx(ring.mbar + c, len);
    bulk_g2s(ring.buf + (size_t)c * SB, src + c * SB, len, ring.mbar + c);
  }
  bool ok = true;
  for (unsigned long long c = 0; c < nch; ++c) {
    const unsigned s = (unsigned)(c % S);
    const unsigned parity = (unsigned)((c / S) & 1);
    if (!mbar_wait(ring.mbar + s, parity, deadline)) {
      ok = false;
      break;
    }
    unsigned len = (unsigned)((bytes - c * SB) < SB ? (bytes - c * SB) : SB);
    bulk_s2g(dst + c * SB, ring.buf + (size_t)s * SB, len);
    bulk_commit();
    // refill the stage the previous store read, not this one: that store has
    // had a whole load wait to finish reading, while this one just started
    const unsigned long long n = c - 1 + S;
    if (c >= 1 && n < nch) {
      bulk_wait_read1();
      const unsigned ps = (unsigned)((c - 1) % S);
      unsigned nlen = (unsigned)((bytes - n * SB) < SB ? (bytes - n * SB) : SB);
      mbar_expect_tx(ring.mbar + ps, nlen);
      bulk_g2s(ring.buf + (size_t)ps * SB, src + n * SB, nlen, ring.mbar + ps);
    }
  }
  bulk_wait_all();
  if (ok) {
    for (unsigned s = 0; s < S; ++s) mbar_inval(ring.mbar + s);
  }
  return ok;
}

// Block-cooperative bulk copy: thread 0 drives the TMA ring over the
// 16-aligned body while the other threads copy the unaligned head and tail.
// Falls back to the generic copy when dst/src alignments differ mod 16 or the
// ring has no room.  Every thread of the block must call it.
// One issuer per CTA streams the body as one sequential range: measured on
// B200 this keeps DRAM accesses more local than splitting the range across
// per-warp rings (which lost 6-7% on 16-256 MiB all-to-all rounds).
__device__ __forceinline__ void bulk_copy_block(const Cfg &c, char *dst, const char *src,
                                                unsigned long long bytes, void *smem,
                                                unsigned smem_bytes) {
  const unsigned r = block_rank(), n = block_size();
  BulkRing ring = make_ring(smem, smem_bytes, 6);
  if ((((uintptr_t)dst ^ (uintptr_t)src) & 15) != 0 || ring.stage_bytes < 1024 || bytes < 4096 ||
      n < 64) {
    copy_coop<16, 4>(dst, src, bytes, r, n);
    __syncthreads();
    return;
  }
  unsigned long long head = (16 - ((uintptr_t)dst & 15)) & 15;
  unsigned long long body = (bytes - head) & ~15ull;
  unsigned long long tail = bytes - head - body;
  if (r == 0) {
    unsigned long long deadline = gtimer() + (unsigned long long)c.wait_timeout_ns;
    if (!bulk_copy_1t(ring, dst + head, src + head, body, deadline))
      record_error(c, NVSHMEMX_ERR_TIMEOUT, -2);
  } else if (r >= 32) {
    // warps 1.. handle head and tail bytes
    unsigned rr = r - 32, nn = n - 32;
    for (unsigned long long i = rr; i < head; i += nn) dst[i] = src[i];
    for (unsigned long long i = rr; i < tail; i += nn) dst[head + body + i] = src[head + body + i];
  }
  __syncthreads();
}

// ---------------------------------------------------------------- waits
__device__ __forceinline__ bool cmp_ok(int v, int cmp, int x) {
  switch (cmp) {
    case NVSHMEMX_CMP_EQ: return v == x;
    case NVSHMEMX_CMP_NE: return v != x;
    case NVSHMEMX_CMP_GT: return v > x;
    case NVSHMEMX_CMP_GE: return v >= x;
    case NVSHMEMX_CMP_LT: return v < x;
    default: return v <= x;
  }
}

// Polls *p with ld.acquire.gpu until cmp_ok; tight polling first, then
// __nanosleep backoff (32 ns doubling to 256 ns) so idle waiters leave L2
// bandwidth to the copies.  Gives up after timeout_ns (library default when
// <= 0), records NVSHMEMX_ERR_TIMEOUT and returns it.
__device__ __forceinline__ int wait_cmp(const Cfg &c, const int *p, int cmp, int val,
                                        long long timeout_ns) {
  if (((uintptr_t)p & 3) != 0 || (in_arena(c, p) && slice_off(c, p) + 4 > c.slice_bytes)) {
    record_error(c, NVSHMEMX_ERR_BOUNDS, (long long)((const char *)p - c.arena));
    return NVSHMEMX_ERR_BOUNDS;
  }
  if (cmp_ok(ld_acquire(p), cmp, val)) return NVSHMEMX_SUCCESS;
  if (timeout_ns <= 0) timeout_ns = c.wait_timeout_ns;
  const unsigned long long t0 = gtimer();
  unsigned ns = 0;
  for (unsigned spins = 1;; ++spins) {
    if (cmp_ok(ld_acquire(p), cmp, val)) return NVSHMEMX_SUCCESS;
    if (spins > 64) {
      ns = ns == 0 ? 32 : (ns >= 256 ? 256 : ns * 2);
      __nanosleep(ns);
    }
    if ((spins & 15) == 0 && (long long)(gtimer() - t0) > timeout_ns) {
      record_error(c, NVSHMEMX_ERR_TIMEOUT, (long long)((const char *)p - c.arena));
      return NVSHMEMX_ERR_TIMEOUT;
    }
  }
}

// ---------------------------------------------------------------- barriers
// Ticket barrier over P CTAs on a monotonically increasing 64-bit counter:
// each CTA's leader adds 1 (acq_rel) and the CTAs of episode e = ticket / P
// leave once the counter reaches (e+1)*P.  One atomic per CTA and no reset
// between episodes; P must stay the same for the counter's lifetime (the
// launcher zeroes it before each launch).
__device__ __forceinline__ int ticket_barrier(const Cfg &c, unsigned long long *ctr,
                                              unsigned long long P) {
  __syncthreads();
  int rc = 0;
  if (block_rank() == 0) {
    // bar.sync orders the CTA's earlier writes before this thread's
    // operations; the acq_rel atomic releases them at GPU scope (cumulative),
    // so no separate fence is needed.
    const unsigned long long t = atom_add_acq_rel_u64(ctr, 1ull);
    const unsigned long long target = (t / P + 1ull) * P;
    if (ld_acquire_u64(ctr) < target) {
      const unsigned long long t0 = gtimer();
      for (unsigned spins = 1;; ++spins) {
        if (ld_acquire_u64(ctr) >= target) break;
        if (spins > 256) __nanosleep(64);
        if ((spins & 15) == 0 && (long long)(gtimer() - t0) > c.wait_timeout_ns) {
          record_error(c, NVSHMEMX_ERR_TIMEOUT, -1);
          rc = NVSHMEMX_ERR_TIMEOUT;
          break;
        }
      }
    }
  }
  rc = __syncthreads_or(rc) ? NVSHMEMX_ERR_TIMEOUT : 0;
  return rc;
}

__device__ __forceinline__ void red_add_release_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// The same barrier when every CTA knows which barrier of the launch this is
// (episode 0, 1, 2 ...): the leader arrives with a fire-and-forget
// red.release and polls for (episode+1)*P, so the last arriver does not wait
// for an atomic's return value before its first poll -- one L2 round trip
// less on the critical path.  Interoperates with ticket_barrier on the same
// counter as long as every CTA passes the true episode number.
__device__ __forceinline__ int episode_barrier(const Cfg &c, unsigned long long *ctr, unsigned long long P,
                                               unsigned long long episode) {
  __syncthreads();
  int rc = 0;
  if (block_rank() == 0) {
    red_add_release_u64(ctr, 1ull);  // releases the CTA's writes (see ticket_barrier)
    const unsigned long long target = (episode + 1ull) * P;
    if (ld_acquire_u64(ctr) < target) {
      const unsigned long long t0 = gtimer();
      for (unsigned spins = 1;; ++spins) {
        if (ld_acquire_u64(ctr) >= target) break;
        if (spins > 256) __nanosleep(64);
        if ((spins & 15) == 0 && (long long)(gtimer() - t0) > c.wait_timeout_ns) {
          record_error(c, NVSHMEMX_ERR_TIMEOUT, -1);
          rc = NVSHMEMX_ERR_TIMEOUT;
          break;
        }
      }
    }
  }
  rc = __syncthreads_or(rc) ? NVSHMEMX_ERR_TIMEOUT : 0;
  return rc;
}

__device__ __forceinline__ int barrier_all(const Cfg &c) {
  const unsigned long long P = (unsigned long long)gridDim.x * gridDim.y * gridDim.z;
  return ticket_barrier(c, c.coll_bar, P);
}

__device__ __forceinline__ int barrier_pe(const Cfg &c) {
  int pe = my_pe(c);
  if ((unsigned)pe >= (unsigned)c.npes) pe = 0;
  const unsigned long long P = (unsigned long long)gridDim.x * gridDim.y;
  return ticket_barrier(c, c.pe_bar + (size_t)pe * 16, P);  // counters 128 bytes apart
}

// ------------------------------------------------------- typed RMA (one thread)
// Scalar accesses must be naturally aligned; a misaligned address is recorded
// as a bounds error and skipped rather than executed (it would fault).
__device__ __forceinline__ bool check_align(const Cfg &c, const void *p, unsigned width) {
  if (((uintptr_t)p & (width - 1)) == 0) return true;
  record_error(c, NVSHMEMX_ERR_BOUNDS, (long long)((const char *)p - c.arena));
  return false;
}

template <typename T>
__device__ __forceinline__ void p_one(const Cfg &c, T *target, T value, int pe) {
  if (!check_remote(c, target, sizeof(T), pe) || !check_align(c, target, sizeof(T))) return;
  char *dst = xlate(c, target, pe);
  if (sizeof(T) == 8) {
    st_relaxed_b64(dst, *reinterpret_cast<unsigned long long *>(&value));
  } else {
    st_relaxed_b32(dst, *reinterpret_cast<unsigned int *>(&value));
  }
}

template <typename T>
__device__ __forceinline__ T g_one(const Cfg &c, const T *source, int pe) {
  if (!check_remote(c, source, sizeof(T), pe) || !check_align(c, source, sizeof(T))) return T(0);
  const char *src = xlate(c, source, pe);
  if (sizeof(T) == 8) {
    unsigned long long v = ld_relaxed_b64(src);
    return *reinterpret_cast<T *>(&v);
  } else {
    unsigned int v = ld_relaxed_b32(src);
    return *reinterpret_cast<T *>(&v);
  }
}

// Bytes of a put/get of `len` elements; a negative len copies nothing, as the
// prototype's `for (i = 0; i < len; i++)` loop.
template <typename T>
__device__ __forceinline__ unsigned long long elem_bytes(int len) {
  return len > 0 ? (unsigned long long)len * sizeof(T) : 0ull;
}

}  // namespace nvshm
