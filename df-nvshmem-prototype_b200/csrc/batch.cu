// batch.cu -- batched one-sided traffic (nvshmemx_batch.h).
//
// A batch runs as a CUDA graph of three nodes on the batch's own stream:
//   memset   zero the 32-byte control block (chunk count, cursor, status)
//   plan     one thread per request: validate, translate to arena addresses,
//            cut into chunks of <= chunk_bytes; a CTA-wide scan plus one
//            atomicAdd per CTA places each CTA's chunks in the work table
//            (CTA order is arbitrary, which is fine: requests are disjoint)
//   exec     persistent grid (SM count x CTAs per SM); each warp claims
//            `grab` chunks per atomicAdd on the cursor, prefetches the next
//            claim and the next 32-byte work item while it copies the current
//            chunk with VB-byte accesses, U in flight per lane.
// Every chunk is a contiguous copy, so the exec kernel is pure streaming:
// its roofline is HBM copy bandwidth (2 bytes moved per payload byte).
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "batch.h"
#include "nvshmemx_batch.h"

namespace nvshm {

struct WorkItem {          // 32 bytes
  unsigned long long dst;  // absolute destination address
  unsigned long long src;  // absolute source address (P: the element bits)
  unsigned int len;        // bytes
  unsigned int kind;       // kCopy, kSignal, kStore
  int value;               // SIGNAL value
  unsigned int pad;
};
enum { kCopy = 0, kSignal = 1, kStore = 2 };

struct BatchCtl {  // 32 bytes, zeroed before every execution
  unsigned long long total_chunks;  // chunks of this piece of the batch
  unsigned long long cursor;
  int status;
  int bad_request;
  unsigned long long item_base;     // index of the piece's first work item
};

__device__ __forceinline__ void set_status(BatchCtl *ctl, int code, int req) {
  if (atomicCAS(&ctl->status, 0, code) == 0) ctl->bad_request = req;
}

// Programmatic dependent launch: the plan kernel lets the exec kernel start
// as soon as every plan CTA is running; the exec kernel sets up its rings,
// then waits until the plan grid has completed and its writes are visible.
// Both are no-ops for a launch without the programmatic attribute.
__device__ __forceinline__ void pdl_release_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait_prerequisites() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Start of an exec kernel: `ctl` holds the piece's plan status, `sctl` the
// status the host reads (the same block for one piece; the first piece's
// for the second piece of a pipelined submit, which runs after the first
// piece is done).  A plan error of this piece is copied to `sctl` (first
// error wins); the piece runs only if neither reports an error.
__device__ __forceinline__ bool piece_may_run(BatchCtl *ctl, BatchCtl *sctl) {
  const int own = *(volatile int *)&ctl->status;
  if (ctl != sctl && own != 0 && blockIdx.x == 0 && threadIdx.x == 0)
    set_status(sctl, own, *(volatile int *)&ctl->bad_request);
  return own == 0 && *(volatile int *)&sctl->status == 0;
}

// ------------------------------------------------------------------- plan
// [off, off + bytes) lies inside the mapped part of a slice.  Written so that
// no sum can wrap: off and bytes are caller-supplied 64-bit values, and
// off + bytes may overflow (off = 2^64 - 4, bytes = 8 would pass a test of
// the sum and address memory below the slice).
__device__ __forceinline__ bool range_in_slice(const Cfg &c, unsigned long long off, unsigned long long bytes) {
  return off <= c.slice_bytes && bytes <= c.slice_bytes - off;
}

// A compact request (nvshmemx_request_compact) in its full form; one that
// the compact form cannot hold (bits outside its fields, a PUT/GET of 4 GiB
// or more, P of a double) gets an invalid op, which planning reports.
__device__ __forceinline__ nvshmemx_request expand_compact(const uint4 q) {
  nvshmemx_request r;
  const unsigned op = (q.w >> 20) & 7u, dt = (q.w >> 23) & 3u;
  r.src_off = (unsigned long long)q.x * 4;
  r.dst_off = (unsigned long long)q.y * 4;
  r.bytes = 0;
  r.src_pe = (uint16_t)(q.w & 1023u);
  r.dst_pe = (uint16_t)((q.w >> 10) & 1023u);
  r.op = (uint8_t)op;
  r.dtype = (uint8_t)dt;
  r.flags = 0;
  r.value = 0;
  bool ok = (q.w >> 25) == 0;
  if (op == NVSHMEMX_REQ_PUT || op == NVSHMEMX_REQ_GET) {
    ok = ok && q.z < (1u << 30);
    r.bytes = q.z * 4u;
  } else if (op == NVSHMEMX_REQ_SIGNAL) {
    r.value = (int)q.z;
  } else if (op == NVSHMEMX_REQ_P) {
    ok = ok && dt != NVSHMEMX_DT_DOUBLE;
    r.src_off = q.x;  // the element's bits
  }
  if (!ok) r.op = 0xff;
  return r;
}

// A batch is planned as one piece, or (pipelined submit) as consecutive
// pieces planned in order on one stream: piece k appends its items after
// those of piece k-1 (`prev`) and reports errors, with request indices offset
// by `req_base`, in its own control block `sctl`.  COMPACT: `reqs_in` holds
// compact requests, and each is also stored in full form at keep[i].
// Threads (one per request) of a plan CTA; each CTA reserves its chunks with
// one atomicAdd on the piece's counter.  256, 512 and 1024 threads measured
// the same C4 step (206.5-206.8 us) and end-to-end call (237.9-239.6 us), so
// the contention of those atomics is not what the plan kernel waits on.
constexpr int kPlanThreads = 256;

template <bool COMPACT>
__global__ void __launch_bounds__(kPlanThreads) batch_plan_kernel(Cfg c, const void *__restrict__ reqs_in, int n,
                                                         unsigned chunk, WorkItem *__restrict__ items,
                                                         unsigned long long cap, BatchCtl *ctl, BatchCtl *sctl,
                                                         const BatchCtl *prev, int req_base,
                                                         nvshmemx_request *__restrict__ keep) {
  __shared__ unsigned warp_sums[kPlanThreads / 32];
  __shared__ unsigned long long block_base;
  pdl_release_dependents();
  const unsigned long long ibase = prev ? prev->item_base + prev->total_chunks : 0ull;
  if (blockIdx.x == 0 && threadIdx.x == 0) ctl->item_base = ibase;
  const int i = blockIdx.x * kPlanThreads + threadIdx.x;
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  unsigned cnt = 0;
  WorkItem w;
  w.dst = w.src = 0;
  w.len = 0;
  w.kind = kCopy;
  w.value = 0;
  w.pad = 0;
  if (i < n) {
    nvshmemx_request r;
    if (COMPACT) {
      r = expand_compact(reinterpret_cast<const uint4 *>(reqs_in)[i]);
      uint4 lo, hi;
      memcpy(&lo, &r, 16);
      memcpy(&hi, reinterpret_cast<const char *>(&r) + 16, 16);
      reinterpret_cast<uint4 *>(keep + i)[0] = lo;
      reinterpret_cast<uint4 *>(keep + i)[1] = hi;
    } else {
      r = reinterpret_cast<const nvshmemx_request *>(reqs_in)[i];
    }
    const unsigned width = r.dtype == NVSHMEMX_DT_DOUBLE ? 8u : 4u;
    const bool pe_ok = r.src_pe < c.npes && r.dst_pe < c.npes && r.dtype <= NVSHMEMX_DT_DOUBLE;
    const unsigned long long dst = (unsigned long long)c.arena + ((unsigned long long)r.dst_pe << c.log2_stride) + r.dst_off;
    const unsigned long long src = (unsigned long long)c.arena + ((unsigned long long)r.src_pe << c.log2_stride) + r.src_off;
    switch (r.op) {
      case NVSHMEMX_REQ_PUT:
      case NVSHMEMX_REQ_GET:
      case NVSHMEMX_REQ_G: {
        const unsigned long long bytes = r.op == NVSHMEMX_REQ_G ? width : r.bytes;
        if (!pe_ok || !range_in_slice(c, r.src_off, bytes) || !range_in_slice(c, r.dst_off, bytes)) {
          set_status(sctl, NVSHMEMX_ERR_BOUNDS, req_base + i);
          break;
        }
        w.dst = dst;
        w.src = src;
        w.len = (unsigned)bytes;
        cnt = bytes ? (unsigned)((bytes + chunk - 1) / chunk) : 0u;
        break;
      }
      case NVSHMEMX_REQ_SIGNAL:
      case NVSHMEMX_REQ_P: {
        const unsigned bytes = r.op == NVSHMEMX_REQ_SIGNAL ? 4u : width;
        if (!pe_ok || !range_in_slice(c, r.dst_off, bytes) || (r.dst_off & (bytes - 1))) {
          set_status(sctl, NVSHMEMX_ERR_BOUNDS, req_base + i);
          break;
        }
        w.dst = dst;
        w.src = r.src_off;
        w.len = bytes;
        w.kind = r.op == NVSHMEMX_REQ_SIGNAL ? kSignal : kStore;
        w.value = r.value;
        cnt = 1;
        break;
      }
      default:
        set_status(sctl, NVSHMEMX_ERR_INVALID, req_base + i);
    }
  }
  // CTA-wide exclusive scan of cnt
  unsigned incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= (unsigned)o) incl += v;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned acc = 0;
    for (int k = 0; k < kPlanThreads / 32; ++k) {
      unsigned s = warp_sums[k];
      warp_sums[k] = acc;
      acc += s;
    }
    block_base = acc ? atomicAdd(&ctl->total_chunks, (unsigned long long)acc) : 0ull;
    if (acc && ibase + block_base + acc > cap) set_status(sctl, NVSHMEMX_ERR_NOMEM, -1);
  }
  __syncthreads();
  if (cnt == 0) return;
  const unsigned long long first = ibase + block_base + warp_sums[warp] + (incl - cnt);
  if (first + cnt > cap) return;
  if (cnt == 1) {
    items[first] = w;
    return;
  }
  for (unsigned k = 0; k < cnt; ++k) {
    WorkItem p = w;
    const unsigned long long off = (unsigned long long)k * chunk;
    p.dst += off;
    p.src += off;
    p.len = (unsigned)((w.len - off) < chunk ? (w.len - off) : chunk);
    items[first + k] = p;
  }
}

// ------------------------------------------------------------------- exec
// Items are read through L2 (the exec kernel may start before the plan
// kernel that writes them has finished; see pdl_wait_prerequisites).
__device__ __forceinline__ WorkItem load_item(const WorkItem *p) {
  const uint4 *q = reinterpret_cast<const uint4 *>(p);
  uint4 a = __ldcg(q), b = __ldcg(q + 1);
  WorkItem w;
  w.dst = ((unsigned long long)a.y << 32) | a.x;
  w.src = ((unsigned long long)a.w << 32) | a.z;
  w.len = b.x;
  w.kind = b.y;
  w.value = (int)b.z;
  w.pad = b.w;
  return w;
}

template <int VB, int U>
__device__ __forceinline__ void run_item(const WorkItem &w, unsigned lane) {
  if (w.kind == kCopy) {
    copy_coop<VB, U>(reinterpret_cast<char *>(w.dst), reinterpret_cast<const char *>(w.src), w.len, lane, 32);
  } else if (lane == 0) {
    // Requests of one batch are unordered with respect to each other (they
    // touch disjoint bytes), so a SIGNAL is a plain 4-byte store like
    // nvshmem_int_p; completion of the batch orders it before later work.
    if (w.kind == kSignal) {
      st_relaxed_b32(reinterpret_cast<void *>(w.dst), (unsigned)w.value);
    } else if (w.len == 8) {
      st_relaxed_b64(reinterpret_cast<void *>(w.dst), w.src);
    } else {
      st_relaxed_b32(reinterpret_cast<void *>(w.dst), (unsigned)w.src);
    }
  }
}

template <int VB, int U>
__global__ void __launch_bounds__(1024) batch_exec_kernel(const WorkItem *__restrict__ items, BatchCtl *ctl,
                                                          BatchCtl *sctl, unsigned long long cap, int grab) {
  const unsigned lane = threadIdx.x & 31u;
  pdl_release_dependents();
  pdl_wait_prerequisites();
  if (!piece_may_run(ctl, sctl)) return;
  unsigned long long C = *(volatile unsigned long long *)&ctl->total_chunks;
  const unsigned long long ib = *(volatile unsigned long long *)&ctl->item_base;
  if (ib + C > cap) return;
  items += ib;
  unsigned long long base = 0;
  if (lane == 0) base = atomicAdd(&ctl->cursor, (unsigned long long)grab);
  base = __shfl_sync(0xffffffffu, base, 0);
  while (base < C) {
    unsigned long long nxt = 0;
    if (lane == 0) nxt = atomicAdd(&ctl->cursor, (unsigned long long)grab);
    const unsigned long long end = base + grab < C ? base + grab : C;
    WorkItem cur = load_item(items + base);
    for (unsigned long long k = base; k < end; ++k) {
      WorkItem nx;
      if (k + 1 < end) nx = load_item(items + k + 1);
      run_item<VB, U>(cur, lane);
      cur = nx;
    }
    base = __shfl_sync(0xffffffffu, nxt, 0);
  }
}

// ------------------------------------------------------- exec through TMA
// A per-warp ring of S shared-memory stages: lane 0 issues cp.async.bulk
// global->shared (completion counted on the stage's mbarrier) and, once a
// stage has landed, cp.async.bulk shared->global as one bulk group.  The ring
// spans work items, so each warp keeps up to S loads in flight across chunk
// boundaries without holding the data in registers; lanes 1..31 copy the
// unaligned head and tail bytes.  Chunks whose source and destination differ
// in alignment modulo 16, or that are shorter than min_bulk, take the
// register copy.  Every mbarrier wait is bounded by `deadline`.
__device__ __forceinline__ void bulk_wait_read_le(unsigned n) {
  switch (n) {
    case 0: asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); break;
    case 1: asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); break;
    case 2: asm volatile("cp.async.bulk.wait_group.read 2;" ::: "memory"); break;
    default: asm volatile("cp.async.bulk.wait_group.read 3;" ::: "memory"); break;
  }
}

template <int S>
struct WarpTma {
  unsigned long long *mbar;  // S mbarriers
  unsigned long long *pdst;  // destination of the piece in each stage
  unsigned *plen;            // length of the piece in each stage
  char *buf;                 // S * SB bytes
  unsigned SB, min_bulk;
  unsigned issued, retired;  // pieces (lane 0's view)
  bool ok;
  unsigned long long deadline;

  // Per-warp region: 256 bytes of mbarriers and piece records, then the stages.
  __device__ __forceinline__ void init(char *smem, unsigned stage_bytes, unsigned minb, long long timeout_ns,
                                       unsigned lane) {
    const unsigned warp = threadIdx.x >> 5;
    char *base = smem + (size_t)warp * (256 + (size_t)S * stage_bytes);
    mbar = reinterpret_cast<unsigned long long *>(base);
    pdst = reinterpret_cast<unsigned long long *>(base + 64);
    plen = reinterpret_cast<unsigned *>(base + 128);
    buf = base + 256;
    SB = stage_bytes;
    min_bulk = minb;
    issued = retired = 0;
    ok = true;
    deadline = gtimer() + (unsigned long long)timeout_ns;
    if (lane == 0) {
      for (int s = 0; s < S; ++s) mbar_init(mbar + s, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncwarp();
  }

  // lane 0: wait for the oldest piece to land, then store it from its stage
  __device__ __forceinline__ void retire_one() {
    const unsigned p = retired, s = p % S;
    if (ok && !mbar_wait(mbar + s, (p / S) & 1u, deadline)) ok = false;
    if (ok) {
      bulk_s2g(reinterpret_cast<void *>(pdst[s]), buf + (size_t)s * SB, plen[s]);
      bulk_commit();
    }
    ++retired;
  }

  // One work item, all lanes of the warp.
  __device__ __forceinline__ void run(const WorkItem &w, unsigned lane) {
    char *d = reinterpret_cast<char *>(w.dst);
    const char *s = reinterpret_cast<const char *>(w.src);
    if (w.kind != kCopy || (((uintptr_t)d ^ (uintptr_t)s) & 15) != 0 || w.len < min_bulk) {
      run_item<16, 4>(w, lane);
      return;
    }
    unsigned head = (unsigned)((16 - ((uintptr_t)d & 15)) & 15);
    if (head > w.len) head = w.len;
    const unsigned body = (w.len - head) & ~15u;
    const unsigned tail = w.len - head - body;
    if (lane != 0) {
      for (unsigned i = lane - 1; i < head; i += 31) d[i] = s[i];
      for (unsigned i = lane - 1; i < tail; i += 31) d[head + body + i] = s[head + body + i];
    } else if (ok) {
      for (unsigned off = 0; off < body && ok; off += SB) {
        const unsigned len = body - off < SB ? body - off : SB;
        if (issued - retired == (unsigned)S) retire_one();
        const unsigned st = issued % S;
        // the store that last read this stage (piece issued - S) must be
        // done reading: at most `after` younger stores may still be pending
        if (issued >= (unsigned)S) bulk_wait_read_le(retired - 1u - (issued - (unsigned)S));
        pdst[st] = (unsigned long long)(d + head + off);
        plen[st] = len;
        mbar_expect_tx(mbar + st, len);
        bulk_g2s(buf + (size_t)st * SB, s + head + off, len, mbar + st);
        ++issued;
      }
    }
    __syncwarp();
  }

  // lane 0: store what is still in flight and wait for every store.
  // Returns false if an mbarrier wait passed the deadline.
  __device__ __forceinline__ bool drain(unsigned lane) {
    if (lane == 0) {
      while (retired < issued) retire_one();
      bulk_wait_all();
      if (ok)
        for (int s = 0; s < S; ++s) mbar_inval(mbar + s);
    }
    return __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
  }
};

template <int S>
__global__ void __launch_bounds__(256) batch_exec_tma_kernel(const WorkItem *__restrict__ items, BatchCtl *ctl,
                                                              BatchCtl *sctl, unsigned long long cap, int grab,
                                                              unsigned SB, unsigned min_bulk, long long timeout_ns) {
  extern __shared__ __align__(128) char smem[];
  const unsigned lane = threadIdx.x & 31u;
  WarpTma<S> ring;
  ring.init(smem, SB, min_bulk, timeout_ns, lane);  // overlaps the plan kernel
  pdl_release_dependents();
  pdl_wait_prerequisites();
  unsigned long long C = *(volatile unsigned long long *)&ctl->total_chunks;
  const unsigned long long ib = *(volatile unsigned long long *)&ctl->item_base;
  if (!piece_may_run(ctl, sctl) || ib + C > cap) C = 0;  // nothing to run
  items += ib;
  unsigned long long bse = 0;
  if (lane == 0) bse = atomicAdd(&ctl->cursor, (unsigned long long)grab);
  bse = __shfl_sync(0xffffffffu, bse, 0);
  while (bse < C) {
    unsigned long long nxt = 0;
    if (lane == 0) nxt = atomicAdd(&ctl->cursor, (unsigned long long)grab);
    const unsigned long long end = bse + grab < C ? bse + grab : C;
    for (unsigned long long k = bse; k < end; ++k) ring.run(load_item(items + k), lane);
    bse = __shfl_sync(0xffffffffu, nxt, 0);
  }
  if (!ring.drain(lane) && lane == 0) {
    if (atomicCAS(&sctl->status, 0, NVSHMEMX_ERR_TIMEOUT) == 0) sctl->bad_request = -2;
  }
}

// ------------------------------------------------ streaming: one launch
// Planning and execution in one persistent cooperative launch.  The first
// `planners` warps of every CTA claim groups of 32 requests in request order
// (ctl->plan_cursor), validate and translate them, reserve their chunks with
// one atomicAdd per group on ctl->total_chunks, write the work items and,
// after one fence per group, tag each item with the launch's generation
// number in its last word.  Every warp (planners too, once no group is left)
// claims chunk indices from ctl->cursor and waits for the item's tag before
// running it through its TMA ring; once a warp has seen every planner done
// (ctl->plan_done) it knows the final chunk count and checks no more tags.
// All waits are bounded.  Unlike the graph path, an invalid request is
// skipped on its own (and reported); the valid ones still run.
struct StreamCtl {                 // the first 32 bytes match BatchCtl
  unsigned long long total_chunks;
  unsigned long long cursor;
  int status;
  int bad_request;
  unsigned long long pad0;
  unsigned int plan_done;
  unsigned int gen;                // generation of the current launch; outside
                                   // the 32 bytes the graph path zeroes, so it
                                   // only ever grows
  unsigned int plan_cursor;        // next group of 32 requests to plan
  unsigned int pad1;
  unsigned long long pad[2];
};
static_assert(sizeof(StreamCtl) == 64, "StreamCtl is one 64-byte block");

__device__ __forceinline__ void plan_one(const Cfg &c, const nvshmemx_request &r, int i, unsigned chunk,
                                         BatchCtl *ctl, WorkItem &w, unsigned &cnt) {
  cnt = 0;
  w.dst = w.src = 0;
  w.len = 0;
  w.kind = kCopy;
  w.value = 0;
  w.pad = 0;
  const unsigned width = r.dtype == NVSHMEMX_DT_DOUBLE ? 8u : 4u;
  const bool pe_ok = r.src_pe < c.npes && r.dst_pe < c.npes && r.dtype <= NVSHMEMX_DT_DOUBLE;
  const unsigned long long dst = (unsigned long long)c.arena + ((unsigned long long)r.dst_pe << c.log2_stride) + r.dst_off;
  const unsigned long long src = (unsigned long long)c.arena + ((unsigned long long)r.src_pe << c.log2_stride) + r.src_off;
  switch (r.op) {
    case NVSHMEMX_REQ_PUT:
    case NVSHMEMX_REQ_GET:
    case NVSHMEMX_REQ_G: {
      const unsigned long long bytes = r.op == NVSHMEMX_REQ_G ? width : r.bytes;
      if (!pe_ok || !range_in_slice(c, r.src_off, bytes) || !range_in_slice(c, r.dst_off, bytes)) {
        set_status(ctl, NVSHMEMX_ERR_BOUNDS, i);
        return;
      }
      w.dst = dst;
      w.src = src;
      w.len = (unsigned)bytes;
      cnt = bytes ? (unsigned)((bytes + chunk - 1) / chunk) : 0u;
      return;
    }
    case NVSHMEMX_REQ_SIGNAL:
    case NVSHMEMX_REQ_P: {
      const unsigned bytes = r.op == NVSHMEMX_REQ_SIGNAL ? 4u : width;
      if (!pe_ok || !range_in_slice(c, r.dst_off, bytes) || (r.dst_off & (bytes - 1))) {
        set_status(ctl, NVSHMEMX_ERR_BOUNDS, i);
        return;
      }
      w.dst = dst;
      w.src = r.src_off;
      w.len = bytes;
      w.kind = r.op == NVSHMEMX_REQ_SIGNAL ? kSignal : kStore;
      w.value = r.value;
      cnt = 1;
      return;
    }
    default:
      set_status(ctl, NVSHMEMX_ERR_INVALID, i);
  }
}

// The item's payload (its first 28 bytes), written with plain stores; the
// generation tag in the last word is stored separately, after a fence.
__device__ __forceinline__ void write_item_body(WorkItem *p, const WorkItem &w) {
  uint4 a = make_uint4((unsigned)w.dst, (unsigned)(w.dst >> 32), (unsigned)w.src, (unsigned)(w.src >> 32));
  *reinterpret_cast<uint4 *>(p) = a;
  uint2 b = make_uint2(w.len, w.kind);
  *reinterpret_cast<uint2 *>(reinterpret_cast<char *>(p) + 16) = b;
  *reinterpret_cast<int *>(reinterpret_cast<char *>(p) + 24) = w.value;
}

__device__ __forceinline__ void *item_tag(WorkItem *p) { return reinterpret_cast<char *>(p) + 28; }

__device__ __forceinline__ WorkItem read_item(const WorkItem *p) {
  const uint4 a = __ldcg(reinterpret_cast<const uint4 *>(p));
  const uint4 b = __ldcg(reinterpret_cast<const uint4 *>(p) + 1);
  WorkItem w;
  w.dst = ((unsigned long long)a.y << 32) | a.x;
  w.src = ((unsigned long long)a.w << 32) | a.z;
  w.len = b.x;
  w.kind = b.y;
  w.value = (int)b.z;
  w.pad = b.w;
  return w;
}

__device__ __forceinline__ nvshmemx_request load_request(const nvshmemx_request *p) {
  const uint4 a = __ldcg(reinterpret_cast<const uint4 *>(p));
  const uint4 b = __ldcg(reinterpret_cast<const uint4 *>(p) + 1);
  nvshmemx_request r;
  memcpy(&r, &a, 16);
  memcpy(reinterpret_cast<char *>(&r) + 16, &b, 16);
  return r;
}

// 1: item k is ready; 2: there is no item k (all planning done and k is past
// the end, or past the table); 3: the deadline passed.  `final_total` is the
// calling lane's cache of the chunk count: ~0 until it has seen every planner
// finish (an acquire of plan_done, which orders every published item before
// this lane's later reads), after which no item needs a check at all.
__device__ __forceinline__ int wait_item(StreamCtl *ctl, const WorkItem *items, unsigned long long k,
                                         unsigned long long cap, unsigned gen, unsigned planners,
                                         unsigned long long deadline, unsigned long long &final_total) {
  if (k >= cap) return 2;
  if (final_total != ~0ull) return k < final_total ? 1 : 2;
  const int *tag = reinterpret_cast<const int *>(reinterpret_cast<const char *>(items + k) + 28);
  unsigned ns = 0;
  for (unsigned spins = 0;; ++spins) {
    // both loads in flight at once: a relaxed read of plan_done that sees
    // every planner done is followed by a fence (the acquire pattern)
    const unsigned pd = ld_relaxed_b32(&ctl->plan_done);
    const unsigned tg = (unsigned)ld_acquire(tag);
    if (pd == planners) {
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
      final_total = ld_acquire_u64(&ctl->total_chunks);
      return k < final_total ? 1 : 2;
    }
    if (tg == gen) return 1;
    if (spins > 8) {
      ns = ns == 0 ? 32 : (ns >= 512 ? 512 : ns * 2);
      __nanosleep(ns);
    }
    if ((spins & 15) == 15 && gtimer() > deadline) return 3;
  }
}

template <int S>
__global__ void __launch_bounds__(256) batch_stream_kernel(Cfg c, const nvshmemx_request *reqs, int n,
                                                           unsigned chunk, WorkItem *__restrict__ items,
                                                           unsigned long long cap, StreamCtl *ctl, int grab,
                                                           unsigned SB, unsigned min_bulk, int planners_per_cta) {
  extern __shared__ __align__(128) char smem[];
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  BatchCtl *bctl = reinterpret_cast<BatchCtl *>(ctl);
  const unsigned gen = *(volatile unsigned *)&ctl->gen;
  const unsigned planners = gridDim.x * (unsigned)planners_per_cta;
  WarpTma<S> ring;
  ring.init(smem, SB, min_bulk, c.wait_timeout_ns, lane);
  // ---- planning (the first planners_per_cta warps of each CTA)
  if (warp < (unsigned)planners_per_cta) {
    const int ngroups = (n + 31) / 32;
    // groups are claimed in request order, so items are published roughly
    // in request order (the order in which executing warps claim them)
    auto claim = [&]() -> int {
      int v = 0;
      if (lane == 0) v = (int)atomicAdd(&ctl->plan_cursor, 1u);
      return __shfl_sync(0xffffffffu, v, 0);
    };
    int g = claim();
    nvshmemx_request r;
    if (g < ngroups && g * 32 + (int)lane < n) r = load_request(reqs + g * 32 + lane);
    while (g < ngroups) {
      const int i = g * 32 + (int)lane;
      // claim the next group and fetch it while this one is planned
      const int gn = claim();
      nvshmemx_request rn;
      if (gn < ngroups && gn * 32 + (int)lane < n) rn = load_request(reqs + gn * 32 + lane);
      WorkItem w;
      unsigned cnt = 0;
      if (i < n) plan_one(c, r, i, chunk, bctl, w, cnt);
      unsigned incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (unsigned)o) incl += v;
      }
      const unsigned tot = __shfl_sync(0xffffffffu, incl, 31);
      unsigned long long base = 0;
      if (lane == 31 && tot) {
        base = atomicAdd(&ctl->total_chunks, (unsigned long long)tot);
        if (base + tot > cap) set_status(bctl, NVSHMEMX_ERR_NOMEM, -1);
      }
      base = __shfl_sync(0xffffffffu, base, 31);
      const unsigned long long first = base + incl - cnt;
      const unsigned last = first + cnt <= cap ? cnt : (first < cap ? (unsigned)(cap - first) : 0u);
      for (unsigned k = 0; k < last; ++k) {
        WorkItem p = w;
        const unsigned long long off = (unsigned long long)k * chunk;
        p.dst += off;
        p.src += off;
        if (w.kind == kCopy) p.len = (unsigned)((w.len - off) < chunk ? (w.len - off) : chunk);
        write_item_body(items + first + k, p);
      }
      // one fence per group orders every payload before its tag (a release
      // pattern: fence, then strong stores); consumers acquire the tag
      __threadfence();
      for (unsigned k = 0; k < last; ++k) st_relaxed_b32(item_tag(items + first + k), gen);
      g = gn;
      r = rn;
    }
    __syncwarp();
    if (lane == 0) {
      __threadfence();
      atomicAdd(&ctl->plan_done, 1u);
    }
  }
  // ---- execution (every warp); the next claim is in flight while the
  // current one runs, as in the graph path
  unsigned long long final_total = ~0ull;
  int st = 1;
  unsigned long long bse = 0;
  if (lane == 0) bse = atomicAdd(&ctl->cursor, (unsigned long long)grab);
  bse = __shfl_sync(0xffffffffu, bse, 0);
  while (st == 1) {
    unsigned long long nxt = 0;
    if (lane == 0) nxt = atomicAdd(&ctl->cursor, (unsigned long long)grab);
    for (unsigned long long k = bse; k < bse + (unsigned long long)grab; ++k) {
      if (lane == 0) st = wait_item(ctl, items, k, cap, gen, planners, ring.deadline, final_total);
      st = __shfl_sync(0xffffffffu, st, 0);
      if (st != 1) break;
      ring.run(read_item(items + k), lane);
    }
    bse = __shfl_sync(0xffffffffu, nxt, 0);
  }
  const bool ok = ring.drain(lane);
  if ((st == 3 || !ok) && lane == 0) {
    if (atomicCAS(&ctl->status, 0, NVSHMEMX_ERR_TIMEOUT) == 0) ctl->bad_request = -2;
  }
}

// End of a pipelined submit: once the last exec kernel is done (it lets this
// kernel start early; griddepcontrol.wait holds it until the exec grid has
// completed and its writes are visible), writes the batch status word and
// the first bad request into the caller-visible pinned host words.
__global__ void status_to_host_kernel(const BatchCtl *ctl, volatile int *host_status) {
  pdl_wait_prerequisites();
  if (threadIdx.x == 0) {
    host_status[0] = *(volatile const int *)&ctl->status;
    host_status[1] = *(volatile const int *)&ctl->bad_request;
    __threadfence_system();
  }
}

// Zeroes the control block of a streaming launch and moves its generation
// on (one thread; a graph node in place of a memset).
__global__ void stream_reset_kernel(StreamCtl *ctl) {
  const unsigned g = ctl->gen + 1u;
  ctl->total_chunks = 0;
  ctl->cursor = 0;
  ctl->status = 0;
  ctl->bad_request = 0;
  ctl->plan_done = 0;
  ctl->plan_cursor = 0;
  ctl->gen = g == 0 ? 1u : g;
}

typedef void (*TmaFn)(const WorkItem *, BatchCtl *, BatchCtl *, unsigned long long, int, unsigned, unsigned,
                      long long);

static TmaFn pick_tma(int stages) {
  switch (stages) {
    case 2: return batch_exec_tma_kernel<2>;
    case 3: return batch_exec_tma_kernel<3>;
    case 4: return batch_exec_tma_kernel<4>;
    default: return nullptr;
  }
}

static size_t tma_smem_bytes(const nvshmemx_batch_config &k) {
  return (size_t)(k.threads / 32) * (256 + (size_t)k.tma_stages * (size_t)k.tma_stage_bytes);
}

// Cooperative launch of the streaming kernel (every CTA must be resident:
// executing warps wait for items that planning warps of other CTAs publish).
static cudaError_t launch_stream(int stages, dim3 grid, dim3 block, size_t smem, cudaStream_t st, const Cfg &c,
                                 const nvshmemx_request *src, int n, unsigned chunk, WorkItem *items,
                                 unsigned long long cap, StreamCtl *ctl, int grab, unsigned SB, unsigned min_bulk,
                                 int planners) {
  cudaLaunchConfig_t lc = {};
  lc.gridDim = grid;
  lc.blockDim = block;
  lc.dynamicSmemBytes = smem;
  lc.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  switch (stages) {
    case 2: return cudaLaunchKernelEx(&lc, batch_stream_kernel<2>, c, src, n, chunk, items, cap, ctl, grab, SB, min_bulk, planners);
    case 3: return cudaLaunchKernelEx(&lc, batch_stream_kernel<3>, c, src, n, chunk, items, cap, ctl, grab, SB, min_bulk, planners);
    case 4: return cudaLaunchKernelEx(&lc, batch_stream_kernel<4>, c, src, n, chunk, items, cap, ctl, grab, SB, min_bulk, planners);
    default: return cudaErrorInvalidValue;
  }
}

static const void *stream_fn(int stages) {
  switch (stages) {
    case 2: return (const void *)batch_stream_kernel<2>;
    case 3: return (const void *)batch_stream_kernel<3>;
    case 4: return (const void *)batch_stream_kernel<4>;
    default: return nullptr;
  }
}

typedef void (*ExecFn)(const WorkItem *, BatchCtl *, BatchCtl *, unsigned long long, int);

static ExecFn pick_exec(int vb, int u) {
#define NVSHM_PICK(V, UU) \
  if (vb == V && u == UU) return batch_exec_kernel<V, UU>;
  NVSHM_PICK(16, 1) NVSHM_PICK(16, 2) NVSHM_PICK(16, 4) NVSHM_PICK(16, 8)
  NVSHM_PICK(8, 1) NVSHM_PICK(8, 2) NVSHM_PICK(8, 4) NVSHM_PICK(8, 8)
  NVSHM_PICK(4, 1) NVSHM_PICK(4, 2) NVSHM_PICK(4, 4) NVSHM_PICK(4, 8)
#undef NVSHM_PICK
  return nullptr;
}

int check_batch_config(const nvshmemx_batch_config &c) {
  const bool ok = (c.vec_bytes == 4 || c.vec_bytes == 8 || c.vec_bytes == 16) && c.chunk_bytes >= 256 &&
                  c.chunk_bytes <= (1 << 20) && (c.chunk_bytes % 256) == 0 &&
                  (c.unroll == 1 || c.unroll == 2 || c.unroll == 4 || c.unroll == 8) &&
                  (c.threads == 128 || c.threads == 256 || c.threads == 512 || c.threads == 1024) &&
                  c.ctas_per_sm >= 0 && c.ctas_per_sm <= 16 && c.grab >= 1 && c.grab <= 16;
  if (!ok) return NVSHMEMX_ERR_INVALID;
  if (c.tma_stages == 0) return c.stream == 0 ? 0 : NVSHMEMX_ERR_INVALID;
  // TMA rings: at most 256 threads per CTA (8 warps, one ring each), stage
  // sizes in whole KiB, and the CTA's rings must fit in 227 KiB of shared
  // memory.
  const bool tma_ok = (c.tma_stages >= 2 && c.tma_stages <= 4) && c.threads <= 256 && c.tma_stage_bytes >= 1024 &&
                      c.tma_stage_bytes <= 32768 && (c.tma_stage_bytes % 1024) == 0 && c.tma_min_bytes >= 0 &&
                      tma_smem_bytes(c) <= 227u * 1024u;
  if (!tma_ok) return NVSHMEMX_ERR_INVALID;
  // streaming needs the TMA rings and at least one executing-only warp
  if (c.stream != 0 && (c.stream != 1 || c.stream_planners < 1 || c.stream_planners > 4 ||
                        c.stream_planners >= c.threads / 32))
    return NVSHMEMX_ERR_INVALID;
  return 0;
}

}  // namespace nvshm

using namespace nvshm;

struct nvshmemx_batch {
  int max_n = 0;
  int min_chunk = 256;
  unsigned long long cap = 0;
  nvshmemx_request *d_reqs = nullptr;
  nvshmemx_request_compact *d_reqs_compact = nullptr;  // compact submits: what crossed the host link
  WorkItem *d_items = nullptr;
  BatchCtl *d_ctl = nullptr;
  nvshmemx_request *h_reqs = nullptr;  // pinned
  int *h_status = nullptr;             // pinned
  int *h_status_dev = nullptr;         // h_status as the device sees it
  int n = 0;
  nvshmemx_batch_config cfg{};
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // pipelined submit: copies and plans of the pieces
  cudaEvent_t ev_reset = nullptr, ev_copied = nullptr;
  cudaEvent_t ev_piece[3] = {nullptr, nullptr, nullptr};  // piece k planned
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int graph_n = -1;
  const nvshmemx_request *graph_src = nullptr;  // request array the graph reads
  nvshmemx_batch_config graph_cfg{};
  Cfg graph_arena{};
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr, ev_plan0 = nullptr, ev_exec0 = nullptr, ev_exec1 = nullptr;
  bool timed_direct = false;  // ev_plan0/ev_exec0/ev_exec1 hold the last direct execution
  int last_pieces = 1;        // pieces of the last execution (pipelined submit: 2)
};

// Control block of piece k of a pipelined submit: bytes 0..31, 64..95 and
// 96..127 of the batch's 128-byte control allocation (bytes 32..63 hold the
// streaming generation, which must never be zeroed).
static BatchCtl *piece_ctl(nvshmemx_batch *b, int k) {
  static const int off[3] = {0, 64, 96};
  return reinterpret_cast<BatchCtl *>(reinterpret_cast<char *>(b->d_ctl) + off[k]);
}

// Pieces of a pipelined submit (ends[k] = end of piece k, in requests): one
// below 8192 requests, where the copy is too short to be worth hiding, else
// two, a quarter (in whole 256-request plan blocks) and the rest.  (Three
// pieces, an eighth / three eighths / a half, measured 6 us slower on the
// 100,000-request batch: each extra exec launch costs more than it hides.)
static int split_pieces(int n, int ends[3]) {
  if (n < 8192) {
    ends[0] = n;
    return 1;
  }
  ends[0] = (n / 4) & ~255;
  ends[1] = n;
  return 2;
}

static void drop_graph(nvshmemx_batch *b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->gexec = nullptr;
  b->graph = nullptr;
  b->graph_n = -1;
}

// Stream mode: reset + the streaming kernel reading the requests at `src`.
static int enqueue_stream(nvshmemx_batch *b, bool with_events, const nvshmemx_request *src) {
  const Runtime &r = rt();
  const Cfg c = r.cfg;
  const nvshmemx_batch_config &k = b->cfg;
  const void *sfn = stream_fn(k.tma_stages);
  if (!sfn) return fail(NVSHMEMX_ERR_INVALID, "batch: no streaming kernel for %d stages", k.tma_stages);
  (void)cudaGetLastError();
  const size_t smem = tma_smem_bytes(k);
  cudaFuncSetAttribute(sfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sfn, k.threads, smem);
  if (per_sm < 1) return fail(NVSHMEMX_ERR_COOP, "batch: streaming kernel does not fit an SM");
  const int ctas = k.ctas_per_sm > 0 && k.ctas_per_sm < per_sm ? k.ctas_per_sm : per_sm;
  StreamCtl *sctl = reinterpret_cast<StreamCtl *>(b->d_ctl);
  if (with_events) cudaEventRecord(b->ev_plan0, b->stream);
  stream_reset_kernel<<<1, 1, 0, b->stream>>>(sctl);
  if (with_events) cudaEventRecord(b->ev_exec0, b->stream);
  cudaError_t e = launch_stream(k.tma_stages, dim3(r.sm_count * ctas), dim3(k.threads), smem, b->stream, c, src,
                                b->n, (unsigned)k.chunk_bytes, b->d_items, b->cap, sctl, k.grab,
                                (unsigned)k.tma_stage_bytes, (unsigned)k.tma_min_bytes, k.stream_planners);
  if (e != cudaSuccess) return check_cuda(e, "batch streaming launch");
  if (with_events) cudaEventRecord(b->ev_exec1, b->stream);
  return check_cuda(cudaGetLastError(), "batch streaming launch");
}

// Plan (parts & 1) and/or exec (parts & 2) of one piece of a batch (n
// requests at `src`) on stream `st`, with the piece's control block `ctl`,
// errors into `sctl`, and its items appended after those of `prev`.
// kCompact: `src` holds compact requests; the plan stores their full form at
// b->d_reqs + req_base.
enum { kPlan = 1, kExec = 2, kCompact = 4 };
static int enqueue_piece(nvshmemx_batch *b, bool with_events, const void *src, int n, BatchCtl *ctl,
                         BatchCtl *sctl, const BatchCtl *prev, int req_base, cudaStream_t st, int parts) {
  const Runtime &r = rt();
  const Cfg c = r.cfg;
  const nvshmemx_batch_config &k = b->cfg;
  const unsigned long long cap_end = b->cap;
  ExecFn fn = pick_exec(k.vec_bytes, k.unroll);
  TmaFn tfn = k.tma_stages ? pick_tma(k.tma_stages) : nullptr;
  if (!fn || (k.tma_stages && !tfn))
    return fail(NVSHMEMX_ERR_INVALID, "batch: no kernel for vec %d unroll %d stages %d", k.vec_bytes, k.unroll,
                k.tma_stages);
  (void)cudaGetLastError();  // report only this enqueue's own launch errors
  if (with_events) cudaEventRecord(b->ev_plan0, st);
  if ((parts & kPlan) && n > 0) {
    if (parts & kCompact)
      batch_plan_kernel<true><<<(n + kPlanThreads - 1) / kPlanThreads, kPlanThreads, 0, st>>>(c, src, n, (unsigned)k.chunk_bytes, b->d_items, cap_end,
                                                              ctl, sctl, prev, req_base, b->d_reqs + req_base);
    else
      batch_plan_kernel<false><<<(n + kPlanThreads - 1) / kPlanThreads, kPlanThreads, 0, st>>>(c, src, n, (unsigned)k.chunk_bytes, b->d_items,
                                                               cap_end, ctl, sctl, prev, req_base, nullptr);
  }
  if (with_events) cudaEventRecord(b->ev_exec0, st);
  if (!(parts & kExec)) return check_cuda(cudaGetLastError(), "batch plan launch");
  const size_t smem = tfn ? tma_smem_bytes(k) : 0;
  int per_sm = 0;
  if (tfn) {
    cudaFuncSetAttribute((const void *)tfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // the rings are all the shared memory a CTA uses: ask for the largest
    // shared-memory carveout, so the CTAs the occupancy query counts on fit
    cudaFuncSetAttribute((const void *)tfn, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)tfn, k.threads, smem);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn, k.threads, 0);
  }
  if (per_sm < 1) per_sm = 1;
  int ctas = k.ctas_per_sm > 0 && k.ctas_per_sm < per_sm ? k.ctas_per_sm : per_sm;
  // Right after the plan kernel (no event between them), the exec kernel is
  // a programmatic dependent launch: its set-up overlaps the plan's tail.
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(r.sm_count * ctas);
  lc.blockDim = dim3(k.threads);
  lc.dynamicSmemBytes = smem;
  lc.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = attr;
  lc.numAttrs = ((parts & kPlan) && n > 0 && !with_events) ? 1 : 0;
  cudaError_t e;
  if (tfn)
    e = cudaLaunchKernelEx(&lc, tfn, (const WorkItem *)b->d_items, ctl, sctl, cap_end, k.grab,
                           (unsigned)k.tma_stage_bytes, (unsigned)k.tma_min_bytes, (long long)c.wait_timeout_ns);
  else
    e = cudaLaunchKernelEx(&lc, fn, (const WorkItem *)b->d_items, ctl, sctl, cap_end, k.grab);
  if (with_events) cudaEventRecord(b->ev_exec1, st);
  if (e != cudaSuccess) return check_cuda(e, "batch exec launch");
  return check_cuda(cudaGetLastError(), "batch launch");
}

// Enqueues memset + plan + exec (or, in stream mode, reset + the streaming
// kernel) reading the requests at `src` on b->stream (used both for capture
// and for the direct path).
static int enqueue_batch(nvshmemx_batch *b, bool with_events, const nvshmemx_request *src) {
  if (b->cfg.stream) return enqueue_stream(b, with_events, src);
  cudaMemsetAsync(b->d_ctl, 0, sizeof(BatchCtl), b->stream);
  return enqueue_piece(b, with_events, src, b->n, b->d_ctl, b->d_ctl, nullptr, 0, b->stream, kPlan | kExec);
}

static int ensure_graph(nvshmemx_batch *b, const nvshmemx_request *src) {
  const Cfg &c = rt().cfg;
  if (b->gexec && b->graph_n == b->n && b->graph_src == src && memcmp(&b->graph_cfg, &b->cfg, sizeof b->cfg) == 0 &&
      memcmp(&b->graph_arena, &c, sizeof c) == 0)
    return 0;
  drop_graph(b);
  int rc;
  if ((rc = check_cuda(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture")))
    return rc;
  int erc = enqueue_batch(b, false, src);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (erc) {
    if (g) cudaGraphDestroy(g);
    return erc;
  }
  if ((rc = check_cuda(e, "cudaStreamEndCapture"))) return rc;
  b->graph = g;
  if ((rc = check_cuda(cudaGraphInstantiate(&b->gexec, g, 0), "cudaGraphInstantiate"))) {
    drop_graph(b);
    return rc;
  }
  b->graph_n = b->n;
  b->graph_src = src;
  b->graph_cfg = b->cfg;
  b->graph_arena = c;
  return 0;
}

// ------------------------------------------------ grouped runs (picker.cu)
// A run's plan or exec error, copied into the sticky word at byte 128 of the
// control allocation unless that already holds one (first error wins).
__global__ void sticky_status_kernel(const BatchCtl *ctl, int *sticky) {
  if (threadIdx.x == 0 && ctl->status != 0 && sticky[0] == 0) {
    sticky[0] = ctl->status;
    sticky[1] = ctl->bad_request;
  }
}

static int *sticky_word(nvshmemx_batch *b) {
  return reinterpret_cast<int *>(reinterpret_cast<char *>(b->d_ctl) + 128);
}

namespace nvshm {
cudaStream_t batch_stream(const nvshmemx_batch *b) { return b->stream; }
nvshmemx_request *batch_device_requests(nvshmemx_batch *b) { return b->d_reqs; }
int batch_capacity(const nvshmemx_batch *b) { return b->max_n; }
int batch_min_chunk(const nvshmemx_batch *b) { return b->min_chunk; }

int batch_enqueue_range(nvshmemx_batch *b, int first, int n, const nvshmemx_batch_config &cfg) {
  if (first < 0 || n < 0 || first > b->max_n || n > b->max_n - first || cfg.stream != 0 || check_batch_config(cfg) ||
      cfg.chunk_bytes < b->min_chunk)
    return fail(NVSHMEMX_ERR_INVALID, "batch range run: bad range or configuration");
  if (n == 0) return 0;
  const nvshmemx_batch_config saved = b->cfg;
  b->cfg = cfg;
  int rc = check_cuda(cudaMemsetAsync(b->d_ctl, 0, sizeof(BatchCtl), b->stream), "cudaMemsetAsync");
  if (!rc) rc = enqueue_piece(b, false, b->d_reqs + first, n, b->d_ctl, b->d_ctl, nullptr, 0, b->stream, kPlan | kExec);
  b->cfg = saved;
  if (!rc) {
    sticky_status_kernel<<<1, 32, 0, b->stream>>>(b->d_ctl, sticky_word(b));
    rc = check_cuda(cudaGetLastError(), "sticky status kernel");
  }
  return rc;
}

int batch_clear_sticky(nvshmemx_batch *b) {
  return check_cuda(cudaMemsetAsync(sticky_word(b), 0, 8, b->stream), "cudaMemsetAsync(sticky)");
}

int batch_sticky_status(nvshmemx_batch *b, int *status, int *bad_request) {
  int st[2] = {0, 0};
  int rc = check_cuda(cudaMemcpy(st, sticky_word(b), 8, cudaMemcpyDeviceToHost), "read sticky status");
  *status = st[0];
  *bad_request = st[1];
  return rc;
}
}  // namespace nvshm

extern "C" {

// Per-warp TMA rings of 3 x 8 KiB, 8 warps per CTA, 16 KiB chunks, 2 chunks
// per claim, register copy below 512 bytes: one of the autotuner's leading
// shapes on the 64-PE / 100,000-request workload (4th of 112, 1% behind the
// table's best, 2 x 8 KiB rings with 4 warps per CTA; the first eight lie
// within 1.5% of each other and their order changes from box to box).
void nvshmemx_batch_default_config(nvshmemx_batch_config *c) {
  c->vec_bytes = 16;
  c->chunk_bytes = 16384;
  c->unroll = 4;
  c->threads = 256;
  c->ctas_per_sm = 0;
  c->grab = 2;
  c->tma_stages = 3;
  c->tma_stage_bytes = 8192;
  c->tma_min_bytes = 512;
  c->stream = 0;
  c->stream_planners = 2;
}

int nvshmemx_batch_create(int max_requests, unsigned long long max_payload_bytes, int min_chunk_bytes,
                          nvshmemx_batch **out) {
  if (!is_started()) return fail(NVSHMEMX_ERR_STATE, "batch before nvstart_pes");
  if (!out || max_requests < 1) return fail(NVSHMEMX_ERR_INVALID, "batch_create: bad arguments");
  if (min_chunk_bytes < 256) min_chunk_bytes = 256;
  nvshmemx_batch *b = new nvshmemx_batch();
  b->max_n = max_requests;
  b->min_chunk = min_chunk_bytes;
  b->cap = (unsigned long long)max_requests + max_payload_bytes / (unsigned long long)min_chunk_bytes + 1;
  nvshmemx_batch_default_config(&b->cfg);
  if (b->cfg.chunk_bytes < min_chunk_bytes) b->cfg.chunk_bytes = (min_chunk_bytes + 255) / 256 * 256;
  int rc = 0;
  if ((rc = check_cuda(cudaMalloc(&b->d_reqs, (size_t)max_requests * sizeof(nvshmemx_request)), "cudaMalloc(reqs)")) ||
      (rc = check_cuda(cudaMalloc(&b->d_reqs_compact, (size_t)max_requests * sizeof(nvshmemx_request_compact)),
                       "cudaMalloc(compact reqs)")) ||
      (rc = check_cuda(cudaMalloc(&b->d_items, (size_t)b->cap * sizeof(WorkItem)), "cudaMalloc(items)")) ||
      (rc = check_cuda(cudaMalloc(&b->d_ctl, 256), "cudaMalloc(ctl)")) ||
      (rc = check_cuda(cudaMallocHost(&b->h_reqs, (size_t)max_requests * sizeof(nvshmemx_request)),
                       "cudaMallocHost(reqs)")) ||
      (rc = check_cuda(cudaMallocHost(&b->h_status, 64), "cudaMallocHost(status)")) ||
      (rc = check_cuda(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate")) ||
      (rc = check_cuda(cudaStreamCreateWithFlags(&b->copy_stream, cudaStreamNonBlocking), "cudaStreamCreate"))) {
    nvshmemx_batch_destroy(b);
    return rc;
  }
  cudaEventCreate(&b->ev_start);
  cudaEventCreate(&b->ev_stop);
  cudaEventCreate(&b->ev_plan0);
  cudaEventCreate(&b->ev_exec0);
  cudaEventCreate(&b->ev_exec1);
  cudaEventCreateWithFlags(&b->ev_reset, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&b->ev_copied, cudaEventDisableTiming);
  for (auto &e : b->ev_piece) cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
  void *hs = nullptr;
  if ((rc = check_cuda(cudaHostGetDevicePointer(&hs, b->h_status, 0), "cudaHostGetDevicePointer(status)"))) {
    nvshmemx_batch_destroy(b);
    return rc;
  }
  b->h_status_dev = static_cast<int *>(hs);
  // control block (BatchCtl or StreamCtl) and every work item's generation
  // tag start at zero; streaming generations start at 1
  cudaMemset(b->d_ctl, 0, 256);
  cudaMemset(b->d_items, 0, (size_t)b->cap * sizeof(WorkItem));
  *out = b;
  return 0;
}

int nvshmemx_batch_destroy(nvshmemx_batch *b) {
  if (!b) return 0;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->copy_stream) cudaStreamSynchronize(b->copy_stream);
  drop_graph(b);
  if (b->d_reqs) cudaFree(b->d_reqs);
  if (b->d_reqs_compact) cudaFree(b->d_reqs_compact);
  if (b->d_items) cudaFree(b->d_items);
  if (b->d_ctl) cudaFree(b->d_ctl);
  if (b->h_reqs) cudaFreeHost(b->h_reqs);
  if (b->h_status) cudaFreeHost(b->h_status);
  cudaEvent_t evs[] = {b->ev_start,    b->ev_stop,     b->ev_plan0,    b->ev_exec0,   b->ev_exec1,
                       b->ev_reset,    b->ev_copied,   b->ev_piece[0], b->ev_piece[1], b->ev_piece[2]};
  for (auto e : evs)
    if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  if (b->copy_stream) cudaStreamDestroy(b->copy_stream);
  delete b;
  return 0;
}

int nvshmemx_batch_set_config(nvshmemx_batch *b, const nvshmemx_batch_config *cfg) {
  if (!b || !cfg || check_batch_config(*cfg) || cfg->chunk_bytes < b->min_chunk)
    return fail(NVSHMEMX_ERR_INVALID, "batch_set_config: invalid configuration");
  b->cfg = *cfg;
  return 0;
}

int nvshmemx_batch_get_config(const nvshmemx_batch *b, nvshmemx_batch_config *cfg) {
  if (!b || !cfg) return NVSHMEMX_ERR_INVALID;
  *cfg = b->cfg;
  return 0;
}

nvshmemx_request *nvshmemx_batch_host_buffer(nvshmemx_batch *b) { return b ? b->h_reqs : nullptr; }

int nvshmemx_batch_upload(nvshmemx_batch *b, const nvshmemx_request *reqs, int n) {
  if (!b || n < 0 || n > b->max_n) return fail(NVSHMEMX_ERR_INVALID, "batch_upload: n outside [0, max]");
  int rc;
  if (n &&
      (rc = check_cuda(cudaMemcpyAsync(b->d_reqs, reqs, (size_t)n * sizeof(nvshmemx_request), cudaMemcpyHostToDevice,
                                       b->stream),
                       "cudaMemcpyAsync(requests)")))
    return rc;
  b->n = n;
  return check_cuda(cudaStreamSynchronize(b->stream), "batch_upload");
}

int nvshmemx_batch_execute(nvshmemx_batch *b, int reps, float *out_ms) {
  if (!b || reps < 1) return fail(NVSHMEMX_ERR_INVALID, "batch_execute: bad arguments");
  int rc;
  if ((rc = ensure_graph(b, b->d_reqs))) return rc;
  b->last_pieces = 1;
  cudaEventRecord(b->ev_start, b->stream);
  for (int i = 0; i < reps; ++i)
    if ((rc = check_cuda(cudaGraphLaunch(b->gexec, b->stream), "cudaGraphLaunch"))) return rc;
  cudaEventRecord(b->ev_stop, b->stream);
  if ((rc = check_cuda(cudaStreamSynchronize(b->stream), "batch_execute"))) return rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, b->ev_start, b->ev_stop);
  if (out_ms) *out_ms = ms;
  int st[2] = {0, 0};
  cudaMemcpy(st, &b->d_ctl->status, sizeof st, cudaMemcpyDeviceToHost);
  if (st[0]) return fail(st[0], "batch_execute: request %d rejected (%s)", st[1], nvshmemx_strerror(st[0]));
  return 0;
}

// The pieces of a submit (graph configuration): see nvshmemx_batch_submit.
// `host` holds n requests of `elem` bytes (full or compact form, `flag` 0 or
// kCompact), copied piece by piece to `dev`.
static int submit_pieces(nvshmemx_batch *b, const void *host, void *dev, size_t elem, int flag, int pieces,
                         const int ends[3]) {
  int rc = 0;
  // The copy stream copies and plans the pieces in order (each plan
  // appends its items after the previous piece's); the batch's stream
  // executes piece k once it is planned and piece k-1 has run.  Each piece
  // has its own control block; the execs report into the first.
  rc = check_cuda(cudaStreamWaitEvent(b->copy_stream, b->ev_start, 0), "cudaStreamWaitEvent");
  if (!rc)
    rc = check_cuda(cudaMemsetAsync(piece_ctl(b, 0), 0, sizeof(BatchCtl), b->copy_stream), "cudaMemsetAsync");
  if (!rc)  // blocks 1 and 2 are contiguous (bytes 64..127)
    rc = check_cuda(cudaMemsetAsync(piece_ctl(b, 1), 0, 2 * sizeof(BatchCtl), b->copy_stream), "cudaMemsetAsync");
  for (int k = 0, at = 0; k < pieces && !rc; at = ends[k++]) {
    const int m = ends[k] - at;
    BatchCtl *ck = piece_ctl(b, k);
    const char *hsrc = static_cast<const char *>(host) + (size_t)at * elem;
    char *dsrc = static_cast<char *>(dev) + (size_t)at * elem;
    if ((rc = check_cuda(cudaMemcpyAsync(dsrc, hsrc, (size_t)m * elem, cudaMemcpyHostToDevice, b->copy_stream),
                         "cudaMemcpyAsync(requests)")) ||
        (rc = enqueue_piece(b, false, dsrc, m, ck, ck, k ? piece_ctl(b, k - 1) : nullptr, at, b->copy_stream,
                            kPlan | flag)) ||
        (rc = check_cuda(cudaEventRecord(b->ev_piece[k], b->copy_stream), "cudaEventRecord")))
      break;
  }
  for (int k = 0, at = 0; k < pieces && !rc; at = ends[k++]) {
    if ((rc = check_cuda(cudaStreamWaitEvent(b->stream, b->ev_piece[k], 0), "cudaStreamWaitEvent")) ||
        (rc = enqueue_piece(b, false, nullptr, ends[k] - at, piece_ctl(b, k), piece_ctl(b, 0), nullptr, at,
                            b->stream, kExec)))
      break;
  }
  if (rc) {
    cudaStreamSynchronize(b->copy_stream);
    cudaStreamSynchronize(b->stream);
    return rc;
  }
  BatchCtl *c0 = piece_ctl(b, 0);
  // the status word reaches the host from a kernel that starts while the
  // last exec runs and writes as soon as it is done (no copy to schedule)
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3(1);
  lc.blockDim = dim3(32);
  lc.stream = b->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  if ((rc = check_cuda(cudaLaunchKernelEx(&lc, status_to_host_kernel, (const BatchCtl *)c0,
                                          (volatile int *)b->h_status_dev),
                       "status kernel launch")))
    return rc;
  return 0;
}

int nvshmemx_batch_submit(nvshmemx_batch *b, const nvshmemx_request *reqs, int n, int *out_status, float *out_ms) {
  if (!b || n < 0 || n > b->max_n || (n && !reqs)) return fail(NVSHMEMX_ERR_INVALID, "batch_submit: bad arguments");
  int rc;
  b->n = n;
  int ends[3];
  const int pieces = b->cfg.stream ? 1 : split_pieces(n, ends);
  if (pieces == 1 && (rc = ensure_graph(b, b->d_reqs))) return rc;
  b->last_pieces = pieces;
  b->timed_direct = false;
  cudaEventRecord(b->ev_start, b->stream);
  if (pieces > 1) {
    if ((rc = submit_pieces(b, reqs, b->d_reqs, sizeof(nvshmemx_request), 0, pieces, ends))) return rc;
  } else {
    if (n && (rc = check_cuda(cudaMemcpyAsync(b->d_reqs, reqs, (size_t)n * sizeof(nvshmemx_request),
                                              cudaMemcpyHostToDevice, b->stream),
                              "cudaMemcpyAsync(requests)")))
      return rc;
    if ((rc = check_cuda(cudaGraphLaunch(b->gexec, b->stream), "cudaGraphLaunch"))) return rc;
    if ((rc = check_cuda(cudaMemcpyAsync(b->h_status, &b->d_ctl->status, 8, cudaMemcpyDeviceToHost, b->stream),
                         "cudaMemcpyAsync(status)")))
      return rc;
  }
  cudaEventRecord(b->ev_stop, b->stream);
  if ((rc = check_cuda(cudaStreamSynchronize(b->stream), "batch_submit"))) return rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, b->ev_start, b->ev_stop);
  if (out_ms) *out_ms = ms;
  if (out_status) *out_status = b->h_status[0];
  return 0;
}

int nvshmemx_batch_submit_compact(nvshmemx_batch *b, const nvshmemx_request_compact *reqs, int n, int *out_status,
                                  float *out_ms) {
  if (!b || n < 0 || n > b->max_n || (n && !reqs))
    return fail(NVSHMEMX_ERR_INVALID, "batch_submit_compact: bad arguments");
  if (b->cfg.stream) return fail(NVSHMEMX_ERR_INVALID, "batch_submit_compact: needs a graph configuration (stream 0)");
  int rc;
  b->n = n;
  b->timed_direct = false;
  if (out_status) *out_status = 0;
  if (out_ms) *out_ms = 0.f;
  if (n == 0) {
    b->last_pieces = 1;
    return 0;
  }
  // every piece count goes through the copy stream: the plan kernels expand
  // the compact requests and leave the full form in b->d_reqs
  int ends[3];
  const int pieces = split_pieces(n, ends);
  b->last_pieces = pieces;
  cudaEventRecord(b->ev_start, b->stream);
  if ((rc = submit_pieces(b, reqs, b->d_reqs_compact, sizeof(nvshmemx_request_compact), kCompact, pieces, ends)))
    return rc;
  cudaEventRecord(b->ev_stop, b->stream);
  if ((rc = check_cuda(cudaStreamSynchronize(b->stream), "batch_submit_compact"))) return rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, b->ev_start, b->ev_stop);
  if (out_ms) *out_ms = ms;
  if (out_status) *out_status = b->h_status[0];
  return 0;
}

int nvshmemx_batch_last_stats(const nvshmemx_batch *b, unsigned long long *chunks, float *plan_ms, float *exec_ms) {
  if (!b) return NVSHMEMX_ERR_INVALID;
  if (chunks) {
    BatchCtl h[4];  // bytes 0..127: piece 0, (streaming state), pieces 1 and 2
    if (cudaMemcpy(h, b->d_ctl, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess)
      return check_cuda(cudaGetLastError(), "batch_last_stats");
    *chunks = h[0].total_chunks;
    if (b->last_pieces > 1) *chunks += h[2].total_chunks;
    if (b->last_pieces > 2) *chunks += h[3].total_chunks;
  }
  float p = 0, e = 0;
  if (b->timed_direct) {
    cudaEventElapsedTime(&p, b->ev_plan0, b->ev_exec0);
    cudaEventElapsedTime(&e, b->ev_exec0, b->ev_exec1);
  }
  if (plan_ms) *plan_ms = p;
  if (exec_ms) *exec_ms = e;
  return 0;
}

// Same work as one graph launch, enqueued directly with CUDA events around
// the plan and exec kernels on the batch's stream, so the exec kernel's own
// duration can be read (events recorded inside a captured graph are not used
// for timing).  *out_exec_ms sums the exec kernel over all reps.
int nvshmemx_batch_execute_direct(nvshmemx_batch *b, int reps, float *out_ms, float *out_exec_ms) {
  if (!b || reps < 1) return fail(NVSHMEMX_ERR_INVALID, "batch_execute_direct: bad arguments");
  int rc;
  float total = 0, exec = 0;
  b->last_pieces = 1;
  for (int i = 0; i < reps; ++i) {
    cudaEventRecord(b->ev_start, b->stream);
    if ((rc = enqueue_batch(b, true, b->d_reqs))) return rc;
    cudaEventRecord(b->ev_stop, b->stream);
    if ((rc = check_cuda(cudaStreamSynchronize(b->stream), "batch_execute_direct"))) return rc;
    float t = 0, e = 0;
    cudaEventElapsedTime(&t, b->ev_start, b->ev_stop);
    cudaEventElapsedTime(&e, b->ev_exec0, b->ev_exec1);
    total += t;
    exec += e;
  }
  b->timed_direct = true;
  if (out_ms) *out_ms = total;
  if (out_exec_ms) *out_exec_ms = exec;
  int st[2] = {0, 0};
  cudaMemcpy(st, &b->d_ctl->status, sizeof st, cudaMemcpyDeviceToHost);
  if (st[0]) return fail(st[0], "batch_execute_direct: request %d rejected (%s)", st[1], nvshmemx_strerror(st[0]));
  return 0;
}

unsigned long long nvshmemx_requests_bytes(const nvshmemx_request *reqs, int n) {
  unsigned long long t = 0;
  for (int i = 0; i < n; ++i) {
    const nvshmemx_request &r = reqs[i];
    const unsigned w = r.dtype == NVSHMEMX_DT_DOUBLE ? 8u : 4u;
    switch (r.op) {
      case NVSHMEMX_REQ_PUT:
      case NVSHMEMX_REQ_GET: t += 2ull * r.bytes; break;
      case NVSHMEMX_REQ_G: t += 2ull * w; break;
      case NVSHMEMX_REQ_SIGNAL: t += 4; break;
      case NVSHMEMX_REQ_P: t += w; break;
      default: break;
    }
  }
  return t;
}

// Per-call path on the batch's device-resident requests: one caller unit per
// request through the public device API (nvshmemx_exec_requests' kernel).
int nvshmemx_batch_execute_percall(nvshmemx_batch *b, int mode, int reps, float *out_ms) {
  if (!b || reps < 1 || mode < 0 || mode > NVSHMEMX_MODE_BULK)
    return fail(NVSHMEMX_ERR_INVALID, "batch_execute_percall: bad arguments");
  int rc;
  cudaEventRecord(b->ev_start, b->stream);
  for (int i = 0; i < reps; ++i)
    if ((rc = launch_exec_requests(mode, b->d_reqs, b->n, b->stream))) return rc;
  cudaEventRecord(b->ev_stop, b->stream);
  if ((rc = check_cuda(cudaStreamSynchronize(b->stream), "batch_execute_percall"))) return rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, b->ev_start, b->ev_stop);
  if (out_ms) *out_ms = ms;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free batch execution (nvshmemx_batch_execute_noalloc).
//
// A batch normally gets its scratch -- the 32-byte control block and the
// table of 32-byte work items the plan kernel fills -- from cudaMalloc in
// nvshmemx_batch_create.  Some callers cannot do that: a serving loop that
// must not take the device-wide synchronisation and unbounded latency of
// cudaMalloc between requests, a process whose device memory belongs to
// another allocator (a framework's caching pool, or a budget fixed at start-up
// that leaves nothing to allocate later), or a foreign-language caller that
// has no way to release device memory it would have to own.  For them the
// scratch below is a file-scope device array that every GPU loading this
// library holds until the process exits.
//
// Host code must not pass g_noalloc_scratch itself to a kernel: on the host
// that name is only a stand-in, not a device address.  The device address is
// looked up once per device with cudaGetSymbolAddress, with that device
// current, on the first call made on it.
namespace nvshm {

static const unsigned long long kNoallocMaxItems = NVSHMEMX_NOALLOC_MAX_CHUNKS;
static const size_t kNoallocCtlBytes = 256;  // BatchCtl, padded to keep the table aligned

static __device__ __align__(256) unsigned char
    g_noalloc_scratch[kNoallocCtlBytes + NVSHMEMX_NOALLOC_MAX_CHUNKS * sizeof(WorkItem)];

static std::mutex g_noalloc_mu;
static void *g_noalloc_addr[128];  // device address of g_noalloc_scratch per device ordinal

static int noalloc_scratch(void **out) {
  int dev = 0;
  int rc;
  if ((rc = check_cuda(cudaGetDevice(&dev), "cudaGetDevice"))) return rc;
  if (dev < 0 || dev >= 128) return fail(NVSHMEMX_ERR_UNSUPPORTED, "batch_execute_noalloc: device ordinal %d", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void *p = nullptr;
    if ((rc = check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(noalloc scratch)")))
      return rc;
    g_noalloc_addr[dev] = p;
  }
  *out = g_noalloc_addr[dev];
  return 0;
}

}  // namespace nvshm

extern "C" int nvshmemx_batch_execute_noalloc(const nvshmemx_request *d_reqs, int n, const nvshmemx_batch_config *cfg,
                                              void *stream) {
  if (!is_started()) return fail(NVSHMEMX_ERR_STATE, "batch_execute_noalloc before nvstart_pes");
  if (n < 0 || (n > 0 && !d_reqs)) return fail(NVSHMEMX_ERR_INVALID, "batch_execute_noalloc: bad request array");
  if ((unsigned long long)n > kNoallocMaxItems)
    return fail(NVSHMEMX_ERR_NOMEM,
                "batch_execute_noalloc: %d requests exceed the fixed scratch of %llu work items; use "
                "nvshmemx_batch_create for larger batches",
                n, kNoallocMaxItems);
  nvshmemx_batch_config k;
  if (cfg) {
    if (check_batch_config(*cfg)) return fail(NVSHMEMX_ERR_INVALID, "batch_execute_noalloc: invalid configuration");
    k = *cfg;
  } else {
    nvshmemx_batch_default_config(&k);
  }
  // Streaming mode keeps a launch generation and per-item tags that must
  // outlive a call; the shared scratch cannot hold them for every caller.
  if (k.stream != 0)
    return fail(NVSHMEMX_ERR_INVALID, "batch_execute_noalloc: stream mode is not available here (set stream = 0)");
  ExecFn fn = pick_exec(k.vec_bytes, k.unroll);
  TmaFn tfn = k.tma_stages ? pick_tma(k.tma_stages) : nullptr;
  if (!fn || (k.tma_stages && !tfn))
    return fail(NVSHMEMX_ERR_INVALID, "batch_execute_noalloc: no kernel for this configuration");
  void *scratch = nullptr;
  int rc;
  if ((rc = noalloc_scratch(&scratch))) return rc;
  BatchCtl *ctl = reinterpret_cast<BatchCtl *>(scratch);
  WorkItem *items = reinterpret_cast<WorkItem *>(static_cast<char *>(scratch) + kNoallocCtlBytes);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const Runtime &r = rt();
  (void)cudaGetLastError();
  // The array keeps the previous call's contents: the control block (chunk
  // count, cursor, status) must start at zero; the work-item table is fully
  // rewritten by the plan kernel before the exec kernel reads it.
  if ((rc = check_cuda(cudaMemsetAsync(ctl, 0, sizeof(BatchCtl), s), "cudaMemsetAsync(noalloc control)"))) return rc;
  if (n > 0)
    batch_plan_kernel<false><<<(n + kPlanThreads - 1) / kPlanThreads, kPlanThreads, 0, s>>>(r.cfg, d_reqs, n, (unsigned)k.chunk_bytes, items,
                                                             kNoallocMaxItems, ctl, ctl, nullptr, 0, nullptr);
  // The exec kernel the configuration names: TMA rings (their stages are
  // shared memory, not scratch) or the register copy.
  int per_sm = 0;
  const size_t smem = tfn ? tma_smem_bytes(k) : 0;
  if (tfn) {
    cudaFuncSetAttribute((const void *)tfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // the rings are all the shared memory a CTA uses: ask for the largest
    // shared-memory carveout, so the CTAs the occupancy query counts on fit
    cudaFuncSetAttribute((const void *)tfn, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)tfn, k.threads, smem);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn, k.threads, 0);
  }
  if (per_sm < 1) per_sm = 1;
  const int ctas = k.ctas_per_sm > 0 && k.ctas_per_sm < per_sm ? k.ctas_per_sm : per_sm;
  if (tfn)
    tfn<<<r.sm_count * ctas, k.threads, smem, s>>>(items, ctl, ctl, kNoallocMaxItems, k.grab,
                                                    (unsigned)k.tma_stage_bytes, (unsigned)k.tma_min_bytes,
                                                    (long long)r.cfg.wait_timeout_ns);
  else
    fn<<<r.sm_count * ctas, k.threads, 0, s>>>(items, ctl, ctl, kNoallocMaxItems, k.grab);
  if ((rc = check_cuda(cudaGetLastError(), "batch_execute_noalloc launch"))) return rc;
  int st[2] = {0, 0};
  if ((rc = check_cuda(cudaMemcpyAsync(st, &ctl->status, sizeof st, cudaMemcpyDeviceToHost, s),
                       "cudaMemcpyAsync(noalloc status)")))
    return rc;
  if ((rc = check_cuda(cudaStreamSynchronize(s), "batch_execute_noalloc"))) return rc;
  if (st[0] == NVSHMEMX_ERR_NOMEM)
    return fail(NVSHMEMX_ERR_NOMEM,
                "batch_execute_noalloc: the batch needs more than %llu chunks of %d bytes; nothing was executed",
                kNoallocMaxItems, k.chunk_bytes);
  if (st[0])
    return fail(st[0], "batch_execute_noalloc: request %d rejected (%s); nothing was executed", st[1],
                nvshmemx_strerror(st[0]));
  return 0;
}
