// runtime.cu -- host runtime of the virtual-PE library: arena set-up,
// symmetric allocation, address queries, host and offload barriers, the
// collective launcher, SPMD host threads, status and the trace ring.
//
// The prototype's equivalents live in nvshmem.cu (nvstart_pes :472-773,
// nvshmalloc :775-802, nvshmcleanup :805-819, nvstop_pes :821-856,
// nvshmem_barrier_all :858-867, nvshmem_barrier_all_offload :869-878,
// nvshmem_ptr :880-883) and nvshmem_kernels.cu:56-102.  There, every PE is a
// process that maps its peers' heaps over CUDA IPC after an MPI exchange.
// Here every PE is a slice of one arena on one GPU, so the exchange and the
// IPC mappings disappear: set-up is one reservation of address space, one
// physical allocation per slice and one upload of the configuration.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "procs.h"

#include <chrono>
#include <condition_variable>
#include <string>
#include <thread>

#include "nvshmem.h"
#include "nvshmemx.h"
#include "runtime.h"

namespace nvshm {

thread_local int t_pe = 0;
thread_local bool t_spmd = false;

Runtime &rt() {
  static Runtime r;
  return r;
}
const Cfg &cfg() { return rt().cfg; }
bool is_started() { return rt().started; }

static bool env_error_mode_read = false;

static void read_env_error_mode() {
  if (env_error_mode_read) return;
  env_error_mode_read = true;
  const char *m = getenv("NVSHMEM_ERROR_MODE");
  if (m && strcmp(m, "return") == 0) rt().error_mode = NVSHMEMX_ERRORS_RETURN;
}

static char g_last_msg[512];

int fail(int code, const char *fmt, ...) {
  Runtime &r = rt();
  read_env_error_mode();
  char msg[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(msg, sizeof msg, fmt, ap);
  va_end(ap);
  memcpy(g_last_msg, msg, sizeof msg);
  if (r.host_err == 0) r.host_err = code;
  if (r.error_mode == NVSHMEMX_ERRORS_EXIT) {
    fprintf(stderr, "[nvshmem %d] %s\n", t_pe, msg);
    exit(-1);
  }
  if (getenv("NVSHMEM_DEBUG")) fprintf(stderr, "[nvshmem %d] %s\n", t_pe, msg);
  return code;
}

int check_cuda(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return NVSHMEMX_SUCCESS;
  return fail(NVSHMEMX_ERR_CUDA, "%s failed: %s", what, cudaGetErrorString(e));
}

// Driver entry points for the virtual-memory calls, resolved through the
// runtime (cudaGetDriverEntryPoint) so the shared library carries no link-time
// dependency on libcuda and loads on machines without a GPU driver.
struct DriverApi {
  PFN_cuGetErrorString get_error_string = nullptr;
  PFN_cuMemGetAllocationGranularity granularity = nullptr;
  PFN_cuMemAddressReserve reserve = nullptr;
  PFN_cuMemAddressFree address_free = nullptr;
  PFN_cuMemCreate create = nullptr;
  PFN_cuMemRelease release = nullptr;
  PFN_cuMemMap map = nullptr;
  PFN_cuMemUnmap unmap = nullptr;
  PFN_cuMemSetAccess set_access = nullptr;
  // process-per-PE mode only
  PFN_cuMemExportToShareableHandle export_handle = nullptr;
  PFN_cuMemImportFromShareableHandle import_handle = nullptr;
  bool loaded = false;
};
static DriverApi g_drv;

static bool get_entry(const char *name, void **fn) {
  cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
  return cudaGetDriverEntryPoint(name, fn, cudaEnableDefault, &q) == cudaSuccess &&
         q == cudaDriverEntryPointSuccess && *fn != nullptr;
}

static int load_driver() {
  if (g_drv.loaded) return 0;
  bool ok = get_entry("cuGetErrorString", (void **)&g_drv.get_error_string) &&
            get_entry("cuMemGetAllocationGranularity", (void **)&g_drv.granularity) &&
            get_entry("cuMemAddressReserve", (void **)&g_drv.reserve) &&
            get_entry("cuMemAddressFree", (void **)&g_drv.address_free) &&
            get_entry("cuMemCreate", (void **)&g_drv.create) &&
            get_entry("cuMemRelease", (void **)&g_drv.release) &&
            get_entry("cuMemMap", (void **)&g_drv.map) &&
            get_entry("cuMemUnmap", (void **)&g_drv.unmap) &&
            get_entry("cuMemSetAccess", (void **)&g_drv.set_access);
  if (!ok) return fail(NVSHMEMX_ERR_CUDA, "cannot resolve the CUDA driver's virtual-memory entry points");
  get_entry("cuMemExportToShareableHandle", (void **)&g_drv.export_handle);
  get_entry("cuMemImportFromShareableHandle", (void **)&g_drv.import_handle);
  g_drv.loaded = true;
  return 0;
}

static int check_cu(CUresult e, const char *what) {
  if (e == CUDA_SUCCESS) return NVSHMEMX_SUCCESS;
  const char *s = nullptr;
  if (g_drv.get_error_string) g_drv.get_error_string(e, &s);
  return fail(NVSHMEMX_ERR_CUDA, "%s failed: %s", what, s ? s : "?");
}

int publish_cfg() { return check_cuda(upload_cfg(rt().cfg), "cudaMemcpyToSymbol(cfg)"); }

// ------------------------------------------------------------ offload barrier
// When every PE lives in this process, all of their kernels are enqueued on
// one device, and a kernel on the legacy default stream starts only after
// every earlier kernel of the default stream and of every blocking stream has
// finished, and makes their writes visible to every later one.  That is the
// whole of what the prototype's offload barrier provides (its kernel
// gathers the PEs' flags through PE 0, nvshmem_kernels.cu:56-102, because its
// PEs are processes whose kernels run independently).  So here the barrier is
// an action on the legacy default stream: with tracing on, one small kernel
// launched normally, one CTA whose lanes write a BARRIER trace record for
// each PE; with tracing off, a wait on an event that has already completed
// (cudaStreamWaitEvent is one of the actions that the legacy stream orders
// against every blocking stream), which launches nothing.  (A cooperative
// launch of one CTA per PE meeting on a ticket counter cost 3.6 to 4.6 us per
// call, most of it the cooperative launch; the one-CTA kernel 2.6-4.1 us.)
__global__ void offload_barrier_kernel(Cfg c, int npes) {
  if (!c.trace) return;
  const unsigned long long t = gtimer();
  for (int pe = threadIdx.x; pe < npes; pe += blockDim.x) {
    unsigned long long idx = atomicAdd(&c.trace_head[pe], 1ull);
    nvshmemx_trace_record *rec = c.trace + (size_t)pe * c.trace_cap + (size_t)(idx & (c.trace_cap - 1));
    rec->t_ns = (long long)t;
    rec->spin_ns = 0;
    rec->local_addr = 0;
    rec->remote_addr = 0;
    rec->bytes = 0;
    rec->op = NVSHMEMX_TRACE_BARRIER;
    rec->pe = (unsigned short)pe;
    rec->peer = (unsigned short)pe;
    rec->tid = 0;
    rec->block = 0;
  }
}

// -------------------------------------------------------------- host barrier
// Meeting point of the SPMD PE threads (stands in for MPI_Barrier).  A PE
// thread that has returned, or a wait longer than the host deadline, fails the
// barrier instead of hanging the others.
struct HostBarrier {
  std::mutex m;
  std::condition_variable cv;
  int n = 0, count = 0, departed = 0;
  unsigned long long gen = 0;
  int wait(double timeout_s) {
    std::unique_lock<std::mutex> lk(m);
    if (departed > 0) return NVSHMEMX_ERR_STATE;
    unsigned long long g = gen;
    if (++count == n) {
      count = 0;
      ++gen;
      cv.notify_all();
      return 0;
    }
    bool ok = cv.wait_for(lk, std::chrono::duration<double>(timeout_s),
                          [&] { return gen != g || departed > 0; });
    if (gen != g) return 0;
    --count;
    return ok ? NVSHMEMX_ERR_STATE : NVSHMEMX_ERR_TIMEOUT;
  }
  void depart() {
    std::lock_guard<std::mutex> lk(m);
    ++departed;
    cv.notify_all();
  }
};
static HostBarrier g_hbar;
static std::vector<cudaEvent_t> g_spmd_events;

static double host_barrier_timeout_s() {
  const char *v = getenv("NVSHMEM_HOST_BARRIER_TIMEOUT_S");
  return v ? atof(v) : 120.0;
}

// ---------------------------------------------------------------- set-up
static size_t next_pow2(size_t x) {
  size_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Completed event that an untraced offload barrier waits on (see
// nvshmem_barrier_all_offload); created at its first use after a start.
static cudaEvent_t g_offload_ev = nullptr;

static void release_all() {
  Runtime &r = rt();
  if (g_offload_ev) cudaEventDestroy(g_offload_ev);
  g_offload_ev = nullptr;
  if (r.d_trace) cudaFree(r.d_trace);
  if (r.d_trace_head) cudaFree(r.d_trace_head);
  r.d_trace = nullptr;
  r.d_trace_head = nullptr;
  r.trace_cap = 0;
  if (r.ctrl) cudaFree(r.ctrl);
  r.ctrl = nullptr;
  if (r.arena) {
    for (int p = 0; p < (int)r.handles.size(); ++p) {
      if (!r.handles[p]) continue;
      g_drv.unmap((CUdeviceptr)(r.arena + (size_t)p * r.stride), r.slice_mapped);
      g_drv.release(r.handles[p]);
    }
    g_drv.address_free((CUdeviceptr)r.arena, (size_t)r.npes * r.stride);
  }
  r.handles.clear();
  r.arena = nullptr;
  r.started = false;
}

// Process-per-PE mode: create this process's slice as an exportable
// allocation, exchange descriptors with the other PE processes, and map every
// slice at its place in the arena.  The own slice is zeroed, then all PEs
// meet, so no PE writes into a slice before its owner has cleared it.
static int map_process_slices(int pe, int npes, const char *dir, const CUmemAllocationProp &prop,
                              const CUmemAccessDesc &acc) {
  Runtime &r = rt();
  int rc;
  if ((rc = proc_open(pe, npes, dir))) return rc;
  const double timeout = host_barrier_timeout_s();
  CUdeviceptr base = (CUdeviceptr)r.arena;
  if ((rc = check_cu(g_drv.create(&r.handles[pe], r.slice_mapped, &prop, 0), "cuMemCreate"))) return rc;
  int my_fd = -1;
  if ((rc = check_cu(g_drv.export_handle(&my_fd, r.handles[pe], CU_MEM_HANDLE_TYPE_POSIX_FILE_DESCRIPTOR, 0),
                     "cuMemExportToShareableHandle")))
    return rc;
  std::vector<int> fds;
  rc = proc_exchange_fds(my_fd, fds, timeout);
  for (int q = 0; q < npes && !rc; ++q) {
    if (q != pe &&
        (rc = check_cu(g_drv.import_handle(&r.handles[q], (void *)(uintptr_t)fds[q],
                                           CU_MEM_HANDLE_TYPE_POSIX_FILE_DESCRIPTOR),
                       "cuMemImportFromShareableHandle")))
      break;
    CUdeviceptr at = base + (size_t)q * r.stride;
    if ((rc = check_cu(g_drv.map(at, r.slice_mapped, 0, r.handles[q], 0), "cuMemMap")) ||
        (rc = check_cu(g_drv.set_access(at, r.slice_mapped, &acc, 1), "cuMemSetAccess"))) {
      g_drv.release(r.handles[q]);
      r.handles[q] = 0;
      break;
    }
  }
  for (int fd : fds)
    if (fd >= 0) close(fd);
  if (rc) return rc;
  if ((rc = check_cuda(cudaMemset(r.arena + (size_t)pe * r.stride, 0, r.slice_mapped), "cudaMemset(slice)")) ||
      (rc = check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize")))
    return rc;
  return proc_barrier(timeout);
}

// proc_pe < 0: every PE in this process (one arena, one collective launch);
// proc_pe >= 0: this process is PE proc_pe of npes processes meeting in the
// rendezvous directory `dir` (procs.cu).
static int init_impl(int npes, size_t heap, int proc_pe = -1, const char *dir = nullptr) {
  Runtime &r = rt();
  std::lock_guard<std::recursive_mutex> lk(r.mu);
  read_env_error_mode();
  if (r.started) return fail(NVSHMEMX_ERR_STATE, "nvstart_pes: already started");
  if (npes < 1 || npes > NVSHMEMX_MAX_NPES)
    return fail(NVSHMEMX_ERR_INVALID, "nvstart_pes: npes %d outside [1, %d]", npes, NVSHMEMX_MAX_NPES);
  if (heap == 0) return fail(NVSHMEMX_ERR_INVALID, "nvstart_pes: heap size 0");
  const char *to = getenv("NVSHMEM_WAIT_TIMEOUT_NS");
  if (to) r.wait_timeout_ns = atoll(to);

  int rc;
  // one process per PE may put its PE on a device of its own (the launcher's
  // --devices); the slices of PEs on other devices are then mapped over the
  // GPUs' peer links with the same exchanged handles
  const char *dv = getenv("NVSHMEM_DEVICE");
  if (proc_pe >= 0 && dv && (rc = check_cuda(cudaSetDevice(atoi(dv)), "cudaSetDevice(NVSHMEM_DEVICE)"))) return rc;
  if ((rc = check_cuda(cudaFree(0), "cudaFree(0)"))) return rc;  // create the context
  if ((rc = check_cuda(cudaGetDevice(&r.device), "cudaGetDevice"))) return rc;
  if ((rc = load_driver())) return rc;
  if ((rc = check_cuda(cudaDeviceGetAttribute(&r.sm_count, cudaDevAttrMultiProcessorCount, r.device),
                       "cudaDeviceGetAttribute")))
    return rc;

  const bool procs = proc_pe >= 0;
  if (procs && (!g_drv.export_handle || !g_drv.import_handle))
    return fail(NVSHMEMX_ERR_UNSUPPORTED, "process mode: the driver cannot share VMM allocations");
  CUmemAllocationProp prop;
  memset(&prop, 0, sizeof prop);
  prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
  prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  prop.location.id = r.device;
  if (procs) prop.requestedHandleTypes = CU_MEM_HANDLE_TYPE_POSIX_FILE_DESCRIPTOR;
  size_t gran = 0;
  if ((rc = check_cu(g_drv.granularity(&gran, &prop, CU_MEM_ALLOC_GRANULARITY_RECOMMENDED),
                     "cuMemGetAllocationGranularity")))
    return rc;
  r.npes = npes;
  r.heap_bytes = heap;
  r.slice_mapped = (heap + gran - 1) / gran * gran;
  r.stride = next_pow2(r.slice_mapped);
  r.log2_stride = 0;
  while ((size_t(1) << r.log2_stride) < r.stride) ++r.log2_stride;

  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  if ((size_t)(procs ? 1 : npes) * r.slice_mapped > free_b)
    return fail(NVSHMEMX_ERR_NOMEM, "nvstart_pes: %d PEs x %zu bytes exceed free device memory (%zu)", npes,
                r.slice_mapped, free_b);

  CUdeviceptr base = 0;
  if ((rc = check_cu(g_drv.reserve(&base, (size_t)npes * r.stride, r.stride, 0, 0),
                     "cuMemAddressReserve")))
    return rc;
  r.arena = (char *)base;
  r.handles.assign(npes, 0);
  CUmemAccessDesc acc;
  memset(&acc, 0, sizeof acc);
  acc.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  acc.location.id = r.device;
  acc.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
  if (!procs) {
    for (int p = 0; p < npes; ++p) {
      CUdeviceptr at = base + (size_t)p * r.stride;
      if ((rc = check_cu(g_drv.create(&r.handles[p], r.slice_mapped, &prop, 0), "cuMemCreate")) ||
          (rc = check_cu(g_drv.map(at, r.slice_mapped, 0, r.handles[p], 0), "cuMemMap")) ||
          (rc = check_cu(g_drv.set_access(at, r.slice_mapped, &acc, 1), "cuMemSetAccess"))) {
        r.handles.resize(p + 1);
        if (r.handles[p] == 0) r.handles.resize(p);
        release_all();
        return rc;
      }
    }
    // The prototype leaves its heap uninitialised (cuMemAlloc, nvshmem.cu:504);
    // zeroing it makes every run start from the same heap image.
    for (int p = 0; p < npes; ++p) {
      if ((rc = check_cuda(cudaMemset(r.arena + (size_t)p * r.stride, 0, r.slice_mapped), "cudaMemset(arena)"))) {
        release_all();
        return rc;
      }
    }
  } else if ((rc = map_process_slices(proc_pe, npes, dir, prop, acc))) {
    release_all();
    proc_close();
    return rc;
  }

  // control block: status (64 B), collective counter and per-PE counters each
  // on its own 128-byte line.
  const size_t line = 128;
  size_t ctrl_bytes = line + line + (size_t)npes * line;
  if ((rc = check_cuda(cudaMalloc(&r.ctrl, ctrl_bytes), "cudaMalloc(ctrl)"))) {
    release_all();
    return rc;
  }
  cudaMemset(r.ctrl, 0, ctrl_bytes);
  r.d_status = (int *)r.ctrl;
  r.d_coll_bar = (unsigned long long *)(r.ctrl + line);
  r.d_pe_bar = (unsigned long long *)(r.ctrl + 2 * line);
  r.bar_reset_bytes = line + (size_t)npes * line;
  r.tail.assign(npes, 0);

  Cfg &c = r.cfg;
  memset(&c, 0, sizeof c);
  c.arena = r.arena;
  c.arena_bytes = (unsigned long long)npes * r.stride;
  c.mask = r.stride - 1;
  c.slice_bytes = r.heap_bytes;  // accesses stay inside NVSHMEM_HEAP_SIZE
  c.log2_stride = r.log2_stride;
  c.npes = npes;
  c.status = r.d_status;
  c.coll_bar = r.d_coll_bar;
  // per-PE counters are 128 bytes apart: index p*16 in units of u64
  c.pe_bar = r.d_pe_bar;
  c.wait_timeout_ns = r.wait_timeout_ns;
  c.proc_pe = proc_pe;
  if (procs) t_pe = proc_pe;
  r.started = true;
  if ((rc = publish_cfg())) {
    release_all();
    return rc;
  }
  if ((rc = check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize"))) {
    release_all();
    return rc;
  }
  // NVSHMEM_ENABLE_TRACING (nvshmem.cu:611-615) turns tracing on at start;
  // NVSHMEM_LOG_BUFFER_SIZE keeps its unit, bytes (nvshmem.cu:145,618-622),
  // here of trace ring per PE (48-byte records, rounded up to a power of two;
  // default 2 MiB).  The processed trace files are written at stop.
  const char *tv = getenv("NVSHMEM_ENABLE_TRACING");
  if (tv && atol(tv) != 0) {
    long long bytes = 2ll << 20;
    const char *sv = getenv("NVSHMEM_LOG_BUFFER_SIZE");
    if (sv && atoll(sv) > 0) bytes = atoll(sv);
    long long recs = bytes / (long long)sizeof(nvshmemx_trace_record);
    if (recs < 16) recs = 16;
    if (recs > (1ll << 24)) recs = 1ll << 24;
    if ((rc = nvshmemx_trace_enable((unsigned)recs))) {
      release_all();
      return rc;
    }
    r.trace_from_env = true;
  }
  return NVSHMEMX_SUCCESS;
}

int launch_collective(const void *func, dim3 grid, dim3 block, void **args, size_t smem, cudaStream_t stream) {
  Runtime &r = rt();
  if (!r.started) return fail(NVSHMEMX_ERR_STATE, "collective launch before nvstart_pes");
  if (grid.z != 1 || grid.x == 0 || grid.y == 0)
    return fail(NVSHMEMX_ERR_INVALID, "collective launch: grid.z must be 1 (it carries the PE)");
  int threads = (int)(block.x * block.y * block.z);
  int rc;
  if (smem > 48 * 1024) {
    if ((rc = check_cuda(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                         "cudaFuncSetAttribute")))
      return rc;
  }
  int per_sm = 0;
  if ((rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, threads, smem),
                       "cudaOccupancyMaxActiveBlocksPerMultiprocessor")))
    return rc;
  // process mode: the launch carries this process's PE only
  const int pes = proc_mode() ? 1 : r.npes;
  long long total = (long long)grid.x * grid.y * pes;
  if (total > (long long)per_sm * r.sm_count)
    return fail(NVSHMEMX_ERR_COOP, "collective launch: %lld CTAs cannot be co-resident (%d per SM x %d SMs)",
                total, per_sm, r.sm_count);
  if ((rc = check_cuda(cudaMemsetAsync(r.d_coll_bar, 0, r.bar_reset_bytes, stream), "cudaMemsetAsync(barrier)")))
    return rc;
  dim3 g(grid.x, grid.y, (unsigned)pes);
  return check_cuda(cudaLaunchCooperativeKernel(func, g, block, args, smem, stream), "cudaLaunchCooperativeKernel");
}

int max_ctas_per_pe(const void *func, int block_threads, size_t smem) {
  Runtime &r = rt();
  if (!r.started) return 0;
  if (smem > 48 * 1024) cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, block_threads, smem) != cudaSuccess) return 0;
  return per_sm * r.sm_count / r.npes;
}

}  // namespace nvshm

using namespace nvshm;

extern "C" {

// ------------------------------------------------------------------ lifetime
int nvshmemx_init_attr(int npes, size_t heap_bytes_per_pe) { return init_impl(npes, heap_bytes_per_pe); }

void nvstart_pes(void) {
  read_env_error_mode();
  int npes = 2;
  size_t heap = (size_t)1 << 30;  // HEAP_SIZE, nvshmem.cu:107
  const char *v = getenv("NVSHMEM_NPES");
  if (v) npes = atoi(v);
  // The prototype read NVSHMEM_HEAP_SIZE only after allocating its heap
  // (nvshmem.cu:504 vs :532), so the variable moved the bounds check but not
  // the allocation; here it sizes the allocation too.
  v = getenv("NVSHMEM_HEAP_SIZE");
  if (v) heap = (size_t)atoll(v);
  // One process per PE (the launcher sets these), as under the prototype's
  // mpirun; otherwise every PE in this process.
  const char *pp = getenv("NVSHMEM_PROCESS_PE");
  if (pp)
    init_impl(npes, heap, atoi(pp), getenv("NVSHMEM_RENDEZVOUS"));
  else
    init_impl(npes, heap);
}

int nvshmemx_init_process(int pe, int npes, size_t heap_bytes_per_pe, const char *rendezvous_dir) {
  if (pe < 0) return fail(NVSHMEMX_ERR_INVALID, "nvshmemx_init_process: PE %d", pe);
  return init_impl(npes, heap_bytes_per_pe, pe, rendezvous_dir);
}

// The application's launcher (MPI or any other) provides rank, size and an
// allgather: rank 0's rendezvous directory name goes to every rank, every
// rank starts process mode in it, a second allgather tells every rank that
// all started, and rank 0 then empties and removes the directory (the
// sockets and the barrier file are only opened during start-up; the barrier
// stays mapped).
int nvshmemx_init_bootstrap(const nvshmemx_bootstrap *bs, size_t heap_bytes_per_pe) {
  constexpr size_t kName = 256;
  if (!bs || !bs->allgather || bs->size < 1 || bs->rank < 0 || bs->rank >= bs->size)
    return fail(NVSHMEMX_ERR_INVALID, "nvshmemx_init_bootstrap: bad bootstrap description");
  char mine[kName];
  memset(mine, 0, sizeof mine);
  if (bs->rank == 0) {
    const char *t = getenv("TMPDIR");
    std::string tmpl = std::string(t && *t ? t : "/tmp") + "/nvshm-XXXXXX";
    std::vector<char> name(tmpl.begin(), tmpl.end());
    name.push_back('\0');
    if (name.size() < kName && mkdtemp(name.data())) memcpy(mine, name.data(), name.size());
    // on failure the empty name tells every rank to stop
  }
  std::vector<char> all((size_t)bs->size * kName);
  if (bs->allgather(mine, all.data(), kName, bs->ctx) != 0) {
    if (mine[0]) rmdir(mine);  // rank 0's directory, still empty
    return fail(NVSHMEMX_ERR_STATE, "nvshmemx_init_bootstrap: the allgather callback failed");
  }
  const std::string dir(all.data(), strnlen(all.data(), kName - 1));
  if (dir.empty()) return fail(NVSHMEMX_ERR_STATE, "nvshmemx_init_bootstrap: rank 0 could not make a rendezvous directory");
  int rc = nvshmemx_init_process(bs->rank, bs->size, heap_bytes_per_pe, dir.c_str());
  const int started = rc == 0 ? 1 : 0;
  std::vector<int> all_started((size_t)bs->size, 0);
  const int grc = bs->allgather(&started, all_started.data(), sizeof(int), bs->ctx);
  if (bs->rank == 0) {
    for (int p = 0; p < bs->size; ++p) unlink((dir + "/pe" + std::to_string(p) + ".sock").c_str());
    unlink((dir + "/barrier").c_str());
    rmdir(dir.c_str());
  }
  bool everyone = grc == 0;
  for (int s : all_started) everyone = everyone && s == 1;
  if (!everyone) {
    if (rc == 0) {
      nvshmemx_finalize();
      rc = fail(NVSHMEMX_ERR_STATE, "nvshmemx_init_bootstrap: another rank did not start");
    }
    return rc;
  }
  return 0;
}

int nvshmemx_finalize(void) {
  Runtime &r = rt();
  std::lock_guard<std::recursive_mutex> lk(r.mu);
  if (!r.started) return fail(NVSHMEMX_ERR_STATE, "nvstop_pes: not started");
  int rc = check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
  // process mode: nobody unmaps a slice another PE may still write
  if (proc_mode() && rc == 0) rc = proc_barrier(host_barrier_timeout_s());
  if (r.trace_from_env && r.d_trace && rc == 0) {
    // nvshmem_processed_tracefile_<pid>_<pe>, as the prototype's stop wrote
    // (nvshmem.cu:377)
    rc = nvshmemx_trace_write_csv(nullptr);
  }
  r.trace_from_env = false;
  release_all();
  if (proc_mode()) proc_close();
  return rc;
}

void nvstop_pes(void) {
  if (t_spmd) {
    // every PE thread calls it; the launching thread releases after the join
    nvshmem_barrier_all();
    return;
  }
  nvshmemx_finalize();
}

int nvshmemx_is_started(void) { return rt().started ? 1 : 0; }

int nvshmem_my_pe(void) { return proc_mode() ? proc_pe() : t_pe; }
int nvshmem_n_pes(void) { return rt().npes; }

// ---------------------------------------------------------------- allocation
void *nvshmalloc(size_t size) {
  Runtime &r = rt();
  std::lock_guard<std::recursive_mutex> lk(r.mu);
  if (!r.started) {
    fail(NVSHMEMX_ERR_STATE, "nvshmalloc before nvstart_pes");
    return nullptr;
  }
  if (t_spmd) {
    size_t off = r.tail[t_pe];
    if (size > r.heap_bytes - off) {  // off <= heap_bytes; no sum that could wrap
      fail(NVSHMEMX_ERR_NOMEM,
           "Not enough memory on the heap (set to %zu, can be increased by setting NVSHMEM_HEAP_SIZE)",
           r.heap_bytes);
      return nullptr;
    }
    r.tail[t_pe] = off + size;
    return r.arena + (size_t)t_pe * r.stride + off;
  }
  // Called outside SPMD threads the allocation is collective by construction:
  // every slice gets the same offset.
  size_t off = r.tail[0];
  for (int p = 1; p < r.npes; ++p) {
    if (r.tail[p] != off) {
      fail(NVSHMEMX_ERR_INVALID, "nvshmalloc: heap tails differ between PEs (asymmetric allocations)");
      return nullptr;
    }
  }
  if (size > r.heap_bytes - off) {
    fail(NVSHMEMX_ERR_NOMEM,
         "Not enough memory on the heap (set to %zu, can be increased by setting NVSHMEM_HEAP_SIZE)",
         r.heap_bytes);
    return nullptr;
  }
  for (int p = 0; p < r.npes; ++p) r.tail[p] = off + size;
  return r.arena + (size_t)nvshmem_my_pe() * r.stride + off;
}

void nvshmcleanup(void) {
  Runtime &r = rt();
  std::lock_guard<std::recursive_mutex> lk(r.mu);
  if (!r.started) return;
  if (t_spmd)
    r.tail[t_pe] = 0;
  else
    for (auto &t : r.tail) t = 0;
}

void *nvshmem_ptr(void *local, int pe) {
  Runtime &r = rt();
  if (!r.started) return nullptr;
  unsigned long long d = (unsigned long long)((char *)local - r.arena);
  if (d >= (unsigned long long)r.npes * r.stride || pe < 0 || pe >= r.npes) return nullptr;
  return r.arena + (size_t)pe * r.stride + (d & (r.stride - 1));
}

// ------------------------------------------------------------------ barriers
void nvshmem_barrier_all(void) {
  Runtime &r = rt();
  if (!r.started) {
    fail(NVSHMEMX_ERR_STATE, "nvshmem_barrier_all before nvstart_pes");
    return;
  }
  if (check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize")) return;
  if (proc_mode()) {
    proc_barrier(host_barrier_timeout_s());
    return;
  }
  if (t_spmd) {
    int rc = g_hbar.wait(host_barrier_timeout_s());
    if (rc) fail(rc, "nvshmem_barrier_all: a PE thread left or the host barrier timed out");
  }
}

void nvshmem_barrier_all_offload(void) {
  Runtime &r = rt();
  if (!r.started) {
    fail(NVSHMEMX_ERR_STATE, "nvshmem_barrier_all_offload before nvstart_pes");
    return;
  }
  if (proc_mode()) {
    // kernels of different processes cannot wait for each other on one GPU:
    // the PE processes meet on the host
    nvshmem_barrier_all();
    return;
  }
  if (t_spmd) {
    // Each PE thread's stream waits for every PE's earlier work: record, meet
    // on the host (no GPU wait), then wait on all events, then meet again so
    // no event is re-recorded before everyone has enqueued its waits.
    if (check_cuda(cudaEventRecord(g_spmd_events[t_pe], 0), "cudaEventRecord")) return;
    int rc = g_hbar.wait(host_barrier_timeout_s());
    if (rc) {
      fail(rc, "nvshmem_barrier_all_offload: a PE thread left or the host barrier timed out");
      return;
    }
    for (int p = 0; p < r.npes; ++p)
      if (check_cuda(cudaStreamWaitEvent(0, g_spmd_events[p], 0), "cudaStreamWaitEvent")) return;
    rc = g_hbar.wait(host_barrier_timeout_s());
    if (rc) fail(rc, "nvshmem_barrier_all_offload: a PE thread left or the host barrier timed out");
    return;
  }
  // Every PE of this process runs on this GPU, so the legacy default stream
  // already orders each PE's earlier work before its later work; an action on
  // that stream also waits for all blocking streams and makes them wait for
  // it.  Traced, the barrier is a one-CTA kernel that writes each PE's
  // BARRIER record at its GPU time; untraced, it is a wait on a completed
  // event, an action on the legacy stream that needs no kernel.
  if (r.cfg.trace) {
    offload_barrier_kernel<<<1, 32, 0, 0>>>(r.cfg, r.npes);
    check_cuda(cudaGetLastError(), "offload barrier launch");
    return;
  }
  if (!g_offload_ev) {
    if (check_cuda(cudaEventCreateWithFlags(&g_offload_ev, cudaEventDisableTiming), "cudaEventCreate") ||
        check_cuda(cudaEventRecord(g_offload_ev, 0), "cudaEventRecord"))
      return;
  }
  check_cuda(cudaStreamWaitEvent(0, g_offload_ev, 0), "offload barrier");
}

// ---------------------------------------------------------- collective launch
int nvshmemx_collective_launch(const void *func, dim3 grid_per_pe, dim3 block, void **args, size_t smem_bytes,
                               cudaStream_t stream) {
  return launch_collective(func, grid_per_pe, block, args, smem_bytes, stream);
}

int nvshmemx_collective_max_ctas_per_pe(const void *func, int block_threads, size_t smem_bytes) {
  return max_ctas_per_pe(func, block_threads, smem_bytes);
}

// -------------------------------------------------------------------- status
int nvshmemx_status(void) {
  Runtime &r = rt();
  int code = r.host_err;
  long long detail = r.host_detail;
  r.host_err = 0;
  r.host_detail = -1;
  if (r.started) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      if (code == 0) code = NVSHMEMX_ERR_CUDA;
    } else {
      int st[4] = {0, 0, 0, 0};
      if (cudaMemcpy(st, r.d_status, sizeof st, cudaMemcpyDeviceToHost) == cudaSuccess && st[0] != 0) {
        if (code == 0) {
          code = st[0];
          memcpy(&detail, st + 2, sizeof detail);
        }
        cudaMemset(r.d_status, 0, sizeof st);
      }
    }
  }
  r.last_detail = detail;
  return code;
}

long long nvshmemx_status_detail(void) { return rt().last_detail; }

const char *nvshmemx_last_error_string(void) { return nvshm::g_last_msg; }

void nvshmemx_set_error_mode(int mode) {
  env_error_mode_read = true;
  rt().error_mode = mode;
}
int nvshmemx_get_error_mode(void) {
  read_env_error_mode();
  return rt().error_mode;
}

const char *nvshmemx_strerror(int code) {
  switch (code) {
    case NVSHMEMX_SUCCESS: return "success";
    case NVSHMEMX_ERR_INVALID: return "invalid argument";
    case NVSHMEMX_ERR_NOMEM: return "out of symmetric heap or device memory";
    case NVSHMEMX_ERR_CUDA: return "CUDA call failed";
    case NVSHMEMX_ERR_STATE: return "library not started, already started, or a PE left";
    case NVSHMEMX_ERR_TIMEOUT: return "wait or barrier deadline passed";
    case NVSHMEMX_ERR_BOUNDS: return "access outside the symmetric arena (skipped)";
    case NVSHMEMX_ERR_COOP: return "grid too large to be co-resident";
    case NVSHMEMX_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown";
  }
}

// --------------------------------------------------------- arena and queries
void *nvshmemx_arena_base(void) { return rt().arena; }
size_t nvshmemx_slice_stride(void) { return rt().stride; }
size_t nvshmemx_heap_size(void) { return rt().heap_bytes; }
size_t nvshmemx_heap_used(int pe) {
  Runtime &r = rt();
  if (!r.started || pe < 0 || pe >= r.npes) return 0;
  return r.tail[pe];
}
int nvshmemx_sm_count(void) {
  Runtime &r = rt();
  if (r.sm_count) return r.sm_count;
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n;
}
int nvshmemx_device_sync(void) { return check_cuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize"); }

static int heap_range_ok(int pe, size_t off, size_t bytes) {
  Runtime &r = rt();
  if (!r.started) return fail(NVSHMEMX_ERR_STATE, "heap access before nvstart_pes");
  if (pe < 0 || pe >= r.npes || off > r.heap_bytes || bytes > r.heap_bytes - off)
    return fail(NVSHMEMX_ERR_INVALID, "heap access pe %d [%zu, +%zu) outside the slice", pe, off, bytes);
  return 0;
}

int nvshmemx_heap_write(int pe, size_t off, const void *src, size_t bytes) {
  int rc = heap_range_ok(pe, off, bytes);
  if (rc) return rc;
  Runtime &r = rt();
  return check_cuda(cudaMemcpy(r.arena + (size_t)pe * r.stride + off, src, bytes, cudaMemcpyHostToDevice),
                    "cudaMemcpy(H2D)");
}
int nvshmemx_heap_read(int pe, size_t off, void *dst, size_t bytes) {
  int rc = heap_range_ok(pe, off, bytes);
  if (rc) return rc;
  Runtime &r = rt();
  return check_cuda(cudaMemcpy(dst, r.arena + (size_t)pe * r.stride + off, bytes, cudaMemcpyDeviceToHost),
                    "cudaMemcpy(D2H)");
}
int nvshmemx_heap_memset(int pe, size_t off, int value, size_t bytes) {
  int rc = heap_range_ok(pe, off, bytes);
  if (rc) return rc;
  Runtime &r = rt();
  return check_cuda(cudaMemset(r.arena + (size_t)pe * r.stride + off, value, bytes), "cudaMemset");
}

void nvshmemx_set_wait_timeout_ns(long long ns) {
  Runtime &r = rt();
  r.wait_timeout_ns = ns > 0 ? ns : 5000000000LL;
  if (r.started) {
    r.cfg.wait_timeout_ns = r.wait_timeout_ns;
    publish_cfg();
  }
}
long long nvshmemx_get_wait_timeout_ns(void) { return rt().wait_timeout_ns; }

// ------------------------------------------------------------- SPMD threads
int nvshmemx_spmd_run(void (*fn)(void *), void *arg) {
  Runtime &r = rt();
  if (!r.started) return fail(NVSHMEMX_ERR_STATE, "nvshmemx_spmd_run before nvstart_pes");
  if (proc_mode()) return fail(NVSHMEMX_ERR_STATE, "nvshmemx_spmd_run: every PE is a process already");
  if (r.spmd_active) return fail(NVSHMEMX_ERR_STATE, "nvshmemx_spmd_run: already running");
  r.spmd_active = true;
  g_hbar.n = r.npes;
  g_hbar.count = 0;
  g_hbar.departed = 0;
  g_spmd_events.assign(r.npes, nullptr);
  for (int p = 0; p < r.npes; ++p) cudaEventCreateWithFlags(&g_spmd_events[p], cudaEventDisableTiming);
  std::vector<std::thread> th;
  const int dev = r.device;
  for (int p = 0; p < r.npes; ++p) {
    th.emplace_back([=] {
      cudaSetDevice(dev);
      t_pe = p;
      t_spmd = true;
      fn(arg);
      g_hbar.depart();
      t_spmd = false;
      t_pe = 0;
    });
  }
  for (auto &t : th) t.join();
  for (auto e : g_spmd_events) cudaEventDestroy(e);
  g_spmd_events.clear();
  r.spmd_active = false;
  return r.host_err;
}

// ---------------------------------------------------------------- trace ring
int nvshmemx_trace_enable(unsigned int records_per_pe) {
  Runtime &r = rt();
  std::lock_guard<std::recursive_mutex> lk(r.mu);
  if (!r.started) return fail(NVSHMEMX_ERR_STATE, "trace before nvstart_pes");
  unsigned cap = 1;
  while (cap < records_per_pe) cap <<= 1;
  if (cap < 16) cap = 16;
  int rc;
  cudaDeviceSynchronize();
  if (r.d_trace) cudaFree(r.d_trace);
  if (r.d_trace_head) cudaFree(r.d_trace_head);
  r.d_trace = nullptr;
  r.d_trace_head = nullptr;
  if ((rc = check_cuda(cudaMalloc(&r.d_trace, (size_t)r.npes * cap * sizeof(nvshmemx_trace_record)),
                       "cudaMalloc(trace)")))
    return rc;
  if ((rc = check_cuda(cudaMalloc(&r.d_trace_head, (size_t)r.npes * sizeof(unsigned long long)),
                       "cudaMalloc(trace head)")))
    return rc;
  cudaMemset(r.d_trace, 0, (size_t)r.npes * cap * sizeof(nvshmemx_trace_record));
  cudaMemset(r.d_trace_head, 0, (size_t)r.npes * sizeof(unsigned long long));
  r.trace_cap = cap;
  r.cfg.trace = r.d_trace;
  r.cfg.trace_head = r.d_trace_head;
  r.cfg.trace_cap = cap;
  return publish_cfg();
}

int nvshmemx_trace_disable(void) {
  Runtime &r = rt();
  std::lock_guard<std::recursive_mutex> lk(r.mu);
  if (!r.started) return fail(NVSHMEMX_ERR_STATE, "trace before nvstart_pes");
  cudaDeviceSynchronize();
  r.cfg.trace = nullptr;
  r.cfg.trace_head = nullptr;
  r.cfg.trace_cap = 0;
  int rc = publish_cfg();
  if (r.d_trace) cudaFree(r.d_trace);
  if (r.d_trace_head) cudaFree(r.d_trace_head);
  r.d_trace = nullptr;
  r.d_trace_head = nullptr;
  r.trace_cap = 0;
  return rc;
}

int nvshmemx_trace_reset(void) {
  Runtime &r = rt();
  if (!r.d_trace_head) return fail(NVSHMEMX_ERR_STATE, "trace not enabled");
  cudaDeviceSynchronize();
  return check_cuda(cudaMemset(r.d_trace_head, 0, (size_t)r.npes * sizeof(unsigned long long)), "cudaMemset");
}

long long nvshmemx_trace_read(int pe, nvshmemx_trace_record *out, size_t max_records, long long *dropped) {
  Runtime &r = rt();
  if (!r.d_trace || pe < 0 || pe >= r.npes) return -1;
  if (cudaDeviceSynchronize() != cudaSuccess) return -1;
  unsigned long long head = 0;
  if (cudaMemcpy(&head, r.d_trace_head + pe, sizeof head, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  unsigned long long n = head < r.trace_cap ? head : r.trace_cap;
  unsigned long long first = head - n;  // oldest surviving record
  if (dropped) *dropped = (long long)(head - n);
  if (n > max_records) n = max_records;
  std::vector<nvshmemx_trace_record> ring(r.trace_cap);
  if (cudaMemcpy(ring.data(), r.d_trace + (size_t)pe * r.trace_cap, r.trace_cap * sizeof(nvshmemx_trace_record),
                 cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  for (unsigned long long i = 0; i < n; ++i) out[i] = ring[(first + i) & (r.trace_cap - 1)];
  return (long long)n;
}

// CSV layout of the prototype's processed trace files (nvshmem.cu:390 header,
// :411-433 records): size is in elements for typed ops, 1 for p/g/wait.
static const char *trace_op_name(int op) {
  static const char *names[] = {"put_int", "put_float", "put_double", "get_int", "get_float",
                                "get_double", "wait_int", "wait_until_int", "barrier", "quiet",
                                "p", "g", "trace_begin", "trace_end"};
  return (op >= 0 && op < 14) ? names[op] : "unknown";
}

int nvshmemx_trace_write_csv(const char *prefix) {
  Runtime &r = rt();
  if (!r.d_trace) return fail(NVSHMEMX_ERR_STATE, "trace not enabled");
  std::string pre = prefix ? prefix : ("nvshmem_processed_tracefile_" + std::to_string((long)getpid()));
  std::vector<nvshmemx_trace_record> recs(r.trace_cap);
  for (int pe = 0; pe < r.npes; ++pe) {
    // one process per PE: each process records and writes its own PE only
    if (proc_mode() && pe != proc_pe()) continue;
    long long dropped = 0;
    long long n = nvshmemx_trace_read(pe, recs.data(), recs.size(), &dropped);
    if (n < 0) return fail(NVSHMEMX_ERR_CUDA, "trace read failed");
    std::string fn = pre + "_" + std::to_string(pe);
    FILE *f = fopen(fn.c_str(), "w");
    if (!f) return fail(NVSHMEMX_ERR_INVALID, "cannot open %s", fn.c_str());
    fprintf(f, "# timestamp, gridid, blockid, tid, type, local_address, remote_address, size, remote_pe, timespent\n");
    for (long long i = 0; i < n; ++i) {
      const nvshmemx_trace_record &t = recs[i];
      long long size = t.bytes;
      if (t.op == NVSHMEMX_TRACE_PUT_DOUBLE || t.op == NVSHMEMX_TRACE_GET_DOUBLE)
        size = t.bytes / 8;
      else if (t.op <= NVSHMEMX_TRACE_GET_FLOAT)
        size = t.bytes / 4;
      else if (t.op == NVSHMEMX_TRACE_WAIT_INT || t.op == NVSHMEMX_TRACE_WAIT_UNTIL_INT)
        size = 1;
      fprintf(f, "%lld, %llu, %u, %u, %s, %p, %p, %lld, %u, %lld\n", t.t_ns, 0ull, t.block, (unsigned)t.tid,
              trace_op_name(t.op), (void *)t.local_addr, (void *)t.remote_addr, size, (unsigned)t.peer,
              t.spin_ns);
    }
    fclose(f);
  }
  return NVSHMEMX_SUCCESS;
}

}  // extern "C"
