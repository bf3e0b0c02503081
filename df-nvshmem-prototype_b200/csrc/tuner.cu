// tuner.cu -- measured autotuning of the batch engine's copy shape
// (nvshmemx_tune.h).  Candidates are timed on the device with CUDA events,
// each run preceded by an L2-flushing write, and ranked by median.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "batch.h"
#include "nvshmemx_tune.h"

namespace nvshm {

__global__ void l2_flush_kernel(uint4 *p, size_t n, unsigned v) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride) p[i] = make_uint4(v, v, v, v);
}

struct FlushBuf {
  uint4 *p = nullptr;
  size_t bytes = 0;
};
static FlushBuf g_flush;

// Writes `bytes` of a library-owned buffer and waits, evicting earlier data
// from L2 (B200 L2 is 126 MB).
int l2_flush(size_t bytes) {
  if (bytes == 0) return 0;
  bytes = (bytes + 15) & ~size_t(15);
  if (g_flush.bytes < bytes) {
    if (g_flush.p) cudaFree(g_flush.p);
    g_flush.p = nullptr;
    g_flush.bytes = 0;
    int rc;
    if ((rc = check_cuda(cudaMalloc(&g_flush.p, bytes), "cudaMalloc(flush)"))) return rc;
    g_flush.bytes = bytes;
  }
  static unsigned v = 1;
  l2_flush_kernel<<<rt().sm_count * 4, 512>>>(g_flush.p, bytes / 16, v++);
  return check_cuda(cudaDeviceSynchronize(), "l2 flush");
}

}  // namespace nvshm

using namespace nvshm;

extern "C" {

int nvshmemx_tune_candidates(nvshmemx_batch_config *out, int max, int min_chunk_bytes) {
  int n = 0;
  auto push = [&](const nvshmemx_batch_config &c) {
    if (n < max && c.chunk_bytes >= min_chunk_bytes && check_batch_config(c) == 0) out[n++] = c;
  };
  nvshmemx_batch_config c;
  nvshmemx_batch_default_config(&c);
  // copies through registers: accesses in flight x chunk x threads x claim
  for (int u : {2, 4, 8})
    for (int ch : {4096, 16384, 65536})
      for (int t : {256, 1024})
        for (int g : {1, 2, 4}) {
          c.vec_bytes = 16;
          c.unroll = u;
          c.chunk_bytes = ch;
          c.threads = t;
          c.ctas_per_sm = 0;
          c.grab = g;
          c.tma_stages = 0;
          push(c);
        }
  // TMA rings: stages x stage size x warps per CTA x chunk x bulk threshold
  for (int s : {2, 3, 4})
    for (int sb : {4096, 8192, 16384})
      for (int t : {128, 256})
        for (int ch : {16384, 65536})
          for (int mb : {512, 1024, 2048}) {
            c.vec_bytes = 16;
            c.unroll = 4;
            c.chunk_bytes = ch;
            c.threads = t;
            c.ctas_per_sm = 0;
            c.grab = 2;
            c.tma_stages = s;
            c.tma_stage_bytes = sb;
            c.tma_min_bytes = mb;
            push(c);
          }
  // streaming (plan and execute in one launch): ring shape x planning warps
  struct Ring { int threads, stages, stage_bytes; };
  for (Ring g : {Ring{128, 4, 4096}, Ring{256, 3, 8192}, Ring{256, 4, 4096}})
    for (int pl : {1, 2}) {
      c.vec_bytes = 16;
      c.unroll = 4;
      c.chunk_bytes = 16384;
      c.threads = g.threads;
      c.ctas_per_sm = 0;
      c.grab = 2;
      c.tma_stages = g.stages;
      c.tma_stage_bytes = g.stage_bytes;
      c.tma_min_bytes = 512;
      c.stream = 1;
      c.stream_planners = pl;
      push(c);
    }
  return n;
}

int nvshmemx_tune_batch(nvshmemx_batch *b, const nvshmemx_batch_config *cand, int ncand, int reps, size_t flush_bytes,
                        nvshmemx_tune_result *res, int *best) {
  if (!b || !cand || ncand < 1 || reps < 1 || !res) return fail(NVSHMEMX_ERR_INVALID, "tune_batch: bad arguments");
  int mode = nvshmemx_get_error_mode();
  nvshmemx_set_error_mode(NVSHMEMX_ERRORS_RETURN);  // a bad candidate must not end the process
  int bi = -1;
  int rc = 0;
  for (int i = 0; i < ncand; ++i) {
    res[i].cfg = cand[i];
    res[i].ms_median = res[i].ms_min = res[i].exec_ms_median = -1.f;
    res[i].status = nvshmemx_batch_set_config(b, &cand[i]);
    if (res[i].status) continue;
    std::vector<float> t, e;
    float ms = 0, ex = 0;
    if ((rc = l2_flush(flush_bytes))) break;
    res[i].status = nvshmemx_batch_execute(b, 1, &ms);  // warm-up (builds the graph)
    for (int r = 0; r < reps && res[i].status == 0; ++r) {
      if ((rc = l2_flush(flush_bytes))) break;
      res[i].status = nvshmemx_batch_execute(b, 1, &ms);
      t.push_back(ms);
      if ((rc = l2_flush(flush_bytes))) break;
      float tot = 0;
      if (res[i].status == 0) res[i].status = nvshmemx_batch_execute_direct(b, 1, &tot, &ex);
      e.push_back(ex);
    }
    if (rc) break;
    if (res[i].status || t.empty()) continue;
    std::sort(t.begin(), t.end());
    std::sort(e.begin(), e.end());
    res[i].ms_median = t[t.size() / 2];
    res[i].ms_min = t[0];
    res[i].exec_ms_median = e[e.size() / 2];
    if (bi < 0 || res[i].ms_median < res[bi].ms_median) bi = i;
  }
  nvshmemx_set_error_mode(mode);
  if (rc) return rc;
  if (bi < 0) return fail(NVSHMEMX_ERR_INVALID, "tune_batch: no candidate ran");
  if (best) *best = bi;
  return nvshmemx_batch_set_config(b, &cand[bi]);
}

}  // extern "C"
