// picker.cu -- run-time use of the learned variant picker (nvshmemx_picker.h).
//
// A picker holds the measured variant-timing table a network was trained on
// and the network itself.  For a feature row it returns the network's
// fastest variant while every feature lies inside the table's range, and
// otherwise the best measured variant of the table's nearest class (the
// network is not trusted outside the data it has seen).
// nvshmemx_batch_execute_picked applies it to a request array: it groups
// like requests, picks a variant per group, and runs the groups -- those
// that chose the same variant together: batch-engine shapes one after the
// other on the batch's stream, per-call modes each on a stream of its own
// beside them.
//
// The reference has one transfer method, the calling thread's scalar loop
// (nvshmem_device.cu:498-500); every variant here gives the same heap
// contents, so the choice only changes the time.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <vector>

#include "batch.h"
#include "nvshmemx_picker.h"

using namespace nvshm;

namespace {
constexpr int kNin = NVSHMEMX_PICKER_NIN, kNv = NVSHMEMX_PICKER_VARIANTS;
constexpr int kScalarVariant = 8;  // the batch engine's default configuration

bool measured(float t) { return t > 0.f && isfinite(t); }
}  // namespace

struct nvshmemx_picker {
  nvshmemx_mlp *net = nullptr;
  // picked execution: one stream per per-call mode (those runs overlap the
  // batch runs and each other), and the events that fork and join them
  cudaStream_t aux[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t ev_copied = nullptr, ev_done[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t ev_t[3] = {nullptr, nullptr, nullptr};  // timing: start, requests copied, end
  int nt = 0;
  std::vector<float> tx, tt;  // nt x kNin features, nt x kNv times (ms)
  float mean[kNin], sd[kNin], lo[kNin], hi[kNin];

  // Best measured variant of class c, or -1 if none ran.
  int best_of(int c) const {
    int best = -1;
    for (int v = 0; v < kNv; ++v) {
      const float t = tt[(size_t)c * kNv + v];
      if (measured(t) && (best < 0 || t < tt[(size_t)c * kNv + best])) best = v;
    }
    return best;
  }

  // The nearest class (standardised Euclidean distance) that has a measured
  // variant; its best variant.
  int table_choice(const float *x) const {
    int bc = -1;
    double bd = 0;
    for (int c = 0; c < nt; ++c) {
      if (best_of(c) < 0) continue;
      double d = 0;
      for (int k = 0; k < kNin; ++k) {
        const double z = ((double)x[k] - tx[(size_t)c * kNin + k]) / sd[k];
        d += z * z;
      }
      if (bc < 0 || d < bd) {
        bc = c;
        bd = d;
      }
    }
    return bc < 0 ? kScalarVariant : best_of(bc);
  }

  bool in_range(const float *x) const {
    for (int k = 0; k < kNin; ++k)
      if (x[k] < lo[k] - 1e-6f || x[k] > hi[k] + 1e-6f) return false;
    return true;
  }
};

extern "C" {

int nvshmemx_picker_create(nvshmemx_mlp *net, const float *table_x, const float *table_t, int nt,
                           nvshmemx_picker **out) {
  if (!net || !table_x || !table_t || nt < 1 || !out) return fail(NVSHMEMX_ERR_INVALID, "picker_create: bad arguments");
  nvshmemx_picker *p = new nvshmemx_picker();
  p->net = net;
  p->nt = nt;
  p->tx.assign(table_x, table_x + (size_t)nt * kNin);
  p->tt.assign(table_t, table_t + (size_t)nt * kNv);
  for (int k = 0; k < kNin; ++k) {
    double s = 0, s2 = 0;
    float lo = table_x[k], hi = table_x[k];
    for (int c = 0; c < nt; ++c) {
      const float v = table_x[(size_t)c * kNin + k];
      s += v;
      s2 += (double)v * v;
      lo = std::min(lo, v);
      hi = std::max(hi, v);
    }
    const double m = s / nt, var = std::max(0.0, s2 / nt - m * m);
    p->mean[k] = (float)m;
    p->sd[k] = std::max((float)sqrt(var), 1e-3f);  // a constant feature still divides safely
    p->lo[k] = lo;
    p->hi[k] = hi;
  }
  int rc = nvshmemx_mlp_set_normalization(net, p->mean, p->sd);
  if (!rc) rc = check_cuda(cudaEventCreateWithFlags(&p->ev_copied, cudaEventDisableTiming), "cudaEventCreate");
  for (int k = 0; k < 3 && !rc; ++k) rc = check_cuda(cudaEventCreate(&p->ev_t[k]), "cudaEventCreate");
  for (int m = 0; m < 4 && !rc; ++m) {
    rc = check_cuda(cudaStreamCreateWithFlags(&p->aux[m], cudaStreamNonBlocking), "cudaStreamCreate");
    if (!rc) rc = check_cuda(cudaEventCreateWithFlags(&p->ev_done[m], cudaEventDisableTiming), "cudaEventCreate");
  }
  if (rc) {
    nvshmemx_picker_destroy(p);
    return rc;
  }
  *out = p;
  return 0;
}

int nvshmemx_picker_destroy(nvshmemx_picker *p) {
  if (!p) return 0;
  for (int m = 0; m < 4; ++m) {
    if (p->aux[m]) {
      cudaStreamSynchronize(p->aux[m]);
      cudaStreamDestroy(p->aux[m]);
    }
    if (p->ev_done[m]) cudaEventDestroy(p->ev_done[m]);
  }
  if (p->ev_copied) cudaEventDestroy(p->ev_copied);
  for (int k = 0; k < 3; ++k)
    if (p->ev_t[k]) cudaEventDestroy(p->ev_t[k]);
  delete p;
  return 0;
}

int nvshmemx_picker_table_pick(nvshmemx_picker *p, const float *X, int n, int *variant) {
  if (!p || n < 0 || (n && (!X || !variant))) return fail(NVSHMEMX_ERR_INVALID, "picker_table_pick: bad arguments");
  for (int i = 0; i < n; ++i) variant[i] = p->table_choice(X + (size_t)i * kNin);
  return 0;
}

int nvshmemx_picker_pick(nvshmemx_picker *p, const float *X, int n, int *variant, int *source) {
  if (!p || n < 0 || (n && (!X || !variant))) return fail(NVSHMEMX_ERR_INVALID, "picker_pick: bad arguments");
  if (n == 0) return 0;
  int rc;
  if ((rc = nvshmemx_mlp_pick(p->net, X, n, variant, nullptr))) return rc;
  for (int i = 0; i < n; ++i) {
    const float *x = X + (size_t)i * kNin;
    const bool net_ok = p->in_range(x);
    if (!net_ok) variant[i] = p->table_choice(x);
    if (source) source[i] = net_ok ? 0 : 1;
  }
  return 0;
}

}  // extern "C"

namespace {

// The host-side checks of the plan kernel, so that an invalid request fails
// the call before anything runs: PEs, op and type, every range inside its
// slice (written so that no sum wraps), SIGNAL/P natural alignment.
int validate(const nvshmemx_request &q, const Runtime &r) {
  const unsigned long long slice = r.heap_bytes;
  auto inside = [&](unsigned long long off, unsigned long long bytes) {
    return off <= slice && bytes <= slice - off;
  };
  if (q.src_pe >= r.npes || q.dst_pe >= r.npes || q.dtype > NVSHMEMX_DT_DOUBLE) return NVSHMEMX_ERR_BOUNDS;
  const unsigned width = q.dtype == NVSHMEMX_DT_DOUBLE ? 8u : 4u;
  switch (q.op) {
    case NVSHMEMX_REQ_PUT:
    case NVSHMEMX_REQ_GET:
    case NVSHMEMX_REQ_G: {
      const unsigned long long bytes = q.op == NVSHMEMX_REQ_G ? width : q.bytes;
      return inside(q.src_off, bytes) && inside(q.dst_off, bytes) ? 0 : NVSHMEMX_ERR_BOUNDS;
    }
    case NVSHMEMX_REQ_SIGNAL:
    case NVSHMEMX_REQ_P: {
      const unsigned bytes = q.op == NVSHMEMX_REQ_SIGNAL ? 4u : width;
      return inside(q.dst_off, bytes) && (q.dst_off & (bytes - 1)) == 0 ? 0 : NVSHMEMX_ERR_BOUNDS;
    }
    default:
      return NVSHMEMX_ERR_INVALID;
  }
}

struct Group {
  std::vector<int> idx;  // request indices
  double bytes = 0;
  int width = 4, align = 16, scalar = 0;
  int variant = 0, source = 0;
  float f[kNin];
};

}  // namespace

extern "C" int nvshmemx_batch_execute_picked(nvshmemx_batch *b, nvshmemx_picker *p, const nvshmemx_request *reqs,
                                             int n, int pattern, nvshmemx_picked_group *groups, int max_groups,
                                             int *ngroups, int *out_status, float *out_ms, float *out_run_ms) {
  if (!is_started()) return fail(NVSHMEMX_ERR_STATE, "batch_execute_picked before nvstart_pes");
  if (!b || !p || n < 0 || (n && !reqs) || n > batch_capacity(b) || pattern < 0 || pattern > 3 ||
      (max_groups > 0 && !groups))
    return fail(NVSHMEMX_ERR_INVALID, "batch_execute_picked: bad arguments");
  if (ngroups) *ngroups = 0;
  if (out_status) *out_status = 0;
  if (out_ms) *out_ms = 0.f;
  if (out_run_ms) *out_run_ms = 0.f;
  if (n == 0) return 0;
  const Runtime &r = rt();
  for (int i = 0; i < n; ++i) {
    const int code = validate(reqs[i], r);
    if (code)
      return fail(code, "batch_execute_picked: request %d rejected (%s); nothing was executed", i,
                  nvshmemx_strerror(code));
  }
  // ---- group like requests
  std::map<unsigned, Group> by_key;
  for (int i = 0; i < n; ++i) {
    const nvshmemx_request &q = reqs[i];
    unsigned key;
    Group *g;
    if (q.op == NVSHMEMX_REQ_PUT || q.op == NVSHMEMX_REQ_GET) {
      const int width = q.dtype == NVSHMEMX_DT_DOUBLE ? 8 : 4;
      const unsigned long long rel = (q.src_off ^ q.dst_off) | 16ull;
      const int align = (int)(rel & (~rel + 1));  // lowest set bit, at most 16
      const int cls = q.bytes ? 31 - __builtin_clz(q.bytes) : 0;
      key = ((unsigned)cls << 16) | ((unsigned)align << 4) | (unsigned)width;
      g = &by_key[key];
      g->width = width;
      g->align = align;
    } else {
      key = 0xffffffffu;  // SIGNAL, P, G: one element each (their `bytes` field is not used)
      g = &by_key[key];
      g->scalar = 1;
    }
    g->idx.push_back(i);
    g->bytes += g->scalar ? (q.op != NVSHMEMX_REQ_SIGNAL && q.dtype == NVSHMEMX_DT_DOUBLE ? 8 : 4) : q.bytes;
  }
  std::vector<Group> gs;
  gs.reserve(by_key.size());
  for (auto &kv : by_key) gs.push_back(std::move(kv.second));
  // ---- features and picks (one network pass for every copy group)
  std::vector<float> X;
  std::vector<int> which;
  for (size_t k = 0; k < gs.size(); ++k) {
    Group &g = gs[k];
    const double cnt = (double)g.idx.size();
    g.f[0] = (float)log2(std::max(1.0, g.bytes / cnt));
    g.f[1] = (float)g.width;
    g.f[2] = (float)log2((double)g.align);
    g.f[3] = (float)log2((double)r.npes);
    g.f[4] = (float)pattern;
    g.f[5] = (float)log2(cnt);
    if (g.scalar) {
      g.variant = kScalarVariant;
      g.source = 2;
    } else {
      X.insert(X.end(), g.f, g.f + kNin);
      which.push_back((int)k);
    }
  }
  if (!which.empty()) {
    std::vector<int> v(which.size()), src(which.size());
    int rc;
    if ((rc = nvshmemx_picker_pick(p, X.data(), (int)which.size(), v.data(), src.data()))) return rc;
    for (size_t j = 0; j < which.size(); ++j) {
      gs[which[j]].variant = v[j];
      gs[which[j]].source = src[j];
    }
  }
  // ---- grouped order: groups sorted by variant, so each variant is one run
  std::stable_sort(gs.begin(), gs.end(), [](const Group &a, const Group &c) { return a.variant < c.variant; });
  // The grouped order is written into the batch's pinned host buffer, so the
  // copy to the device runs at the host link's speed (from pageable memory
  // the driver would stage it at a fraction of that); when the caller's
  // requests already sit in that buffer, they are gathered through a
  // temporary array first.
  nvshmemx_request *pinned = nvshmemx_batch_host_buffer(b);
  const uintptr_t pin0 = reinterpret_cast<uintptr_t>(pinned), req0 = reinterpret_cast<uintptr_t>(reqs);
  const bool aliased = req0 < pin0 + (size_t)batch_capacity(b) * sizeof(nvshmemx_request) &&
                       pin0 < req0 + (size_t)n * sizeof(nvshmemx_request);
  std::vector<nvshmemx_request> tmp;
  nvshmemx_request *perm = pinned;
  if (aliased) {
    tmp.resize((size_t)n);
    perm = tmp.data();
  }
  std::vector<int> first(gs.size());
  size_t at = 0;
  for (size_t k = 0; k < gs.size(); ++k) {
    first[k] = (int)at;
    for (int i : gs[k].idx) perm[at++] = reqs[i];
  }
  if (aliased) memcpy(pinned, tmp.data(), (size_t)n * sizeof(nvshmemx_request));
  if (ngroups) *ngroups = (int)gs.size();
  for (size_t k = 0; k < gs.size() && (int)k < max_groups; ++k) {
    groups[k].first = first[k];
    groups[k].count = (int)gs[k].idx.size();
    groups[k].variant = gs[k].variant;
    groups[k].source = gs[k].source;
    memcpy(groups[k].features, gs[k].f, sizeof gs[k].f);
  }
  // ---- run: one request copy, then one launch or batch run per variant
  cudaStream_t st = batch_stream(b);
  nvshmemx_request *d = batch_device_requests(b);
  int rc = check_cuda(cudaEventRecord(p->ev_t[0], st), "cudaEventRecord");
  if (!rc)
    rc = check_cuda(cudaMemcpyAsync(d, pinned, (size_t)n * sizeof(nvshmemx_request), cudaMemcpyHostToDevice, st),
                    "cudaMemcpyAsync(requests)");
  if (!rc) rc = batch_clear_sticky(b);
  if (!rc) rc = check_cuda(cudaEventRecord(p->ev_copied, st), "cudaEventRecord");
  if (!rc) rc = check_cuda(cudaEventRecord(p->ev_t[1], st), "cudaEventRecord");
  nvshmemx_batch_config own;
  nvshmemx_batch_get_config(b, &own);
  if (own.stream) nvshmemx_batch_default_config(&own);  // runs here are plan-then-exec
  bool used[4] = {false, false, false, false};
  for (size_t k = 0; k < gs.size() && !rc;) {
    size_t e = k;
    int count = 0;
    while (e < gs.size() && gs[e].variant == gs[k].variant) count += (int)gs[e++].idx.size();
    int mode = -1;
    nvshmemx_batch_config c;
    nvshmemx_variant_describe(gs[k].variant, &mode, &c);
    if (mode >= 0) {
      // a per-call run on its own stream, beside the batch runs (requests of
      // one call touch disjoint bytes, so the runs may overlap)
      rc = check_cuda(cudaStreamWaitEvent(p->aux[mode], p->ev_copied, 0), "cudaStreamWaitEvent");
      if (!rc) rc = launch_exec_requests(mode, d + first[k], count, p->aux[mode]);
      if (!rc) rc = check_cuda(cudaEventRecord(p->ev_done[mode], p->aux[mode]), "cudaEventRecord");
      used[mode] = true;
    } else {
      // a shape whose chunk is below the batch's smallest chunk would not
      // fit its chunk table: run it with the batch's own configuration
      if (c.chunk_bytes < batch_min_chunk(b)) c = own;
      if (c.chunk_bytes < batch_min_chunk(b)) c.chunk_bytes = (batch_min_chunk(b) + 255) / 256 * 256;
      rc = batch_enqueue_range(b, first[k], count, c);
    }
    k = e;
  }
  for (int m = 0; m < 4; ++m)
    if (used[m]) {
      const int wr = check_cuda(cudaStreamWaitEvent(st, p->ev_done[m], 0), "cudaStreamWaitEvent");
      if (!rc) rc = wr;
    }
  if (!rc) rc = check_cuda(cudaEventRecord(p->ev_t[2], st), "cudaEventRecord");
  if (!rc) rc = check_cuda(cudaStreamSynchronize(st), "batch_execute_picked");
  if (rc) {
    // let whatever was enqueued finish before the caller reuses the buffers
    for (int m = 0; m < 4; ++m)
      if (used[m]) cudaStreamSynchronize(p->aux[m]);
    cudaStreamSynchronize(st);
    return rc;
  }
  float ms = 0, run_ms = 0;
  cudaEventElapsedTime(&ms, p->ev_t[0], p->ev_t[2]);
  cudaEventElapsedTime(&run_ms, p->ev_t[1], p->ev_t[2]);
  int s0 = 0, bad = 0;
  if ((rc = batch_sticky_status(b, &s0, &bad))) return rc;
  if (out_status) *out_status = s0;
  if (out_ms) *out_ms = ms;
  if (out_run_ms) *out_run_ms = run_ms;
  return 0;
}
