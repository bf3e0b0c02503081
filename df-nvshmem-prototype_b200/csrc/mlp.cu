// mlp.cu -- the learned variant picker (nvshmemx_picker.h): an FP32 MLP
// 6 -> 64 -> 64 -> 64 -> 12 (ReLU) with this library's own forward, backward
// and Adam kernels, and the executor of the 12 transfer variants it chooses
// between.
//
// Kernel shape: one CTA of 64 threads per tile of 32 samples; all weights sit
// in shared memory with rows padded by one float, so the forward pass (thread
// = output unit, reading its weight row) and the backward pass (thread = input
// unit, reading a weight column) are both free of bank conflicts.  Per-tile
// weight gradients are summed over the tile's samples in registers and added
// to the global gradient with one atomicAdd per weight per tile.  The network
// is tiny (9,548 parameters); the work is latency-bound, not a contraction
// worth the tensor cores.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "batch.h"
#include "nvshmemx_picker.h"

namespace nvshm {

constexpr int NI = NVSHMEMX_PICKER_NIN, NH = NVSHMEMX_PICKER_HIDDEN, NO = NVSHMEMX_PICKER_VARIANTS, TS = 32;
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NH * NI, OFF_W2 = OFF_B1 + NH, OFF_B2 = OFF_W2 + NH * NH,
              OFF_W3 = OFF_B2 + NH, OFF_B3 = OFF_W3 + NH * NH, OFF_W4 = OFF_B3 + NH, OFF_B4 = OFF_W4 + NO * NH,
              NPARAM = OFF_B4 + NO;
// shared-memory floats: padded weights, biases, inputs, three activations,
// outputs, two gradient buffers
constexpr int SM_FLOATS = NH * (NI + 1) + 2 * NH * (NH + 1) + NO * (NH + 1) + 3 * NH + 16 + TS * NI + 3 * TS * NH +
                          TS * NO + 2 * TS * NH;

template <bool BWD>
__global__ void __launch_bounds__(64) mlp_kernel(const float *__restrict__ P, const float *__restrict__ X,
                                                 const float *__restrict__ Y, const float *__restrict__ M,
                                                 const int *__restrict__ idx, int n, const float *__restrict__ norm,
                                                 float inv_count, float *__restrict__ out, float *__restrict__ grad,
                                                 float *__restrict__ loss) {
  extern __shared__ float sm[];
  float *W1 = sm;
  float *W2 = W1 + NH * (NI + 1);
  float *W3 = W2 + NH * (NH + 1);
  float *W4 = W3 + NH * (NH + 1);
  float *b1 = W4 + NO * (NH + 1);
  float *b2 = b1 + NH;
  float *b3 = b2 + NH;
  float *b4 = b3 + NH;
  float *Xs = b4 + 16;
  float *A1 = Xs + TS * NI;
  float *A2 = A1 + TS * NH;
  float *A3 = A2 + TS * NH;
  float *Os = A3 + TS * NH;
  float *dZ = Os + TS * NO;
  float *dA = dZ + TS * NH;
  const int t = threadIdx.x;
  for (int i = t; i < NH * NI; i += 64) W1[(i / NI) * (NI + 1) + i % NI] = P[OFF_W1 + i];
  for (int i = t; i < NH * NH; i += 64) {
    W2[(i / NH) * (NH + 1) + i % NH] = P[OFF_W2 + i];
    W3[(i / NH) * (NH + 1) + i % NH] = P[OFF_W3 + i];
  }
  for (int i = t; i < NO * NH; i += 64) W4[(i / NH) * (NH + 1) + i % NH] = P[OFF_W4 + i];
  b1[t] = P[OFF_B1 + t];
  b2[t] = P[OFF_B2 + t];
  b3[t] = P[OFF_B3 + t];
  if (t < NO) b4[t] = P[OFF_B4 + t];
  const int s0 = blockIdx.x * TS;
  const int ns = min(TS, n - s0);
  for (int i = t; i < TS * NI; i += 64) {
    const int s = i / NI, f = i % NI;
    float v = 0.f;
    if (s < ns) {
      const int g = idx ? idx[s0 + s] : s0 + s;
      v = (X[g * NI + f] - norm[f]) / norm[NI + f];
    }
    Xs[i] = v;
  }
  __syncthreads();
  // forward: thread t is output unit t
  for (int s = 0; s < TS; ++s) {
    float a = b1[t];
#pragma unroll
    for (int i = 0; i < NI; ++i) a += W1[t * (NI + 1) + i] * Xs[s * NI + i];
    A1[s * NH + t] = fmaxf(a, 0.f);
  }
  __syncthreads();
  for (int s = 0; s < TS; ++s) {
    float a = b2[t];
    for (int i = 0; i < NH; ++i) a += W2[t * (NH + 1) + i] * A1[s * NH + i];
    A2[s * NH + t] = fmaxf(a, 0.f);
  }
  __syncthreads();
  for (int s = 0; s < TS; ++s) {
    float a = b3[t];
    for (int i = 0; i < NH; ++i) a += W3[t * (NH + 1) + i] * A2[s * NH + i];
    A3[s * NH + t] = fmaxf(a, 0.f);
  }
  __syncthreads();
  if (t < NO) {
    for (int s = 0; s < TS; ++s) {
      float a = b4[t];
      for (int i = 0; i < NH; ++i) a += W4[t * (NH + 1) + i] * A3[s * NH + i];
      Os[s * NO + t] = a;
    }
  }
  __syncthreads();
  if (!BWD) {
    for (int i = t; i < ns * NO; i += 64) out[(size_t)(s0 + i / NO) * NO + i % NO] = Os[i];
    return;
  }
  // loss and dL/dO = 2 m (o - y) / count, in place
  float lsum = 0.f;
  for (int i = t; i < TS * NO; i += 64) {
    const int s = i / NO, k = i % NO;
    float d = 0.f;
    if (s < ns) {
      const int g = idx ? idx[s0 + s] : s0 + s;
      const float m = M[g * NO + k], diff = Os[i] - Y[g * NO + k];
      d = 2.f * m * diff * inv_count;
      lsum += m * diff * diff;
    }
    Os[i] = d;
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if ((t & 31) == 0) atomicAdd(loss, lsum * inv_count);
  __syncthreads();
  // layer 4: thread t is input column t
  for (int k = 0; k < NO; ++k) {
    float acc = 0.f;
    for (int s = 0; s < TS; ++s) acc += Os[s * NO + k] * A3[s * NH + t];
    atomicAdd(&grad[OFF_W4 + k * NH + t], acc);
  }
  if (t < NO) {
    float acc = 0.f;
    for (int s = 0; s < TS; ++s) acc += Os[s * NO + t];
    atomicAdd(&grad[OFF_B4 + t], acc);
  }
  for (int s = 0; s < TS; ++s) {
    float acc = 0.f;
    for (int k = 0; k < NO; ++k) acc += Os[s * NO + k] * W4[k * (NH + 1) + t];
    dZ[s * NH + t] = A3[s * NH + t] > 0.f ? acc : 0.f;
  }
  __syncthreads();
  // layer 3 (dZ holds dL/dz3)
  for (int j = 0; j < NH; ++j) {
    float acc = 0.f;
    for (int s = 0; s < TS; ++s) acc += dZ[s * NH + j] * A2[s * NH + t];
    atomicAdd(&grad[OFF_W3 + j * NH + t], acc);
  }
  {
    float acc = 0.f;
    for (int s = 0; s < TS; ++s) acc += dZ[s * NH + t];
    atomicAdd(&grad[OFF_B3 + t], acc);
  }
  for (int s = 0; s < TS; ++s) {
    float acc = 0.f;
    for (int j = 0; j < NH; ++j) acc += dZ[s * NH + j] * W3[j * (NH + 1) + t];
    dA[s * NH + t] = A2[s * NH + t] > 0.f ? acc : 0.f;
  }
  __syncthreads();
  // layer 2 (dA holds dL/dz2)
  for (int j = 0; j < NH; ++j) {
    float acc = 0.f;
    for (int s = 0; s < TS; ++s) acc += dA[s * NH + j] * A1[s * NH + t];
    atomicAdd(&grad[OFF_W2 + j * NH + t], acc);
  }
  {
    float acc = 0.f;
    for (int s = 0; s < TS; ++s) acc += dA[s * NH + t];
    atomicAdd(&grad[OFF_B2 + t], acc);
  }
  for (int s = 0; s < TS; ++s) {
    float acc = 0.f;
    for (int j = 0; j < NH; ++j) acc += dA[s * NH + j] * W2[j * (NH + 1) + t];
    dZ[s * NH + t] = A1[s * NH + t] > 0.f ? acc : 0.f;
  }
  __syncthreads();
  // layer 1 (dZ holds dL/dz1): thread t is output unit t
  for (int f = 0; f < NI; ++f) {
    float acc = 0.f;
    for (int s = 0; s < TS; ++s) acc += dZ[s * NH + t] * Xs[s * NI + f];
    atomicAdd(&grad[OFF_W1 + t * NI + f], acc);
  }
  {
    float acc = 0.f;
    for (int s = 0; s < TS; ++s) acc += dZ[s * NH + t];
    atomicAdd(&grad[OFF_B1 + t], acc);
  }
}

__global__ void adam_kernel(float *P, const float *G, float *m, float *v, int n, float lr, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = G[i];
  const float mi = 0.9f * m[i] + 0.1f * g;
  const float vi = 0.999f * v[i] + 0.001f * g * g;
  m[i] = mi;
  v[i] = vi;
  P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
}

// Deterministic host RNG for initialisation and shuffles.
static unsigned long long mix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

}  // namespace nvshm

using namespace nvshm;

struct nvshmemx_mlp {
  float *P = nullptr, *G = nullptr, *Am = nullptr, *Av = nullptr;  // params, grad, Adam moments
  float *norm = nullptr;                                           // mean[6], std[6]
  float *loss = nullptr;
  long long step = 0;
};

static int mlp_launch(nvshmemx_mlp *m, bool bwd, const float *dX, const float *dY, const float *dM, const int *didx,
                      int n, float inv_count, float *dout) {
  const size_t smem = (size_t)SM_FLOATS * sizeof(float);
  const void *fn = bwd ? (const void *)mlp_kernel<true> : (const void *)mlp_kernel<false>;
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int blocks = (n + TS - 1) / TS;
  if (bwd)
    mlp_kernel<true><<<blocks, 64, smem>>>(m->P, dX, dY, dM, didx, n, m->norm, inv_count, dout, m->G, m->loss);
  else
    mlp_kernel<false><<<blocks, 64, smem>>>(m->P, dX, dY, dM, didx, n, m->norm, inv_count, dout, m->G, m->loss);
  return check_cuda(cudaGetLastError(), "mlp kernel");
}

struct DevArr {
  void *p = nullptr;
  ~DevArr() {
    if (p) cudaFree(p);
  }
};

// Device copy of a host array; h == nullptr only allocates (an output).
static int upload(DevArr &a, const void *h, size_t bytes) {
  if (cudaMalloc(&a.p, bytes ? bytes : 4) != cudaSuccess) return fail(NVSHMEMX_ERR_NOMEM, "mlp: cudaMalloc");
  if (bytes && h) return check_cuda(cudaMemcpy(a.p, h, bytes, cudaMemcpyHostToDevice), "mlp: upload");
  return 0;
}

extern "C" {

int nvshmemx_mlp_num_params(void) { return NPARAM; }

int nvshmemx_mlp_create(unsigned long long seed, nvshmemx_mlp **out) {
  if (!out) return fail(NVSHMEMX_ERR_INVALID, "mlp_create: null out");
  nvshmemx_mlp *m = new nvshmemx_mlp();
  int rc;
  if ((rc = check_cuda(cudaMalloc(&m->P, NPARAM * 4), "cudaMalloc(mlp)")) ||
      (rc = check_cuda(cudaMalloc(&m->G, NPARAM * 4), "cudaMalloc(mlp)")) ||
      (rc = check_cuda(cudaMalloc(&m->Am, NPARAM * 4), "cudaMalloc(mlp)")) ||
      (rc = check_cuda(cudaMalloc(&m->Av, NPARAM * 4), "cudaMalloc(mlp)")) ||
      (rc = check_cuda(cudaMalloc(&m->norm, 2 * NI * 4), "cudaMalloc(mlp)")) ||
      (rc = check_cuda(cudaMalloc(&m->loss, 16), "cudaMalloc(mlp)"))) {
    nvshmemx_mlp_destroy(m);
    return rc;
  }
  // He initialisation: N(0, 2 / fan_in) by Box-Muller on a splitmix64 stream
  std::vector<float> p(NPARAM, 0.f);
  unsigned long long ctr = seed;
  auto normal = [&]() {
    const double u1 = ((mix64(ctr++) >> 11) + 1.0) * (1.0 / 9007199254740993.0);
    const double u2 = (mix64(ctr++) >> 11) * (1.0 / 9007199254740992.0);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
  };
  auto fill = [&](int off, int count, int fan_in) {
    const double sd = sqrt(2.0 / fan_in);
    for (int i = 0; i < count; ++i) p[off + i] = (float)(sd * normal());
  };
  fill(OFF_W1, NH * NI, NI);
  fill(OFF_W2, NH * NH, NH);
  fill(OFF_W3, NH * NH, NH);
  fill(OFF_W4, NO * NH, NH);
  cudaMemcpy(m->P, p.data(), NPARAM * 4, cudaMemcpyHostToDevice);
  cudaMemset(m->Am, 0, NPARAM * 4);
  cudaMemset(m->Av, 0, NPARAM * 4);
  const float norm[2 * NI] = {0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1};
  cudaMemcpy(m->norm, norm, sizeof norm, cudaMemcpyHostToDevice);
  *out = m;
  return check_cuda(cudaDeviceSynchronize(), "mlp_create");
}

int nvshmemx_mlp_destroy(nvshmemx_mlp *m) {
  if (!m) return 0;
  float *bufs[] = {m->P, m->G, m->Am, m->Av, m->norm, m->loss};
  for (float *b : bufs)
    if (b) cudaFree(b);
  delete m;
  return 0;
}

int nvshmemx_mlp_get_params(const nvshmemx_mlp *m, float *h) {
  if (!m || !h) return fail(NVSHMEMX_ERR_INVALID, "mlp_get_params");
  return check_cuda(cudaMemcpy(h, m->P, NPARAM * 4, cudaMemcpyDeviceToHost), "mlp_get_params");
}

int nvshmemx_mlp_set_params(nvshmemx_mlp *m, const float *h) {
  if (!m || !h) return fail(NVSHMEMX_ERR_INVALID, "mlp_set_params");
  return check_cuda(cudaMemcpy(m->P, h, NPARAM * 4, cudaMemcpyHostToDevice), "mlp_set_params");
}

int nvshmemx_mlp_set_normalization(nvshmemx_mlp *m, const float *mean, const float *sd) {
  if (!m || !mean || !sd) return fail(NVSHMEMX_ERR_INVALID, "mlp_set_normalization");
  float h[2 * NI];
  for (int i = 0; i < NI; ++i) {
    h[i] = mean[i];
    h[NI + i] = sd[i] > 1e-12f ? sd[i] : 1.f;
  }
  return check_cuda(cudaMemcpy(m->norm, h, sizeof h, cudaMemcpyHostToDevice), "mlp_set_normalization");
}

int nvshmemx_mlp_forward(nvshmemx_mlp *m, const float *X, int n, float *Y) {
  if (!m || n < 0 || (n && (!X || !Y))) return fail(NVSHMEMX_ERR_INVALID, "mlp_forward");
  if (n == 0) return 0;
  DevArr dX, dY;
  int rc;
  if ((rc = upload(dX, X, (size_t)n * NI * 4)) || (rc = upload(dY, nullptr, (size_t)n * NO * 4))) return rc;
  if ((rc = mlp_launch(m, false, (float *)dX.p, nullptr, nullptr, nullptr, n, 0.f, (float *)dY.p))) return rc;
  return check_cuda(cudaMemcpy(Y, dY.p, (size_t)n * NO * 4, cudaMemcpyDeviceToHost), "mlp_forward");
}

int nvshmemx_mlp_loss_grad(nvshmemx_mlp *m, const float *X, const float *Y, const float *M, int n, float *loss,
                           float *grad) {
  if (!m || n < 1 || !X || !Y || !M) return fail(NVSHMEMX_ERR_INVALID, "mlp_loss_grad");
  double cnt = 0;
  for (size_t i = 0; i < (size_t)n * NO; ++i) cnt += M[i];
  if (cnt <= 0) return fail(NVSHMEMX_ERR_INVALID, "mlp_loss_grad: empty mask");
  DevArr dX, dY, dM;
  int rc;
  if ((rc = upload(dX, X, (size_t)n * NI * 4)) || (rc = upload(dY, Y, (size_t)n * NO * 4)) ||
      (rc = upload(dM, M, (size_t)n * NO * 4)))
    return rc;
  cudaMemset(m->G, 0, NPARAM * 4);
  cudaMemset(m->loss, 0, 4);
  if ((rc = mlp_launch(m, true, (float *)dX.p, (float *)dY.p, (float *)dM.p, nullptr, n, (float)(1.0 / cnt),
                       nullptr)))
    return rc;
  if (loss && (rc = check_cuda(cudaMemcpy(loss, m->loss, 4, cudaMemcpyDeviceToHost), "mlp loss"))) return rc;
  if (grad) return check_cuda(cudaMemcpy(grad, m->G, NPARAM * 4, cudaMemcpyDeviceToHost), "mlp grad");
  return 0;
}

int nvshmemx_mlp_train(nvshmemx_mlp *m, const float *X, const float *Y, const float *M, int n, int epochs, int batch,
                       float lr, unsigned long long seed, float *curve) {
  if (!m || n < 1 || epochs < 1 || batch < 1 || !X || !Y || !M) return fail(NVSHMEMX_ERR_INVALID, "mlp_train");
  DevArr dX, dY, dM, dI;
  int rc;
  if ((rc = upload(dX, X, (size_t)n * NI * 4)) || (rc = upload(dY, Y, (size_t)n * NO * 4)) ||
      (rc = upload(dM, M, (size_t)n * NO * 4)) || (rc = upload(dI, nullptr, (size_t)n * 4)))
    return rc;
  std::vector<int> perm(n);
  std::vector<double> rowm(n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < NO; ++k) rowm[i] += M[(size_t)i * NO + k];
  for (int e = 0; e < epochs; ++e) {
    for (int i = 0; i < n; ++i) perm[i] = i;
    unsigned long long st = seed * 0x100000001b3ull + (unsigned long long)e;
    for (int i = n - 1; i > 0; --i) std::swap(perm[i], perm[mix64(st++) % (unsigned long long)(i + 1)]);
    if ((rc = check_cuda(cudaMemcpy(dI.p, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice), "mlp idx"))) return rc;
    cudaMemset(m->loss, 0, 4);
    int nb = 0;
    for (int b0 = 0; b0 < n; b0 += batch, ++nb) {
      const int cnt = std::min(batch, n - b0);
      double c = 0;
      for (int i = b0; i < b0 + cnt; ++i) c += rowm[perm[i]];
      if (c <= 0) continue;
      cudaMemsetAsync(m->G, 0, NPARAM * 4);
      if ((rc = mlp_launch(m, true, (float *)dX.p, (float *)dY.p, (float *)dM.p, (int *)dI.p + b0, cnt,
                           (float)(1.0 / c), nullptr)))
        return rc;
      ++m->step;
      const float c1 = 1.f - powf(0.9f, (float)m->step), c2 = 1.f - powf(0.999f, (float)m->step);
      adam_kernel<<<(NPARAM + 255) / 256, 256>>>(m->P, m->G, m->Am, m->Av, NPARAM, lr, c1, c2);
    }
    if (curve) {
      float l = 0;
      if ((rc = check_cuda(cudaMemcpy(&l, m->loss, 4, cudaMemcpyDeviceToHost), "mlp loss"))) return rc;
      curve[e] = nb ? l / nb : 0.f;
    }
  }
  return check_cuda(cudaDeviceSynchronize(), "mlp_train");
}

int nvshmemx_mlp_pick(nvshmemx_mlp *m, const float *X, int n, int *variant, float *margin) {
  if (!m || n < 0 || (n && (!X || !variant))) return fail(NVSHMEMX_ERR_INVALID, "mlp_pick");
  std::vector<float> y((size_t)n * NO);
  int rc;
  if ((rc = nvshmemx_mlp_forward(m, X, n, y.data()))) return rc;
  for (int i = 0; i < n; ++i) {
    const float *r = &y[(size_t)i * NO];
    int best = 0;
    for (int k = 1; k < NO; ++k)
      if (r[k] < r[best]) best = k;
    float second = 1e30f;
    for (int k = 0; k < NO; ++k)
      if (k != best && r[k] < second) second = r[k];
    variant[i] = best;
    if (margin) margin[i] = second - r[best];
  }
  return 0;
}

// ------------------------------------------------------------------ variants
int nvshmemx_variant_describe(int v, int *percall_mode, nvshmemx_batch_config *cfg) {
  if (v < 0 || v >= NO) return NVSHMEMX_ERR_INVALID;
  nvshmemx_batch_config c;
  nvshmemx_batch_default_config(&c);
  int mode = -1;
  struct Shape {
    int chunk, unroll, threads, grab, stages, stage, minb;
  };
  static const Shape shapes[8] = {
      {4096, 4, 1024, 4, 0, 8192, 512},   {16384, 8, 256, 2, 0, 8192, 512},   {65536, 4, 256, 2, 0, 8192, 512},
      {16384, 4, 128, 2, 2, 8192, 2048},  {16384, 4, 256, 2, 3, 8192, 512},   {16384, 4, 128, 2, 4, 4096, 512},
      {65536, 4, 256, 2, 3, 8192, 512},   {65536, 4, 128, 2, 2, 16384, 2048},
  };
  if (v < 4) {
    mode = v;  // NVSHMEMX_MODE_THREAD, WARP, BLOCK, BULK
  } else {
    const Shape &s = shapes[v - 4];
    c.vec_bytes = 16;
    c.chunk_bytes = s.chunk;
    c.unroll = s.unroll;
    c.threads = s.threads;
    c.ctas_per_sm = 0;
    c.grab = s.grab;
    c.tma_stages = s.stages;
    c.tma_stage_bytes = s.stage;
    c.tma_min_bytes = s.minb;
  }
  if (percall_mode) *percall_mode = mode;
  if (cfg) *cfg = c;
  return 0;
}

int nvshmemx_variant_time(nvshmemx_batch *b, int v, int reps, size_t flush_bytes, float *out_ms) {
  int mode;
  nvshmemx_batch_config c, saved;
  if (!b || reps < 1 || nvshmemx_variant_describe(v, &mode, &c)) return fail(NVSHMEMX_ERR_INVALID, "variant_time");
  nvshmemx_batch_get_config(b, &saved);
  int rc = 0;
  if (mode < 0 && (rc = nvshmemx_batch_set_config(b, &c))) return rc;
  std::vector<float> t;
  for (int r = 0; r <= reps && rc == 0; ++r) {  // r == 0 warms up (graph build)
    if ((rc = l2_flush(flush_bytes))) break;
    float ms = 0;
    rc = mode >= 0 ? nvshmemx_batch_execute_percall(b, mode, 1, &ms) : nvshmemx_batch_execute(b, 1, &ms);
    if (r > 0) t.push_back(ms);
  }
  nvshmemx_batch_set_config(b, &saved);
  if (rc) return rc;
  std::sort(t.begin(), t.end());
  if (out_ms) *out_ms = t[t.size() / 2];
  return 0;
}

}  // extern "C"
