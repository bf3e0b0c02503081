/*
 * shmem_model.c -- sequential CPU restatement of the prototype's one-sided
 * path over per-PE heap images.  TEST INFRASTRUCTURE ONLY (see shmem_model.h).
 *
 * Every data movement in the prototype is a bit copy: nvshmem_T_put is
 * `for (i = 0; i < len; i++) target_actual[i] = source[i]`
 * (nvshmem_device.cu:498-500), nvshmem_T_get the mirror image (:525-527),
 * nvshmem_T_p one store (:449), nvshmem_T_g one load (:474).  The element type
 * only sets the width.  So the model is memcpy over heap images; what it adds
 * is the order in which the scenario drivers perform those copies, which is
 * the order the device code enforces with quiet + flag + wait + barrier.
 */
#include "shmem_model.h"

#include <stdlib.h>
#include <string.h>

om_model *om_create(int npes, size_t slice, size_t heap_limit) {
  if (npes < 1 || slice == 0) return NULL;
  om_model *m = (om_model *)calloc(1, sizeof *m);
  if (!m) return NULL;
  m->npes = npes;
  m->slice = slice;
  m->heap_limit = heap_limit ? heap_limit : slice;
  m->heap = (unsigned char *)calloc((size_t)npes, slice);
  m->tail = (size_t *)calloc((size_t)npes, sizeof(size_t));
  if (!m->heap || !m->tail) {
    om_destroy(m);
    return NULL;
  }
  return m;
}

void om_destroy(om_model *m) {
  if (!m) return;
  free(m->heap);
  free(m->tail);
  free(m);
}

unsigned char *om_slice(om_model *m, int pe) { return m->heap + (size_t)pe * m->slice; }

/* nvshmem.cu:780-787: fail when tail + size passes the heap end, otherwise
 * return the tail and advance it by exactly `size` (no alignment). */
long long om_alloc(om_model *m, int pe, size_t size) {
  if (pe >= 0) {
    size_t off = m->tail[pe];
    if (off + size > m->heap_limit) return -1;
    m->tail[pe] = off + size;
    return (long long)off;
  }
  size_t off = m->tail[0];
  for (int p = 1; p < m->npes; ++p)
    if (m->tail[p] != off) return -1;
  if (off + size > m->heap_limit) return -1;
  for (int p = 0; p < m->npes; ++p) m->tail[p] = off + size;
  return (long long)off;
}

/* nvshmem.cu:805-819: drop the region list and reset the tail. */
void om_cleanup(om_model *m, int pe) {
  if (pe >= 0)
    m->tail[pe] = 0;
  else
    for (int p = 0; p < m->npes; ++p) m->tail[p] = 0;
}

/* nvshmem.cu:880-883: heap_pointers[pe] + (local - my_heap); on offsets the
 * offset itself, provided it lies in the heap. */
long long om_ptr(const om_model *m, size_t off, int pe) {
  if (pe < 0 || pe >= m->npes || off >= m->slice) return -1;
  return (long long)off;
}

void om_p(om_model *m, int width, size_t target_off, uint64_t bits, int pe) {
  memcpy(om_slice(m, pe) + target_off, &bits, (size_t)width); /* little-endian low bytes */
}

uint64_t om_g(const om_model *m, int width, size_t source_off, int pe) {
  uint64_t v = 0;
  memcpy(&v, m->heap + (size_t)pe * m->slice + source_off, (size_t)width);
  return v;
}

/* Element order does not matter for disjoint ranges; memmove also covers a
 * put whose source and target overlap on the same PE, which the prototype's
 * forward loop would smear -- callers never do that. */
void om_put(om_model *m, int width, size_t target_off, int me, size_t source_off, int len, int pe) {
  if (len <= 0) return;
  memmove(om_slice(m, pe) + target_off, om_slice(m, me) + source_off, (size_t)len * (size_t)width);
}

void om_get(om_model *m, int width, int me, size_t target_off, size_t source_off, int len, int pe) {
  if (len <= 0) return;
  memmove(om_slice(m, me) + target_off, om_slice(m, pe) + source_off, (size_t)len * (size_t)width);
}

/* 32-byte nvshmemx_request records (layout of include/nvshmemx_ops.h). */
typedef struct {
  uint64_t src_off, dst_off;
  uint32_t bytes;
  uint16_t src_pe, dst_pe;
  uint8_t op, dtype;
  uint16_t flags;
  int32_t value;
} om_request;

int om_apply_requests(om_model *m, const void *reqs, int n) {
  const om_request *r = (const om_request *)reqs;
  for (int i = 0; i < n; ++i) {
    const om_request q = r[i];
    const int w = q.dtype == 2 ? 8 : 4;
    if (q.src_pe >= m->npes || q.dst_pe >= m->npes) return -1 - i;
    switch (q.op) {
      case 0: /* PUT by src_pe */
        om_put(m, 1, q.dst_off, q.src_pe, q.src_off, (int)q.bytes, q.dst_pe);
        break;
      case 1: /* GET by dst_pe */
        om_get(m, 1, q.dst_pe, q.dst_off, q.src_off, (int)q.bytes, q.src_pe);
        break;
      case 2: { /* SIGNAL: 4-byte store */
        uint32_t v = (uint32_t)q.value;
        om_p(m, 4, q.dst_off, v, q.dst_pe);
        break;
      }
      case 3: /* P: element bits carried in src_off */
        om_p(m, w, q.dst_off, q.src_off, q.dst_pe);
        break;
      case 4: { /* G by dst_pe, result stored at dst_off */
        uint64_t v = om_g(m, w, q.src_off, q.src_pe);
        om_p(m, w, q.dst_off, v, q.dst_pe);
        break;
      }
      default:
        return -1 - i;
    }
  }
  return 0;
}

/* PE p's message k goes to q = (p+1+k) % npes; puts land in q's slot p, gets
 * fill p's slot q from q's block p.  Rounds only rotate buffer sets. */
void om_alltoall(om_model *m, int op, size_t send_off, size_t recv_off, size_t bytes, int rounds, int nsets,
                 size_t set_stride) {
  for (int r = 0; r < rounds; ++r) {
    const size_t so = send_off + (size_t)(r % nsets) * set_stride;
    const size_t ro = recv_off + (size_t)(r % nsets) * set_stride;
    for (int p = 0; p < m->npes; ++p)
      for (int k = 0; k < m->npes - 1; ++k) {
        const int q = (p + 1 + k) % m->npes;
        if (op == 0)
          om_put(m, 1, ro + (size_t)p * bytes, p, so + (size_t)q * bytes, (int)bytes, q);
        else
          om_get(m, 1, p, ro + (size_t)q * bytes, so + (size_t)p * bytes, (int)bytes, q);
      }
  }
}

static int halo_nbr(int pe, int d, int px, int py, int pz) {
  int x = pe % px, y = (pe / px) % py, z = pe / (px * py);
  const int s = (d & 1) ? 1 : -1;
  if (d < 2)
    x = (x + s + px) % px;
  else if (d < 4)
    y = (y + s + py) % py;
  else
    z = (z + s + pz) % pz;
  return x + px * (y + py * z);
}

/* Face d of every sender goes to ghost d^1 of its neighbour in direction d;
 * block element (z, y, x) is double index (z*n + y)*n + x.  Face rows:
 * x faces row j = z=j over y; y faces row j = z=j over x; z faces row j =
 * y=j over x.  Signals end at `iters` (the last it+1). */
void om_halo(om_model *m, int px, int py, int pz, int n, size_t block_off, size_t ghost_off, size_t sig_off,
             int iters) {
  if (iters < 1) return;
  const size_t nn = (size_t)n, face = nn * nn * 8;
  for (int pe = 0; pe < m->npes; ++pe) {
    const double *blk = (const double *)(om_slice(m, pe) + block_off);
    for (int d = 0; d < 6; ++d) {
      const int nb = halo_nbr(pe, d, px, py, pz);
      double *g = (double *)(om_slice(m, nb) + ghost_off + (size_t)(d ^ 1) * face);
      const int e = (d & 1) ? n - 1 : 0;
      for (size_t j = 0; j < nn; ++j)
        for (size_t k = 0; k < nn; ++k) {
          size_t idx;
          if (d < 2)
            idx = (j * nn + k) * nn + (size_t)e;
          else if (d < 4)
            idx = (j * nn + (size_t)e) * nn + k;
          else
            idx = ((size_t)e * nn + j) * nn + k;
          memcpy(&g[j * nn + k], &blk[idx], 8);
        }
    }
  }
  for (int pe = 0; pe < m->npes; ++pe)
    for (int d = 0; d < 6; ++d) {
      int32_t v = iters;
      memcpy(om_slice(m, pe) + sig_off + 4 * (size_t)d, &v, 4);
    }
}

/* PE 0 puts len ints then sets PE 1's flag to i+1; PE 1 waits for its flag
 * to change, echoes its data and then PE 0's flag = i+1. */
void om_pingpong(om_model *m, size_t flag_off, size_t data_off, int len, int total, int32_t *seen0, int32_t *seen1) {
  for (int i = 0; i < total; ++i) {
    int32_t v = i + 1;
    om_put(m, 4, data_off, 0, data_off, len, 1);
    om_p(m, 4, flag_off, (uint32_t)v, 1);
    if (seen1) seen1[i] = (int32_t)om_g(m, 4, flag_off, 1);
    om_put(m, 4, data_off, 1, data_off, len, 0);
    om_p(m, 4, flag_off, (uint32_t)v, 0);
    if (seen0) seen0[i] = (int32_t)om_g(m, 4, flag_off, 0);
  }
}

uint64_t om_splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

void om_fill_random(om_model *m, int pe, size_t off, size_t bytes, uint64_t seed) {
  unsigned char *s = om_slice(m, pe);
  const uint64_t key = om_splitmix64(seed ^ ((uint64_t)pe << 48));
  size_t b = off;
  /* ragged head byte by byte, whole words, ragged tail byte by byte */
  while (b < off + bytes && (b & 7)) {
    const uint64_t v = om_splitmix64(key + (b >> 3));
    s[b] = (unsigned char)(v >> (8 * (b & 7)));
    ++b;
  }
  for (; b + 8 <= off + bytes; b += 8) {
    const uint64_t v = om_splitmix64(key + (b >> 3));
    memcpy(s + b, &v, 8);
  }
  while (b < off + bytes) {
    const uint64_t w = b >> 3;
    const uint64_t v = om_splitmix64(key + w);
    const size_t lo = (size_t)w << 3;
    for (size_t k = b - lo; k < 8 && b < off + bytes; ++k, ++b) s[b] = (unsigned char)(v >> (8 * k));
  }
}

uint64_t om_checksum(const unsigned char *p, size_t bytes) {
  uint64_t sum = 0;
  for (size_t i = 0; i < bytes / 8; ++i) {
    uint64_t w;
    memcpy(&w, p + 8 * i, 8);
    sum += om_splitmix64(w ^ ((uint64_t)i * 0x9E3779B97F4A7C15ull));
  }
  return sum;
}

uint64_t om_fnv1a(const unsigned char *p, size_t bytes) {
  uint64_t h = 0xcbf29ce484222325ull;
  for (size_t i = 0; i < bytes; ++i) {
    h ^= p[i];
    h *= 0x100000001b3ull;
  }
  return h;
}
