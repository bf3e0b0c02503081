// Calls every function of nvshmem.h, nvshmem_device.h and nvshmemx.h once so
// that compiling with -rdc=true and linking against libnvshmem.a proves the
// static library provides each symbol (the way applications of the
// prototype link, microbench/Makefile:38-45).  Built by the tests; never run.
#include <cuda_runtime.h>
#include <stdio.h>

#include "nvshmem.h"
#include "nvshmem_device.h"
#include "nvshmemx.h"

__global__ void every_device_call(int *ia, float *fa, double *da, char *smem_unused) {
  __shared__ __align__(128) char ring[8192];
  int pe = nvshmemx_my_pe();
  int peer = (pe + 1) % nvshmemx_n_pes();
  nvshmem_trace_begin();
  nvshmem_int_p(ia, 1, peer);
  nvshmem_float_p(fa, 1.0f, peer);
  nvshmem_double_p(da, 1.0, peer);
  int a = nvshmem_int_g(ia, peer);
  float b = nvshmem_float_g(fa, peer);
  double c = nvshmem_double_g(da, peer);
  int *li = (int *)nvshmemx_local_ptr(ia);
  float *lf = (float *)nvshmemx_ptr(fa, pe);
  double *ld = (double *)nvshmemx_local_ptr(da);
  nvshmem_int_put(ia + 4, li, 4, peer);
  nvshmem_float_put(fa + 4, lf, 4, peer);
  nvshmem_double_put(da + 4, ld, 4, peer);
  nvshmem_int_get(li + 8, ia, 4, peer);
  nvshmem_float_get(lf + 8, fa, 4, peer);
  nvshmem_double_get(ld + 8, da, 4, peer);
  nvshmemx_int_put_warp(ia, li, 1, peer);
  nvshmemx_float_put_warp(fa, lf, 1, peer);
  nvshmemx_double_put_warp(da, ld, 1, peer);
  nvshmemx_int_get_warp(li, ia, 1, peer);
  nvshmemx_float_get_warp(lf, fa, 1, peer);
  nvshmemx_double_get_warp(ld, da, 1, peer);
  nvshmemx_int_put_block(ia, li, 1, peer);
  nvshmemx_float_put_block(fa, lf, 1, peer);
  nvshmemx_double_put_block(da, ld, 1, peer);
  nvshmemx_int_get_block(li, ia, 1, peer);
  nvshmemx_float_get_block(lf, fa, 1, peer);
  nvshmemx_double_get_block(ld, da, 1, peer);
  nvshmemx_putmem_warp(ia, li, 4, peer);
  nvshmemx_getmem_warp(li, ia, 4, peer);
  nvshmemx_putmem_block(ia, li, 4, peer);
  nvshmemx_getmem_block(li, ia, 4, peer);
  nvshmemx_putmem_bulk_block(ia, li, 4096, peer, ring, sizeof ring);
  nvshmemx_getmem_bulk_block(li, ia, 4096, peer, ring, sizeof ring);
  nvshmem_quiet();
  nvshmemx_int_signal(ia, a + (int)b + (int)c, peer);
  nvshmem_int_wait(li, 0);
  nvshmem_int_wait_until(li, 0, 1);
  nvshmemx_int_wait_until_cmp(li, NVSHMEMX_CMP_GE, 1, 1000);
  nvshmemx_barrier_pe();
  nvshmemx_barrier_all();
  nvshmemx_barrier_all_ep(1);
  nvshmem_trace_end();
}

static void spmd_body(void *) {
  nvshmem_my_pe();
  nvshmem_barrier_all();
}

int main() {
  nvstart_pes();
  int *ia = (int *)nvshmalloc(4096);
  float *fa = (float *)nvshmalloc(4096);
  double *da = (double *)nvshmalloc(4096);
  void *args[] = {&ia, &fa, &da, &ia};
  nvshmemx_collective_launch((const void *)every_device_call, dim3(1), dim3(64), args, 0, 0);
  nvshmemx_collective_max_ctas_per_pe((const void *)every_device_call, 64, 0);
  nvshmem_barrier_all();
  nvshmem_barrier_all_offload();
  nvshmemx_spmd_run(spmd_body, nullptr);
  printf("%p %d %d\n", nvshmem_ptr(ia, 1), nvshmem_n_pes(), nvshmemx_status());
  nvshmcleanup();
  nvstop_pes();
  nvshmemx_init_process(0, 2, 1 << 20, "/nonexistent");  // process-per-PE start (returns an error here)
  return 0;
}
