"""ctypes binding of libnvshmem_b200.so (the C ABI of include/nvshmemx_ops.h,
include/nvshmemx_batch.h, include/nvshmemx.h and include/nvshmem.h).

There is no fallback: if the shared library is missing this module raises at
import, so nothing can silently run on the CPU instead of the GPU kernels.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, c_char_p, c_double, c_float, c_int, c_longlong,
                    c_size_t, c_uint, c_uint64, c_ulonglong, c_void_p)

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
LIB_PATH = os.environ.get("NVSHMEM_B200_LIB",
                          os.path.join(PKG_ROOT, "lib", "libnvshmem_b200.so"))

from ._abi import (  # noqa: F401  (re-exported)
    SUCCESS, ERR_INVALID, ERR_NOMEM, ERR_CUDA, ERR_STATE, ERR_TIMEOUT, ERR_BOUNDS, ERR_COOP, ERR_UNSUPPORTED,
    ERRORS_EXIT, ERRORS_RETURN, CMP_EQ, CMP_NE, CMP_GT, CMP_GE, CMP_LT, CMP_LE,
    REQ_PUT, REQ_GET, REQ_SIGNAL, REQ_P, REQ_G, DT_INT, DT_FLOAT, DT_DOUBLE, DT_WIDTH,
    MODE_THREAD, MODE_WARP, MODE_BLOCK, MODE_BULK, REQUEST_DTYPE, REQUEST_COMPACT_DTYPE, TRACE_DTYPE,
    PICKED_GROUP_DTYPE, PATTERN_PAIRS, PATTERN_ALLTOALL, PATTERN_NEIGHBOR, PATTERN_RANDOM)


class BatchConfig(ctypes.Structure):
    _fields_ = [("vec_bytes", c_int), ("chunk_bytes", c_int), ("unroll", c_int),
                ("threads", c_int), ("ctas_per_sm", c_int), ("grab", c_int),
                ("tma_stages", c_int), ("tma_stage_bytes", c_int), ("tma_min_bytes", c_int),
                ("stream", c_int), ("stream_planners", c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneResult(ctypes.Structure):
    _fields_ = [("cfg", BatchConfig), ("ms_median", c_float), ("ms_min", c_float),
                ("exec_ms_median", c_float), ("status", c_int)]


class ShmemError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        detail = lib.nvshmemx_last_error_string()
        detail = detail.decode(errors="replace") if detail else ""
        super().__init__(f"{what}: {strerror(code)} ({code}) {detail}")


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"native library {LIB_PATH} is missing: build it with "
            f"`make -C {PKG_ROOT}` (or __graft_entry__.build())")
    return ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)


lib = _load()

_P = POINTER
_SIGS = {
    # nvshmem.h
    "nvstart_pes": (None, []), "nvstop_pes": (None, []),
    "nvshmem_my_pe": (c_int, []), "nvshmem_n_pes": (c_int, []),
    "nvshmalloc": (c_void_p, [c_size_t]), "nvshmcleanup": (None, []),
    "nvshmem_barrier_all": (None, []), "nvshmem_barrier_all_offload": (None, []),
    "nvshmem_ptr": (c_void_p, [c_void_p, c_int]),
    # nvshmemx.h host
    "nvshmemx_init_attr": (c_int, [c_int, c_size_t]), "nvshmemx_finalize": (c_int, []),
    "nvshmemx_init_process": (c_int, [c_int, c_int, c_size_t, c_char_p]),
    "nvshmemx_is_started": (c_int, []), "nvshmemx_status": (c_int, []),
    "nvshmemx_status_detail": (c_longlong, []),
    "nvshmemx_set_error_mode": (None, [c_int]), "nvshmemx_get_error_mode": (c_int, []),
    "nvshmemx_strerror": (c_char_p, [c_int]),
    "nvshmemx_last_error_string": (c_char_p, []),
    "nvshmemx_arena_base": (c_void_p, []), "nvshmemx_slice_stride": (c_size_t, []),
    "nvshmemx_heap_size": (c_size_t, []), "nvshmemx_heap_used": (c_size_t, [c_int]),
    "nvshmemx_heap_write": (c_int, [c_int, c_size_t, c_void_p, c_size_t]),
    "nvshmemx_heap_read": (c_int, [c_int, c_size_t, c_void_p, c_size_t]),
    "nvshmemx_heap_memset": (c_int, [c_int, c_size_t, c_int, c_size_t]),
    "nvshmemx_sm_count": (c_int, []), "nvshmemx_device_sync": (c_int, []),
    "nvshmemx_set_wait_timeout_ns": (None, [c_longlong]),
    "nvshmemx_get_wait_timeout_ns": (c_longlong, []),
    "nvshmemx_spmd_run": (c_int, [c_void_p, c_void_p]),
    "nvshmemx_trace_enable": (c_int, [c_uint]), "nvshmemx_trace_disable": (c_int, []),
    "nvshmemx_trace_read": (c_longlong, [c_int, c_void_p, c_size_t, _P(c_longlong)]),
    "nvshmemx_trace_reset": (c_int, []), "nvshmemx_trace_write_csv": (c_int, [c_char_p]),
    # nvshmemx_ops.h
    "nvshmemx_exec_requests": (c_int, [c_void_p, c_int, c_int, _P(c_float)]),
    "nvshmemx_fill_random": (c_int, [c_int, c_size_t, c_size_t, c_uint64]),
    "nvshmemx_compare": (c_int, [c_int, c_size_t, c_int, c_size_t, c_size_t, _P(c_ulonglong)]),
    "nvshmemx_checksum": (c_int, [c_int, c_size_t, c_size_t, _P(c_ulonglong)]),
    "nvshmemx_op_pingpong": (c_int, [c_size_t, c_size_t, c_int, c_int, c_int, _P(c_double), _P(c_double)]),
    "nvshmemx_op_barrier_latency": (c_int, [c_int, c_int, c_int, _P(c_double), _P(c_double)]),
    "nvshmemx_op_offload_barrier": (c_int, [c_int, _P(c_double)]),
    "nvshmemx_op_alltoall": (c_int, [c_int, c_int, c_size_t, c_size_t, c_size_t, c_int, c_int,
                                     c_size_t, c_int, c_int, _P(c_float)]),
    "nvshmemx_op_alltoall_host": (c_int, [c_int, c_int, c_size_t, c_size_t, c_size_t, c_int, c_int,
                                          c_size_t, c_int, c_int, _P(c_float)]),
    "nvshmemx_op_halo": (c_int, [c_int, c_int, c_int, c_int, c_size_t, c_size_t, c_size_t, c_int,
                                 c_int, _P(c_float)]),
    "nvshmemx_op_halo_offload": (c_int, [c_int, c_int, c_int, c_int, c_size_t, c_size_t, c_size_t, c_int,
                                         c_int, _P(c_float)]),
    "nvshmemx_op_strided_read": (c_int, [c_size_t, c_size_t, c_int, c_size_t, c_size_t, c_int, c_int, _P(c_float)]),
    "nvshmemx_op_wait_test": (c_int, [c_size_t, c_int, c_longlong, _P(c_int)]),
    "nvshmemx_op_barrier_fault_test": (c_int, [c_int, c_longlong, _P(c_int)]),
    # nvshmemx_batch.h
    "nvshmemx_batch_default_config": (None, [_P(BatchConfig)]),
    "nvshmemx_batch_create": (c_int, [c_int, c_ulonglong, c_int, _P(c_void_p)]),
    "nvshmemx_batch_destroy": (c_int, [c_void_p]),
    "nvshmemx_batch_set_config": (c_int, [c_void_p, _P(BatchConfig)]),
    "nvshmemx_batch_get_config": (c_int, [c_void_p, _P(BatchConfig)]),
    "nvshmemx_batch_host_buffer": (c_void_p, [c_void_p]),
    "nvshmemx_batch_upload": (c_int, [c_void_p, c_void_p, c_int]),
    "nvshmemx_batch_execute": (c_int, [c_void_p, c_int, _P(c_float)]),
    "nvshmemx_batch_execute_direct": (c_int, [c_void_p, c_int, _P(c_float), _P(c_float)]),
    "nvshmemx_batch_submit": (c_int, [c_void_p, c_void_p, c_int, _P(c_int), _P(c_float)]),
    "nvshmemx_batch_submit_compact": (c_int, [c_void_p, c_void_p, c_int, _P(c_int), _P(c_float)]),
    "nvshmemx_batch_last_stats": (c_int, [c_void_p, _P(c_ulonglong), _P(c_float), _P(c_float)]),
    "nvshmemx_requests_bytes": (c_ulonglong, [c_void_p, c_int]),
    "nvshmemx_batch_execute_percall": (c_int, [c_void_p, c_int, c_int, _P(c_float)]),
    "nvshmemx_batch_execute_noalloc": (c_int, [c_void_p, c_int, _P(BatchConfig), c_void_p]),
    # nvshmemx_picker.h
    "nvshmemx_mlp_num_params": (c_int, []),
    "nvshmemx_mlp_create": (c_int, [c_ulonglong, _P(c_void_p)]),
    "nvshmemx_mlp_destroy": (c_int, [c_void_p]),
    "nvshmemx_mlp_get_params": (c_int, [c_void_p, c_void_p]),
    "nvshmemx_mlp_set_params": (c_int, [c_void_p, c_void_p]),
    "nvshmemx_mlp_set_normalization": (c_int, [c_void_p, c_void_p, c_void_p]),
    "nvshmemx_mlp_forward": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "nvshmemx_mlp_loss_grad": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, _P(c_float), c_void_p]),
    "nvshmemx_mlp_train": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_float,
                                   c_ulonglong, c_void_p]),
    "nvshmemx_mlp_pick": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "nvshmemx_variant_time": (c_int, [c_void_p, c_int, c_int, c_size_t, _P(c_float)]),
    "nvshmemx_variant_describe": (c_int, [c_int, _P(c_int), _P(BatchConfig)]),
    "nvshmemx_picker_create": (c_int, [c_void_p, c_void_p, c_void_p, c_int, _P(c_void_p)]),
    "nvshmemx_picker_destroy": (c_int, [c_void_p]),
    "nvshmemx_picker_pick": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "nvshmemx_picker_table_pick": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "nvshmemx_batch_execute_picked": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_int,
                                              _P(c_int), _P(c_int), _P(c_float), _P(c_float)]),
    # nvshmemx_tune.h
    "nvshmemx_tune_candidates": (c_int, [_P(BatchConfig), c_int, c_int]),
    "nvshmemx_tune_batch": (c_int, [c_void_p, _P(BatchConfig), c_int, c_int, c_size_t, _P(TuneResult),
                                    _P(c_int)]),
}

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def strerror(code: int) -> str:
    s = lib.nvshmemx_strerror(int(code))
    return s.decode() if s else "unknown"


def check(rc: int, what: str) -> None:
    if rc != SUCCESS:
        raise ShmemError(rc, what)


def ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data
