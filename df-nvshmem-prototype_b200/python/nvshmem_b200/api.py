"""Python view of the B200 virtual-PE library for tests and benchmarks.

Thin wrappers over the C ABI in _lib: every call reaches the CUDA kernels in
libnvshmem_b200.so; results come back as numpy arrays.
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_double, c_float, c_int, c_longlong, c_ulonglong, c_void_p

import numpy as np

from . import _lib as L
from ._lib import check, lib, ptr


class Shmem:
    """One started instance: `npes` virtual PEs with `heap_bytes` each."""

    def __init__(self, npes: int, heap_bytes: int, error_mode: int = L.ERRORS_RETURN,
                 wait_timeout_ns: int | None = None):
        lib.nvshmemx_set_error_mode(error_mode)
        if lib.nvshmemx_is_started():
            lib.nvshmemx_finalize()
        lib.nvshmemx_status()  # clear anything left by an earlier instance
        check(lib.nvshmemx_init_attr(int(npes), int(heap_bytes)), "nvshmemx_init_attr")
        self.npes = npes
        self.heap_bytes = heap_bytes
        self.base = lib.nvshmemx_arena_base()
        self.stride = lib.nvshmemx_slice_stride()
        if wait_timeout_ns:
            lib.nvshmemx_set_wait_timeout_ns(int(wait_timeout_ns))

    # -- lifetime --------------------------------------------------------
    def close(self):
        if lib.nvshmemx_is_started():
            check(lib.nvshmemx_finalize(), "nvshmemx_finalize")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- host API --------------------------------------------------------
    def alloc(self, size: int) -> int:
        """nvshmalloc on the launching thread; returns the slice offset."""
        p = lib.nvshmalloc(int(size))
        if not p:
            raise L.ShmemError(self.status() or L.ERR_NOMEM, "nvshmalloc")
        return p - self.base

    def cleanup(self):
        lib.nvshmcleanup()

    def ptr(self, off: int, pe: int) -> int | None:
        return lib.nvshmem_ptr(c_void_p(self.base + off), pe)

    def status(self) -> int:
        return lib.nvshmemx_status()

    def status_detail(self) -> int:
        return lib.nvshmemx_status_detail()

    def sync(self):
        check(lib.nvshmemx_device_sync(), "device sync")

    # -- heap access -----------------------------------------------------
    def write(self, pe: int, off: int, data) -> None:
        a = np.ascontiguousarray(data)
        check(lib.nvshmemx_heap_write(pe, off, ptr(a), a.nbytes), "heap_write")

    def read(self, pe: int, off: int, nbytes: int, dtype=np.uint8) -> np.ndarray:
        out = np.empty(nbytes, dtype=np.uint8)
        check(lib.nvshmemx_heap_read(pe, off, ptr(out), nbytes), "heap_read")
        return out.view(dtype)

    def memset(self, pe: int, off: int, value: int, nbytes: int) -> None:
        check(lib.nvshmemx_heap_memset(pe, off, value, nbytes), "heap_memset")

    def fill_random(self, pe: int, off: int, nbytes: int, seed: int) -> None:
        check(lib.nvshmemx_fill_random(pe, off, nbytes, seed), "fill_random")

    def compare(self, a_pe, a_off, b_pe, b_off, nbytes) -> int:
        out = c_ulonglong(0)
        check(lib.nvshmemx_compare(a_pe, a_off, b_pe, b_off, nbytes, byref(out)), "compare")
        return out.value

    def checksum(self, pe: int, off: int, nbytes: int) -> int:
        out = c_ulonglong(0)
        check(lib.nvshmemx_checksum(pe, off, nbytes, byref(out)), "checksum")
        return out.value

    # -- operations ------------------------------------------------------
    def exec_requests(self, reqs: np.ndarray, mode: int = L.MODE_THREAD) -> float:
        r = np.ascontiguousarray(reqs, dtype=L.REQUEST_DTYPE)
        ms = c_float(0)
        check(lib.nvshmemx_exec_requests(ptr(r), len(r), mode, byref(ms)), "exec_requests")
        return ms.value

    def pingpong(self, flag_off, data_off, len_elems, iters, skip=20):
        out = np.zeros(iters, dtype=np.float64)
        total = c_double(0)
        check(lib.nvshmemx_op_pingpong(flag_off, data_off, len_elems, iters, skip,
                                       out.ctypes.data_as(ctypes.POINTER(c_double)), byref(total)),
              "pingpong")
        return out, total.value

    def barrier_latency(self, ctas_per_pe, iters, counted=False):
        out = np.zeros(iters, dtype=np.float64)
        total = c_double(0)
        check(lib.nvshmemx_op_barrier_latency(ctas_per_pe, iters, int(counted),
                                              out.ctypes.data_as(ctypes.POINTER(c_double)),
                                              byref(total)), "barrier_latency")
        return out, total.value

    def offload_barrier(self, iters) -> float:
        us = c_double(0)
        check(lib.nvshmemx_op_offload_barrier(iters, byref(us)), "offload_barrier")
        return us.value

    def alltoall(self, op, dtype, send_off, recv_off, nbytes, rounds=1, nsets=1, set_stride=0,
                 mode=L.MODE_BLOCK, ctas_per_pe=1, host_rounds=False) -> float:
        """C2 rounds; host_rounds=True runs one launch per round followed by the
        host's nvshmem_barrier_all, as the prototype structures it."""
        ms = c_float(0)
        fn = lib.nvshmemx_op_alltoall_host if host_rounds else lib.nvshmemx_op_alltoall
        check(fn(op, dtype, send_off, recv_off, nbytes, rounds, nsets, set_stride, mode, ctas_per_pe, byref(ms)),
              "alltoall")
        return ms.value

    def halo(self, px, py, pz, n, block_off, ghost_off, sig_off, iters, ctas_per_pe, offload=False) -> float:
        """C3 exchange; offload=True runs one launch per iteration followed by
        nvshmem_barrier_all_offload, as the prototype structures it."""
        ms = c_float(0)
        fn = lib.nvshmemx_op_halo_offload if offload else lib.nvshmemx_op_halo
        check(fn(px, py, pz, n, block_off, ghost_off, sig_off, iters, ctas_per_pe, byref(ms)), "halo")
        return ms.value

    def strided_read(self, off, set_off, nsets, rows, stride, ctas_per_pe, iters) -> float:
        """nvshmemx_op_strided_read: device ms of `iters` scattered-read launches."""
        ms = c_float(0)
        check(lib.nvshmemx_op_strided_read(off, set_off, nsets, rows, stride, ctas_per_pe, iters, byref(ms)),
              "strided_read")
        return ms.value

    def wait_test(self, flag_off, value, timeout_ns) -> int:
        st = c_int(0)
        check(lib.nvshmemx_op_wait_test(flag_off, value, timeout_ns, byref(st)), "wait_test")
        return st.value

    def barrier_fault_test(self, skip_pe, timeout_ns) -> int:
        st = c_int(0)
        check(lib.nvshmemx_op_barrier_fault_test(skip_pe, timeout_ns, byref(st)), "barrier_fault_test")
        return st.value

    # -- trace -----------------------------------------------------------
    def trace_enable(self, records_per_pe: int):
        check(lib.nvshmemx_trace_enable(records_per_pe), "trace_enable")

    def trace_disable(self):
        check(lib.nvshmemx_trace_disable(), "trace_disable")

    def trace_read(self, pe: int, max_records: int = 1 << 16):
        out = np.zeros(max_records, dtype=L.TRACE_DTYPE)
        dropped = c_longlong(0)
        n = lib.nvshmemx_trace_read(pe, ptr(out), max_records, byref(dropped))
        if n < 0:
            raise L.ShmemError(L.ERR_STATE, "trace_read")
        return out[:n], dropped.value

    def trace_write_csv(self, prefix: str):
        check(lib.nvshmemx_trace_write_csv(prefix.encode()), "trace_write_csv")

    # -- batches ---------------------------------------------------------
    def batch(self, max_requests: int, max_payload_bytes: int, min_chunk_bytes: int = 256) -> "Batch":
        return Batch(self, max_requests, max_payload_bytes, min_chunk_bytes)


def default_batch_config() -> L.BatchConfig:
    c = L.BatchConfig()
    lib.nvshmemx_batch_default_config(byref(c))
    return c


class Batch:
    def __init__(self, sh: Shmem, max_requests: int, max_payload_bytes: int, min_chunk_bytes: int):
        self.h = c_void_p(0)
        check(lib.nvshmemx_batch_create(max_requests, max_payload_bytes, min_chunk_bytes,
                                        byref(self.h)), "batch_create")
        self.max_requests = max_requests
        self.n = 0

    def close(self):
        if self.h:
            lib.nvshmemx_batch_destroy(self.h)
            self.h = c_void_p(0)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_config(self, cfg: L.BatchConfig | dict):
        """A BatchConfig, or a dict of fields over the defaults; a dict without
        `tma_stages` selects the register copy."""
        if isinstance(cfg, dict):
            c = default_batch_config()
            c.tma_stages = 0
            c.stream = 0
            for k, v in cfg.items():
                setattr(c, k, int(v))
            cfg = c
        check(lib.nvshmemx_batch_set_config(self.h, byref(cfg)), "batch_set_config")

    def config(self) -> dict:
        c = L.BatchConfig()
        check(lib.nvshmemx_batch_get_config(self.h, byref(c)), "batch_get_config")
        return c.as_dict()

    def host_buffer(self) -> np.ndarray:
        """The batch's pinned request buffer as a numpy structured array."""
        p = lib.nvshmemx_batch_host_buffer(self.h)
        raw = (ctypes.c_char * (self.max_requests * 32)).from_address(p)
        return np.frombuffer(raw, dtype=L.REQUEST_DTYPE)

    def upload(self, reqs: np.ndarray):
        r = np.ascontiguousarray(reqs, dtype=L.REQUEST_DTYPE)
        check(lib.nvshmemx_batch_upload(self.h, ptr(r), len(r)), "batch_upload")
        self.n = len(r)

    def execute(self, reps: int = 1) -> float:
        ms = c_float(0)
        check(lib.nvshmemx_batch_execute(self.h, reps, byref(ms)), "batch_execute")
        return ms.value

    def execute_direct(self, reps: int = 1):
        """(total ms, exec-kernel ms) of `reps` executions without the graph."""
        ms, ex = c_float(0), c_float(0)
        check(lib.nvshmemx_batch_execute_direct(self.h, reps, byref(ms), byref(ex)), "batch_execute_direct")
        return ms.value, ex.value

    def submit(self, reqs: np.ndarray, n: int | None = None):
        """End-to-end: H2D of the requests, execution, D2H of the status."""
        n = len(reqs) if n is None else n
        st = c_int(0)
        ms = c_float(0)
        check(lib.nvshmemx_batch_submit(self.h, ptr(reqs), n, byref(st), byref(ms)), "batch_submit")
        self.n = n
        return st.value, ms.value

    def submit_compact(self, reqs: np.ndarray, n: int | None = None):
        """submit() for requests in the 16-byte compact form (to_compact)."""
        n = len(reqs) if n is None else n
        st = c_int(0)
        ms = c_float(0)
        check(lib.nvshmemx_batch_submit_compact(self.h, ptr(reqs), n, byref(st), byref(ms)), "batch_submit_compact")
        self.n = n
        return st.value, ms.value

    def host_buffer_compact(self) -> np.ndarray:
        """The batch's pinned request buffer viewed as compact requests."""
        p = lib.nvshmemx_batch_host_buffer(self.h)
        raw = (ctypes.c_char * (self.max_requests * 32)).from_address(p)
        return np.frombuffer(raw, dtype=L.REQUEST_COMPACT_DTYPE)

    def percall(self, mode: int = L.MODE_THREAD, reps: int = 1) -> float:
        ms = c_float(0)
        check(lib.nvshmemx_batch_execute_percall(self.h, mode, reps, byref(ms)), "batch_percall")
        return ms.value

    def execute_picked(self, picker, reqs: np.ndarray, pattern: int = L.PATTERN_RANDOM, max_groups: int = 256):
        """nvshmemx_batch_execute_picked: (status, device ms with the request
        copy, device ms after it, groups) for the host requests `reqs` run
        group by group with the picker's variants."""
        r = np.ascontiguousarray(reqs, dtype=L.REQUEST_DTYPE)
        groups = np.zeros(max_groups, L.PICKED_GROUP_DTYPE)
        ng, st, ms, run = c_int(0), c_int(0), c_float(0), c_float(0)
        check(lib.nvshmemx_batch_execute_picked(self.h, picker.h, ptr(r), len(r), pattern, ptr(groups), max_groups,
                                                byref(ng), byref(st), byref(ms), byref(run)), "batch_execute_picked")
        return st.value, ms.value, run.value, groups[:min(ng.value, max_groups)]

    def stats(self):
        ch = c_ulonglong(0)
        p = c_float(0)
        e = c_float(0)
        check(lib.nvshmemx_batch_last_stats(self.h, byref(ch), byref(p), byref(e)), "batch_stats")
        return ch.value, p.value, e.value


def to_compact(reqs: np.ndarray) -> np.ndarray:
    """The 16-byte compact form of full requests (nvshmemx_request_compact);
    ValueError for a request it cannot hold (offsets or PUT/GET sizes not
    multiples of 4 or too large, PEs of 1024 and more, P of a double)."""
    r = np.ascontiguousarray(reqs, dtype=L.REQUEST_DTYPE)
    op, dt = r["op"].astype(np.uint32), r["dtype"].astype(np.uint32)
    is_p = op == L.REQ_P
    is_copy = (op == L.REQ_PUT) | (op == L.REQ_GET)
    off_src = np.where(is_p, 0, r["src_off"])
    bad = ((off_src % 4 != 0) | (r["dst_off"] % 4 != 0) | (off_src >= (16 << 30)) | (r["dst_off"] >= (16 << 30))
           | (r["src_pe"] >= 1024) | (r["dst_pe"] >= 1024) | (op > 7) | (dt > 3)
           | (is_copy & (r["bytes"] % 4 != 0)) | (is_p & ((dt == L.DT_DOUBLE) | (r["src_off"] >= (1 << 32)))))
    if bad.any():
        raise ValueError(f"request {int(np.flatnonzero(bad)[0])} has no compact form")
    out = np.zeros(len(r), dtype=L.REQUEST_COMPACT_DTYPE)
    out["src_off4"] = np.where(is_p, r["src_off"], r["src_off"] // 4).astype(np.uint32)
    out["dst_off4"] = (r["dst_off"] // 4).astype(np.uint32)
    arg = np.zeros(len(r), dtype=np.uint32)
    arg = np.where(is_copy, r["bytes"] // 4, arg)
    arg = np.where(op == L.REQ_SIGNAL, r["value"].astype(np.int64) & 0xFFFFFFFF, arg)
    out["arg"] = arg.astype(np.uint32)
    out["meta"] = (r["src_pe"].astype(np.uint32) | (r["dst_pe"].astype(np.uint32) << 10) | (op << 20) | (dt << 23))
    return out


def requests_bytes(reqs: np.ndarray) -> int:
    r = np.ascontiguousarray(reqs, dtype=L.REQUEST_DTYPE)
    return int(lib.nvshmemx_requests_bytes(ptr(r), len(r)))
