"""ctypes view of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The library never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_int, c_int32, c_longlong, c_size_t, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
HOST_BENCH = os.path.join(HERE, "_build", "host_shmem_bench")


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


if not os.path.exists(LIB):
    build()

_o = ctypes.CDLL(LIB)


class _Model(ctypes.Structure):
    _fields_ = [("npes", c_int), ("slice", c_size_t), ("heap_limit", c_size_t),
                ("heap", c_void_p), ("tail", POINTER(c_size_t))]


_sig = {
    "om_create": (POINTER(_Model), [c_int, c_size_t, c_size_t]),
    "om_destroy": (None, [POINTER(_Model)]),
    "om_alloc": (c_longlong, [POINTER(_Model), c_int, c_size_t]),
    "om_cleanup": (None, [POINTER(_Model), c_int]),
    "om_ptr": (c_longlong, [POINTER(_Model), c_size_t, c_int]),
    "om_p": (None, [POINTER(_Model), c_int, c_size_t, c_uint64, c_int]),
    "om_g": (c_uint64, [POINTER(_Model), c_int, c_size_t, c_int]),
    "om_put": (None, [POINTER(_Model), c_int, c_size_t, c_int, c_size_t, c_int, c_int]),
    "om_get": (None, [POINTER(_Model), c_int, c_int, c_size_t, c_size_t, c_int, c_int]),
    "om_apply_requests": (c_int, [POINTER(_Model), c_void_p, c_int]),
    "om_alltoall": (None, [POINTER(_Model), c_int, c_size_t, c_size_t, c_size_t, c_int, c_int, c_size_t]),
    "om_halo": (None, [POINTER(_Model), c_int, c_int, c_int, c_int, c_size_t, c_size_t, c_size_t, c_int]),
    "om_pingpong": (None, [POINTER(_Model), c_size_t, c_size_t, c_int, c_int, POINTER(c_int32), POINTER(c_int32)]),
    "om_fill_random": (None, [POINTER(_Model), c_int, c_size_t, c_size_t, c_uint64]),
    "om_splitmix64": (c_uint64, [c_uint64]),
    "om_checksum": (c_uint64, [c_void_p, c_size_t]),
    "om_fnv1a": (c_uint64, [c_void_p, c_size_t]),
}
for _n, (_r, _a) in _sig.items():
    _f = getattr(_o, _n)
    _f.restype = _r
    _f.argtypes = _a


class Model:
    """npes heap images of `slice` bytes; allocator limit heap_limit."""

    def __init__(self, npes: int, slice_bytes: int, heap_limit: int | None = None):
        self.m = _o.om_create(npes, slice_bytes, heap_limit or slice_bytes)
        if not self.m:
            raise MemoryError("om_create")
        self.npes, self.slice = npes, slice_bytes
        buf = (ctypes.c_uint8 * (npes * slice_bytes)).from_address(self.m.contents.heap)
        self.heap = np.frombuffer(buf, dtype=np.uint8).reshape(npes, slice_bytes)

    def close(self):
        if self.m:
            _o.om_destroy(self.m)
            self.m = None

    def __del__(self):
        self.close()

    # allocator
    def alloc(self, size, pe=-1):
        return _o.om_alloc(self.m, pe, size)

    def cleanup(self, pe=-1):
        _o.om_cleanup(self.m, pe)

    def ptr(self, off, pe):
        return _o.om_ptr(self.m, off, pe)

    # one-sided ops
    def p(self, width, target_off, bits, pe):
        _o.om_p(self.m, width, target_off, bits, pe)

    def g(self, width, source_off, pe):
        return _o.om_g(self.m, width, source_off, pe)

    def put(self, width, target_off, me, source_off, nelems, pe):
        _o.om_put(self.m, width, target_off, me, source_off, nelems, pe)

    def get(self, width, me, target_off, source_off, nelems, pe):
        _o.om_get(self.m, width, me, target_off, source_off, nelems, pe)

    def apply_requests(self, reqs: np.ndarray):
        r = np.ascontiguousarray(reqs)
        assert r.dtype.itemsize == 32
        rc = _o.om_apply_requests(self.m, r.ctypes.data, len(r))
        if rc:
            raise ValueError(f"request {-rc - 1} invalid")

    def alltoall(self, op, send_off, recv_off, nbytes, rounds=1, nsets=1, set_stride=0):
        _o.om_alltoall(self.m, op, send_off, recv_off, nbytes, rounds, nsets, set_stride)

    def halo(self, px, py, pz, n, block_off, ghost_off, sig_off, iters):
        _o.om_halo(self.m, px, py, pz, n, block_off, ghost_off, sig_off, iters)

    def pingpong(self, flag_off, data_off, nelems, total):
        s0 = np.zeros(total, dtype=np.int32)
        s1 = np.zeros(total, dtype=np.int32)
        _o.om_pingpong(self.m, flag_off, data_off, nelems, total,
                       s0.ctypes.data_as(POINTER(c_int32)), s1.ctypes.data_as(POINTER(c_int32)))
        return s0, s1

    def fill_random(self, pe, off, nbytes, seed):
        _o.om_fill_random(self.m, pe, off, nbytes, seed)


def splitmix64(x: int) -> int:
    return _o.om_splitmix64(x)


def checksum(a: np.ndarray) -> int:
    a = np.ascontiguousarray(a)
    return _o.om_checksum(a.ctypes.data, a.nbytes)


def fnv1a(a: np.ndarray) -> int:
    a = np.ascontiguousarray(a)
    return _o.om_fnv1a(a.ctypes.data, a.nbytes)
