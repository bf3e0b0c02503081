"""The allocation-free batch entry point, nvshmemx_batch_execute_noalloc.

Some callers of the batch engine cannot allocate device memory while they
run: a serving loop that cannot afford cudaMalloc's device-wide
synchronisation between requests, a process whose device memory belongs to
another allocator or to a budget fixed at start-up, a foreign-language caller
that cannot release device memory it would own.  This entry point takes its
scratch from a fixed array inside the library instead.  The test calls it
through the C ABI twice in a row (the second call finds the first call's
leftovers in the shared scratch) and checks that each call leaves every heap
bit-identical to the existing entry point, nvshmemx_batch_execute, run on the
same requests from the same starting heap.  It lives in its own file, which
pytest collects last.
"""
import ctypes

import numpy as np
import pytest

from nvshmem_b200 import ERR_BOUNDS, ERR_INVALID, ERR_NOMEM, REQ_PUT, _lib as L, default_batch_config
from nvshmem_b200.traffic import c4_batch
from _util import heap_images, requests  # noqa: E402

pytestmark = pytest.mark.gpu


def _device_copy(reqs):
    import torch
    d = torch.from_numpy(np.ascontiguousarray(reqs).view(np.uint8).copy()).cuda()
    torch.cuda.synchronize()
    return d


def _noalloc(d, n, cfg=None):
    return L.lib.nvshmemx_batch_execute_noalloc(ctypes.c_void_p(d.data_ptr()), n,
                                                ctypes.byref(cfg) if cfg is not None else None, None)


def _register_config():
    cfg = default_batch_config()
    cfg.tma_stages = 0
    return cfg


@pytest.mark.parametrize("which", ["default (TMA rings)", "register copy"])
def test_noalloc_matches_batch_execute_on_two_calls(shmem_factory, which):
    npes, heap = 8, 8 << 20
    sh = shmem_factory(npes, heap)
    cfg = default_batch_config() if which.startswith("default") else _register_config()
    for call, seed in enumerate((21, 22)):
        reqs = c4_batch(seed=seed, n=2000, npes=npes, heap=heap, hi=128 << 10)
        for pe in range(npes):
            sh.fill_random(pe, 0, heap, 100 + call)
        with sh.batch(len(reqs), int(reqs["bytes"].sum()), 256) as b:
            b.upload(reqs)
            b.execute(1)
        want = heap_images(sh, npes, heap)
        for pe in range(npes):
            sh.fill_random(pe, 0, heap, 100 + call)
        d = _device_copy(reqs)
        rc = _noalloc(d, len(reqs), cfg)
        assert rc == 0, L.lib.nvshmemx_last_error_string()
        assert sh.status() == 0
        got = heap_images(sh, npes, heap)
        assert np.array_equal(got, want), f"call {call + 1} differs from nvshmemx_batch_execute"


def test_noalloc_rejects_batches_beyond_its_scratch(shmem_factory):
    npes, heap = 2, 8 << 20
    sh = shmem_factory(npes, heap)
    for pe in range(npes):
        sh.fill_random(pe, 0, heap, 5)
    before = heap_images(sh, npes, heap)
    too_many = np.zeros(32769, dtype=L.REQUEST_DTYPE)
    too_many["dst_off"] = heap // 2 + 16 * np.arange(32769)
    too_many["bytes"] = 4
    too_many["dst_pe"] = 1
    assert _noalloc(_device_copy(too_many), len(too_many)) == ERR_NOMEM
    # 4 MiB in 256-byte chunks needs 16384 chunks per request: two overflow the table
    cfg = default_batch_config()
    cfg.chunk_bytes = 256
    big = requests([dict(src_off=0, dst_off=heap // 2, bytes=4 << 20, src_pe=0, dst_pe=1, op=REQ_PUT, dtype=0),
                    dict(src_off=0, dst_off=heap // 2, bytes=4 << 20, src_pe=1, dst_pe=0, op=REQ_PUT, dtype=0),
                    dict(src_off=0, dst_off=heap // 2 - 16, bytes=4, src_pe=1, dst_pe=1, op=REQ_PUT, dtype=0)])
    assert _noalloc(_device_copy(big), len(big), cfg) == ERR_NOMEM
    sh.status()
    assert np.array_equal(heap_images(sh, npes, heap), before)


def test_noalloc_rejects_stream_mode_and_wrapping_offsets(shmem_factory):
    """stream = 1 is refused (its state outlives a call, which the shared
    scratch cannot hold), and an offset whose sum with the size wraps past
    2^64 is a bounds error; in both cases no heap byte changes."""
    npes, heap = 2, 1 << 20
    sh = shmem_factory(npes, heap)
    for pe in range(npes):
        sh.fill_random(pe, 0, heap, 6)
    before = heap_images(sh, npes, heap)
    ok = requests([dict(src_off=0, dst_off=heap // 2, bytes=4096, src_pe=0, dst_pe=1, op=REQ_PUT, dtype=0)])
    cfg = default_batch_config()
    cfg.stream = 1
    assert _noalloc(_device_copy(ok), 1, cfg) == ERR_INVALID
    wrap = requests([dict(src_off=(1 << 64) - 4, dst_off=heap // 2, bytes=8, src_pe=0, dst_pe=1, op=REQ_PUT,
                          dtype=0),
                     dict(src_off=0, dst_off=heap // 2 + 64, bytes=4096, src_pe=0, dst_pe=1, op=REQ_PUT, dtype=0)])
    assert _noalloc(_device_copy(wrap), len(wrap)) == ERR_BOUNDS
    sh.status()
    assert np.array_equal(heap_images(sh, npes, heap), before)
