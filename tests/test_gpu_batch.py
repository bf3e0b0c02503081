"""Parity of the batched engine against the CPU oracle and against the
per-call path: uneven request batches (C4 traffic) must leave every heap
bit-identical whatever the batch configuration, at small sizes byte for byte
and at the full 64-PE x 64 MiB size through per-PE checksums."""
import numpy as np
import pytest

from nvshmem_b200 import (ERR_BOUNDS, ERR_NOMEM, MODE_THREAD, MODE_WARP, REQ_G, REQ_GET, REQ_PUT,
                          requests_bytes)
from nvshmem_b200.traffic import c4_batch, check_disjoint
from oracle.model import Model, checksum
from _util import first_diff, heap_images, random_requests, requests

pytestmark = pytest.mark.gpu

CONFIGS = [
    dict(vec_bytes=16, chunk_bytes=16384, unroll=4, threads=512, ctas_per_sm=2, grab=2),
    dict(vec_bytes=16, chunk_bytes=256, unroll=1, threads=128, ctas_per_sm=1, grab=1),
    dict(vec_bytes=8, chunk_bytes=4096, unroll=8, threads=1024, ctas_per_sm=0, grab=16),
    dict(vec_bytes=4, chunk_bytes=65536, unroll=2, threads=256, ctas_per_sm=4, grab=4),
    # TMA rings: every aligned chunk streamed through shared memory
    dict(vec_bytes=16, chunk_bytes=16384, unroll=4, threads=256, ctas_per_sm=0, grab=2,
         tma_stages=3, tma_stage_bytes=8192, tma_min_bytes=0),
    dict(vec_bytes=16, chunk_bytes=65536, unroll=4, threads=128, ctas_per_sm=0, grab=4,
         tma_stages=4, tma_stage_bytes=4096, tma_min_bytes=2048),
    dict(vec_bytes=16, chunk_bytes=1024, unroll=4, threads=256, ctas_per_sm=1, grab=1,
         tma_stages=2, tma_stage_bytes=1024, tma_min_bytes=16),
    # streaming: planning warps feed executing warps inside one launch
    dict(vec_bytes=16, chunk_bytes=16384, unroll=4, threads=256, ctas_per_sm=0, grab=2,
         tma_stages=3, tma_stage_bytes=8192, tma_min_bytes=512, stream=1, stream_planners=2),
    dict(vec_bytes=16, chunk_bytes=1024, unroll=4, threads=128, ctas_per_sm=1, grab=1,
         tma_stages=2, tma_stage_bytes=4096, tma_min_bytes=0, stream=1, stream_planners=1),
]

STREAM = dict(vec_bytes=16, chunk_bytes=16384, unroll=4, threads=256, ctas_per_sm=0, grab=2,
              tma_stages=3, tma_stage_bytes=8192, tma_min_bytes=512, stream=1, stream_planners=2)


def setup(shmem_factory, npes, heap, seed=7):
    sh = shmem_factory(npes, heap)
    om = Model(npes, heap)
    for pe in range(npes):
        sh.fill_random(pe, 0, heap, seed)
        om.fill_random(pe, 0, heap, seed)
    return sh, om


@pytest.mark.parametrize("cfg", CONFIGS)
def test_c4_small_bit_exact(shmem_factory, cfg):
    npes, heap = 16, 4 << 20
    reqs = c4_batch(seed=4, n=3000, npes=npes, heap=heap, hi=256 << 10)
    assert check_disjoint(reqs)
    sh, om = setup(shmem_factory, npes, heap)
    with sh.batch(len(reqs), int(reqs["bytes"].sum()), 256) as b:
        b.set_config(cfg)
        b.upload(reqs)
        b.execute(1)
        b.execute(2)  # idempotent: sources never overlap destinations
        total, exec_ms = b.execute_direct(1)
        assert 0 < exec_ms <= total
        chunks, _, _ = b.stats()
        assert chunks >= len(reqs) - np.count_nonzero(reqs["bytes"] == 0) // 2
    assert sh.status() == 0
    om.apply_requests(reqs)
    assert first_diff(heap_images(sh, npes, heap), om.heap) is None


@pytest.mark.parametrize("tma", [0, 3])
def test_mixed_ops_and_alignments(shmem_factory, tma):
    npes, heap = 8, 2 << 20
    reqs = random_requests(77, 800, npes, heap, max_bytes=40000)
    sh, om = setup(shmem_factory, npes, heap)
    with sh.batch(len(reqs), int(reqs["bytes"].sum()) + 8 * len(reqs), 256) as b:
        b.set_config(dict(vec_bytes=16, chunk_bytes=1024, unroll=4, threads=256, ctas_per_sm=2, grab=2,
                          tma_stages=tma, tma_stage_bytes=2048, tma_min_bytes=0))
        b.upload(reqs)
        b.execute(1)
    assert sh.status() == 0
    om.apply_requests(reqs)
    assert first_diff(heap_images(sh, npes, heap), om.heap) is None


@pytest.mark.parametrize("mode", [MODE_THREAD, MODE_WARP])
def test_percall_equals_batch(shmem_factory, mode):
    npes, heap = 8, 4 << 20
    reqs = c4_batch(seed=9, n=2000, npes=npes, heap=heap, hi=128 << 10)
    sh, om = setup(shmem_factory, npes, heap)
    with sh.batch(len(reqs), int(reqs["bytes"].sum()), 4096) as b:
        b.upload(reqs)
        b.percall(mode, 1)
        assert sh.status() == 0
        om.apply_requests(reqs)
        assert first_diff(heap_images(sh, npes, heap), om.heap) is None
        b.execute(1)
        assert first_diff(heap_images(sh, npes, heap), om.heap) is None


def test_submit_end_to_end(shmem_factory):
    npes, heap = 8, 4 << 20
    reqs = c4_batch(seed=10, n=2000, npes=npes, heap=heap, hi=128 << 10)
    sh, om = setup(shmem_factory, npes, heap)
    with sh.batch(len(reqs), int(reqs["bytes"].sum()), 4096) as b:
        buf = b.host_buffer()
        buf[:len(reqs)] = reqs
        st, ms = b.submit(buf, len(reqs))
        assert st == 0 and ms > 0
    om.apply_requests(reqs)
    assert first_diff(heap_images(sh, npes, heap), om.heap) is None


def expected_chunks(reqs, chunk):
    """Work items of a batch: ceil(bytes / chunk) per PUT/GET, one per G,
    SIGNAL and P."""
    copies = np.isin(reqs["op"], (REQ_PUT, REQ_GET))
    by = reqs["bytes"].astype(np.int64)
    return int(((by[copies] + chunk - 1) // chunk).sum() + np.count_nonzero(~copies))


@pytest.mark.parametrize("tma", [0, 3])
def test_large_mixed_batch_and_small_table(shmem_factory, tma):
    """6000 requests of mixed ops, widths and alignments (more than one plan
    wave): the heaps match the oracle and the plan makes exactly one work
    item per chunk; a bad request stops the batch, and so does a work-item
    table too small for its chunks (nothing runs)."""
    npes, heap = 8, 32 << 20
    reqs = random_requests(78, 6000, npes, heap, max_bytes=40000)
    assert len(reqs) >= 4096
    chunk = 1024
    cfg = dict(vec_bytes=16, chunk_bytes=chunk, unroll=4, threads=256, ctas_per_sm=2, grab=2,
               tma_stages=tma, tma_stage_bytes=2048, tma_min_bytes=0)
    sh, om = setup(shmem_factory, npes, heap)
    payload = int(reqs["bytes"].sum()) + 8 * len(reqs)
    with sh.batch(len(reqs), payload, 256) as b:
        b.set_config(cfg)
        b.upload(reqs)
        b.execute(1)
        assert b.stats()[0] == expected_chunks(reqs, chunk)
        assert sh.status() == 0
        om.apply_requests(reqs)
        assert first_diff(heap_images(sh, npes, heap), om.heap) is None
        before = heap_images(sh, npes, heap)
        bad = reqs.copy()
        bad[len(bad) // 2]["dst_pe"] = 99
        b.upload(bad)
        with pytest.raises(Exception) as ei:
            b.execute(1)
        assert ei.value.code == ERR_BOUNDS
        sh.status()
        assert np.array_equal(heap_images(sh, npes, heap), before)
    # a table of len(reqs) + 1 items cannot hold the 1 KiB chunks
    with sh.batch(len(reqs), 0, 256) as b:
        b.set_config(cfg)
        b.upload(reqs)
        with pytest.raises(Exception) as ei:
            b.execute(1)
        assert ei.value.code == ERR_NOMEM
    sh.status()
    assert np.array_equal(heap_images(sh, npes, heap), before)


def test_large_arena_offsets(shmem_factory):
    """16 PEs x 1 GiB (a 16 GiB arena: work-item addresses far above 4 GiB
    from the base). The batch leaves the same heaps as one call per
    request."""
    npes, heap = 16, 1 << 30
    reqs = c4_batch(seed=51, n=20000, npes=npes, heap=heap, hi=64 << 10)
    sh = shmem_factory(npes, heap)
    with sh.batch(len(reqs), int(reqs["bytes"].sum()), 256) as b:
        for pe in range(npes):
            sh.fill_random(pe, 0, heap, 12)
        b.upload(reqs)
        b.execute(1)
        batched = [sh.checksum(pe, 0, heap) for pe in range(npes)]
        for pe in range(npes):
            sh.fill_random(pe, 0, heap, 12)
        b.percall(MODE_WARP, 1)
        assert [sh.checksum(pe, 0, heap) for pe in range(npes)] == batched
    assert sh.status() == 0


def split_ends(n):
    """Piece boundaries of a pipelined submit, as the library splits."""
    return [n] if n < 8192 else [(n // 4) & ~255, n]


@pytest.mark.parametrize("n", [8191, 8192, 8193, 12345, 40000])
def test_submit_at_the_split_point(shmem_factory, n):
    """One piece below 8192 requests, two from 8192 on (the first a quarter
    in whole 256-request blocks); same heaps either way."""
    npes, heap = 8, 32 << 20
    reqs = c4_batch(seed=50 + n, n=n, npes=npes, heap=heap, hi=8 << 10)
    sh, om = setup(shmem_factory, npes, heap)
    with sh.batch(len(reqs), int(reqs["bytes"].sum()), 256) as b:
        st, _ = b.submit(reqs.copy())
        assert st == 0
        om.apply_requests(reqs)
        assert first_diff(heap_images(sh, npes, heap), om.heap) is None
        chunks = b.stats()[0]
        b.execute(1)
        assert b.stats()[0] == chunks


@pytest.mark.parametrize("n", [20000, 40000])
@pytest.mark.parametrize("cfg", [None, CONFIGS[0]], ids=["tma", "register"])
def test_submit_pipelined(shmem_factory, cfg, n):
    """A submit of 8192 or more requests in a graph configuration runs in
    pieces: each executes while the next is copied and planned (appending its
    chunks after the previous piece's)."""
    npes, heap = 16, 32 << 20
    reqs = c4_batch(seed=48, n=n, npes=npes, heap=heap, hi=16 << 10)
    sh, om = setup(shmem_factory, npes, heap)
    with sh.batch(len(reqs), int(reqs["bytes"].sum()), 256) as b:
        if cfg:
            b.set_config(cfg)
        buf = b.host_buffer()
        buf[:] = reqs
        st, ms = b.submit(buf, len(reqs))
        assert st == 0 and ms > 0
        chunks = b.stats()[0]
        om.apply_requests(reqs)
        assert first_diff(heap_images(sh, npes, heap), om.heap) is None
        # the requests stay resident; one-piece execution plans the same chunks
        b.execute(1)
        assert b.stats()[0] == chunks
        assert first_diff(heap_images(sh, npes, heap), om.heap) is None
        # a bad request in the last piece: the pieces before it have run, the
        # last has not
        n0 = split_ends(len(reqs))[-2]
        for pe in range(npes):
            sh.fill_random(pe, 0, heap, 8)
        om2 = Model(npes, heap)
        for pe in range(npes):
            om2.fill_random(pe, 0, heap, 8)
        bad = reqs.copy()
        bad[n0 + 100]["dst_pe"] = 99
        st, _ = b.submit(bad)
        assert st == ERR_BOUNDS
        om2.apply_requests(reqs[:n0])
        assert first_diff(heap_images(sh, npes, heap), om2.heap) is None
    sh.status()


@pytest.mark.parametrize("n", [5000, 20000], ids=["one_piece", "two_pieces"])
@pytest.mark.parametrize("cfg", [None, CONFIGS[0]], ids=["tma", "register"])
def test_submit_compact(shmem_factory, cfg, n):
    """The 16-byte compact form through the pinned buffer: the same heaps as
    the oracle, the full form left resident for later executions, and an
    invalid compact request in the last piece reported after the pieces
    before it have run."""
    from nvshmem_b200 import ERR_INVALID, to_compact
    npes, heap = 16, 32 << 20
    reqs = c4_batch(seed=49, n=n, npes=npes, heap=heap, hi=16 << 10)
    sh, om = setup(shmem_factory, npes, heap)
    with sh.batch(len(reqs), int(reqs["bytes"].sum()), 256) as b:
        if cfg:
            b.set_config(cfg)
        buf = b.host_buffer_compact()
        buf[:n] = to_compact(reqs)
        st, ms = b.submit_compact(buf, n)
        assert st == 0 and ms > 0
        om.apply_requests(reqs)
        assert first_diff(heap_images(sh, npes, heap), om.heap) is None
        b.execute(1)  # runs the expanded requests the plan kernels left
        assert sh.status() == 0
        assert first_diff(heap_images(sh, npes, heap), om.heap) is None
        # bits outside the fields of one request of the last piece
        last = split_ends(n)
        n0 = last[-2] if len(last) > 1 else 0
        for pe in range(npes):
            sh.fill_random(pe, 0, heap, 8)
        om2 = Model(npes, heap)
        for pe in range(npes):
            om2.fill_random(pe, 0, heap, 8)
        bad = to_compact(reqs)
        bad[n0 + 7]["meta"] |= 1 << 30
        buf[:n] = bad
        st, _ = b.submit_compact(buf, n)
        assert st == ERR_INVALID
        om2.apply_requests(reqs[:n0])
        assert first_diff(heap_images(sh, npes, heap), om2.heap) is None
    sh.status()


@pytest.mark.parametrize("where", ["pinned", "pageable"])
def test_submit_compact_first_piece_error_and_host_memory(shmem_factory, where):
    """Two pieces of compact requests, from the batch's pinned buffer (the
    first piece planned straight from host memory) or from ordinary host
    memory (copied first): a valid batch matches the oracle, and an invalid
    request in the first piece stops everything."""
    from nvshmem_b200 import ERR_INVALID, to_compact
    npes, heap, n = 16, 32 << 20, 30000
    reqs = c4_batch(seed=50, n=n, npes=npes, heap=heap, hi=16 << 10)
    sh, om = setup(shmem_factory, npes, heap)
    with sh.batch(len(reqs), int(reqs["bytes"].sum()), 256) as b:
        comp = to_compact(reqs)
        if where == "pinned":
            buf = b.host_buffer_compact()
            buf[:n] = comp
            src = buf[:n]
        else:
            src = comp.copy()
        st, ms = b.submit_compact(src, n)
        assert st == 0 and ms > 0
        om.apply_requests(reqs)
        assert first_diff(heap_images(sh, npes, heap), om.heap) is None
        for pe in range(npes):
            sh.fill_random(pe, 0, heap, 9)
        before = heap_images(sh, npes, heap)
        bad = comp.copy()
        bad[123]["meta"] |= 1 << 31
        if where == "pinned":
            buf[:n] = bad
            src = buf[:n]
        else:
            src = bad
        st, _ = b.submit_compact(src, n)
        assert st == ERR_INVALID
        assert np.array_equal(heap_images(sh, npes, heap), before)
    sh.status()


def test_submit_compact_needs_a_graph_configuration(shmem_factory):
    from nvshmem_b200 import ShmemError, to_compact
    sh, _ = setup(shmem_factory, 4, 1 << 20)
    reqs = c4_batch(seed=50, n=100, npes=4, heap=1 << 20, hi=1024)
    with sh.batch(len(reqs), int(reqs["bytes"].sum()), 256) as b:
        b.set_config(STREAM)
        with pytest.raises(ShmemError):
            b.submit_compact(to_compact(reqs))
    sh.status()


def test_stream_submit(shmem_factory):
    """End-to-end in stream mode (copy, then the streaming kernel): batches of
    several sizes in a row through the pinned buffer and from ordinary
    (pageable) host memory, then graph-mode and stream-mode executions of the
    resident requests on the same object."""
    npes, heap = 16, 16 << 20
    sh, om = setup(shmem_factory, npes, heap)
    with sh.batch(30000, 256 << 20, 4096) as b:
        b.set_config(STREAM)
        buf = b.host_buffer()
        for seed, n, pinned in ((41, 30000, True), (42, 9000, False), (46, 777, False), (47, 8192, True)):
            reqs = c4_batch(seed=seed, n=n, npes=npes, heap=heap, hi=16 << 10)
            if pinned:
                buf[:len(reqs)] = reqs
                st, ms = b.submit(buf, len(reqs))
            else:
                st, ms = b.submit(reqs.copy())
            assert st == 0 and ms > 0
            om.apply_requests(reqs)
            assert first_diff(heap_images(sh, npes, heap), om.heap) is None, (seed, n)
        # the submitted requests stay resident: device-resident execution (the
        # graph of the streaming kernel) of the last batch
        b.execute(2)
        om.apply_requests(reqs)
        assert first_diff(heap_images(sh, npes, heap), om.heap) is None
        # switching between graph and stream modes on one object stays exact
        reqs = c4_batch(seed=43, n=2500, npes=npes, heap=heap, hi=128 << 10)
        b.upload(reqs)
        b.set_config(dict(STREAM, stream=0))
        b.execute(1)
        b.set_config(STREAM)
        b.execute(1)
        om.apply_requests(reqs)
        om.apply_requests(reqs)
        assert first_diff(heap_images(sh, npes, heap), om.heap) is None
        # an empty submit does nothing
        st, _ = b.submit(buf, 0)
        assert st == 0
    assert sh.status() == 0


def test_stream_skips_invalid_requests_individually(shmem_factory):
    npes, heap = 4, 1 << 20
    sh, om = setup(shmem_factory, npes, heap)
    good = c4_batch(seed=44, n=600, npes=npes, heap=heap, hi=8 << 10)
    bad = requests([dict(src_off=0, dst_off=heap - 16, bytes=64, src_pe=0, dst_pe=1, op=REQ_PUT, dtype=0),
                    dict(src_off=0, dst_off=heap // 2, bytes=64, src_pe=0, dst_pe=9, op=REQ_PUT, dtype=0)])
    reqs = np.concatenate([good[:300], bad, good[300:]])
    with sh.batch(len(reqs), int(good["bytes"].sum()) + 128, 256) as b:
        b.set_config(dict(STREAM, chunk_bytes=4096))
        b.upload(reqs)
        with pytest.raises(Exception):
            b.execute(1)  # reports the first bad request ...
    sh.status()
    om.apply_requests(good)  # ... but the valid ones ran
    assert first_diff(heap_images(sh, npes, heap), om.heap) is None


def test_bad_request_rejected_not_executed(shmem_factory):
    npes, heap = 4, 1 << 20
    sh, om = setup(shmem_factory, npes, heap)
    reqs = requests([dict(src_off=0, dst_off=heap - 16, bytes=64, src_pe=0, dst_pe=1, op=REQ_PUT, dtype=0),
                     dict(src_off=0, dst_off=heap // 2, bytes=64, src_pe=0, dst_pe=9, op=REQ_PUT, dtype=0)])
    with sh.batch(4, 1 << 16, 256) as b:
        b.upload(reqs)
        with pytest.raises(Exception):
            b.execute(1)
    sh.status()
    assert first_diff(heap_images(sh, npes, heap), om.heap) is None


WRAP = (1 << 64) - 4  # offset + 8 wraps to 4: must be rejected, never executed


@pytest.mark.parametrize("cfg", [CONFIGS[0], CONFIGS[4], STREAM])
@pytest.mark.parametrize("field", ["src_off", "dst_off"])
def test_wrapping_offsets_rejected(shmem_factory, cfg, field):
    """An offset near 2^64 whose sum with the size wraps around is a bounds
    error: the planner rejects it (graph path: nothing runs; stream mode:
    that request alone is skipped) and no byte outside the valid requests
    changes."""
    npes, heap = 4, 1 << 20
    sh, om = setup(shmem_factory, npes, heap)
    good = c4_batch(seed=48, n=200, npes=npes, heap=heap, hi=4 << 10)
    row = dict(src_off=0, dst_off=heap // 2 - 64, bytes=8, src_pe=1, dst_pe=2, op=REQ_PUT, dtype=0)
    row[field] = WRAP
    bad = requests([row])
    reqs = np.concatenate([good[:100], bad, good[100:]])
    with sh.batch(len(reqs), int(good["bytes"].sum()) + 64, 256) as b:
        b.set_config(cfg)
        b.upload(reqs)
        with pytest.raises(Exception) as ei:
            b.execute(1)
        assert ei.value.code == ERR_BOUNDS
    sh.status()
    if cfg.get("stream"):
        om.apply_requests(good)
    assert first_diff(heap_images(sh, npes, heap), om.heap) is None


def test_empty_batch(shmem_factory):
    sh = shmem_factory(2, 1 << 20)
    with sh.batch(16, 1 << 16, 256) as b:
        b.upload(requests([]))
        b.execute(3)
    assert sh.status() == 0


@pytest.mark.parametrize("mode", ["register", "tma", "stream"])
def test_c4_full_size_checksums(shmem_factory, mode):
    """The benchmark's batch: 64 PEs x 64 MiB, 100,000 requests."""
    npes, heap = 64, 64 << 20
    reqs = c4_batch(seed=4, n=100_000, npes=npes, heap=heap)
    assert check_disjoint(reqs)
    sh, om = setup(shmem_factory, npes, heap, seed=44)
    with sh.batch(len(reqs), int(reqs["bytes"].sum()), 4096) as b:
        if mode == "register":
            b.set_config(CONFIGS[0])
        elif mode == "tma":
            b.set_config(dict(vec_bytes=16, chunk_bytes=16384, unroll=4, threads=256, ctas_per_sm=0, grab=2,
                              tma_stages=3, tma_stage_bytes=8192, tma_min_bytes=1024))
        else:
            b.set_config(STREAM)
        b.upload(reqs)
        b.execute(3)
        if mode == "stream":
            buf = b.host_buffer()
            buf[:len(reqs)] = reqs
            assert b.submit(buf, len(reqs))[0] == 0
    assert sh.status() == 0
    om.apply_requests(reqs)
    for pe in range(npes):
        assert sh.checksum(pe, 0, heap) == checksum(om.heap[pe]), f"PE {pe}"
    assert requests_bytes(reqs) > 0
