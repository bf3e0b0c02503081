"""The CPU oracle against independent numpy restatements of the prototype's
semantics (no GPU): allocator offsets, put/get/p/g, request lists, all-to-all,
halo, ping-pong, the deterministic fill and the checksum."""
import numpy as np
import pytest

from nvshmem_b200 import REQ_G, REQ_GET, REQ_P, REQ_PUT, REQ_SIGNAL
from nvshmem_b200.traffic import GOLDEN, c3_block, splitmix64
from oracle.model import Model, checksum, fnv1a
from _util import random_requests


def test_alloc_offsets_no_padding():
    # nvshmem.cu:775-802: cumulative sums, no alignment, -1 past the limit
    m = Model(3, 4096, heap_limit=100)
    sizes = [3, 1, 8, 0, 17, 70]
    offs = [m.alloc(s) for s in sizes]
    assert offs == [0, 3, 4, 12, 12, 29]
    assert m.alloc(2) == -1  # 99 + 2 > 100
    assert m.alloc(1) == 99
    m.cleanup()
    assert m.alloc(5) == 0
    assert m.ptr(5, 2) == 5 and m.ptr(5000, 0) == -1 and m.ptr(0, 3) == -1


def test_alloc_per_pe_then_collective_requires_symmetry():
    m = Model(2, 4096)
    assert m.alloc(10, pe=0) == 0
    assert m.alloc(11, pe=1) == 0
    assert m.alloc(4) == -1  # tails 10 and 11 differ
    m.alloc(1, pe=0)
    assert m.alloc(4) == 11


def test_put_get_p_g_are_bit_copies():
    m = Model(2, 1024)
    rng = np.random.default_rng(0)
    m.heap[:] = rng.integers(0, 256, size=m.heap.shape, dtype=np.uint8)
    ref = m.heap.copy()
    m.put(4, 100, 0, 200, 10, 1)  # PE 0 puts 10 ints from its 200 to PE 1's 100
    ref[1, 100:140] = ref[0, 200:240]
    m.get(8, 1, 500, 16, 3, 0)  # PE 1 gets 3 doubles from PE 0's 16 into its 500
    ref[1, 500:524] = ref[0, 16:40]
    m.p(8, 800, 0x0123456789ABCDEF, 0)
    ref[0, 800:808] = np.frombuffer((0x0123456789ABCDEF).to_bytes(8, "little"), np.uint8)
    assert m.g(4, 800, 0) == 0x89ABCDEF
    m.put(4, 0, 0, 0, 0, 1)  # len 0 and negative lengths copy nothing
    m.put(4, 0, 0, 0, -5, 1)
    assert np.array_equal(m.heap, ref)


def _numpy_apply(heap, reqs):
    for r in reqs:
        op, w = int(r["op"]), 8 if r["dtype"] == 2 else 4
        s, d = int(r["src_off"]), int(r["dst_off"])
        sp, dp = int(r["src_pe"]), int(r["dst_pe"])
        if op in (REQ_PUT, REQ_GET):
            heap[dp, d:d + int(r["bytes"])] = heap[sp, s:s + int(r["bytes"])]
        elif op == REQ_SIGNAL:
            heap[dp, d:d + 4] = np.frombuffer(np.int32(r["value"]).tobytes(), np.uint8)
        elif op == REQ_P:
            heap[dp, d:d + w] = np.frombuffer(int(r["src_off"]).to_bytes(8, "little")[:w], np.uint8)
        elif op == REQ_G:
            heap[dp, d:d + w] = heap[sp, s:s + w]


def test_requests_match_numpy():
    npes, heap = 4, 1 << 18
    reqs = random_requests(5, 200, npes, heap, max_bytes=4000)
    m = Model(npes, heap)
    for pe in range(npes):
        m.fill_random(pe, 0, heap, 3)
    ref = m.heap.copy()
    m.apply_requests(reqs)
    _numpy_apply(ref, reqs)
    assert np.array_equal(m.heap, ref)


@pytest.mark.parametrize("op", [0, 1])
def test_alltoall_matches_numpy(op):
    npes, nbytes = 5, 24
    heap = 2 * npes * nbytes
    m = Model(npes, heap)
    for pe in range(npes):
        m.fill_random(pe, 0, heap, 1)
    ref = m.heap.copy()
    m.alltoall(op, 0, npes * nbytes, nbytes)
    for p in range(npes):
        for q in range(npes):
            if p != q:
                ref[q, npes * nbytes + p * nbytes:npes * nbytes + (p + 1) * nbytes] = ref[p, q * nbytes:(q + 1) * nbytes]
    assert np.array_equal(m.heap, ref)


def test_halo_matches_numpy():
    n, npes = 6, 8
    block = n ** 3 * 8
    heap = block + 6 * n * n * 8 + 64
    m = Model(npes, heap)
    blocks = [c3_block(n, pe) for pe in range(npes)]
    for pe in range(npes):
        m.heap[pe, :block] = blocks[pe].view(np.uint8)
    m.halo(2, 2, 2, n, 0, block, block + 6 * n * n * 8, 3)

    def nbr(pe, d):
        x, y, z = pe % 2, (pe // 2) % 2, pe // 4
        s = 1 if d & 1 else -1
        if d < 2:
            x = (x + s) % 2
        elif d < 4:
            y = (y + s) % 2
        else:
            z = (z + s) % 2
        return x + 2 * (y + 2 * z)

    for pe in range(npes):
        b = blocks[pe].reshape(n, n, n)  # [z][y][x]
        faces = [b[:, :, 0], b[:, :, -1], b[:, 0, :], b[:, -1, :], b[0, :, :], b[-1, :, :]]
        for d in range(6):
            nb = nbr(pe, d)
            g = m.heap[nb, block + (d ^ 1) * n * n * 8: block + ((d ^ 1) + 1) * n * n * 8].view(np.float64)
            assert np.array_equal(g.reshape(n, n), faces[d])
    sig = m.heap[:, block + 6 * n * n * 8: block + 6 * n * n * 8 + 24].copy().view(np.int32)
    assert np.all(sig == 3)


def test_pingpong_sequence():
    m = Model(2, 4096)
    m.fill_random(0, 64, 400, 1)
    m.fill_random(1, 64, 400, 2)
    d0 = m.heap[0, 64:464].copy()
    s0, s1 = m.pingpong(0, 64, 100, 50)
    assert list(s1) == list(range(1, 51)) and list(s0) == list(range(1, 51))
    assert np.array_equal(m.heap[1, 64:464], d0) and np.array_equal(m.heap[0, 64:464], d0)


def test_fill_random_is_the_splitmix_stream():
    m = Model(3, 256)
    m.fill_random(2, 5, 200, 99)
    key = splitmix64(np.uint64(99) ^ np.uint64(2 << 48))
    words = splitmix64(key + np.arange(32, dtype=np.uint64))
    expect = words.view(np.uint8)
    assert np.array_equal(m.heap[2, 5:205], expect[5:205])
    assert not m.heap[2, :5].any() and not m.heap[2, 205:].any()


def test_checksum_definition():
    a = np.arange(64, dtype=np.uint64) * np.uint64(0x1234567)
    with np.errstate(over="ignore"):
        s = splitmix64(a ^ (np.arange(64, dtype=np.uint64) * GOLDEN)).sum(dtype=np.uint64)
    assert checksum(a.view(np.uint8)) == int(s)
    assert fnv1a(np.frombuffer(b"a", np.uint8)) == 0xaf63dc4c8601ec8c
