"""Parity of the collective-launch patterns against the CPU oracle: the C1
ping-pong, C2 all-to-all rounds (every mode, put and get, every element type,
sizes from 8 B up) and the C3 halo exchange; plus the bounded-wait and
barrier failure paths, which must end with NVSHMEMX_ERR_TIMEOUT, never hang."""
import numpy as np
import pytest

from nvshmem_b200 import (DT_DOUBLE, DT_FLOAT, DT_INT, ERR_INVALID, ERR_TIMEOUT, MODE_BLOCK,
                          MODE_BULK, MODE_THREAD, MODE_WARP, REQ_GET, REQ_PUT)
from nvshmem_b200.traffic import c3_block
from oracle.model import Model, checksum
from _util import first_diff, heap_images

pytestmark = pytest.mark.gpu


def test_pingpong_flags_and_data(shmem_factory):
    heap = 1 << 20
    sh = shmem_factory(2, heap)
    om = Model(2, heap)
    flag = sh.alloc(4)
    data = sh.alloc(4096 * 4)
    assert (flag, data) == (om.alloc(4), om.alloc(4096 * 4))
    for pe in range(2):
        sh.fill_random(pe, data, 4096 * 4, 5)
        om.fill_random(pe, data, 4096 * 4, 5)
    iters, skip = 1000, 20
    ns, total = sh.pingpong(flag, data, 4096, iters, skip)
    assert sh.status() == 0
    om.pingpong(flag, data, 4096, iters + skip)
    assert first_diff(heap_images(sh, 2, heap), om.heap) is None
    assert total > 0 and np.all(ns > 0)


def test_pingpong_flag_only_latency(shmem_factory):
    sh = shmem_factory(2, 1 << 20)
    flag = sh.alloc(4)
    ns, total = sh.pingpong(flag, 0, 0, 10000, 20)
    assert sh.status() == 0
    assert sh.read(0, flag, 4, np.int32)[0] == 10020
    assert sh.read(1, flag, 4, np.int32)[0] == 10020
    p50 = float(np.median(ns))
    assert 0 < p50 < 50_000  # a round trip through L2, far below 50 us
    # the flags are reset by the call: a second exchange on the same words
    # still waits for every echo (it would run far faster if the waits passed
    # on the values the first one left)
    ns2, _ = sh.pingpong(flag, 0, 0, 10000, 20)
    assert sh.status() == 0
    assert 0.5 * p50 < float(np.median(ns2)) < 2 * p50
    assert sh.read(1, flag, 4, np.int32)[0] == 10020


@pytest.mark.parametrize("counted", [False, True])
@pytest.mark.parametrize("ctas", [1, 4])
def test_barrier_latency(shmem_factory, ctas, counted):
    sh = shmem_factory(8, 1 << 20)
    ns, total = sh.barrier_latency(ctas, 2000, counted)
    assert sh.status() == 0
    assert 0 < np.median(ns) < 100_000


def test_offload_barrier(shmem_factory):
    sh = shmem_factory(8, 1 << 20)
    us = sh.offload_barrier(200)
    assert sh.status() == 0 and us > 0


@pytest.mark.parametrize("mode", [MODE_THREAD, MODE_WARP, MODE_BLOCK, MODE_BULK])
@pytest.mark.parametrize("op", [REQ_PUT, REQ_GET])
def test_alltoall_small_sizes(shmem_factory, mode, op):
    npes, heap = 8, 4 << 20
    sh = shmem_factory(npes, heap)
    om = Model(npes, heap)
    for pe in range(npes):
        sh.fill_random(pe, 0, heap, 1)
        om.fill_random(pe, 0, heap, 1)
    for dtype, nbytes in [(DT_INT, 8), (DT_FLOAT, 4100), (DT_DOUBLE, 65536), (DT_INT, 123456)]:
        send, recv = 0, heap // 2
        sh.alltoall(op, dtype, send, recv, nbytes, rounds=2, mode=mode, ctas_per_pe=3)
        assert sh.status() == 0
        om.alltoall(1 if op == REQ_GET else 0, send, recv, nbytes, rounds=2)
    assert first_diff(heap_images(sh, npes, heap), om.heap) is None


@pytest.mark.parametrize("host_rounds", [False, True], ids=["device_barrier", "host_barrier"])
def test_alltoall_rotating_sets(shmem_factory, host_rounds):
    """Rounds over rotating buffer sets, in one launch with the device barrier
    and in the prototype's structure (a launch per round, then the host's
    nvshmem_barrier_all)."""
    npes, heap = 8, 8 << 20
    sh = shmem_factory(npes, heap)
    om = Model(npes, heap)
    for pe in range(npes):
        sh.fill_random(pe, 0, heap, 9)
        om.fill_random(pe, 0, heap, 9)
    nbytes, stride = 65536, 1 << 20
    sh.alltoall(REQ_PUT, DT_FLOAT, 0, 4 << 20, nbytes, rounds=5, nsets=3, set_stride=stride,
                mode=MODE_BULK, ctas_per_pe=4, host_rounds=host_rounds)
    om.alltoall(0, 0, 4 << 20, nbytes, rounds=5, nsets=3, set_stride=stride)
    assert sh.status() == 0
    assert first_diff(heap_images(sh, npes, heap), om.heap) is None


def test_alltoall_large_on_device_compare(shmem_factory):
    """64 MiB messages: every received block equals the sender's block."""
    npes, nbytes = 8, 64 << 20
    heap = 2 * npes * nbytes
    sh = shmem_factory(npes, heap)
    for pe in range(npes):
        sh.fill_random(pe, 0, npes * nbytes, 21)
        sh.memset(pe, npes * nbytes, 0, npes * nbytes)
    sh.alltoall(REQ_PUT, DT_DOUBLE, 0, npes * nbytes, nbytes, mode=MODE_BLOCK, ctas_per_pe=18)
    assert sh.status() == 0
    for p in range(npes):
        for q in range(npes):
            if p == q:
                continue
            assert sh.compare(q, npes * nbytes + p * nbytes, p, q * nbytes, nbytes) == 0


@pytest.mark.parametrize("env", [None, "5"], ids=["default", "NVSHMEM_CTAS_PER_PE=5"])
def test_ctas_per_pe_zero_picks_a_default(shmem_factory, monkeypatch, env):
    """ctas_per_pe 0: NVSHMEM_CTAS_PER_PE when set, else the operation's own
    default; the heaps match the oracle either way."""
    if env:
        monkeypatch.setenv("NVSHMEM_CTAS_PER_PE", env)
    else:
        monkeypatch.delenv("NVSHMEM_CTAS_PER_PE", raising=False)
    npes, heap = 8, 4 << 20
    sh = shmem_factory(npes, heap)
    om = Model(npes, heap)
    for pe in range(npes):
        sh.fill_random(pe, 0, heap, 3)
        om.fill_random(pe, 0, heap, 3)
    for mode in (MODE_BLOCK, MODE_BULK):
        sh.alltoall(REQ_PUT, DT_FLOAT, 0, heap // 2, 65536 + 4, rounds=2, mode=mode, ctas_per_pe=0)
        om.alltoall(0, 0, heap // 2, 65536 + 4, rounds=2)
    assert sh.status() == 0
    assert first_diff(heap_images(sh, npes, heap), om.heap) is None


def test_alltoall_every_c2_size(shmem_factory):
    """The whole C2 sweep, 26 message sizes from 8 B to 256 MiB (int, float
    and double in turn), put and get through the TMA form: after each call
    PE q's receive slot p holds exactly PE p's send slot q, and no other byte
    of the receive area changed."""
    from nvshmem_b200 import DT_DOUBLE
    from nvshmem_b200.traffic import c2_sizes
    npes, top = 8, 256 << 20
    heap = 2 * npes * top + (2 << 20)
    sh = shmem_factory(npes, heap)
    dts = (DT_INT, DT_FLOAT, DT_DOUBLE)
    for i, nbytes in enumerate(c2_sizes()):
        dt = dts[i % 3]
        for op in (REQ_PUT, REQ_GET):
            recv = npes * nbytes
            for pe in range(npes):
                sh.fill_random(pe, 0, npes * nbytes, 100 + i)
                sh.memset(pe, recv, 0, npes * nbytes + 64)
            sh.alltoall(op, dt, 0, recv, nbytes, mode=MODE_BULK, ctas_per_pe=18)
            assert sh.status() == 0
            zero = checksum(np.zeros(nbytes, np.uint8))
            for p in range(npes):
                for q in range(npes):
                    if p != q:
                        assert sh.compare(q, recv + p * nbytes, p, q * nbytes, nbytes) == 0, (nbytes, op, p, q)
                # its own slot and the 64 bytes past the area stay zero
                assert sh.checksum(p, recv + p * nbytes, nbytes) == zero, (nbytes, op, p)
                assert sh.checksum(p, recv + npes * nbytes, 64) == checksum(np.zeros(64, np.uint8))


@pytest.mark.parametrize("offload", [False, True], ids=["persistent", "offload_barrier"])
@pytest.mark.parametrize("n", [8, 32, 40])
def test_halo_bit_exact(shmem_factory, n, offload):
    npes = 8
    block = n * n * n * 8
    heap = block + 6 * n * n * 8 + 4096
    heap = (heap + 4095) // 4096 * 4096
    sh = shmem_factory(npes, heap)
    om = Model(npes, heap)
    block_off, ghost_off, sig_off = 0, block, block + 6 * n * n * 8
    for pe in range(npes):
        b = c3_block(n, pe)
        sh.write(pe, block_off, b)
        om.heap[pe, block_off:block_off + block] = b.view(np.uint8)
    sh.halo(2, 2, 2, n, block_off, ghost_off, sig_off, iters=5, ctas_per_pe=4, offload=offload)
    assert sh.status() == 0
    om.halo(2, 2, 2, n, block_off, ghost_off, sig_off, 5)
    assert first_diff(heap_images(sh, npes, heap), om.heap) is None


@pytest.mark.parametrize("offload", [False, True], ids=["persistent", "offload_barrier"])
def test_halo_benchmark_size_bit_exact(shmem_factory, offload):
    """The benchmark's halo: 8 PEs, 256^3 float64 blocks (N(0,1), seed 3),
    3 iterations, as many CTAs per PE as stay co-resident; every PE's heap
    (block, ghosts, signal words and the bytes past them) is compared with the
    oracle through per-PE checksums."""
    npes, n, iters = 8, 256, 3
    block = n * n * n * 8
    ghosts = 6 * n * n * 8
    heap = block + ghosts + 4096
    sh = shmem_factory(npes, heap)
    om = Model(npes, heap)
    for pe in range(npes):
        b = c3_block(n, pe)
        sh.write(pe, 0, b)
        om.heap[pe, :block] = b.view(np.uint8)
        sh.memset(pe, block, 0, heap - block)
    sh.halo(2, 2, 2, n, 0, block, block + ghosts, iters=iters, ctas_per_pe=0, offload=offload)
    assert sh.status() == 0
    om.halo(2, 2, 2, n, 0, block, block + ghosts, iters)
    for pe in range(npes):
        assert sh.checksum(pe, 0, heap) == checksum(om.heap[pe]), f"PE {pe}"


def test_host_checks_reject_wrapping_arguments(shmem_factory):
    """Offsets and counts whose sums or products wrap past 2^64 are invalid
    arguments, refused on the host before any launch."""
    sh = shmem_factory(8, 1 << 20)
    huge = (1 << 64) - 8
    with pytest.raises(Exception) as ei:
        sh.alltoall(REQ_PUT, DT_INT, huge, 0, 64)
    assert ei.value.code == ERR_INVALID
    with pytest.raises(Exception) as ei:  # (nsets - 1) * set_stride wraps
        sh.alltoall(REQ_PUT, DT_INT, 0, 4096, 64, rounds=2, nsets=3, set_stride=1 << 63)
    assert ei.value.code == ERR_INVALID
    with pytest.raises(Exception) as ei:  # n^3 * 8 wraps
        sh.halo(2, 2, 2, 1 << 22, 0, 0, 0, 1, 1)
    assert ei.value.code == ERR_INVALID
    with pytest.raises(Exception) as ei:
        sh.halo(2, 2, 2, 4, 0, 4096, huge, 1, 1)
    assert ei.value.code == ERR_INVALID
    with pytest.raises(Exception) as ei:
        sh.wait_test(huge, 1, 1000)
    assert ei.value.code == ERR_INVALID
    with pytest.raises(Exception) as ei:  # (rows - 1) * stride + 8 wraps to 0
        sh.strided_read(0, 8, 1, (1 << 61), 8, 1, 1)
    assert ei.value.code == ERR_INVALID
    with pytest.raises(Exception) as ei:  # one row past the heap
        sh.strided_read(0, 8, 1, (1 << 20) // 8 + 1, 8, 1, 1)
    assert ei.value.code == ERR_INVALID
    # the status word reports the first host-side refusal once, and no device
    # error: nothing was launched
    assert sh.status() == ERR_INVALID
    assert sh.status() == 0
    sh2 = shmem_factory(2, 1 << 20)
    with pytest.raises(Exception) as ei:
        sh2.pingpong(huge, 0, 0, 1)
    assert ei.value.code == ERR_INVALID


def test_strided_read_reads_the_rows_it_is_given(shmem_factory):
    """nvshmemx_op_strided_read (the halo's x-face read ceiling): a valid
    call over the last row of the heap runs and leaves the status clean."""
    heap = 1 << 20
    sh = shmem_factory(8, heap)
    n = 64
    ms = sh.strided_read(0, (n - 1) * 8, 2, heap // (8 * n), 8 * n, 4, 3)
    assert ms > 0
    assert sh.status() == 0


def test_wait_timeout_reports_and_returns(shmem_factory):
    sh = shmem_factory(2, 1 << 20)
    flag = sh.alloc(4)
    st = sh.wait_test(flag, 12345, 2_000_000)  # 2 ms, nothing ever sets it
    assert st == ERR_TIMEOUT
    assert sh.status() == ERR_TIMEOUT
    sh.write(0, flag, np.array([12345], np.int32))
    assert sh.wait_test(flag, 12345, 2_000_000) == 0
    assert sh.status() == 0


def test_barrier_with_missing_pe_times_out(shmem_factory):
    sh = shmem_factory(4, 1 << 20)
    st = sh.barrier_fault_test(2, 5_000_000)
    assert st == ERR_TIMEOUT
    assert sh.status() == ERR_TIMEOUT
    # the context is still usable afterwards
    ns, _ = sh.barrier_latency(1, 100)
    assert sh.status() == 0
