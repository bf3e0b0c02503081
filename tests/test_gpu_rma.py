"""Parity of the one-sided device API (p/g/put/get/signal) against the CPU
oracle: request lists executed through nvshmem_{int,float,double}_{p,g,put,get}
and the warp / block / TMA-bulk cooperative forms must leave heap images
bit-identical to the oracle's."""
import numpy as np
import pytest

from nvshmem_b200 import (DT_DOUBLE, DT_FLOAT, DT_INT, ERR_BOUNDS, MODE_BLOCK,
                          MODE_BULK, MODE_THREAD, MODE_WARP, REQ_G, REQ_GET,
                          REQ_P, REQ_PUT, REQ_SIGNAL)
from oracle.model import Model
from _util import first_diff, heap_images, random_requests, requests

pytestmark = pytest.mark.gpu

HEAP = 1 << 20
MODES = [MODE_THREAD, MODE_WARP, MODE_BLOCK, MODE_BULK]


def start(shmem_factory, npes, heap=HEAP, seed=11):
    sh = shmem_factory(npes, heap)
    om = Model(npes, heap)
    for pe in range(npes):
        sh.fill_random(pe, 0, heap, seed)
        om.fill_random(pe, 0, heap, seed)
    return sh, om


def test_fill_matches_oracle(shmem_factory):
    sh, om = start(shmem_factory, 3, seed=123)
    got = heap_images(sh, 3, HEAP)
    assert first_diff(got, om.heap) is None


@pytest.mark.parametrize("mode", MODES)
def test_random_requests_bit_exact(shmem_factory, mode):
    npes = 4
    sh, om = start(shmem_factory, npes)
    reqs = random_requests(100 + mode, 300, npes, HEAP, max_bytes=20000)
    sh.exec_requests(reqs, mode)
    assert sh.status() == 0
    om.apply_requests(reqs)
    got = heap_images(sh, npes, HEAP)
    assert first_diff(got, om.heap) is None


@pytest.mark.parametrize("dtype", [DT_INT, DT_FLOAT, DT_DOUBLE])
@pytest.mark.parametrize("nelems", [0, 1, 2, 3, 5, 31, 32, 33, 257, 4099, 65536])
def test_put_get_lengths(shmem_factory, dtype, nelems):
    """Every length, including 0 and lengths that leave ragged heads/tails."""
    w = 8 if dtype == DT_DOUBLE else 4
    heap = 4 << 20
    sh, om = start(shmem_factory, 2, heap=heap)
    rows = [dict(src_off=64 + 4, dst_off=heap // 2 + 8, bytes=nelems * w, src_pe=0, dst_pe=1,
                 op=REQ_PUT, dtype=dtype),
            dict(src_off=128, dst_off=3 * heap // 4 + 4 * (w == 4), bytes=nelems * w, src_pe=1,
                 dst_pe=0, op=REQ_GET, dtype=dtype)]
    reqs = requests(rows)
    for mode in MODES:
        sh.exec_requests(reqs, mode)
        assert sh.status() == 0
    om.apply_requests(reqs)
    assert first_diff(heap_images(sh, 2, heap), om.heap) is None


@pytest.mark.parametrize("mode", MODES)
def test_long_copies_every_alignment(shmem_factory, mode):
    """Copies long enough for the thread and warp forms' L2 prefetch (32 KiB
    and up, and just below), at every 4-byte relative alignment of source and
    destination, put and get, all in one launch: bit-exact against the
    oracle (the prefetch is a hint; it must never change a byte)."""
    heap = 32 << 20
    sh, om = start(shmem_factory, 2, heap=heap)
    rows, cur = [], heap // 4
    for nbytes in (32768 - 4, 32768, 65536 + 12, 1 << 20, (1 << 20) + 4):
        for mis in (0, 4, 8, 12):
            for op, (sp, dp) in ((REQ_PUT, (0, 1)), (REQ_GET, (1, 0))):
                cur = (cur + 63) // 64 * 64
                rows.append(dict(src_off=64 + 4 * (len(rows) % 4), dst_off=cur + mis + 4 * (len(rows) % 4),
                                 bytes=nbytes, src_pe=sp, dst_pe=dp, op=op, dtype=DT_INT))
                cur += nbytes + 64 + 16
    assert cur < heap
    reqs = requests(rows)
    sh.exec_requests(reqs, mode)
    assert sh.status() == 0
    om.apply_requests(reqs)
    assert first_diff(heap_images(sh, 2, heap), om.heap) is None


def test_p_g_all_types(shmem_factory):
    sh, om = start(shmem_factory, 2)
    rows = []
    for i, dt in enumerate([DT_INT, DT_FLOAT, DT_DOUBLE] * 4):
        bits = (0x7FF8000000000001 if dt == DT_DOUBLE else 0x7FC00001) + i  # NaN payloads too
        rows.append(dict(src_off=bits, dst_off=HEAP // 2 + 16 * i, bytes=0, src_pe=i % 2, dst_pe=(i + 1) % 2,
                         op=REQ_P, dtype=dt))
        rows.append(dict(src_off=1024 + 16 * i, dst_off=HEAP // 2 + 4096 + 16 * i, bytes=0, src_pe=(i + 1) % 2,
                         dst_pe=i % 2, op=REQ_G, dtype=dt))
    reqs = requests(rows)
    sh.exec_requests(reqs, MODE_THREAD)
    assert sh.status() == 0
    om.apply_requests(reqs)
    assert first_diff(heap_images(sh, 2, HEAP), om.heap) is None


def test_out_of_bounds_is_skipped_and_reported(shmem_factory):
    sh, om = start(shmem_factory, 2)
    bad = requests([dict(src_off=0, dst_off=HEAP - 8, bytes=64, src_pe=0, dst_pe=1, op=REQ_PUT, dtype=DT_INT),
                    dict(src_off=0, dst_off=HEAP // 2 + 2, bytes=0, src_pe=0, dst_pe=1, op=REQ_SIGNAL,
                         dtype=DT_INT, value=7)])
    for mode in (MODE_THREAD, MODE_WARP, MODE_BLOCK):
        sh.exec_requests(bad, mode)
        assert sh.status() == ERR_BOUNDS
    # nothing was written
    assert first_diff(heap_images(sh, 2, HEAP), om.heap) is None


def test_signal_values(shmem_factory):
    sh, om = start(shmem_factory, 3)
    rows = [dict(src_off=0, dst_off=HEAP // 2 + 4 * i, bytes=0, src_pe=i % 3, dst_pe=(i + 1) % 3, op=REQ_SIGNAL,
                 dtype=DT_INT, value=-5 + 1000 * i) for i in range(64)]
    reqs = requests(rows)
    sh.exec_requests(reqs, MODE_WARP)
    om.apply_requests(reqs)
    assert sh.status() == 0
    assert first_diff(heap_images(sh, 3, HEAP), om.heap) is None


@pytest.mark.parametrize("link", ["plain", "dlto"])
def test_direct_loads_and_stores_through_nvshmem_ptr(tmp_path, link):
    """A CUDA application compiled against libnvshmem.a dereferences the
    addresses nvshmem_ptr (host) and nvshmemx_ptr (device) return: plain
    stores into the next PE's slice, quiet + device barrier, plain loads from
    the previous PE's slice, then ordinary launches copying between slices
    through host-side nvshmem_ptr pointers (tests/native/ptr_direct.cu).  The
    heap images must equal the oracle's for the same puts and gets."""
    import os
    import subprocess
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = tmp_path / "ptr_direct"
    src = os.path.join(repo, "tests", "native", "ptr_direct.cu")
    libs = ["-L", os.path.join(repo, "df-nvshmem-prototype_b200", "lib"), "-lnvshmem",
            "-L/usr/local/cuda/lib64/stubs", "-lcuda"]
    inc = ["-I", os.path.join(repo, "include")]
    if link == "plain":
        cmds = [["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-rdc=true", *inc, src, "-o", str(exe), *libs]]
    else:  # the application's kernels and the library's device code optimised together
        obj = str(tmp_path / "ptr_direct.o")
        cmds = [["nvcc", "-gencode", "arch=compute_100a,code=lto_100a", "-rdc=true", *inc, "-c", src, "-o", obj],
                ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-dlto", "-rdc=true", obj, "-o", str(exe),
                 *libs]]
    for cmd in cmds:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]
    npes, heap = 4, 1 << 20
    env = dict(os.environ, NVSHMEM_NPES=str(npes), NVSHMEM_HEAP_SIZE=str(heap))
    out = tmp_path / "heaps.bin"
    r = subprocess.run([str(exe), str(out)], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    send, recv, got, copy2, n, np_, heap_ = map(int, r.stdout.split())
    assert (np_, heap_) == (npes, heap)
    images = np.fromfile(out, dtype=np.uint8).reshape(npes, heap)
    om = Model(npes, heap)
    i = np.arange(heap, dtype=np.int64)
    for pe in range(npes):
        om.heap[pe][:] = ((pe * 131 + i * 7 + (i >> 8)) & 0xff).astype(np.uint8)
    ring = [dict(src_off=send, dst_off=recv, bytes=n, src_pe=p, dst_pe=(p + 1) % npes, op=REQ_PUT, dtype=DT_INT)
            for p in range(npes)]
    pull = [dict(src_off=send, dst_off=got, bytes=n, src_pe=(p - 1) % npes, dst_pe=p, op=REQ_GET, dtype=DT_INT)
            for p in range(npes)]
    host = [dict(src_off=recv, dst_off=copy2, bytes=n, src_pe=(q + 1) % npes, dst_pe=q, op=REQ_PUT, dtype=DT_INT)
            for q in range(npes)]
    for batch in (ring, pull, host):
        om.apply_requests(requests(batch))
    assert first_diff(images, om.heap) is None
    assert not np.array_equal(images[0, recv:recv + n], images[0, send:send + n])  # the exchange moved data
