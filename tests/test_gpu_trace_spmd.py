"""The %globaltimer trace ring with its CSV export in the prototype's
processed-trace format, and the SPMD host threads that stand in for the
prototype's MPI processes (per-thread my_pe, per-PE allocation tails, host and
offload barriers, and a PE thread that leaves early failing the barrier
instead of hanging it)."""
import ctypes
import os
import threading

import numpy as np
import pytest

from nvshmem_b200 import ERR_STATE, _lib as L

pytestmark = pytest.mark.gpu

lib = L.lib


def test_trace_ring_records_and_csv(shmem_factory, tmp_path):
    sh = shmem_factory(2, 1 << 20)
    flag = sh.alloc(4)
    data = sh.alloc(1024)
    sh.trace_enable(4096)
    sh.pingpong(flag, data, 64, 50, skip=0)
    assert sh.status() == 0
    rec0, dropped0 = sh.trace_read(0)
    rec1, _ = sh.trace_read(1)
    assert dropped0 == 0
    # PE 0 per iteration: one int put (256 B), one int p (recorded as put_int
    # of one element, as the prototype does) and one wait
    assert ((rec0["op"] == 0) & (rec0["bytes"] == 256)).sum() == 50
    assert ((rec0["op"] == 0) & (rec0["bytes"] == 4)).sum() == 50
    assert (rec0["op"] == 6).sum() == 50  # wait_int
    assert (rec1["op"] == 6).sum() == 50
    assert np.all(np.diff(rec0["t_ns"]) >= 0)
    assert np.all(rec0["pe"] == 0) and np.all(rec1["pe"] == 1)
    prefix = str(tmp_path / "trace")
    sh.trace_write_csv(prefix)
    lines = open(prefix + "_0").read().splitlines()
    assert lines[0] == ("# timestamp, gridid, blockid, tid, type, local_address, remote_address, size, remote_pe, "
                        "timespent")
    row = [x.strip() for x in lines[1].split(",")]
    assert len(row) == 10 and row[4] in ("put_int", "wait_int", "put_float")
    assert len(lines) - 1 == len(rec0)
    # a small ring keeps the newest records and counts the dropped ones
    sh.trace_enable(16)
    sh.pingpong(flag, data, 0, 40, skip=0)
    sh.status()
    rec, dropped = sh.trace_read(0)
    assert len(rec) == 16 and dropped == 40 * 2 - 16
    sh.trace_disable()


def test_offload_barrier_and_halo_trace_records(shmem_factory):
    """Every nvshmem_barrier_all_offload leaves one BARRIER record per PE, and
    the halo records one PUT per face row (x rows as put_double)."""
    npes, n = 8, 32
    block, ghosts = n ** 3 * 8, 6 * n * n * 8
    sh = shmem_factory(npes, block + ghosts + 4096)
    sh.trace_enable(1 << 14)
    for _ in range(3):
        lib.nvshmem_barrier_all_offload()
    sh.sync()
    for pe in range(npes):
        rec, dropped = sh.trace_read(pe)
        assert dropped == 0 and (rec["op"] == 8).sum() == 3 and np.all(rec["pe"] == pe)
    sh.trace_enable(1 << 14)  # a fresh ring
    sh.halo(2, 2, 2, n, 0, block, block + ghosts, 1, 2)
    assert sh.status() == 0
    for pe in range(npes):
        rec, _ = sh.trace_read(pe)
        assert ((rec["op"] == 2) & (rec["bytes"] == n * 8)).sum() == 2 * n  # x-face rows
        assert ((rec["op"] == 0) & (rec["bytes"] == n * 8)).sum() == 4 * n  # y and z rows
    sh.trace_disable()


CB = ctypes.CFUNCTYPE(None, ctypes.c_void_p)


def test_trace_from_environment(tmp_path):
    """NVSHMEM_ENABLE_TRACING=1 at nvstart_pes turns the ring on (sized by
    NVSHMEM_LOG_BUFFER_SIZE bytes per PE) and nvstop_pes writes one processed
    trace file per PE, named as the prototype named them."""
    import subprocess
    import sys
    pkg = os.path.dirname(os.path.dirname(L.__file__))
    code = "\n".join([
        "import os, sys",
        f"sys.path.insert(0, {pkg!r})",
        "from nvshmem_b200 import Shmem",
        "from nvshmem_b200 import _lib as L",
        "L.lib.nvstart_pes()",
        "sh = Shmem.__new__(Shmem)",
        "sh.npes, sh.heap_bytes = 2, 1 << 20",
        "sh.base = L.lib.nvshmemx_arena_base()",
        "flag = sh.alloc(4); data = sh.alloc(1024)",
        "sh.pingpong(flag, data, 64, 20, skip=0)",
        "assert L.lib.nvshmemx_status() == 0",
        "L.lib.nvstop_pes()",
        "print(os.getpid())",
    ])
    env = dict(os.environ, NVSHMEM_ENABLE_TRACING="1", NVSHMEM_LOG_BUFFER_SIZE=str(48 * 1024),
               NVSHMEM_NPES="2", NVSHMEM_HEAP_SIZE=str(1 << 20), NVSHMEM_ERROR_MODE="return")
    out = subprocess.run([sys.executable, "-c", code], cwd=tmp_path, env=env, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    pid = out.stdout.strip().splitlines()[-1]
    for pe in range(2):
        lines = (tmp_path / f"nvshmem_processed_tracefile_{pid}_{pe}").read_text().splitlines()
        assert lines[0].startswith("# timestamp, gridid, blockid, tid, type")
        ops = [ln.split(", ")[4] for ln in lines[1:]]
        assert ops.count("wait_int") == 20


def test_spmd_threads(shmem_factory):
    npes = 4
    sh = shmem_factory(npes, 1 << 20)
    seen, lock = [], threading.Lock()
    base = lib.nvshmemx_arena_base()
    stride = lib.nvshmemx_slice_stride()

    def body(_):
        pe = lib.nvshmem_my_pe()
        a = lib.nvshmalloc(100 + 0)
        b = lib.nvshmalloc(28)
        lib.nvshmem_barrier_all()
        lib.nvshmem_barrier_all_offload()
        lib.nvshmem_barrier_all()
        with lock:
            seen.append((pe, a, b))

    cb = CB(body)
    assert lib.nvshmemx_spmd_run(cb, None) == 0
    assert sorted(p for p, _, _ in seen) == list(range(npes))
    for pe, a, b in seen:
        assert a == base + pe * stride and b == a + 100  # per-PE tail, no padding
    assert sh.status() == 0


def test_spmd_departed_pe_fails_barrier(shmem_factory):
    os.environ["NVSHMEM_HOST_BARRIER_TIMEOUT_S"] = "20"
    sh = shmem_factory(3, 1 << 20)
    results, lock = [], threading.Lock()

    def body(_):
        pe = lib.nvshmem_my_pe()
        if pe == 1:
            return  # this PE leaves without reaching the barrier
        lib.nvshmem_barrier_all()
        with lock:
            results.append(pe)

    cb = CB(body)
    rc = lib.nvshmemx_spmd_run(cb, None)
    assert rc == ERR_STATE
    assert sorted(results) == [0, 2]  # both returned (with an error) instead of hanging
    assert sh.status() == ERR_STATE
