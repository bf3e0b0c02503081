"""Process-per-PE mode, the prototype's own execution model: a prototype-style
application (tests/native/proc_pes.cu, linked against libnvshmem.a) runs as
one process per PE under python -m nvshmem_b200.launch.  Every process maps
every PE's slice through exchanged VMM handles; puts and gets between the
processes must leave the heaps equal to the oracle's, and a PE process that
leaves must make the others' nvshmem_barrier_all fail instead of waiting."""
import os
import subprocess

import numpy as np
import pytest

from nvshmem_b200 import DT_INT, REQ_GET, REQ_PUT
from nvshmem_b200.launch import launch
from oracle.model import Model
from _util import first_diff, requests

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build(tmp_path, name="proc_pes"):
    exe = tmp_path / name
    r = subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-rdc=true",
                        "-I", os.path.join(REPO, "include"), os.path.join(REPO, "tests", "native", name + ".cu"),
                        "-o", str(exe), "-L", os.path.join(REPO, "df-nvshmem-prototype_b200", "lib"), "-lnvshmem",
                        "-L/usr/local/cuda/lib64/stubs", "-lcuda"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return str(exe)


def pattern(pe, n):
    i = np.arange(n, dtype=np.uint64)
    return ((pe * 2654435761 + i * 40503 + 7) & 0xFFFFFFFF).astype(np.uint32)


def visible_devices():
    import torch
    return torch.cuda.device_count()


def check_exchange(tmp_path, npes, heap):
    """The heaps the exchange of proc_pes.cu / boot_pes.cu wrote, against the
    oracle: PE p's block in PE p+1's slot p and in PE p+1's `got` area."""
    rows = [list(map(int, (tmp_path / f"pe{pe}.txt").read_text().split())) for pe in range(npes)]
    assert sorted(r[0] for r in rows) == list(range(npes))
    _, send, recv, got, n = rows[0]
    assert all(r[1:] == [send, recv, got, n] for r in rows)  # symmetric offsets in every process
    images = np.stack([np.fromfile(tmp_path / f"pe{pe}.bin", dtype=np.uint8) for pe in range(npes)])
    om = Model(npes, heap)
    for pe in range(npes):
        om.heap[pe][send:send + 4 * n] = pattern(pe, n).view(np.uint8)
    ring = [dict(src_off=send, dst_off=recv + p * 4 * n, bytes=4 * n, src_pe=p, dst_pe=(p + 1) % npes, op=REQ_PUT,
                 dtype=DT_INT) for p in range(npes)]
    pull = [dict(src_off=send, dst_off=got, bytes=4 * n, src_pe=(p - 1) % npes, dst_pe=p, op=REQ_GET, dtype=DT_INT)
            for p in range(npes)]
    om.apply_requests(requests(ring))
    om.apply_requests(requests(pull))
    assert first_diff(images, om.heap) is None


@pytest.mark.parametrize("npes,spread", [(2, False), (4, False), (4, True)])
def test_processes_exchange_blocks(tmp_path, npes, spread):
    """spread: the launcher's --devices over every visible GPU (contiguous
    blocks of PEs per device; on a one-GPU box every PE names device 0)."""
    exe = build(tmp_path)
    heap = 4 << 20
    codes = launch([exe, "exchange", str(tmp_path)], npes, heap=heap, timeout=240,
                   env=dict(os.environ, NVSHMEM_HOST_BARRIER_TIMEOUT_S="60"),
                   devices=visible_devices() if spread else None)
    assert codes == [0] * npes, codes
    check_exchange(tmp_path, npes, heap)


def test_departed_process_fails_the_barrier(tmp_path):
    exe = build(tmp_path)
    codes = launch([exe, "depart", str(tmp_path)], 3, heap=4 << 20, timeout=240, stop_on_failure=False,
                   env=dict(os.environ, NVSHMEM_HOST_BARRIER_TIMEOUT_S="3"))
    assert codes == [3, 0, 3], codes


def test_process_start_failures_leave_the_library_usable(tmp_path):
    """nvshmemx_init_process fails cleanly -- an unusable rendezvous
    directory, or a peer that never arrives (bounded by the host timeout) --
    and a one-process start works afterwards in the same process."""
    import subprocess
    import sys
    pkg = os.path.join(REPO, "df-nvshmem-prototype_b200", "python")
    code = "\n".join([
        "import os, sys, time",
        f"sys.path.insert(0, {pkg!r})",
        "from nvshmem_b200 import _lib as L",
        "lib = L.lib",
        "lib.nvshmemx_set_error_mode(1)",
        "rc1 = lib.nvshmemx_init_process(0, 2, 1 << 20, b'/nonexistent/rendezvous')",
        "assert not lib.nvshmemx_is_started()",
        "t0 = time.time()",
        f"rc2 = lib.nvshmemx_init_process(0, 2, 1 << 20, {str(tmp_path).encode()!r})",
        "dt = time.time() - t0",
        "assert not lib.nvshmemx_is_started()",
        "lib.nvshmemx_status()",
        "rc3 = lib.nvshmemx_init_attr(2, 1 << 20)",
        "assert lib.nvshmemx_is_started() and lib.nvshmemx_finalize() == 0",
        "print(rc1, rc2, rc3, round(dt, 1))",
    ])
    env = dict(os.environ, NVSHMEM_HOST_BARRIER_TIMEOUT_S="2")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    rc1, rc2, rc3, dt = r.stdout.split()
    assert int(rc1) != 0 and int(rc2) != 0 and int(rc3) == 0
    assert 1.5 <= float(dt) <= 30  # the missing peer is given up on after the timeout


@pytest.mark.parametrize("npes", [2, 4])
def test_bootstrap_from_the_applications_own_launcher(tmp_path, npes):
    """nvshmemx_init_bootstrap: the application forks its PE processes and
    provides the allgather (the stand-in for MPI_Allgather), as an MPI program
    would; the same exchange then matches the oracle, and the rendezvous
    directory rank 0 made is gone afterwards."""
    import signal
    exe = build(tmp_path, "boot_pes")
    before = set(os.listdir("/tmp"))
    env = dict(os.environ, NVSHMEM_HOST_BARRIER_TIMEOUT_S="60", TMPDIR="/tmp")
    p = subprocess.Popen([exe, str(npes), str(tmp_path)], env=env, start_new_session=True)
    try:
        rc = p.wait(timeout=240)
    except subprocess.TimeoutExpired:
        os.killpg(p.pid, signal.SIGKILL)  # the group this test started: the app and its PE processes
        p.wait()
        raise
    assert rc == 0, rc
    check_exchange(tmp_path, npes, 4 << 20)
    assert not [d for d in set(os.listdir("/tmp")) - before if d.startswith("nvshm-")]


def test_offload_barrier_orders_blocking_streams(tmp_path):
    """nvshmem_barrier_all_offload is an action on the legacy default stream:
    a kernel on a blocking stream after it runs only once the kernels that
    blocking streams launched before it have finished
    (tests/native/offload_order.cu). Without the barrier the same reader runs
    beside the writer, which shows that the check can fail."""
    exe = build(tmp_path, "offload_order")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr[-2000:])
    counts = dict(kv.split("=") for kv in r.stdout.split() if "=" in kv)
    assert int(counts["misses_with_barrier"]) == 0
    assert int(counts["races_without"]) >= 1
