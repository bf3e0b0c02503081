"""Starts one process per PE for the library's process-per-PE mode, the
stand-in for the prototype's ``mpirun -np N ./app`` (no MPI is needed).

    python -m nvshmem_b200.launch -n 4 [--heap BYTES] [--timeout S] [--devices D] -- ./app args

Every process gets NVSHMEM_NPES, NVSHMEM_PROCESS_PE and NVSHMEM_RENDEZVOUS
(a fresh private directory where the processes exchange their slices' VMM
handles and share the host barrier); ``nvstart_pes()`` in the application
picks them up.  When one process fails the others are stopped, and the exit
status is the failed process's status (the first in PE order, if several).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import tempfile
import time


def launch(cmd: list[str], npes: int, heap: int | None = None, timeout: float | None = None,
           env: dict | None = None, cwd: str | None = None, stop_on_failure: bool = True,
           devices: int | None = None) -> list[int]:
    """Runs `cmd` as `npes` PE processes; returns their exit statuses (a PE
    stopped because another failed -- with stop_on_failure -- or because the
    timeout passed reports -9).  With `devices`, the PEs are split into
    contiguous blocks, one per device: PE k runs on device k * devices // npes
    (NVSHMEM_DEVICE), so neighbouring PEs share a GPU."""
    if npes < 1:
        raise ValueError("npes must be at least 1")
    rdv = tempfile.mkdtemp(prefix="nvshm-")
    procs: list[subprocess.Popen] = []
    try:
        for pe in range(npes):
            e = dict(os.environ if env is None else env)
            e.update(NVSHMEM_NPES=str(npes), NVSHMEM_PROCESS_PE=str(pe), NVSHMEM_RENDEZVOUS=rdv)
            if heap:
                e["NVSHMEM_HEAP_SIZE"] = str(heap)
            if devices:
                e["NVSHMEM_DEVICE"] = str(pe * devices // npes)
            procs.append(subprocess.Popen(cmd, env=e, cwd=cwd))
        deadline = None if timeout is None else time.monotonic() + timeout
        codes: list[int | None] = [None] * npes
        while any(c is None for c in codes):
            for i, p in enumerate(procs):
                if codes[i] is None:
                    codes[i] = p.poll()
            failed = stop_on_failure and any(c not in (None, 0) for c in codes)
            late = deadline is not None and time.monotonic() > deadline
            if failed or late:
                for i, p in enumerate(procs):
                    if codes[i] is None:
                        p.kill()  # this PE process only, by its PID
                        p.wait()
                        codes[i] = -9
                break
            time.sleep(0.01)
        return [int(c) for c in codes]
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
                p.wait()
        shutil.rmtree(rdv, ignore_errors=True)


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("-n", "--npes", type=int, required=True)
    ap.add_argument("--heap", type=int, default=None, help="bytes per PE (NVSHMEM_HEAP_SIZE)")
    ap.add_argument("--timeout", type=float, default=None, help="seconds before every PE is stopped")
    ap.add_argument("--devices", type=int, default=None,
                    help="spread the PEs over this many GPUs in contiguous blocks (PE k on device k * D // n)")
    ap.add_argument("cmd", nargs=argparse.REMAINDER)
    a = ap.parse_args()
    cmd = a.cmd[1:] if a.cmd and a.cmd[0] == "--" else a.cmd
    if not cmd:
        ap.error("no command")
    codes = launch(cmd, a.npes, a.heap, a.timeout, devices=a.devices)
    # the PE that failed, not one the launcher stopped because of it (-9)
    failed = [c for c in codes if c not in (0, -9)]
    return failed[0] if failed else next((c for c in codes if c != 0), 0)


if __name__ == "__main__":
    sys.exit(main())
