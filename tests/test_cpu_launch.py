"""The process-per-PE launcher (the stand-in for the prototype's mpirun) on
CPU: every process gets its PE, the PE count and one shared rendezvous
directory; a failing PE stops the others; a timeout stops every PE."""
import sys

from nvshmem_b200.launch import launch

WRITE_ENV = ("import os, sys; e = os.environ; "
             "open(os.path.join(sys.argv[1], 'pe' + e['NVSHMEM_PROCESS_PE']), 'w').write(' '.join(["
             "e['NVSHMEM_PROCESS_PE'], e['NVSHMEM_NPES'], e['NVSHMEM_RENDEZVOUS'], e.get('NVSHMEM_HEAP_SIZE', '')]))")


def test_each_process_gets_its_pe(tmp_path):
    codes = launch([sys.executable, "-c", WRITE_ENV, str(tmp_path)], 4, heap=1 << 20)
    assert codes == [0, 0, 0, 0]
    rows = [(tmp_path / f"pe{k}").read_text().split() for k in range(4)]
    assert [r[0] for r in rows] == ["0", "1", "2", "3"]
    assert {r[1] for r in rows} == {"4"} and {r[3] for r in rows} == {str(1 << 20)}
    assert len({r[2] for r in rows}) == 1  # one rendezvous directory for all


def test_failing_pe_stops_the_others():
    code = "import os, sys, time; pe = int(os.environ['NVSHMEM_PROCESS_PE']); sys.exit(5) if pe == 2 else time.sleep(60)"
    codes = launch([sys.executable, "-c", code], 3, timeout=120)
    assert codes[2] == 5 and codes[0] == -9 and codes[1] == -9


def test_timeout_stops_every_pe():
    codes = launch([sys.executable, "-c", "import time; time.sleep(60)"], 2, timeout=1.0)
    assert codes == [-9, -9]


def test_devices_spread_the_pes(tmp_path):
    code = ("import os, sys; open(os.path.join(sys.argv[1], 'pe' + os.environ['NVSHMEM_PROCESS_PE']), 'w')"
            ".write(os.environ.get('NVSHMEM_DEVICE', '-'))")
    assert launch([sys.executable, "-c", code, str(tmp_path)], 5, devices=2) == [0] * 5
    assert [(tmp_path / f"pe{k}").read_text() for k in range(5)] == ["0", "0", "0", "1", "1"]


def test_command_line_runs_the_pes_and_returns_the_first_failure(tmp_path):
    """python -m nvshmem_b200.launch -n N [--devices D] -- cmd: every PE runs
    with its environment, and the exit status is the first non-zero one."""
    import os
    import subprocess
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "df-nvshmem-prototype_b200",
                       "python")
    env = dict(os.environ, PYTHONPATH=pkg + os.pathsep + os.environ.get("PYTHONPATH", ""))
    # PE 3 fails once the others have written their files (bounded wait)
    code = ("import os, sys, time; e = os.environ; pe = int(e['NVSHMEM_PROCESS_PE']); d = sys.argv[1]; "
            "open(os.path.join(d, 'pe%d' % pe), 'w').write(e['NVSHMEM_DEVICE']); "
            "t = time.time() + 30\n"
            "while pe == 3 and time.time() < t and not all(os.path.exists(os.path.join(d, 'pe%d' % k)) for k in range(3)):"
            " time.sleep(0.01)\n"
            "sys.exit(7 if pe == 3 else 0)")
    r = subprocess.run([sys.executable, "-m", "nvshmem_b200.launch", "-n", "4", "--devices", "2", "--timeout", "60",
                        "--", sys.executable, "-c", code, str(tmp_path)], env=env, capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 7, r.stderr
    assert [(tmp_path / f"pe{k}").read_text() for k in range(4)] == ["0", "0", "1", "1"]
