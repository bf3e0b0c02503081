"""bench.py --impl reference runs on the host cores alone (no GPU) and prints
the one JSON line the benchmark contract asks for."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    # the arm must not load the GPU library: point its path at nothing
    env = dict(os.environ, NVSHMEM_B200_LIB=os.path.join(REPO, "no-such-library.so"))
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "3"], capture_output=True, text=True, timeout=600, cwd=REPO, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["warmup"] == 3 and line["value"] > 0
    assert line["steps"] == 2  # exactly the requested steps
    sys.path.insert(0, REPO)
    import bench
    assert line["config"] == bench.line_config(line["config"]["alg_bytes_per_step"], 1)  # the GPU arm's config
    assert line["cpu_baseline"]["kind"] in ("port", "reference") and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_c3_full_size_check_matches_the_oracle():
    """bench.py checks the 256^3 halo by comparing every ghost face with the
    faces of the neighbours' blocks (c3_faces / c3_nbr); on a small grid those
    expected ghosts must equal what the oracle's halo writes."""
    import numpy as np
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    import bench
    from oracle.model import Model
    n, npes = 6, 8
    block, ghosts = n ** 3 * 8, 6 * n * n * 8
    heap = block + ghosts + 64
    om = Model(npes, heap)
    rng = np.random.default_rng(5)
    blocks = [rng.normal(size=n ** 3) for _ in range(npes)]
    for pe in range(npes):
        om.heap[pe, :block] = blocks[pe].view(np.uint8)
    om.halo(2, 2, 2, n, 0, block, block + ghosts, 4)
    for q in range(npes):
        got = om.heap[q, block:block + ghosts]
        for g in range(6):
            want = np.ascontiguousarray(bench.c3_faces(blocks[bench.c3_nbr(q, g)], n)[g ^ 1]).view(np.uint8).reshape(-1)
            assert np.array_equal(got[g * n * n * 8:(g + 1) * n * n * 8], want), (q, g)
        assert np.array_equal(om.heap[q, block + ghosts:block + ghosts + 24].view(np.int32), np.full(6, 4, np.int32))


def test_startup_rows_keep_an_eight_warp_shape():
    """The startup tune re-times the most robust shapes of the tuned table
    and always keeps an 8-warp one among them."""
    sys.path.insert(0, REPO)
    import bench

    def row(threads, worst, mb=512):
        return {"cfg": {"threads": threads, "tma_min_bytes": mb}, "worst_ratio": worst, "mean_ratio": worst}

    table = {"robust": {"candidates": [row(128, 1.00), row(128, 1.01, 1024), row(128, 1.02), row(128, 1.03, 2048),
                                       row(256, 1.05), row(256, 1.04, 1024)]}}
    rows = bench.startup_rows(table, 4)
    assert [r["cfg"]["threads"] for r in rows] == [128, 128, 128, 256]
    assert rows[-1]["worst_ratio"] == 1.04  # the best-ranked 8-warp shape
    assert rows[0]["worst_ratio"] == 1.00
    with open(bench.TUNED) as f:
        committed = bench.startup_rows(json.load(f), 4)
    assert len(committed) == 4 and any(r["cfg"]["threads"] >= 256 for r in committed)


def test_reference_arm_under_torchrun_prints_one_line():
    """Launched as the driver launches N > 1 (torchrun, 2 ranks here, on the
    host cores): rank 0 alone runs and prints one line, the other rank exits
    0 without work."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ, NVSHMEM_B200_LIB=os.path.join(REPO, "no-such-library.so"))
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(REPO, "bench.py"),
                        "--impl", "reference", "--gpus", "2", "--steps", "2", "--warmup", "3"],
                       capture_output=True, text=True, timeout=600, cwd=REPO, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["steps"] == 2
