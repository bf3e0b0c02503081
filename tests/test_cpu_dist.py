"""The benchmark's multi-process plumbing on CPU with the gloo backend
(world size 2): max-over-ranks timing and barriers agree across ranks, and a
rank that fails before a collective makes the other rank's next collective end
with an error after the short process-group timeout, not hang."""
import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, mode, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    try:
        if mode == "ok":
            m = bench.reduce_max(dist, 1.5 + rank)
            bench.barrier(dist)
            q.put((rank, m))
        else:
            if rank == 1:
                q.put((rank, "left"))
                q.close()
                q.join_thread()  # flush the message before leaving
                os._exit(0)  # leaves between steps, before the next collective
            try:
                bench.reduce_max(dist, 1.0)
                q.put((rank, "no error"))
            except Exception as e:  # noqa: BLE001
                q.put((rank, "error:" + type(e).__name__))
    finally:
        if mode == "ok":
            dist.destroy_process_group()


def _run(mode):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, mode, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_reduce_max_and_barrier_two_ranks():
    out = _run("ok")
    assert out == {0: 2.5, 1: 2.5}


def test_departed_rank_ends_collective_with_error():
    out = _run("fail")
    assert out[1] == "left"
    assert out[0].startswith("error:")


def test_dist_env_defaults(monkeypatch):
    sys.path.insert(0, REPO)
    import bench
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert bench.dist_env() == (0, 1, 0)
    assert bench.dist_init(1) is None
    assert bench.reduce_max(None, 3.0) == 3.0


@pytest.mark.parametrize("x", [0])
def test_bench_importable_without_gpu(x):
    sys.path.insert(0, REPO)
    import bench
    assert bench.METRIC.startswith("batched put/get GB/s")
