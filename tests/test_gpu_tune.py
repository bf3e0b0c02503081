"""The autotuner measures every candidate, ranks them by median time, leaves
the batch configured with the best one, and tuning never changes results
(every candidate re-executes the same idempotent batch)."""
import numpy as np
import pytest

from nvshmem_b200 import tune
from nvshmem_b200.traffic import c4_batch
from oracle.model import Model
from _util import first_diff, heap_images

pytestmark = pytest.mark.gpu


def test_tuner_ranks_and_keeps_results_exact(shmem_factory):
    npes, heap = 8, 4 << 20
    reqs = c4_batch(seed=12, n=2000, npes=npes, heap=heap, hi=256 << 10)
    sh = shmem_factory(npes, heap)
    om = Model(npes, heap)
    for pe in range(npes):
        sh.fill_random(pe, 0, heap, 2)
        om.fill_random(pe, 0, heap, 2)
    om.apply_requests(reqs)
    cands = tune.candidates(min_chunk=4096)[:12]
    with sh.batch(len(reqs), int(reqs["bytes"].sum()), 4096) as b:
        b.upload(reqs)
        rows, best = tune.tune_batch(b, cands, reps=3, flush_bytes=64 << 20)
        assert len(rows) == len(cands)
        ok = [r for r in rows if r["status"] == 0]
        assert len(ok) == len(cands)
        assert best["ms_median"] == min(r["ms_median"] for r in ok)
        assert all(r["exec_ms_median"] > 0 and r["exec_ms_median"] <= r["ms_median"] * 1.5 for r in ok)
        assert b.config() == best["cfg"]
    assert sh.status() == 0
    assert first_diff(heap_images(sh, npes, heap), om.heap) is None


def test_candidate_grid():
    c = tune.candidates(min_chunk=256)
    assert len(c) == 138 and sum(1 for x in c if x.tma_stages) == 84 and sum(x.stream for x in c) == 6
    assert sorted({x.tma_min_bytes for x in c if x.tma_stages and not x.stream}) == [512, 1024, 2048]
    assert all(x.chunk_bytes >= 4096 for x in tune.candidates(min_chunk=4096))
