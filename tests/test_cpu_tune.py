"""The tuner's robust choice (nvshmem_b200.tune.robust_choice) and the
committed table it wrote: the configuration kept is the one whose worst
slowdown over several C4 batches is smallest, not the fastest on one batch."""
import json
import os

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TABLE = os.path.join(REPO, "df-nvshmem-prototype_b200", "tuned", "batch_c4.json")


class _FakeBatch:
    def __init__(self, seed):
        self.seed = seed

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False

    def upload(self, reqs):
        self.n = len(reqs)


class _FakeShmem:
    """Hands out one batch per seed, in the order robust_choice asks."""

    def __init__(self, seeds):
        self.seeds = list(seeds)

    def batch(self, n, payload, min_chunk):
        return _FakeBatch(self.seeds.pop(0))


def test_robust_choice_prefers_the_smallest_worst_slowdown(monkeypatch):
    from nvshmem_b200 import tune

    # ms per seed for three configurations: A is fastest on seed 4 but 10%
    # slower on seed 5; B is never fastest but never more than 2% behind
    ms = {4: [1.00, 1.01, 1.05], 5: [1.10, 1.02, 1.00], 6: [1.00, 1.01, 1.03]}
    calls = []

    def fake_tune_batch(b, cands=None, reps=5, flush_bytes=0):
        calls.append((b.seed, len(cands)))
        rows = [dict(cfg=c.as_dict(), ms_median=ms[b.seed][i], ms_min=ms[b.seed][i], exec_ms_median=0.0,
                     status=0) for i, c in enumerate(cands)]
        return rows, rows[0]

    monkeypatch.setattr(tune, "tune_batch", fake_tune_batch)
    base = dict(vec_bytes=16, chunk_bytes=16384, unroll=4, threads=128, ctas_per_sm=0, grab=2, tma_stages=2,
                tma_stage_bytes=8192, tma_min_bytes=512, stream=0, stream_planners=2)
    top = [dict(base, tma_min_bytes=m) for m in (512, 2048, 4096)]
    seeds = [4, 5, 6]
    spec = dict(seed=4, n=200, npes=4, heap=1 << 20)
    out = tune.robust_choice(_FakeShmem(seeds), spec, top, seeds, reps=2, rounds=3)
    assert out["chosen"] == top[1]
    worst = [c["worst_ratio"] for c in out["candidates"]]
    assert worst == [pytest.approx(1.10 / 1.00, abs=1e-3), pytest.approx(1.02 / 1.00, abs=1e-3),
                     pytest.approx(1.05 / 1.00, abs=1e-3)]
    assert calls == [(s, 3) for s in seeds for _ in range(3)]  # interleaved rounds per seed


def test_committed_table_is_consistent():
    with open(TABLE) as f:
        t = json.load(f)
    cfgs = [r["cfg"] for r in t["results"]]
    assert t["best"] in cfgs and t["sweep_best"] == cfgs[0]
    rob = t["robust"]
    assert rob["seeds"][0] == t["key"]["seed"] and len(rob["seeds"]) >= 3
    ranked = sorted(rob["candidates"], key=lambda c: (c["worst_ratio"], c["mean_ratio"]))
    assert ranked[0]["cfg"] == rob["chosen"] == t["best"]
    # the candidates are the sweep's leading configurations
    assert [c["cfg"] for c in rob["candidates"]] == cfgs[:len(rob["candidates"])]


def test_robust_choice_refuses_a_batch_where_nothing_ran(monkeypatch):
    from nvshmem_b200 import tune

    def failing(b, cands=None, reps=5, flush_bytes=0):
        rows = [dict(cfg=c.as_dict(), ms_median=-1.0, ms_min=-1.0, exec_ms_median=-1.0, status=1) for c in cands]
        return rows, rows[0]

    monkeypatch.setattr(tune, "tune_batch", failing)
    base = dict(vec_bytes=16, chunk_bytes=16384, unroll=4, threads=128, ctas_per_sm=0, grab=2, tma_stages=2,
                tma_stage_bytes=8192, tma_min_bytes=512, stream=0, stream_planners=2)
    with pytest.raises(RuntimeError):
        tune.robust_choice(_FakeShmem([4]), dict(seed=4, n=100, npes=4, heap=1 << 20), [base], [4], reps=1, rounds=1)
