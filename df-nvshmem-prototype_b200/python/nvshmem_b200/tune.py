"""Autotuner driver: measures batch configurations on the GPU (the C++ tuner
in csrc/tuner.cu does the timing) and keeps the measured table as JSON.

  python -m nvshmem_b200.tune [--workload c4] [--reps 5] [--out PATH]

The table ({"key", "results": [...], "best": {...}}) is what bench.py loads,
what the learned picker falls back to, and the yardstick for the picker's regret.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import time

from . import _lib as L
from ._lib import check, lib

TUNED_DIR = os.path.join(L.PKG_ROOT, "tuned")


def candidates(min_chunk: int = 256, max_n: int = 512) -> list[L.BatchConfig]:
    arr = (L.BatchConfig * max_n)()
    n = lib.nvshmemx_tune_candidates(arr, max_n, min_chunk)
    return [arr[i] for i in range(n)]


def tune_batch(batch, cands=None, reps: int = 5, flush_bytes: int = 256 << 20):
    cands = cands or candidates()
    carr = (L.BatchConfig * len(cands))(*cands)
    res = (L.TuneResult * len(cands))()
    best = ctypes.c_int(-1)
    check(lib.nvshmemx_tune_batch(batch.h, carr, len(cands), reps, flush_bytes, res, ctypes.byref(best)),
          "tune_batch")
    rows = [dict(cfg=r.cfg.as_dict(), ms_median=r.ms_median, ms_min=r.ms_min,
                 exec_ms_median=r.exec_ms_median, status=r.status) for r in res]
    return rows, rows[best.value]


def write_table(path: str, key: dict, rows, best, alg_bytes: int):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    for r in rows:
        if r["ms_median"] > 0:
            r["GBps"] = round(alg_bytes / (r["ms_median"] / 1e3) / 1e9, 1)
    table = {"key": key, "alg_bytes": alg_bytes, "measured_at": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
             "results": sorted(rows, key=lambda r: (r["ms_median"] if r["ms_median"] > 0 else 1e9)),
             "best": best["cfg"], "best_ms": best["ms_median"]}
    with open(path, "w") as f:
        json.dump(table, f, indent=1)
    return table


def main():
    from .api import Shmem, requests_bytes
    from .traffic import c4_batch

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c4", choices=["c4"])
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--out", default=os.path.join(TUNED_DIR, "batch_c4.json"))
    a = ap.parse_args()
    spec = dict(seed=4, n=100_000, npes=64, heap=64 << 20)
    reqs = c4_batch(**spec)
    with Shmem(spec["npes"], spec["heap"]) as sh:
        for pe in range(spec["npes"]):
            sh.fill_random(pe, 0, spec["heap"], 44)
        with sh.batch(len(reqs), int(reqs["bytes"].sum()), 256) as b:
            b.upload(reqs)
            rows, best = tune_batch(b, reps=a.reps)
        key = {"workload": "c4", **spec, "requests": len(reqs)}
        t = write_table(a.out, key, rows, best, requests_bytes(reqs))
    print(json.dumps({"best": t["best"], "best_ms": t["best_ms"], "candidates": len(rows),
                      "top5": [(r["cfg"], r["ms_median"]) for r in t["results"][:5]]}))


if __name__ == "__main__":
    main()
