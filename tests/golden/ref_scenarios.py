"""Scenarios used to pin the CPU oracle to the reference's own build.

Each scenario is run (a) through the reference's sources compiled for sm_100a
with every MPI rank on one GPU (oracle/_ref/ref_driver, by make_ref_golden.py
on a GPU machine; the printed per-rank heap hashes are committed in
ref_heaps.json), (b) through the CPU oracle, and (c) through this library;
all three must agree bit for bit.  Inputs are regenerated from the seeds
below, so nothing but the hashes needs to be stored.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "df-nvshmem-prototype_b200", "python"))
sys.path.insert(0, REPO)

from nvshmem_b200 import REQUEST_DTYPE  # noqa: E402
from nvshmem_b200.traffic import Stream, c3_block  # noqa: E402

SCENARIOS = [
    dict(name="alloc", npes=2),
    dict(name="requests", npes=4, heap=1 << 20, seed=31, nreq=400, req_seed=301),
    dict(name="requests", npes=8, heap=1 << 20, seed=32, nreq=800, req_seed=302),
    dict(name="alltoall", npes=8, bytes=4096, rounds=2, seed=33),
    dict(name="alltoall", npes=4, bytes=65536, rounds=1, seed=34),
    dict(name="halo", npes=8, n=16, iters=3),
    dict(name="pingpong", npes=2, len=256, iters=20, seed=35),
]

ALLOC_SIZES = [3, 1, 8, 0, 17, 70, 4096, 5]


def scenario_id(s: dict) -> str:
    return "_".join(f"{k}={v}" for k, v in s.items())


def request_list(npes: int, heap: int, n: int, seed: int) -> np.ndarray:
    """PUT/GET/SIGNAL/P/G requests with element-aligned offsets (the
    reference's typed loads and stores need natural alignment), disjoint
    destinations in the upper half of each heap, sources in the lower half."""
    st = Stream(seed)
    half = heap // 2
    out = np.zeros(n, dtype=REQUEST_DTYPE)
    cursor = [half] * npes
    k = 0
    for _ in range(n):
        op = int(st.randint(1, 5)[0])
        dt = int(st.randint(1, 3)[0])
        w = 8 if dt == 2 else 4
        sp, dp = int(st.randint(1, npes)[0]), int(st.randint(1, npes)[0])
        nb = int(st.randint(1, 2048)[0]) * w if op in (0, 1) else 0
        wb = 4 if op == 2 else (w if op in (3, 4) else nb)
        src = int(st.randint(1, (half - nb - 64) // w)[0]) * w
        dst = (cursor[dp] + w - 1) // w * w
        if dst + wb > heap:
            break
        cursor[dp] = dst + wb + 8 * int(st.randint(1, 4)[0])
        bits = int(st.u64(1)[0]) & ((1 << (8 * w)) - 1)
        out[k] = (bits if op == 3 else src, dst, nb, sp, dp, op, dt, 0, int(st.randint(1, 1 << 30)[0]))
        k += 1
    return out[:k]


def halo_blocks(n: int, npes: int = 8):
    return [c3_block(n, pe) for pe in range(npes)]


def oracle_hashes(s: dict) -> dict:
    """Per-rank FNV-1a hashes the CPU oracle predicts for scenario s."""
    from oracle.model import Model, fnv1a
    name, npes = s["name"], s["npes"]
    if name == "alloc":
        m = Model(npes, 1 << 20)
        offs = [m.alloc(x) for x in ALLOC_SIZES]
        m.cleanup()
        return {"offsets": offs, "after_cleanup": m.alloc(16)}
    if name == "requests":
        m = Model(npes, s["heap"])
        for pe in range(npes):
            m.fill_random(pe, 0, s["heap"], s["seed"])
        m.apply_requests(request_list(npes, s["heap"], s["nreq"], s["req_seed"]))
    elif name == "alltoall":
        heap = 2 * npes * s["bytes"]
        m = Model(npes, heap)
        for pe in range(npes):
            m.fill_random(pe, 0, heap, s["seed"])
        m.alltoall(0, 0, npes * s["bytes"], s["bytes"], rounds=s["rounds"])
    elif name == "halo":
        n = s["n"]
        block, ghosts = n ** 3 * 8, 6 * n * n * 8
        heap = (block + ghosts + 64 + 4095) // 4096 * 4096
        m = Model(npes, heap)
        for pe, b in enumerate(halo_blocks(n, npes)):
            m.heap[pe, :block] = b.view(np.uint8)
        m.halo(2, 2, 2, n, 0, block, block + ghosts, s["iters"])
    elif name == "pingpong":
        heap = (4096 + s["len"] * 4 + 4095) // 4096 * 4096
        m = Model(2, heap)
        for pe in range(2):
            m.fill_random(pe, 0, heap, s["seed"])
            m.heap[pe, :4] = 0
        m.pingpong(0, 64, s["len"], s["iters"])
    else:
        raise ValueError(name)
    return {str(pe): f"{fnv1a(m.heap[pe]):016x}" for pe in range(npes)}
