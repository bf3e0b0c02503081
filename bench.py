"""Benchmark of the virtual-PE one-sided path on B200.

Headline (one JSON line on rank 0): batched put/get throughput of the C4
workload -- 64 virtual PEs x 64 MiB heap, 100,000 requests per batch with
log-normal sizes (median 2 KiB, sigma 1.5, 4 B..4 MiB), put 45% / get 45% /
signal 10%, uniform PE pairs, disjoint destinations -- in GB/s counting 2
bytes per payload byte (read + write), with L2 flushed between steps.
Beside it: the per-call path on the same batch, the end-to-end call with
host-resident requests (16-byte compact requests; the 32-byte form beside
it), the C2 all-to-all bulk throughput, the C1 ping-pong
round trip and the device barrier latency, the roofline of the batch's exec
kernel and the CPU baseline (forked processes + memcpy + process-shared
barrier, the stand-in for the reference's MPI host path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "df-nvshmem-prototype_b200", "python"))
sys.path.insert(0, ROOT)

METRIC = "batched put/get GB/s (% HBM peak) vs per-call path; p50 wait/barrier ns; 1 B200"
UNIT = "GB/s"
C4 = dict(seed=4, n=100_000, npes=64, heap=64 << 20)
# a quarter-size case of the same kernel for ncu captures (1 GiB arena)
C4_SMALL = dict(seed=4, n=25_000, npes=16, heap=64 << 20)
WORKLOAD = ("C4 batched uneven traffic: 64 virtual PEs x 64 MiB heap, 100,000 put/get/signal "
            "requests per batch, log-normal sizes median 2 KiB sigma 1.5 clipped 4 B..4 MiB, "
            "put 45%/get 45%/signal 10%, uniform PE pairs, disjoint 16-B-aligned destinations, seed 4")
TUNED = os.path.join(ROOT, "df-nvshmem-prototype_b200", "tuned", "batch_c4.json")


def line_config(alg, world):
    """The `config` object of both arms' JSON lines (identical by design)."""
    return {"workload": WORKLOAD,
            "l2": "inputs larger than L2 (64 x 64 MiB heap); the GPU arm also flushes L2 between steps "
                  "(256 MiB write)",
            "alg_bytes_per_step": int(alg), "parallelism": f"replicas x{world}"}
NCU_SUMMARY = os.path.join(ROOT, "profiles", "batch_exec_c4.json")


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev: int):
        self.dev = dev
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.dev)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        load = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------ distributed
def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def dist_init(world):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group("nccl" if os.environ.get("BENCH_BACKEND", "nccl") == "nccl" else "gloo",
                            timeout=datetime.timedelta(seconds=120))
    return dist


def reduce_max(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


# ------------------------------------------------------------ CPU baseline
def cpu_baseline(reqs, npes, heap, max_seconds=12.0, warmup=1, reps=1000000):
    """The host path timed on this machine's cores: `reps` executions of the
    batch (at most `max_seconds` of them) by npes forked ranks."""
    from oracle import model as om  # the checker package; only this leg runs it
    if not os.path.exists(om.HOST_BENCH):
        om.build()
    with tempfile.NamedTemporaryFile(suffix=".req", delete=False) as f:
        f.write(reqs.tobytes())
        path = f.name
    try:
        out = subprocess.run([om.HOST_BENCH, "batch", path, str(npes), str(heap), str(reps), str(max_seconds), "44",
                              str(warmup)],
                             capture_output=True, text=True, timeout=600, check=True).stdout
    finally:
        os.unlink(path)
    r = json.loads(out.strip().splitlines()[-1])
    return {"value": round(r["gbs"], 3), "unit": UNIT, "cores": r["cores"], "kind": "port",
            "ms_per_step": 1e3 * r["seconds_per_rep"], "reps": r["reps"],
            "sample": f"the full {r['requests']}-request batch, {r['npes']} forked ranks, {r['reps']} reps "
                      f"in {r['reps'] * r['seconds_per_rep']:.1f} s (host has {r['host_cores']} cores)",
            "heap_checksum": r["heap_checksum"]}


def run_reference(args, rank, world):
    """--impl reference: the CPU host path on this box's cores (rank 0 only)."""
    if rank != 0:
        return
    import numpy as np  # noqa: F401
    from nvshmem_b200._abi import REQ_GET, REQ_PUT, REQ_SIGNAL  # constants only: the GPU library is not loaded
    from nvshmem_b200.traffic import c4_batch
    reqs = c4_batch(**C4)
    copies = (reqs["op"] == REQ_PUT) | (reqs["op"] == REQ_GET)
    alg = 2 * int(reqs["bytes"][copies].astype(np.int64).sum()) + 4 * int((reqs["op"] == REQ_SIGNAL).sum())
    t0 = time.time()
    # exactly the requested steps, each one execution of the whole batch by
    # 64 forked ranks (about 8 ms each); 600 s is only a safety bound
    cb = cpu_baseline(reqs, C4["npes"], C4["heap"], max_seconds=600.0, warmup=args.warmup, reps=args.steps)
    assert cb["reps"] == args.steps, cb
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": cb["reps"],
            "warmup": args.warmup, "ms_per_step": round(cb["ms_per_step"], 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded)", "impl": "reference",
            "config": line_config(alg, args.gpus),
            "parallelism_detail": "one OS process per PE (64 forked ranks), memcpy into a shared mapping, "
                                  "process-shared pthread barrier",
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": round(time.time() - t0, 1)}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------- GPU arm
def l2_flusher():
    import torch
    buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def flush():
        buf.fill_(1)
        torch.cuda.synchronize()
    return flush


def startup_rows(table, k=4):
    """The k table rows the startup tune re-times: the k most robust
    graph-mode shapes (smallest worst slowdown over the tuner's C4 seeds),
    with the best 8-warp shape in place of the last when none of them has 8
    warps (the 4-warp shapes have a slow mode on some boxes that the 8-warp
    ones do not share); the sweep's first k for a table without that
    ranking."""
    if "robust" in table:
        ranked = sorted(table["robust"]["candidates"], key=lambda r: (r["worst_ratio"], r["mean_ratio"]))
        rows = ranked[:k]
        wide = [r for r in ranked if r["cfg"]["threads"] >= 256]
        if wide and not any(r["cfg"]["threads"] >= 256 for r in rows):
            rows[-1] = wide[0]
        return rows
    return [r for r in table["results"] if r.get("ms_median", -1) > 0 and not r["cfg"].get("stream", 0)][:k]


def startup_tune(b, k=4, reps=7):
    """The tuned table's k best graph-mode configurations (startup_rows),
    re-timed on this box by the library's autotuner
    (nvshmemx_tune_batch: L2 flushed before every run, median of `reps`),
    which leaves the fastest set on the batch.  Done before the warm-up
    steps, outside every timed region: the ranking of the leading shapes
    changes from box to box while the table is measured once."""
    from nvshmem_b200 import _lib as L
    from nvshmem_b200.tune import tune_batch
    if not os.path.exists(TUNED):
        return None
    with open(TUNED) as f:
        table = json.load(f)
    rows = startup_rows(table, k)
    cands = []
    for r in rows:
        c = L.BatchConfig()
        for key, v in r["cfg"].items():
            setattr(c, key, int(v))
        cands.append(c)
    res, best = tune_batch(b, cands, reps=reps)
    return {"candidates": [{"cfg": {key: r["cfg"][key] for key in ("tma_stages", "tma_stage_bytes", "threads",
                                                                     "chunk_bytes", "tma_min_bytes")},
                            "step_ms_median": round(r["ms_median"], 4)} for r in res],
            "chosen": best["cfg"]}


def load_tuned():
    if os.path.exists(TUNED):
        with open(TUNED) as f:
            return json.load(f).get("best")
    return None


def run_extras(peak):
    """Latency metrics (C1 ping-pong, device barrier on 8 PEs) and C2 bulk
    all-to-all throughput (8 PEs, rotating buffer sets larger than 2x L2)."""
    import numpy as np
    from nvshmem_b200 import MODE_BLOCK, MODE_BULK, REQ_PUT, DT_FLOAT, Shmem
    out = {}
    with Shmem(2, 8 << 20) as sh:
        flag = sh.alloc(4)
        ns, _ = sh.pingpong(flag, 0, 0, 10000, 20)
        out["pingpong_rtt_ns"] = {"p50": round(float(np.percentile(ns, 50)), 1),
                                  "p99": round(float(np.percentile(ns, 99)), 1), "iters": 10000}
        # the same exchange with the flag word on 32 other 128-byte lines
        # (other L2 slices): the round trip depends on where the line lives
        p50s = []
        for k in range(32):
            off = (k * 37 * 4096 + k * 640) % (1 << 20) // 128 * 128
            ns, _ = sh.pingpong(off, 2 << 20, 0, 3000, 20)
            p50s.append(round(float(np.percentile(ns, 50)), 1))
        out["pingpong_p50_ns_over_flag_lines"] = {"lines": 32, "iters": 3000, "sorted": sorted(p50s)}
    with Shmem(8, 1 << 20) as sh:
        bar = {}
        for ctas in (1, 16):
            for counted, kind in ((False, "ticket"), (True, "counted")):
                ns, _ = sh.barrier_latency(ctas, 10000, counted)
                bar[f"{kind}_{ctas}_cta_per_pe"] = {"p50": round(float(np.percentile(ns, 50)), 1),
                                                    "p99": round(float(np.percentile(ns, 99)), 1)}
        out["barrier_ns"] = bar
        out["offload_barrier_us_per_call"] = round(sh.offload_barrier(1000), 3)
    # C2 bulk all-to-all: 8 PEs, 1 MiB and 16 MiB messages, rotating sets > 2x L2
    a2a = {}
    for nbytes in (1 << 20, 16 << 20):
        nsets = max(2, (512 << 20) // (2 * 8 * 8 * nbytes) + 1)
        heap = 2 * 8 * nbytes * nsets
        with Shmem(8, heap) as sh:
            for pe in range(8):
                sh.fill_random(pe, 0, heap, 1)
            rounds = 4 * nsets
            for mode, name in ((MODE_BLOCK, "block"), (MODE_BULK, "bulk")):
                ctas = 18 if name == "block" else 18
                sh.alltoall(REQ_PUT, DT_FLOAT, 0, 8 * nbytes, nbytes, rounds=nsets, nsets=nsets,
                            set_stride=16 * nbytes, mode=mode, ctas_per_pe=ctas)
                ms = sh.alltoall(REQ_PUT, DT_FLOAT, 0, 8 * nbytes, nbytes, rounds=rounds, nsets=nsets,
                                 set_stride=16 * nbytes, mode=mode, ctas_per_pe=ctas)
                gbs = 2 * 8 * 7 * nbytes * rounds / (ms / 1e3) / 1e9
                a2a[f"{nbytes >> 20}MiB_{name}"] = {"GBps": round(gbs, 1), "frac": round(gbs / peak, 3)}
            assert sh.status() == 0
    out["alltoall_8pe"] = a2a
    return out


def run_c1_sweep():
    """C1 put sweep: PE 0 puts 4 B .. 1 MiB of float32 payload (uniform in
    [-1, 1), seed 0) to PE 1 with one call: nvshmem_float_put by one thread
    (the prototype's shape), and the CTA and CTA-TMA cooperative forms.  Each
    figure is one launch with one request (launch overhead included)."""
    import numpy as np
    from nvshmem_b200 import DT_FLOAT, MODE_BLOCK, MODE_BULK, MODE_THREAD, REQ_PUT, REQUEST_DTYPE, Shmem
    from nvshmem_b200.traffic import c1_float_payload, c1_sizes
    heap = 8 << 20
    out = {}
    with Shmem(2, heap) as sh:
        payload = c1_float_payload((1 << 20) // 4, seed=0)
        sh.write(0, 0, payload)
        for size in c1_sizes():
            r = np.zeros(1, REQUEST_DTYPE)
            r[0] = (0, 4 << 20, size, 0, 1, REQ_PUT, DT_FLOAT, 0, 0)
            row = {}
            for mode, name in ((MODE_THREAD, "thread"), (MODE_BLOCK, "cta"), (MODE_BULK, "cta_tma")):
                sh.exec_requests(r, mode)
                ts = sorted(sh.exec_requests(r, mode) for _ in range(5))
                us = 1e3 * ts[2]
                row[name] = {"us": round(us, 2), "GBps": round(2 * size / (us * 1e-6) / 1e9, 2)}
            assert sh.compare(1, 4 << 20, 0, 0, size) == 0
            out[str(size)] = row
        assert sh.status() == 0
    return out


C2_SIZES = [8 << k for k in range(26)]  # 8 B .. 256 MiB
C2_TYPES = ((0, "int32"), (1, "float32"), (2, "float64"))


def run_c2_sweep(peak, only_size=0):
    """C2 all-to-all on 8 PEs, every message size from 8 B to 256 MiB in
    powers of two, for int32, float32 and float64 payloads (random bits from
    seed 1): each round every PE puts (or gets) one message to (from) each of
    the 7 others through the CTA-wide TMA ring form (18 CTAs per PE), then
    quiet + device barrier; buffer sets rotate so that large working sets
    exceed 2x L2.  Below 1 MiB a round is mostly its fixed cost, reported as
    us per round.  Every received message is compared with its source on the
    device after each size.  The prototype's structure (a launch per round +
    the host's nvshmem_barrier_all) is timed beside it on float32 at six
    sizes."""
    from nvshmem_b200 import MODE_BULK, REQ_GET, REQ_PUT, Shmem
    out = {}
    sizes = [only_size] if only_size else C2_SIZES
    host_sizes = {8, 512, 32 << 10, 1 << 20, 16 << 20, 256 << 20}
    for nbytes in sizes:
        nsets = max(1, min(8, (512 << 20) // (2 * 8 * 8 * nbytes)))
        heap = max(2 * 8 * nbytes * nsets, 1 << 20)
        rounds = max(nsets, min(400, int(4e9 // max(112 * nbytes, 1))))
        row = {}
        with Shmem(8, heap) as sh:
            for pe in range(8):
                sh.fill_random(pe, 0, heap, 1)
            for dt, tname in C2_TYPES:
                cell = {}
                for op, name in ((REQ_PUT, "put"), (REQ_GET, "get")):
                    kw = dict(rounds=rounds, nsets=nsets, set_stride=16 * nbytes, mode=MODE_BULK, ctas_per_pe=18)
                    sh.alltoall(op, dt, 0, 8 * nbytes, nbytes, **dict(kw, rounds=nsets))
                    ms = sh.alltoall(op, dt, 0, 8 * nbytes, nbytes, **kw)
                    gbs = 2 * 8 * 7 * nbytes * rounds / (ms / 1e3) / 1e9
                    cell[name] = {"GBps": round(gbs, 1), "frac": round(gbs / peak, 3),
                                  "us_per_round": round(1e3 * ms / rounds, 2)}
                row[tname] = cell
            if nbytes in host_sizes:
                kw = dict(rounds=min(rounds, 50), nsets=nsets, set_stride=16 * nbytes, mode=MODE_BULK,
                          ctas_per_pe=18, host_rounds=True)
                ms = sh.alltoall(REQ_PUT, 1, 0, 8 * nbytes, nbytes, **kw)
                gbs = 2 * 8 * 7 * nbytes * kw["rounds"] / (ms / 1e3) / 1e9
                row["put_host_rounds_float32"] = {"GBps": round(gbs, 1), "frac": round(gbs / peak, 3),
                                                  "us_per_round": round(1e3 * ms / kw["rounds"], 2)}
            for p in range(8):
                for q in range(8):
                    if p != q:
                        assert sh.compare(q, 8 * nbytes + p * nbytes, p, q * nbytes, nbytes) == 0
            assert sh.status() == 0
        out[f"{nbytes}B"] = row
    big = [c["frac"] for k, r in out.items() if int(k[:-1]) >= (1 << 20)
           for t, cell in r.items() if t in ("int32", "float32", "float64") for c in cell.values()]
    if big:
        out["min_frac_1MiB_and_up"] = min(big)
    return out


def c3_nbr(pe, d, px=2, py=2, pz=2):
    """Neighbour of `pe` in direction d (0..5 = -x,+x,-y,+y,-z,+z) on the
    periodic px x py x pz grid (PE = x + px*(y + py*z))."""
    x, y, z = pe % px, (pe // px) % py, pe // (px * py)
    s = 1 if d & 1 else -1
    if d < 2:
        x = (x + s) % px
    elif d < 4:
        y = (y + s) % py
    else:
        z = (z + s) % pz
    return x + px * (y + py * z)


def c3_faces(block, n):
    """The six faces of one (z, y, x) block as the halo sends them: face d
    row j is z=j over y (x faces), z=j over x (y faces), y=j over x (z faces)."""
    b = block.reshape(n, n, n)
    return [b[:, :, 0], b[:, :, n - 1], b[:, 0, :], b[:, n - 1, :], b[0, :, :], b[n - 1, :, :]]


def run_c3_halo(peak, iters=100):
    """C3: 8 PEs on a periodic 2x2x2 grid, 256^3 float64 per PE (N(0,1),
    seed 3), 100 iterations of 6 face puts (x faces gathered with stride 256)
    + int_p signals + int_wait + a barrier: the device barrier inside one
    persistent launch (headline), and one launch per iteration followed by
    nvshmem_barrier_all_offload (the prototype's structure).  After each
    timed run every PE's six ghost faces and six signal words are read back
    and checked bit for bit against the faces of its neighbours' blocks."""
    import numpy as np
    from nvshmem_b200 import Shmem
    from nvshmem_b200.traffic import c3_block
    n = 256
    block, ghosts = n ** 3 * 8, 6 * n * n * 8
    heap = block + ghosts + 4096
    sig = block + ghosts
    faces = []
    with Shmem(8, heap) as sh:
        for pe in range(8):
            b = c3_block(n, pe)
            sh.write(pe, 0, b)
            faces.append([np.ascontiguousarray(f).view(np.uint8).reshape(-1) for f in c3_faces(b, n)])
            del b
            sh.memset(pe, block, 0, ghosts + 4096)

        def check(tag):
            for q in range(8):
                got = sh.read(q, block, ghosts + 24)
                for g in range(6):
                    want = faces[c3_nbr(q, g)][g ^ 1]
                    assert np.array_equal(got[g * n * n * 8:(g + 1) * n * n * 8], want), (tag, q, g)
                assert np.array_equal(got[ghosts:].view(np.int32), np.full(6, iters, np.int32)), (tag, q)

        # ctas_per_pe 0: as many CTAs per PE as stay co-resident (the
        # exchange is latency-bound, so more warps in flight help)
        sh.halo(2, 2, 2, n, 0, block, sig, 3, 0)
        for pe in range(8):
            sh.memset(pe, block, 0, ghosts + 64)
        ms = sh.halo(2, 2, 2, n, 0, block, sig, iters, 0)
        assert sh.status() == 0
        check("persistent")
        for pe in range(8):
            sh.memset(pe, block, 0, ghosts + 64)
        ms_off = sh.halo(2, 2, 2, n, 0, block, sig, iters, 0, offload=True)
        assert sh.status() == 0
        check("offload")
        # the x faces' scattered reads alone (one 8-byte element per 2 KiB
        # row, both faces of all 8 PEs at once): the best of a few grid sizes
        gather = min(sh.strided_read(0, (n - 1) * 8, 2, n * n, 8 * n, cp, 50) / 50 for cp in (18, 37, 74, 148))
    face_bytes = 8 * 6 * n * n * 8
    us = 1e3 * ms / iters
    # ceiling of one iteration's data movement: the x-face gather as measured
    # above, plus the four contiguous faces (read + write) and the x faces'
    # contiguous stores at the copy peak; synchronisation is not included
    contig_us = (8 * 4 * n * n * 8 * 2 + 8 * 2 * n * n * 8) / (peak * 1e3)
    ceiling_us = 1e3 * gather + contig_us
    return {"us_per_iter": round(us, 2), "face_GBps": round(2 * face_bytes * iters / (ms / 1e3) / 1e9, 1),
            "iters": iters, "n": n, "ctas_per_pe": "as many as stay co-resident",
            "offload_barrier_us_per_iter": round(1e3 * ms_off / iters, 2),
            "x_face_gather_ceiling_us": round(1e3 * gather, 2), "contiguous_faces_at_peak_us": round(contig_us, 2),
            "frac_of_gather_ceiling": round(ceiling_us / us, 3),
            "bit_exact": "every ghost face and signal word of all 8 PEs after each timed run"}


def run_c5_picker():
    from nvshmem_b200 import picker
    if not os.path.exists(picker.DATA):
        return {"unavailable": "no variant timings measured"}
    summary, _, _ = picker.evaluate(picker.DATA, epochs=400)
    return summary


def run_c4_heldout_seeds(flush, seeds=(8, 9, 10, 11), reps=5):
    """The tuned table's configuration (swept on the seed-4 batch, chosen over
    seeds 4-7) against the library default on C4 batches of seeds the tuner
    never saw: median graph step and exec kernel time, L2 flushed before each
    run."""
    from nvshmem_b200 import Shmem, default_batch_config, requests_bytes
    from nvshmem_b200.traffic import c4_batch
    tuned = load_tuned()
    default = default_batch_config().as_dict()
    out = {}
    with Shmem(C4["npes"], C4["heap"]) as sh:
        for pe in range(C4["npes"]):
            sh.fill_random(pe, 0, C4["heap"], 44)
        for seed in seeds:
            reqs = c4_batch(**dict(C4, seed=seed))
            alg = requests_bytes(reqs)
            row = {}
            with sh.batch(len(reqs), int(reqs["bytes"].sum()), 256) as b:
                b.upload(reqs)
                for name, cfg in (("tuned", tuned), ("default", default)):
                    if not cfg:
                        continue
                    b.set_config(cfg)
                    for _ in range(2):
                        flush()
                        b.execute(1)
                    st, ex = [], []
                    for _ in range(reps):
                        flush()
                        st.append(b.execute(1))
                        flush()
                        ex.append(b.execute_direct(1)[1])
                    row[name] = {"step_us": round(1e3 * statistics.median(st), 1),
                                 "exec_us": round(1e3 * statistics.median(ex), 1),
                                 "GBps": round(alg / (statistics.median(st) / 1e3) / 1e9, 1)}
            if "tuned" in row and "default" in row:
                row["tuned_gain_pct"] = round(100 * (row["default"]["step_us"] / row["tuned"]["step_us"] - 1), 2)
            out[f"seed{seed}"] = row
        assert sh.status() == 0
    return out


def run_c4_picked(steps, flush):
    """The C4 batch through nvshmemx_batch_execute_picked: host requests
    grouped by size class, width and alignment, a variant picked per group by
    the trained network (the measured table outside its range), each variant
    run once; L2 flushed before each step.  Checked against the batch engine's
    result (per-PE heap checksums) and timed beside it."""
    import numpy as np
    from nvshmem_b200 import PATTERN_RANDOM, Shmem, picker, requests_bytes
    from nvshmem_b200.traffic import c4_batch
    if not os.path.exists(picker.DATA):
        return {"unavailable": "no variant timings measured"}
    d = np.load(picker.DATA)
    pk = picker.Picker(d["train_x"], d["train_t"], seed=0)
    pk.fit(epochs=400)
    reqs = c4_batch(**C4)
    alg = requests_bytes(reqs)
    with Shmem(C4["npes"], C4["heap"]) as sh:
        for pe in range(C4["npes"]):
            sh.fill_random(pe, 0, C4["heap"], 44)
        with sh.batch(len(reqs), int(reqs["bytes"].sum()), 256) as b:
            b.upload(reqs)
            b.execute(1)
            want = [sh.checksum(pe, 0, C4["heap"]) for pe in range(C4["npes"])]
            ms, run_ms = [], []
            hb = b.host_buffer()
            hb[:len(reqs)] = reqs
            for i in range(steps + 1):
                flush()
                st, t, tr, groups = b.execute_picked(pk, hb[:len(reqs)], PATTERN_RANDOM)
                assert st == 0, f"picked execution status {st}"
                if i:
                    ms.append(t)
                    run_ms.append(tr)
            got = [sh.checksum(pe, 0, C4["heap"]) for pe in range(C4["npes"])]
            assert got == want, "picked execution differs from the batch engine"
        assert sh.status() == 0
    pk.close()
    per_variant = {}
    for g in groups:
        k = picker.VARIANT_NAMES[int(g["variant"])]
        per_variant[k] = per_variant.get(k, 0) + int(g["count"])
    med, run = statistics.median(ms), statistics.median(run_ms)
    return {"GBps": round(alg / (med / 1e3) / 1e9, 1), "ms": round(med, 4),
            "run_GBps": round(alg / (run / 1e3) / 1e9, 1), "run_ms": round(run, 4), "groups": int(len(groups)),
            "decided_by": {"network": int((groups["source"] == 0).sum()), "table": int((groups["source"] == 1).sum()),
                           "fixed": int((groups["source"] == 2).sum())},
            "requests_per_variant": per_variant,
            "timing": ("GBps / ms: device time from the start of the host-to-device copy of the 32-byte requests "
                       "(from pinned memory) to the end of the last run; run_GBps / run_ms: after the copy")}


def cpu_latency():
    from oracle import model as om
    if not os.path.exists(om.HOST_BENCH):
        om.build()
    pp = json.loads(subprocess.run([om.HOST_BENCH, "pingpong", "10000"], capture_output=True, text=True,
                                   timeout=300, check=True).stdout.strip().splitlines()[-1])
    br = json.loads(subprocess.run([om.HOST_BENCH, "barrier", "8", "10000"], capture_output=True, text=True,
                                   timeout=300, check=True).stdout.strip().splitlines()[-1])
    return {"pingpong_rtt_ns_p50": pp["p50_ns"], "barrier_8_ns_p50": br["p50_ns"], "cores": br["cores"],
            "kind": "port"}


def run_gpu(args, rank, world, local):
    import numpy as np
    import torch

    torch.cuda.set_device(local)
    from nvshmem_b200 import (MODE_BLOCK, MODE_BULK, MODE_THREAD, MODE_WARP, REQ_PUT, DT_FLOAT, Shmem, requests_bytes,
                              to_compact)
    from nvshmem_b200.traffic import c4_batch

    dist = dist_init(world)
    peak, peak_kind = measured_peak()
    flush = l2_flusher()
    C4 = globals()["C4"] if args.workload == "c4" else C4_SMALL
    reqs = c4_batch(**C4)
    alg = requests_bytes(reqs)
    payload = int(reqs["bytes"].sum())
    out = {}
    sampler = ClockSampler(local)
    with sampler:
        with Shmem(C4["npes"], C4["heap"]) as sh:
            for pe in range(C4["npes"]):
                sh.fill_random(pe, 0, C4["heap"], 44)
            with sh.batch(len(reqs), payload, 256) as b:
                tuned = load_tuned()
                if tuned:
                    b.set_config(tuned)
                b.upload(reqs)
                startup = startup_tune(b) if tuned else None
                for _ in range(args.warmup):
                    flush()
                    b.execute(1)
                # device-resident batches: K steps, L2 flushed between steps
                torch.cuda.synchronize()
                barrier(dist)
                step_ms = []
                for _ in range(args.steps):
                    flush()
                    step_ms.append(b.execute(1))
                torch.cuda.synchronize()
                barrier(dist)
                t_batch = reduce_max(dist, sum(step_ms) / 1e3)
                chunks = b.stats()[0]
                # the exec kernel alone (CUDA events around it on its stream)
                exec_ms = []
                for _ in range(args.steps):
                    flush()
                    exec_ms.append(b.execute_direct(1)[1])
                # per-call path on the same batch (one thread per request)
                pc = {}
                for mode, name in ((MODE_THREAD, "thread"), (MODE_WARP, "warp")):
                    flush()
                    b.percall(mode, 1)
                    ts = []
                    for _ in range(max(1, args.steps // 5)):
                        flush()
                        ts.append(b.percall(mode, 1))
                    pc[name] = alg / (statistics.median(ts) / 1e3) / 1e9
                # end to end: host-resident requests each step
                hb = b.host_buffer()
                hb[:len(reqs)] = reqs
                for _ in range(args.warmup):
                    flush()
                    b.submit(hb, len(reqs))
                barrier(dist)
                e2e_ms = []
                for _ in range(args.steps):
                    flush()
                    st, ms = b.submit(hb, len(reqs))
                    assert st == 0, f"batch status {st}"
                    e2e_ms.append(ms)
                barrier(dist)
                t_e2e_full = reduce_max(dist, sum(e2e_ms) / 1e3)
                # the same through the 16-byte compact request form (half the
                # bytes over the host link): the headline end-to-end figure
                hc = b.host_buffer_compact()
                hc[:len(reqs)] = to_compact(reqs)
                for _ in range(args.warmup):
                    flush()
                    b.submit_compact(hc, len(reqs))
                barrier(dist)
                e2e_ms, e2e_wall = [], []
                for _ in range(args.steps):
                    flush()
                    w0 = time.perf_counter()
                    st, ms = b.submit_compact(hc, len(reqs))
                    e2e_wall.append(time.perf_counter() - w0)
                    assert st == 0, f"batch status {st}"
                    e2e_ms.append(ms)
                barrier(dist)
                t_e2e = reduce_max(dist, sum(e2e_ms) / 1e3)
                t_e2e_wall = reduce_max(dist, sum(e2e_wall))
                cfg_used = b.config()
            assert sh.status() == 0
            checks = [sh.checksum(pe, 0, C4["heap"]) for pe in range(C4["npes"])]
        if args.only != "batch":
            out.update(run_extras(peak))
            out["c1_float_put_sweep"] = run_c1_sweep()
            out["c2_alltoall_sweep"] = run_c2_sweep(peak)
            out["c3_halo"] = run_c3_halo(peak)
            out["c5_picker_regret"] = run_c5_picker()
            out["c4_picked"] = run_c4_picked(max(3, args.steps // 4), flush)
            out["c4_heldout_seeds"] = run_c4_heldout_seeds(flush)
    clocks = sampler.summary()

    value = world * alg * args.steps / t_batch / 1e9
    e2e = world * alg * args.steps / t_e2e / 1e9
    e2e_full = world * alg * args.steps / t_e2e_full / 1e9
    e2e_wall = world * alg * args.steps / t_e2e_wall / 1e9
    exec_avg = statistics.mean(exec_ms) / 1e3
    achieved = alg / exec_avg / 1e9
    traffic = None
    if os.path.exists(NCU_SUMMARY):
        with open(NCU_SUMMARY) as f:
            traffic = json.load(f).get("dram_bytes_per_launch")
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1e3 * t_batch / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded)",
        "config": line_config(alg, world),
        "batch_detail": {"batch_config": cfg_used, "chunks": chunks, "startup_tune": startup},
        "frac_of_hbm": round(value / peak, 3),
        "percall_GBps": {k: round(v, 2) for k, v in pc.items()},
        "speedup_vs_percall_thread": round(value / pc["thread"], 2),
        "e2e": {"value": round(e2e, 2), "unit": UNIT, "h2d_bytes_per_step": int(len(reqs) * 16),
                "d2h_bytes_per_step": 8,
                "mode": ("nvshmemx_batch_submit_compact (16-byte requests from pinned host memory), pipelined: "
                         "the first quarter of the requests executes while the rest is copied"),
                "timing": ("CUDA events on the batch stream, from before the request copy to after the "
                           "status word reached host memory"),
                "host_wall": {"value": round(e2e_wall, 2),
                              "timing": "host clock around the Python call (ctypes entry to return, the final "
                                        "stream synchronisation included)"},
                "full_form": {"value": round(e2e_full, 2), "h2d_bytes_per_step": int(len(reqs) * 32),
                              "call": "nvshmemx_batch_submit (32-byte requests)"}},
        # plan + exec per device-resident step; 2 x (plan + exec) + the
        # status kernel per pipelined end-to-end step
        "gpu_launches": 2 * args.steps + 5 * args.steps,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 3), "traffic": traffic,
                     "kernel": ("batch_exec_tma_kernel" if cfg_used.get("tma_stages") else "batch_exec_kernel"),
                     "peak_kind": peak_kind, "alg_bytes_per_launch": alg,
                     "traffic_source": "profiles/batch_exec_c4.json (ncu, full size, 1 pass)"},
        "clocks": clocks,
        "heap_checksum": int(sum(checks) % (1 << 64)),
    }
    line.update(out)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = {k: v for k, v in cpu_baseline(reqs, C4["npes"], C4["heap"]).items()
                                if k in ("value", "unit", "cores", "kind", "sample")}
        if args.only != "batch":
            line["cpu_latency"] = cpu_latency()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="c4", choices=["c4", "c4-small"])
    ap.add_argument("--only", default="all", choices=["all", "batch", "c2", "c3"],
                    help="all: the contract line with every section; batch: the C4 line alone; "
                         "c2 / c3: one diagnostic JSON line for that section alone (for profiling)")
    ap.add_argument("--c2-size", type=int, default=0, help="with --only c2: one message size in bytes")
    ap.add_argument("--c3-iters", type=int, default=100, help="with --only c3: timed iterations")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.only in ("c2", "c3"):
        import torch
        torch.cuda.set_device(local)
        peak, _ = measured_peak()
        out = run_c2_sweep(peak, args.c2_size) if args.only == "c2" else run_c3_halo(peak, args.c3_iters)
        if rank == 0:
            print(json.dumps({"section": args.only, "result": out}), flush=True)
        return
    run_gpu(args, rank, world, local)


if __name__ == "__main__":
    main()
